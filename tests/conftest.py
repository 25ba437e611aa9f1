"""Shared fixtures.  `-m gpu` tests drive the CUDA engine on a B200 and fail
loudly when it is missing; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")
KEM = os.path.join(GOLDEN, "kem")
SETS = (348864, 460896, 6688128, 6960119, 8192128)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA engine)")


def golden_sk(set_id: int) -> bytes:
    with open(os.path.join(KEM, f"sk_{set_id}.bin"), "rb") as f:
        return f.read()


def golden_ct(set_id: int) -> bytes:
    with open(os.path.join(KEM, f"ct_{set_id}.bin"), "rb") as f:
        return f.read()


def golden_errorstream(set_id: int) -> bytes:
    with open(os.path.join(KEM, f"errorstream0_{set_id}.bin"), "rb") as f:
        return f.read()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as o
    o.build(with_reference=None)
    return o


@pytest.fixture(scope="session")
def engine():
    import cm_decrypt__b200 as cmd
    eng = cmd.Engine(0)
    yield eng
    eng.close()


def rng(seed: int = 0) -> np.random.Generator:
    return np.random.default_rng(seed)
