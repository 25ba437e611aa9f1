"""Pins the C restatement (oracle/cmd_oracle.c) before anything is checked
against it:
  * against the reference decoder's own errorstreams for the regenerated kem/
    fixtures (tests/golden/kem, made by gen_kem_vectors.sh from the
    reference's CPU/ binaries);
  * against the reference's own CPU/ sources compiled into oracle/_ref
    (exhaustive field sweeps, support generation, inverse tables, and the
    synd / bm / root stages on random inputs), when that build is present.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from conftest import KEM, SETS, golden_ct, golden_errorstream, golden_sk, rng


def _sha_ok(name: str) -> bool:
    sums = dict(line.split()[::-1] for line in open(os.path.join(KEM, "SHA256SUMS")))
    return hashlib.sha256(open(os.path.join(KEM, name), "rb").read()).hexdigest() == sums[name]


@pytest.mark.parametrize("s", SETS)
def test_fixtures_intact(s):
    for name in (f"sk_{s}.bin", f"ct_{s}.bin", f"errorstream0_{s}.bin"):
        assert _sha_ok(name), name


@pytest.mark.parametrize("s", SETS)
def test_oracle_matches_reference_errorstream(oracle_mod, s):
    o = oracle_mod.Oracle(s)
    cts = np.frombuffer(golden_ct(s), np.uint8).reshape(-1, o.ct_bytes)
    err = o.decrypt(golden_sk(s), cts)
    assert o.errorstream(err) == golden_errorstream(s)


def _ref(oracle_mod, s):
    if not oracle_mod.RefLib.available(s):
        pytest.skip("reference build oracle/_ref absent (needs the reference tree at build time)")
    return oracle_mod.RefLib(s)


@pytest.mark.parametrize("m_set", [348864, 6960119])  # m = 12 and m = 13
def test_field_exhaustive(oracle_mod, m_set):
    o, r = oracle_mod.Oracle(m_set), _ref(oracle_mod, m_set)
    for a in range(1 << o.m):
        assert np.array_equal(o.gf_mul_row(a), r.gf_mul_row(a)), a
    for num in range(0, 1 << o.m, 7):
        assert np.array_equal(o.gf_frac_row(num), r.gf_frac_row(num)), num


@pytest.mark.parametrize("s", SETS)
def test_key_expansion_matches_reference(oracle_mod, s):
    o, r = oracle_mod.Oracle(s), _ref(oracle_mod, s)
    sk = golden_sk(s)
    g, L, tab = o.expand(sk)
    r.load_sk(sk)
    assert np.array_equal(g, r.goppa())
    assert np.array_equal(L, r.support())
    assert np.array_equal(tab, r.inverse_table())
    # arbitrary control bits (support of a derived key)
    cond = rng(s).integers(0, 256, (2 ** (o.m - 4)) * (2 * o.m - 1), dtype=np.uint8).tobytes()
    assert np.array_equal(o.support_from_cond(cond), r.support_from_cond(cond))


@pytest.mark.parametrize("s", SETS)
def test_stages_match_reference(oracle_mod, s):
    o, r = oracle_mod.Oracle(s), _ref(oracle_mod, s)
    sk = golden_sk(s)
    o.expand(sk)
    r.load_sk(sk)
    g = rng(100 + s)
    for _ in range(6):
        ct = g.integers(0, 256, o.ct_bytes, dtype=np.uint8).tobytes()
        s1, s2 = o.synd(ct), r.synd(ct)
        assert np.array_equal(s1, s2)
        l1, l2 = o.bm(s1), r.bm(s2)
        assert np.array_equal(l1, l2)
        assert np.array_equal(o.root(l1), r.root(l2))
    # BM on arbitrary syndromes (exercises L > t paths the decoder can reach)
    for _ in range(6):
        syn = g.integers(0, 1 << o.m, 2 * o.t, dtype=np.uint16)
        assert np.array_equal(o.bm(syn), r.bm(syn))


@pytest.mark.parametrize("s", SETS)
def test_oracle_decrypt_matches_reference_threads(oracle_mod, s):
    o, r = oracle_mod.Oracle(s), _ref(oracle_mod, s)
    cts = rng(7 + s).integers(0, 256, (12, o.ct_bytes), dtype=np.uint8)
    assert np.array_equal(o.decrypt(golden_sk(s), cts, nthreads=3), r.decrypt(golden_sk(s), cts, nthreads=4))


def test_reference_cli_contract(oracle_mod, tmp_path):
    """The unmodified reference CLI, run in its expected directory layout,
    reproduces the committed errorstream (pins the fixture pipeline)."""
    import shutil
    import subprocess
    s = 348864
    exe = os.path.join(os.path.dirname(oracle_mod.__file__), "_ref", "bin", f"decrypt_{s}")
    if not os.path.exists(exe):
        pytest.skip("reference CLI not built")
    work = tmp_path / "CPU" / "param" / f"param{s}"
    work.mkdir(parents=True)
    (tmp_path / "CPU" / "results" / "output").mkdir(parents=True)
    vec = tmp_path / "kem" / "test_vectors" / "Cipher_Sk"
    vec.mkdir(parents=True)
    shutil.copy(os.path.join(KEM, f"sk_{s}.bin"), vec)
    shutil.copy(os.path.join(KEM, f"ct_{s}.bin"), vec)
    subprocess.run([exe, "5"], cwd=work, check=True, capture_output=True)
    got = (tmp_path / "CPU" / "results" / "output" / f"errorstream0_{s}.bin").read_bytes()
    assert got == golden_errorstream(s)
