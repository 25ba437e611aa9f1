"""GPU key generation (cmd_kem_keypair*) against the oracle.

- the seed stored in each shipped secret key regenerates that secret key byte
  for byte on the GPU, and the public key equals the oracle's (which equals the
  reference's own pk_gen; tests/test_keygen_oracle.py);
- a batch of fresh seeds gives, key by key, the oracle's key pairs and attempt
  counts (rejected attempts continue with the next seed, as the reference
  does);
- a generated key decrypts: weight-t vectors encrypted with the generated
  public key under the reference's syndrome rule decode to themselves.
"""
from __future__ import annotations

import numpy as np
import pytest

import cm_decrypt__b200 as cmd
from conftest import SETS, golden_sk, rng
from test_keygen_oracle import pk_syndromes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("s", SETS)
def test_keypair_regenerates_shipped_key(oracle_mod, engine, s):
    sk_ref = golden_sk(s)
    pk, sk, attempts = cmd.kem_keypair(engine, s, sk_ref[:32])
    assert attempts == 1
    assert sk == sk_ref
    pk_o, _, _ = oracle_mod.Oracle(s).keypair(sk_ref[:32])
    assert pk == pk_o


@pytest.mark.parametrize("s", SETS)
def test_keypair_batch_matches_oracle(oracle_mod, engine, s):
    o = oracle_mod.Oracle(s)
    count = 5 if s in (348864, 6960119) else 3
    seeds = np.frombuffer(rng(100 + s % 97).bytes(32 * count), np.uint8).reshape(count, 32)
    pks, sks, att = cmd.kem_keypair_batch(engine, s, seeds)
    for i in range(seeds.shape[0]):
        pk_o, sk_o, a_o = o.keypair(seeds[i].tobytes())
        assert int(att[i]) == a_o, i
        assert sks[i].tobytes() == sk_o, i
        assert pks[i].tobytes() == pk_o, i


@pytest.mark.parametrize("s", [348864, 460896, 6960119, 8192128])
def test_generated_key_decrypts(engine, s):
    info = cmd.set_info(s)
    pk, sk, _ = cmd.kem_keypair(engine, s, rng(5).bytes(32))
    g = rng(6)
    count = 64
    e = np.zeros((count, info.n), np.uint8)
    for i in range(count):
        e[i, g.choice(info.n, info.t, replace=False)] = 1
    cts = pk_syndromes(pk, info.m, info.n, info.t, e)
    key = cmd.Key(engine, s, sk)
    try:
        err, w = cmd.decrypt(engine, key, cts)
        assert np.array_equal(err, np.packbits(e, axis=1, bitorder="little"))
        assert (w == info.t).all()
    finally:
        key.free()


def test_keypair_argument_errors(engine):
    with pytest.raises(Exception):
        cmd.kem_keypair(engine, 6960119, b"short")
    with pytest.raises(Exception):
        cmd.kem_keypair_batch(engine, 6960119, np.zeros((0, 32), np.uint8))


def test_keypair_batch_repeatable_and_matches_oracle(oracle_mod, engine):
    """A larger batch twice: identical results both times (no ordering
    dependence between the chained stages) and equal to the oracle."""
    s = 348864
    o = oracle_mod.Oracle(s)
    seeds = np.frombuffer(rng(4242).bytes(32 * 24), np.uint8).reshape(24, 32)
    first = cmd.kem_keypair_batch(engine, s, seeds)
    again = cmd.kem_keypair_batch(engine, s, seeds)
    for a, b in zip(first, again):
        assert np.array_equal(a, b)
    pks, sks, att = first
    for i in range(seeds.shape[0]):
        pk_o, sk_o, a_o = o.keypair(seeds[i].tobytes())
        assert (int(att[i]), sks[i].tobytes(), pks[i].tobytes()) == (a_o, sk_o, pk_o), i
