"""Key-generation checkers on the CPU.

The oracle's restatement of crypto_kem_keypair (oracle/cmd_oracle.c
o_kg_*, oracle/oracle.py keypair_from_seed) is pinned three ways:
- from the seed stored in each shipped secret key it rebuilds that secret key
  byte for byte (the reference wrote them: kem/common/core/operations.c:36-107);
- it agrees with the reference's own kem/ key generation (oracle/_ref/
  libkeygen_<set>.so: genpoly_gen, pk_gen, controlbitsfrompermutation) on
  fresh seeds, rejected attempts included, and stage by stage;
- its public key re-encrypts the reference's shipped ciphertexts from their
  decoded error vectors with the reference's syndrome rule (encrypt.c:66-96).
  For n < 2^m, kem/ drops error positions >= n (encrypt.c:147-190), so those
  ciphertexts carry fewer than t errors and the decoder also flags the
  support position holding the zero field element; that one position is not
  part of the encrypted vector.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SETS, golden_ct, golden_errorstream, golden_sk, rng


def pk_syndromes(pk: bytes, m: int, n: int, t: int, e_bits: np.ndarray) -> np.ndarray:
    """encrypt.c:66-96: row i = pk row i placed in the last (n-mt+7)/8 bytes of
    an n-bit row, identity bit i set; syndrome bit i = <row i, e>."""
    mt = m * t
    row_b = (n - mt + 7) // 8
    rows = np.zeros((mt, n // 8), np.uint8)
    rows[:, n // 8 - row_b:] = np.frombuffer(pk, np.uint8).reshape(mt, row_b)
    idx = np.arange(mt)
    rows[idx, idx // 8] |= (1 << (idx % 8)).astype(np.uint8)
    H = np.unpackbits(rows, axis=1, bitorder="little")[:, :n].astype(np.int64)
    s = (H @ e_bits.T.astype(np.int64)) % 2  # [mt, count]
    return np.packbits(s.T.astype(np.uint8), axis=1, bitorder="little")


def errors_from_stream(text: bytes, n: int) -> np.ndarray:
    lines = [ln for ln in text.decode().split("\n") if ln.strip()]
    e = np.zeros((len(lines), n), np.uint8)
    for i, ln in enumerate(lines):
        for p in ln.split():
            e[i, int(p)] = 1
    return e


@pytest.mark.parametrize("s", SETS)
def test_oracle_keypair_rebuilds_shipped_sk(oracle_mod, s):
    sk = golden_sk(s)
    pk, sk2, attempts = oracle_mod.Oracle(s).keypair(sk[:32])
    assert attempts == 1
    assert sk2 == sk


@pytest.mark.parametrize("s", SETS)
def test_oracle_pk_reencrypts_shipped_ciphertexts(oracle_mod, s):
    o = oracle_mod.Oracle(s)
    sk = golden_sk(s)
    pk, _, _ = o.keypair(sk[:32])
    assert len(pk) == o.m * o.t * ((o.n - o.m * o.t + 7) // 8)
    _, L, _ = o.expand(sk)
    zero = int(np.nonzero(L == 0)[0][0])  # support position of the field element 0
    e = errors_from_stream(golden_errorstream(s), o.n)
    cts = np.frombuffer(golden_ct(s), np.uint8).reshape(-1, o.ct_bytes)
    assert e.shape[0] == cts.shape[0] > 0
    for i in range(e.shape[0]):
        ei = e[i: i + 1].copy()
        if ei.sum() < o.t + 1 and ei[0, zero] and not np.array_equal(pk_syndromes(pk, o.m, o.n, o.t, ei)[0], cts[i]):
            ei[0, zero] = 0  # the decoder's flag at the zero element when fewer than t errors were sent
        assert np.array_equal(pk_syndromes(pk, o.m, o.n, o.t, ei)[0], cts[i]), (s, i)


@pytest.mark.parametrize("s", SETS)
def test_oracle_keypair_matches_reference_keygen(oracle_mod, s):
    if not oracle_mod.RefKeygen.available(s):
        pytest.skip("reference key generation not built (oracle/_ref)")
    o, r = oracle_mod.Oracle(s), oracle_mod.RefKeygen(s)
    assert o.keypair(golden_sk(s)[:32]) == r.keypair(golden_sk(s)[:32])  # public keys too
    seed = rng(s).bytes(32)
    assert o.keypair(seed) == r.keypair(seed)


@pytest.mark.parametrize("s", [348864, 6960119])
def test_oracle_controlbits_match_reference(oracle_mod, s):
    if not oracle_mod.RefKeygen.available(s):
        pytest.skip("reference key generation not built (oracle/_ref)")
    o, r = oracle_mod.Oracle(s), oracle_mod.RefKeygen(s)
    g = rng(7)
    for pi in (np.arange(1 << o.m), np.arange(1 << o.m)[::-1], g.permutation(1 << o.m), g.permutation(1 << o.m)):
        pi = pi.astype(np.int16)
        assert np.array_equal(o.kg_controlbits(pi), r.kg_controlbits(pi))


@pytest.mark.parametrize("s", [348864, 460896, 6960119])
def test_oracle_genpoly_matches_reference_and_rejects_subfield(oracle_mod, s):
    if not oracle_mod.RefKeygen.available(s):
        pytest.skip("reference key generation not built (oracle/_ref)")
    o, r = oracle_mod.Oracle(s), oracle_mod.RefKeygen(s)
    g = rng(11)
    for _ in range(3):
        f = g.integers(0, 1 << o.m, o.t).astype(np.uint16)
        a, b = o.kg_genpoly(f), r.kg_genpoly(f)
        assert a is not None and np.array_equal(a, b)
    # f in GF(2^m) itself: minimal polynomial of degree 1, rejected
    f = np.zeros(o.t, np.uint16)
    f[0] = 5
    assert o.kg_genpoly(f) is None and r.kg_genpoly(f) is None


def test_oracle_pk_gen_rejects_repeated_words(oracle_mod):
    s = 348864
    o = oracle_mod.Oracle(s)
    irr = np.frombuffer(golden_sk(s)[40: 40 + 2 * o.t], "<u2")
    perm = rng(3).integers(0, 1 << 32, 1 << o.m, dtype=np.uint64).astype(np.uint32)
    perm[17] = perm[4000]
    assert o.kg_pk_gen(irr, perm) is None
    if oracle_mod.RefKeygen.available(s):
        assert oracle_mod.RefKeygen(s).kg_pk_gen(irr, perm) is None


@pytest.mark.parametrize("s", SETS)
def test_oracle_encrypt_matches_syndrome_rule_and_reference_decoder(oracle_mod, s):
    """o_encrypt_batch (the reference-only bench arm's input generator) equals
    the row-wise syndrome rule, re-encrypts the shipped ciphertexts, and its
    weight-t ciphertexts decode to their error vectors in the reference's own
    decoder."""
    o = oracle_mod.Oracle(s)
    sk = golden_sk(s)
    pk, _, _ = o.keypair(sk[:32])
    e = o.random_errors(seed=11 + s, count=6)
    bits = np.unpackbits(e, axis=1, bitorder="little")
    assert (bits.sum(axis=1) == o.t).all()
    assert not np.array_equal(e[0], e[1])
    cts = o.encrypt(pk, e)
    assert np.array_equal(cts, pk_syndromes(pk, o.m, o.n, o.t, bits))
    dec = (oracle_mod.RefLib(s) if oracle_mod.RefLib.available(s) else o).decrypt(sk, cts)
    assert np.array_equal(dec, e)
    # the shipped kem/ ciphertexts from their decoded vectors (zero-element
    # flag dropped when fewer than t errors were sent)
    _, L, _ = o.expand(sk)
    zero = int(np.nonzero(L == 0)[0][0])
    es = errors_from_stream(golden_errorstream(s), o.n)
    shipped = np.frombuffer(golden_ct(s), np.uint8).reshape(-1, o.ct_bytes)
    for i in range(es.shape[0]):
        ei = es[i].copy()
        if ei.sum() < o.t + 1 and ei[zero]:
            alt = ei.copy()
            alt[zero] = 0
            if np.array_equal(o.encrypt(pk, np.packbits(alt, bitorder="little")[None])[0], shipped[i]):
                continue
        assert np.array_equal(o.encrypt(pk, np.packbits(ei, bitorder="little")[None])[0], shipped[i]), (s, i)
