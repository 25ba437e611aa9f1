"""CPU tests of the product library's host side (no GPU calls):
  * libcmd_b200.so loads and exports every function include/cmd_b200.h declares;
  * parameter table, error codes, errorstream text vs the oracle's;
  * the synthetic workload generator: derived keys are valid keys, valid
    ciphertexts decode (oracle) to exactly the planted weight-t error vector,
    malformed ones behave like the reference decoder on them, determinism.
"""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

import cm_decrypt__b200 as cmd
from conftest import REPO, SETS, golden_sk, rng


def declared_functions() -> list[str]:
    src = open(os.path.join(REPO, "include", "cmd_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cmd_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header():
    L = cmd.lib()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n


def test_set_info_table():
    expect = {348864: (12, 3488, 64, 96, 6492), 460896: (13, 4608, 96, 156, 13608),
              6688128: (13, 6688, 128, 208, 13932), 6960119: (13, 6960, 119, 194, 13948),
              8192128: (13, 8192, 128, 208, 14120)}
    for s, (m, n, t, ct, sk) in expect.items():
        i = cmd.set_info(s)
        assert (i.m, i.n, i.t, i.ct_bytes, i.sk_bytes) == (m, n, t, ct, sk)
        assert i.sb == 8 * ct and i.err_bytes == n // 8 and i.err_words == (n + 31) // 32


def test_no_device_is_an_error_not_a_fallback():
    # On a host without a B200 the engine refuses to start (no CPU fallback).
    import torch
    if torch.cuda.is_available():
        pytest.skip("host has a GPU")
    with pytest.raises(cmd.CmdError) as ei:
        cmd.Engine(0)
    assert ei.value.code == cmd.CMD_E_NODEVICE


@pytest.mark.parametrize("s", SETS)
def test_errorstream_text_matches_oracle(oracle_mod, s):
    o = oracle_mod.Oracle(s)
    info = cmd.set_info(s)
    err = rng(s).integers(0, 256, (7, info.err_bytes), dtype=np.uint8)
    err[2] = 0                      # empty decode -> bare newline
    err[3, :] = 0
    err[3, -1] = 0x80               # last position n-1
    err[4, 0] = 1                   # position 0
    assert cmd.errorstream(s, err) == o.errorstream(err)


def test_errorstream_write(tmp_path, oracle_mod):
    s = 6960119
    info = cmd.set_info(s)
    err = rng(1).integers(0, 2, (3, info.err_bytes), dtype=np.uint8)
    p = str(tmp_path / "e.bin")
    cmd.write_errorstream(s, err, p)
    cmd.write_errorstream(s, err[:1], p, append=True)
    assert open(p, "rb").read() == oracle_mod.Oracle(s).errorstream(np.concatenate([err, err[:1]]))
    with pytest.raises(cmd.CmdError) as ei:
        cmd.write_errorstream(s, err, str(tmp_path / "no" / "such" / "dir.bin"))
    assert ei.value.code == cmd.CMD_E_FILE


@pytest.mark.parametrize("s", SETS)
def test_synth_valid_ciphertexts_decode_to_planted_errors(oracle_mod, s):
    o = oracle_mod.Oracle(s)
    sk = cmd.synth_key(s, golden_sk(s), seed=11)
    assert len(sk) == o.sk_bytes and sk != golden_sk(s)
    pk = cmd.PubKey(s, sk)
    cts, err, valid = pk.ciphertexts(seed=5, count=6, malformed_permille=0)
    assert valid.all()
    got = o.decrypt(sk, cts, nthreads=6)
    assert np.array_equal(got, err)
    assert all(int(np.unpackbits(r).sum()) == o.t for r in err)
    # the base key itself also yields a systematic public key
    pk0 = cmd.PubKey(s, golden_sk(s))
    cts0, err0, _ = pk0.ciphertexts(seed=9, count=3)
    assert np.array_equal(o.decrypt(golden_sk(s), cts0), err0)


def test_synth_malformed_and_determinism(oracle_mod):
    s = 6960119
    sk = golden_sk(s)
    pk = cmd.PubKey(s, sk)
    a = pk.ciphertexts(seed=3, count=200, malformed_permille=500)
    b = pk.ciphertexts(seed=3, count=200, malformed_permille=500, nthreads=1)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    cts, err, valid = a
    assert 50 < int(valid.sum()) < 150
    # padding bits (mt..sb-1) are zero: 1547 bits -> top 5 bits of byte 193
    assert not (cts[:, 193] & 0xF8).any()
    assert not err[valid == 0].any()
    bad = cts[valid == 0][:8]
    o = oracle_mod.Oracle(s)
    dec = o.decrypt(sk, bad)
    # malformed strings rarely decode to anything of weight t
    assert all(int(np.unpackbits(r).sum()) < o.t for r in dec)


def test_synth_key_rejects_bad_args():
    with pytest.raises(ValueError):
        cmd.synth_key(99, b"\0" * 10, 1)
    assert cmd.lib().cmd_synth_key(7, None, 1, None) == cmd.CMD_E_ARG


def _sparse_errors(s, rows, seed):
    """Error vectors of weight 0..t (the only weights a decode can produce)."""
    info = cmd.set_info(s)
    g = rng(seed)
    err = np.zeros((rows, info.err_bytes), np.uint8)
    for r in range(rows):
        w = int(g.integers(0, info.t + 1)) if r > 1 else (0 if r == 0 else info.t)
        for p in g.choice(info.n, w, replace=False):
            err[r, p >> 3] |= np.uint8(1 << (p & 7))
    return err


@pytest.mark.parametrize("s", SETS)
def test_positions_text_matches_errorstream(oracle_mod, s):
    err = _sparse_errors(s, 9, s)
    pos = cmd.positions_from_errors(s, err)
    info = cmd.set_info(s)
    assert pos.shape == (9, info.t + 1)
    assert pos[0, 0] == 0 and (pos[0, 1:] == 0xFFFF).all()
    assert pos[1, 0] == info.t and (np.diff(pos[1, 1:].astype(np.int64)) > 0).all()
    assert cmd.positions_text(s, pos) == oracle_mod.Oracle(s).errorstream(err)


def test_binary_errorstream_file_roundtrip(tmp_path, oracle_mod):
    s = 6960119
    err = _sparse_errors(s, 12, 5)
    pos = cmd.positions_from_errors(s, err)
    b = str(tmp_path / "es.pos")
    cmd.write_positions(s, pos[:7], b)
    cmd.write_positions(s, pos[7:], b, append=True)
    raw = open(b, "rb").read()
    assert raw[:8] == b"CMDPOS01"
    assert int.from_bytes(raw[8:12], "little") == s and int.from_bytes(raw[16:24], "little") == 12
    assert len(raw) == 24 + 12 * 120 * 2
    t = str(tmp_path / "es.txt")
    cmd.positions_to_errorstream(b, t)
    assert open(t, "rb").read() == oracle_mod.Oracle(s).errorstream(err)
    # a file of another set, or not a positions file at all, is refused
    with pytest.raises(cmd.CmdError) as ei:
        cmd.write_positions(348864, cmd.positions_from_errors(348864, _sparse_errors(348864, 1, 1)), b, append=True)
    assert ei.value.code == cmd.CMD_E_FILE
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"\0" * 64)
    with pytest.raises(cmd.CmdError) as ei:
        cmd.positions_to_errorstream(str(junk), t)
    assert ei.value.code == cmd.CMD_E_FILE


@pytest.mark.parametrize("s", [348864, 6960119])
def test_pubkey_columns_reencode(s):
    """C = [I | T] e for valid synthetic ciphertexts, with T read back through
    cmd_pubkey_columns (the block the decapsulation kernel checks against)."""
    info = cmd.set_info(s)
    mt = info.m * info.t
    pk = cmd.PubKey(s, golden_sk(s))
    T = pk.columns()
    assert T.shape[0] == info.n - mt
    cts, err, valid = pk.ciphertexts(seed=8, count=6, malformed_permille=0)
    Tb = np.unpackbits(T.view(np.uint8), axis=1, bitorder="little")[:, :mt]   # [n-mt, mt]
    for c in range(6):
        e = np.unpackbits(err[c], bitorder="little")
        ct = np.unpackbits(cts[c], bitorder="little")[:mt]
        enc = (e[:mt] + Tb[e[mt:].astype(bool)].sum(axis=0)) & 1
        assert np.array_equal(enc, ct)


@pytest.mark.parametrize("s", [348864, 6960119])
def test_oracle_decap_matches_encapsulation(oracle_mod, s):
    """The oracle's decapsulation returns the reference encapsulation's key
    K = SHAKE256(1 || e || C) (kem/common/core/operations.c:15-34) for valid
    ciphertexts and rejects malformed ones and the reference's own kem/
    ciphertexts (their error vectors have weight below t)."""
    import hashlib
    o = oracle_mod.Oracle(s)
    sk = golden_sk(s)
    cts, planted, valid = cmd.PubKey(s, sk).ciphertexts(seed=12, count=24, malformed_permille=300)
    keys, acc = o.decap(sk, cts)
    assert np.array_equal(acc, valid)
    for c in range(cts.shape[0]):
        if valid[c]:
            assert keys[c].tobytes() == hashlib.shake_256(b"\x01" + planted[c].tobytes() + cts[c].tobytes()).digest(32)
    from conftest import golden_ct
    _, acc2 = o.decap(sk, np.frombuffer(golden_ct(s), np.uint8).reshape(-1, o.ct_bytes))
    assert not acc2.any()
