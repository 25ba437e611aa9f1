"""GPU parity: the CUDA engine against the oracle, bit-exact, through the C ABI.

Covers key expansion (support, Goppa polynomial, syndrome table), each stage
in isolation (synd / bm / root images / root + pack), and whole decrypts on
both kernel paths for every parameter set: the reference's own kem/ fixtures
(errorstream byte-identical), synthetic valid weight-t ciphertexts (decode to
the planted error vector), malformed random strings (the reference's failure
outcome), ragged batch sizes, derived keys and mixed multi-key batches.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest
import torch

import cm_decrypt__b200 as cmd
from conftest import KEM, SETS, golden_ct, golden_errorstream, golden_sk, rng

pytestmark = pytest.mark.gpu


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def words_to_bytes(err_words: torch.Tensor, n: int) -> np.ndarray:
    w = err_words.cpu().numpy().astype("<u4")
    return w.view(np.uint8).reshape(w.shape[0], -1)[:, : n // 8]


@pytest.fixture(scope="module")
def keys(engine):
    out = {s: cmd.Key(engine, s, golden_sk(s)) for s in SETS}
    yield out
    for k in out.values():
        k.free()


@pytest.mark.parametrize("s", SETS)
def test_key_expansion(oracle_mod, keys, s):
    g, L, tab = oracle_mod.Oracle(s).expand(golden_sk(s))
    k = keys[s]
    assert np.array_equal(k.goppa(), g)
    assert np.array_equal(k.support(), L)
    assert np.array_equal(k.synd_table(), tab)


@pytest.mark.parametrize("s", SETS)
def test_stages(oracle_mod, engine, keys, s):
    o = oracle_mod.Oracle(s)
    o.expand(golden_sk(s))
    k = keys[s]
    info = k.info
    pk = cmd.PubKey(s, golden_sk(s))
    valid, _, _ = pk.ciphertexts(seed=21, count=40)
    junk = rng(s).integers(0, 256, (37, info.ct_bytes), dtype=np.uint8)
    cts = np.concatenate([valid, junk])
    n = cts.shape[0]
    d_ct = dev(cts)
    d_s = torch.zeros((n, 2 * info.t), dtype=torch.int16, device="cuda")
    d_sf = torch.zeros((n, 2 * info.t), dtype=torch.int16, device="cuda")
    d_l = torch.zeros((n, info.t + 1), dtype=torch.int16, device="cuda")
    d_img = torch.zeros((n, info.n), dtype=torch.int16, device="cuda")
    d_e = torch.zeros((n, info.err_words), dtype=torch.int32, device="cuda")
    d_w = torch.zeros(n, dtype=torch.int16, device="cuda")
    cmd.synd(engine, k, d_ct.data_ptr(), n, d_s.data_ptr())
    cmd.synd_fft(engine, k, d_ct.data_ptr(), n, d_sf.data_ptr())
    cmd.bm(engine, s, d_s.data_ptr(), n, d_l.data_ptr())
    cmd.root_images(engine, k, d_l.data_ptr(), n, d_img.data_ptr())
    cmd.root(engine, k, d_l.data_ptr(), n, d_e.data_ptr(), d_w.data_ptr())
    torch.cuda.synchronize()
    S = d_s.cpu().numpy().view(np.uint16)
    SF = d_sf.cpu().numpy().view(np.uint16)
    Lc = d_l.cpu().numpy().view(np.uint16)
    IMG = d_img.cpu().numpy().view(np.uint16)
    E = words_to_bytes(d_e, info.n)
    W = d_w.cpu().numpy().view(np.uint16)
    for i in range(n):
        ct = cts[i].tobytes()
        s_ref = o.synd(ct)
        assert np.array_equal(S[i], s_ref), ("synd", i)
        assert np.array_equal(SF[i], s_ref), ("synd by the transposed FFT", i)
        l_ref = o.bm(s_ref)
        assert np.array_equal(Lc[i], l_ref), ("bm", i)
        img = o.root(l_ref)
        assert np.array_equal(IMG[i], img), ("root", i)
        ebits = np.zeros(info.err_bytes, np.uint8)
        idx = np.nonzero(img == 0)[0]
        np.bitwise_or.at(ebits, idx >> 3, (1 << (idx & 7)).astype(np.uint8))
        assert np.array_equal(E[i], ebits), ("pack", i)
        assert W[i] == idx.size
    # padding bits of the last word stay zero
    if info.n % 32:
        tail = d_e[:, -1].cpu().numpy().astype(np.uint32) >> (info.n % 32)
        assert not tail.any()


@pytest.mark.parametrize("path", ["plain", "fused", "tile"])
@pytest.mark.parametrize("s", SETS)
def test_kem_fixture_errorstream(engine, keys, s, path):
    info = keys[s].info
    cts = np.frombuffer(golden_ct(s), np.uint8).reshape(-1, info.ct_bytes)
    err, w = cmd.decrypt(engine, keys[s], cts, path=path)
    assert cmd.errorstream(s, err) == golden_errorstream(s)


@pytest.mark.parametrize("wpb,balanced", [(8, True), (8, False), (4, True), (4, False)])
def test_fused_round_shares(engine, keys, wpb, balanced):
    """Fused rounds of every fill: whole tiles, rounds spread evenly over the
    CTA's warps (more than 16 ciphertexts a warp) and short tails, for both
    CTA sizes and round schedules.  The fused rows must equal the plain path's
    (itself checked against the oracle) bit for bit, malformed ones included,
    and the valid ones their planted errors."""
    s = 6960119
    pk = cmd.PubKey(s, golden_sk(s))
    before = cmd.fused_config(engine, s)
    try:
        cmd.set_fused_config(engine, s, wpb, balanced)
        for count in (148 * 160, 148 * 224 + 100, 5 * 32 * wpb + 77, 200, 131, 33):
            cts, planted, valid = pk.ciphertexts(seed=500 + count, count=count, malformed_permille=100)
            err_f, w_f = cmd.decrypt(engine, keys[s], cts, path="fused")
            err_p, w_p = cmd.decrypt(engine, keys[s], cts, path="plain")
            assert np.array_equal(err_f, err_p), (wpb, balanced, count)
            assert np.array_equal(w_f, w_p), (wpb, balanced, count)
            assert np.array_equal(err_f[valid == 1], planted[valid == 1]), (wpb, balanced, count)
    finally:
        cmd.set_fused_config(engine, s, before["wpb"], before["balanced"])


@pytest.mark.parametrize("path", ["plain", "fused", "tile"])
@pytest.mark.parametrize("s", SETS)
def test_decrypt_vs_oracle(oracle_mod, engine, keys, s, path):
    o = oracle_mod.Oracle(s)
    info = keys[s].info
    pk = cmd.PubKey(s, golden_sk(s))
    for count, permille in ((1, 0), (33, 0), (300, 100), (97, 1000)):
        cts, planted, valid = pk.ciphertexts(seed=1000 + count, count=count, malformed_permille=permille)
        err, w = cmd.decrypt(engine, keys[s], cts, path=path)
        ref = o.decrypt(golden_sk(s), cts, nthreads=8)
        assert np.array_equal(err, ref), (count, permille)
        assert np.array_equal(err[valid == 1], planted[valid == 1])
        assert np.array_equal(w, np.unpackbits(ref, axis=1).sum(axis=1))
        assert (w[valid == 1] == info.t).all()


@pytest.mark.parametrize("s", [348864, 6960119])
def test_derived_keys(oracle_mod, engine, s):
    o = oracle_mod.Oracle(s)
    for seed in (1, 2):
        sk = cmd.synth_key(s, golden_sk(s), seed)
        key = cmd.Key(engine, s, sk)
        try:
            g, L, tab = o.expand(sk)
            assert np.array_equal(key.support(), L)
            pk = cmd.PubKey(s, sk)
            cts, planted, valid = pk.ciphertexts(seed=seed, count=70, malformed_permille=200)
            for path in ("plain", "fused", "tile"):
                err, _ = cmd.decrypt(engine, key, cts, path=path)
                assert np.array_equal(err, o.decrypt(sk, cts, nthreads=8))
        finally:
            key.free()


def test_mixed_batch(oracle_mod, engine):
    """Ciphertexts of several keys and all five sets interleaved in one launch,
    each in its own slot of a shared byte buffer and error buffer."""
    g = rng(42)
    ks, sks, pks = [], [], []
    for s in SETS:
        for seed in (0, 1):
            sk = golden_sk(s) if seed == 0 else cmd.synth_key(s, golden_sk(s), seed)
            ks.append(cmd.Key(engine, s, sk))
            sks.append((s, sk))
            pks.append(cmd.PubKey(s, sk))
    try:
        count = 700
        key_idx = g.integers(0, len(ks), count).astype(np.uint32)
        blobs = []
        ct_off = np.zeros(count, np.uint64)
        err_off = np.zeros(count, np.uint64)
        off = woff = 0
        for c in range(count):
            s, _ = sks[key_idx[c]]
            info = cmd.set_info(s)
            ct, _, _ = pks[key_idx[c]].ciphertexts(seed=c, count=1, malformed_permille=100)
            blobs.append(ct[0])
            ct_off[c] = off
            off += info.ct_bytes + int(g.integers(0, 5))   # ragged, unaligned placement
            err_off[c] = woff
            woff += info.err_words
        buf = np.zeros(off + 16, np.uint8)
        for c in range(count):
            buf[int(ct_off[c]): int(ct_off[c]) + blobs[c].size] = blobs[c]
        d_ct = dev(buf)
        d_err = torch.zeros(woff, dtype=torch.int32, device="cuda")
        d_w = torch.zeros(count, dtype=torch.int16, device="cuda")
        cmd.decrypt_mixed_device(engine, ks, key_idx, d_ct.data_ptr(), ct_off, d_err.data_ptr(), err_off,
                                 d_w.data_ptr())
        torch.cuda.synchronize()
        E = d_err.cpu().numpy().astype("<u4")
        W = d_w.cpu().numpy().view(np.uint16)
        for c in range(count):
            s, sk = sks[key_idx[c]]
            info = cmd.set_info(s)
            o = oracle_mod.Oracle(s)
            ct = buf[int(ct_off[c]): int(ct_off[c]) + info.ct_bytes]
            ref = o.decrypt(sk, ct.reshape(1, -1))[0]
            row = E[int(err_off[c]): int(err_off[c]) + info.err_words].view(np.uint8)[: info.err_bytes]
            assert np.array_equal(row, ref), c
            assert W[c] == int(np.unpackbits(ref).sum())
    finally:
        for k in ks:
            k.free()


def test_mixed_64_keys_every_row_vs_reference(oracle_mod, engine):
    """The mixed-batch workload at 2^14 ciphertexts: 64 seeded keys spread
    13/13/13/13/12 over the five sets, the set drawn uniformly per ciphertext,
    10% uniformly random mt-bit strings, one cmd_decrypt_mixed_device launch.
    Every row, malformed ones included, equals the reference's own CPU
    decoder's output (oracle/_ref; CPU/param/param<set>/src/decrypt.c), and
    every weight its popcount."""
    g = rng(0x5EED4)
    per_set = [13, 13, 13, 13, 12]
    ring = [(s, cmd.synth_key(s, golden_sk(s), 0xC0FFEE + 97 * i + j)) for i, s in enumerate(SETS)
            for j in range(per_set[i])]
    ks = [cmd.Key(engine, s, sk) for s, sk in ring]
    try:
        count = 1 << 14
        set_of = g.integers(0, 5, count)
        first = np.cumsum([0] + per_set[:-1])
        key_idx = (first[set_of] + (g.random(count) * np.array(per_set)[set_of]).astype(np.int64)).astype(np.uint32)
        buf = np.zeros((count, 208), np.uint8)
        valid = np.zeros(count, np.uint8)
        for k in range(len(ks)):
            idx = np.nonzero(key_idx == k)[0]
            if idx.size:
                c, _, v = cmd.PubKey(*ring[k]).ciphertexts(seed=1000 + k, count=idx.size, malformed_permille=100)
                buf[idx, : c.shape[1]] = c
                valid[idx] = v
        assert 0.05 < 1 - valid.mean() < 0.15
        d_ct = dev(buf.reshape(-1))
        d_err = torch.zeros(count * 256, dtype=torch.int32, device="cuda")
        d_w = torch.zeros(count, dtype=torch.int16, device="cuda")
        cmd.decrypt_mixed_device(engine, ks, key_idx, d_ct.data_ptr(), np.arange(count, dtype=np.uint64) * 208,
                                 d_err.data_ptr(), np.arange(count, dtype=np.uint64) * 256, d_w.data_ptr())
        torch.cuda.synchronize()
        E = d_err.cpu().numpy().astype("<u4").view(np.uint8).reshape(count, 1024)
        W = d_w.cpu().numpy().view(np.uint16)
    finally:
        for k in ks:
            k.free()
    ref, _ = oracle_mod.reference_decrypt_rows(ring, key_idx, buf)
    bad = np.nonzero(~(E == ref).all(axis=1))[0]
    assert bad.size == 0, (bad[:10], int((valid[bad] == 0).sum()))
    assert np.array_equal(W, np.unpackbits(ref, axis=1).sum(axis=1))


@pytest.mark.parametrize("path", ["plain", "fused", "tile"])
def test_full_size_properties(engine, keys, path):
    """Full-size batch at 6960119 (65,536 ciphertexts): every valid
    ciphertext decodes to exactly its planted weight-119 error vector."""
    s = 6960119
    pk = cmd.PubKey(s, golden_sk(s))
    cts, planted, valid = pk.ciphertexts(seed=77, count=65536, malformed_permille=0)
    err, w = cmd.decrypt(engine, keys[s], cts, path=path)
    assert np.array_equal(err, planted)
    assert (w == 119).all()


@pytest.mark.parametrize("s", [460896, 6960119])
def test_host_batch_in_pieces(oracle_mod, engine, keys, s):
    """A ragged host-buffer batch large enough to be split over the engine's
    piece streams (eight concurrent fused launches with their own counters,
    rounds sized as one launch over the batch would size them) equals the
    one-launch device path row for row, for error vectors and for position
    rows."""
    pk = cmd.PubKey(s, golden_sk(s))
    count = 4 * 8192 * 3 + 17
    cts, planted, valid = pk.ciphertexts(seed=5, count=count, malformed_permille=100)
    err, w = cmd.decrypt(engine, keys[s], cts, path="fused")
    assert np.array_equal(err[valid == 1], planted[valid == 1])
    info = keys[s].info
    d_ct = dev(cts)
    d_err = torch.zeros((count, info.err_words), dtype=torch.int32, device="cuda")
    d_w = torch.zeros(count, dtype=torch.int16, device="cuda")
    cmd.decrypt_device(engine, keys[s], d_ct.data_ptr(), count, d_err.data_ptr(), d_w.data_ptr(), 0, "fused")
    torch.cuda.synchronize()
    assert np.array_equal(words_to_bytes(d_err, info.n), err)
    assert np.array_equal(d_w.cpu().numpy().view(np.uint16), w)
    bad = np.nonzero(valid == 0)[0][:64]
    assert np.array_equal(err[bad], oracle_mod.Oracle(s).decrypt(golden_sk(s), cts[bad], nthreads=8))
    assert np.array_equal(cmd.decrypt_positions(engine, keys[s], cts), cmd.positions_from_errors(s, err))


@pytest.mark.parametrize("s", [348864, 6960119, 8192128])
def test_host_batch_into_pinned_rows(engine, keys, s):
    """With pinned error rows, which the GPU can write, the pieces' kernels
    store the packed rows straight into the caller's buffer.  The rows equal
    the staged copy's, both from a 4-byte aligned start and from one 2 bytes
    into a word (6960119's 870-byte rows alternate between the two), and no
    byte outside the rows changes."""
    pk = cmd.PubKey(s, golden_sk(s))
    count = 4 * 8192 * 3 + 17
    cts, planted, valid = pk.ciphertexts(seed=11, count=count, malformed_permille=100)
    ref, w = cmd.decrypt(engine, keys[s], cts, path="fused")  # pageable rows: staged copies
    assert np.array_equal(ref[valid == 1], planted[valid == 1])
    rb = keys[s].info.err_bytes
    base = torch.full((count * rb + 64,), 0xEE, dtype=torch.uint8).pin_memory().numpy()
    for off in (16, 18):
        base[:] = 0xEE
        wts = np.zeros(count, np.uint16)
        cmd._check(cmd.lib().cmd_decrypt_batch(engine.handle, keys[s].handle, cmd.PATHS["fused"], cts.ctypes.data,
                                               count, base.ctypes.data + off, wts.ctypes.data), "cmd_decrypt_batch")
        assert np.array_equal(base[off:off + count * rb].reshape(count, rb), ref)
        assert (base[:off] == 0xEE).all() and (base[off + count * rb:] == 0xEE).all()
        assert np.array_equal(wts, w)


@pytest.mark.parametrize("s", SETS)
def test_positions_output(oracle_mod, engine, keys, s):
    """cmd_decrypt_positions rows equal the positions of the packed error
    vectors (oracle) for the kem fixtures, valid and malformed ciphertexts,
    and their text is the reference errorstream."""
    info = keys[s].info
    kem = np.frombuffer(golden_ct(s), np.uint8).reshape(-1, info.ct_bytes)
    pos = cmd.decrypt_positions(engine, keys[s], kem)
    assert cmd.positions_text(s, pos) == golden_errorstream(s)
    pk = cmd.PubKey(s, golden_sk(s))
    cts, planted, valid = pk.ciphertexts(seed=31, count=333, malformed_permille=300)
    ref = oracle_mod.Oracle(s).decrypt(golden_sk(s), cts, nthreads=8)
    pos = cmd.decrypt_positions(engine, keys[s], cts)
    assert np.array_equal(pos, cmd.positions_from_errors(s, ref))
    assert (pos[valid == 1, 0] == info.t).all()
    # device entry point, same rows
    d_ct = dev(cts)
    d_pos = torch.zeros((cts.shape[0], info.t + 1), dtype=torch.int16, device="cuda")
    cmd.decrypt_positions_device(engine, keys[s], d_ct.data_ptr(), cts.shape[0], d_pos.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(d_pos.cpu().numpy().view(np.uint16), pos)


@pytest.mark.parametrize("s", SETS)
def test_kem_decap(oracle_mod, engine, keys, s):
    """Decapsulation keys and accept flags equal the oracle's for valid and
    malformed ciphertexts, the reference's kem/ ciphertexts and (6960119)
    valid ciphertexts with a padding bit set; accepted keys are the reference
    encapsulation's SHAKE256(1 || e || C)."""
    import hashlib
    info = keys[s].info
    sk = golden_sk(s)
    cts, planted, valid = cmd.PubKey(s, sk).ciphertexts(seed=77, count=300, malformed_permille=200)
    kem = np.frombuffer(golden_ct(s), np.uint8).reshape(-1, info.ct_bytes)
    allc = np.concatenate([cts, kem])
    if 8 * info.ct_bytes > info.m * info.t:
        padded = cts[valid == 1][:5].copy()
        padded[:, -1] |= 0x80
        allc = np.concatenate([allc, padded])
    k, a = cmd.kem_decap(engine, keys[s], allc)
    rk, ra = oracle_mod.Oracle(s).decap(sk, allc, nthreads=8)
    assert np.array_equal(a, ra)
    assert np.array_equal(k, rk)
    assert a[: cts.shape[0]].sum() == valid.sum()
    # kem/ draws error positions from m-bit values without rejecting those >= n
    # (kem/common/core/encrypt.c:147-190): below weight t, so rejected, except
    # for 8192128 where n = 2^m and the weight is always t
    k0 = cts.shape[0]
    assert (a[k0: k0 + kem.shape[0]] == (1 if info.n == 1 << info.m else 0)).all()
    assert not a[k0 + kem.shape[0]:].any()   # padding bit set
    for c in np.nonzero(valid)[0][:40]:
        assert k[c].tobytes() == hashlib.shake_256(b"\x01" + planted[c].tobytes() + cts[c].tobytes()).digest(32)
    d_ct = dev(allc)
    d_k = torch.zeros((allc.shape[0], 32), dtype=torch.uint8, device="cuda")
    cmd.kem_decap_device(engine, keys[s], d_ct.data_ptr(), allc.shape[0], d_k.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(d_k.cpu().numpy(), k)


def test_decap_key_preparation_on_device(oracle_mod, engine):
    """The decapsulation's public-key columns are derived on the device from
    the key's support and Goppa polynomial.  Keys made by flipping one
    control bit of a golden key: one whose parity-check matrix stays
    systematic decapsulates its own valid ciphertexts (made from the host's
    public key) with the oracle's keys; one that has no systematic form (the
    host derivation refuses it) is refused with CMD_E_ARG."""
    s = 460896
    sk = golden_sk(s)
    info = cmd.set_info(s)
    off = 40 + 2 * info.t

    def flipped(i):
        b = bytearray(sk)
        b[off + 37 * i] ^= 0x01
        return bytes(b)

    def systematic(k):
        try:
            cmd.PubKey(s, k)
            return True
        except cmd.CmdError:
            return False

    good = next(flipped(i) for i in range(1, 40) if systematic(flipped(i)))
    bad = next(flipped(i) for i in range(1, 40) if not systematic(flipped(i)))
    key = cmd.Key(engine, s, good)
    cmd.prepare_decap(engine, key)
    cts, planted, valid = cmd.PubKey(s, good).ciphertexts(seed=5, count=96, malformed_permille=100)
    k, a = cmd.kem_decap(engine, key, cts)
    rk, ra = oracle_mod.Oracle(s).decap(good, cts, nthreads=8)
    assert np.array_equal(a, ra) and np.array_equal(k, rk)
    assert a.sum() == valid.sum() > 0
    with pytest.raises(cmd.CmdError) as err:
        cmd.prepare_decap(engine, cmd.Key(engine, s, bad))
    assert err.value.code == cmd.CMD_E_ARG


def test_binary_errorstream_files_and_cli(engine, tmp_path):
    s = 6960119
    b = str(tmp_path / "es.pos")
    cmd.decrypt_files_binary(engine, s, os.path.join(KEM, f"sk_{s}.bin"), os.path.join(KEM, f"ct_{s}.bin"), 5, b)
    t = str(tmp_path / "es.txt")
    r = subprocess.run([cmd.CLI_PATH, "--to-text", b, t], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert open(t, "rb").read() == golden_errorstream(s)
    b2 = str(tmp_path / "cli.pos")
    r = subprocess.run([cmd.CLI_PATH, str(s), "5", "--sk", os.path.join(KEM, f"sk_{s}.bin"), "--ct",
                        os.path.join(KEM, f"ct_{s}.bin"), "--out", b2, "--format", "binary"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert open(b2, "rb").read() == open(b, "rb").read()


def test_decrypt_files_and_cli(engine, tmp_path):
    s = 348864
    out = str(tmp_path / "es.bin")
    cmd.decrypt_files(engine, s, os.path.join(KEM, f"sk_{s}.bin"), os.path.join(KEM, f"ct_{s}.bin"), 5, out)
    assert open(out, "rb").read() == golden_errorstream(s)
    # short ct file -> KAT_FILE_OPEN_ERROR (-1); KATNUM 0 -> KAT_CRYPTO_FAILURE (-4)
    with pytest.raises(cmd.CmdError) as ei:
        cmd.decrypt_files(engine, s, os.path.join(KEM, f"sk_{s}.bin"), os.path.join(KEM, f"ct_{s}.bin"), 6, out)
    assert ei.value.code == cmd.CMD_E_FILE
    with pytest.raises(cmd.CmdError) as ei:
        cmd.decrypt_files(engine, s, os.path.join(KEM, f"sk_{s}.bin"), os.path.join(KEM, f"ct_{s}.bin"), 0, out)
    assert ei.value.code == cmd.CMD_E_ARG
    # the CLI in the reference's directory layout, default relative paths
    for st in SETS:
        work = tmp_path / f"w{st}" / "CPU" / "param" / f"param{st}"
        work.mkdir(parents=True)
        (tmp_path / f"w{st}" / "CPU" / "results" / "output").mkdir(parents=True)
        vec = tmp_path / f"w{st}" / "kem" / "test_vectors" / "Cipher_Sk"
        vec.mkdir(parents=True)
        for name in (f"sk_{st}.bin", f"ct_{st}.bin"):
            (vec / name).write_bytes(open(os.path.join(KEM, name), "rb").read())
        r = subprocess.run([cmd.CLI_PATH, str(st), "5"], cwd=work, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = (tmp_path / f"w{st}" / "CPU" / "results" / "output" / f"errorstream0_{st}.bin").read_bytes()
        assert got == golden_errorstream(st)
    r = subprocess.run([cmd.CLI_PATH, "348864", "0"], capture_output=True)
    assert r.returncode == 256 - 4


def test_bad_key_length_and_budget(engine):
    with pytest.raises(cmd.CmdError) as ei:
        cmd.Key(engine, 348864, golden_sk(348864)[:-1])
    assert ei.value.code == cmd.CMD_E_ARG
    small = cmd.Engine(0, hbm_budget=2 << 20)   # a 6960119 key needs ~1.5 MB
    try:
        base = small.memory()[0]   # the engine's own root-search tables
        assert base < (1 << 17)
        k1 = cmd.Key(small, 6960119, golden_sk(6960119))
        assert 0 < k1.device_bytes() <= small.memory()[0] - base <= (2 << 20)
        with pytest.raises(cmd.CmdError) as ei:
            cmd.Key(small, 6960119, golden_sk(6960119))   # second copy exceeds the budget
        assert ei.value.code == cmd.CMD_E_BUDGET
        k1.free()
        assert small.memory()[0] == base
        k2 = cmd.Key(small, 6960119, golden_sk(6960119))   # fits again once freed
        k2.free()
    finally:
        small.close()
