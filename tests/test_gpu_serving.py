"""GPU tests of the batching layers on top of the kernels: the autotuner, CUDA
graph replay, and the continuous-batching serving loop.

The serving tests check that each request's result is bit-identical whether it
is decrypted alone or inside a large mixed batch of many keys and all five
parameter sets (both the plain multi-key kernels and the fused kernel), equal
to the oracle, and that keys are evicted and re-expanded under a small HBM
budget without changing results.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import cm_decrypt__b200 as cmd
from conftest import SETS, golden_sk, rng

pytestmark = pytest.mark.gpu


def test_tune_per_sample_size(engine):
    """A tuning for a given batch size is cached apart from the default one,
    so tuning at the batch a caller runs does not replace the default choice
    (the winners differ: at 65,536 ciphertexts how the batch fills whole
    rounds decides)."""
    s = 6960119
    key = cmd.Key(engine, s, golden_sk(s))
    try:
        sized = cmd.tune(engine, key, sample_count=65536, force=True)
        default = cmd.tune(engine, key, force=True)
        again = cmd.tune(engine, key, sample_count=65536)  # from the cache, keyed by the size
        assert (again["wpb"], again["balanced"]) == (sized["wpb"], sized["balanced"])
        assert again["ns_per_ct"] == pytest.approx(sized["ns_per_ct"], rel=1e-3)
        back = cmd.tune(engine, key)
        assert (back["wpb"], back["balanced"]) == (default["wpb"], default["balanced"])
        assert back["ns_per_ct"] == pytest.approx(default["ns_per_ct"], rel=1e-3)
    finally:
        key.free()


def test_tune_and_graph_replay(engine):
    s = 6960119
    key = cmd.Key(engine, s, golden_sk(s))
    try:
        cfg = cmd.tune(engine, key, force=True)
        assert cfg["wpb"] in (4, 8) and cfg["ns_per_ct"] > 0
        cached = cmd.tune(engine, key)  # served from the cache
        assert (cached["wpb"], cached["balanced"], cached["tile_below"]) == \
            (cfg["wpb"], cfg["balanced"], cfg["tile_below"])
        assert cached["ns_per_ct"] == pytest.approx(cfg["ns_per_ct"], rel=1e-3)
        # the tuned crossover: small batches take the tile kernels under
        # CMD_PATH_AUTO (the tile path wins on a batch of a few tiles)
        assert cfg["tile_below"] >= 512
        pk = cmd.PubKey(s, golden_sk(s))
        small, small_e, _ = pk.ciphertexts(seed=8, count=100, malformed_permille=100)
        launches = engine.launch_count()
        err, _ = cmd.decrypt(engine, key, small, path="auto")
        assert engine.launch_count() - launches == 4  # tile items + the three tile kernels
        assert np.array_equal(err, cmd.decrypt(engine, key, small, path="fused")[0])
        cts, planted, _ = pk.ciphertexts(seed=4, count=5000)
        d_ct = torch.from_numpy(cts).cuda()
        for path in ("fused", "plain"):
            d_err = torch.zeros((5000, key.info.err_words), dtype=torch.int32, device="cuda")
            d_w = torch.zeros(5000, dtype=torch.int16, device="cuda")
            g = cmd.Graph(engine, key, d_ct.data_ptr(), 5000, d_err.data_ptr(), d_w.data_ptr(), path=path)
            try:
                for _ in range(2):
                    d_err.zero_()
                    before = engine.launch_count()
                    g.launch()
                    torch.cuda.synchronize()
                    assert engine.launch_count() > before
                    got = d_err.cpu().numpy().astype("<u4").view(np.uint8).reshape(5000, -1)[:, :870]
                    assert np.array_equal(got, planted), path
            finally:
                g.close()
    finally:
        key.free()


def _keyring():
    """Two keys per set: the reference kem key and one derived key."""
    ring = []
    for s in SETS:
        ring.append((s, golden_sk(s)))
        ring.append((s, cmd.synth_key(s, golden_sk(s), 7)))
    return ring


@pytest.fixture(scope="module")
def workload(oracle_mod):
    ring = _keyring()
    g = rng(5)
    n = 1200
    key_of = g.integers(0, len(ring), n)
    cts = np.zeros((n, 208), np.uint8)
    expect = {}
    pks = [cmd.PubKey(s, sk) for s, sk in ring]
    for i in range(n):
        s, sk = ring[key_of[i]]
        c, _, _ = pks[key_of[i]].ciphertexts(seed=1000 + i, count=1, malformed_permille=50)
        cts[i, : c.shape[1]] = c[0]
    # oracle results grouped per key
    for k, (s, sk) in enumerate(ring):
        idx = np.nonzero(key_of == k)[0]
        if idx.size:
            info = cmd.set_info(s)
            ref = oracle_mod.Oracle(s).decrypt(sk, cts[idx, : info.ct_bytes], nthreads=8)
            for j, i in enumerate(idx):
                expect[int(i)] = ref[j]
    return ring, key_of, cts, expect


@pytest.mark.parametrize("fused_threshold", [0, 1, 300])
def test_server_alone_equals_in_mix(engine, workload, fused_threshold):
    ring, key_of, cts, expect = workload
    n = cts.shape[0]
    with cmd.Server(engine, max_batch=512, slots=3, max_wait_us=300, fused_threshold=fused_threshold) as srv:
        ids = [srv.add_key(s, sk) for s, sk in ring]
        # alone: one request at a time, waiting for each
        alone = {}
        for i in (0, 1, 2, 3, 17, 99):
            out = np.zeros(1024, np.uint8)
            assert srv.submit(ids[key_of[i]], cts[i], out, i) == cmd.CMD_OK
            srv.drain()
            alone[i] = out.copy()
        srv.poll()
        # in the mix: everything at once (batches of mixed keys and sets)
        outs = np.zeros((n, 1024), np.uint8)
        for i in range(n):
            assert srv.submit(ids[key_of[i]], cts[i], outs[i], 100000 + i) == cmd.CMD_OK
        srv.drain()
        comps = srv.poll(max_n=n + 10)
        assert len(comps) == n and all(c[1] == cmd.CMD_OK for c in comps)
        st = srv.stats()
        assert st["batches"] >= 3
        if fused_threshold == 1:
            assert st["fused_batches"] == st["batches"]
        if fused_threshold == 0:
            assert st["fused_batches"] == 0
    for i in range(n):
        s, _ = ring[key_of[i]]
        nb = cmd.set_info(s).err_bytes
        assert np.array_equal(outs[i, :nb], expect[i]), i
    for i, a in alone.items():
        s, _ = ring[key_of[i]]
        nb = cmd.set_info(s).err_bytes
        assert np.array_equal(a[:nb], outs[i, :nb]), ("alone vs mix", i)
        assert np.array_equal(a[:nb], expect[i])


def test_server_submit_many(engine, workload):
    """Requests queued in groups under one lock give the oracle's results,
    with their tags, and a group larger than the queue is cut where it fills."""
    ring, key_of, cts, expect = workload
    n = cts.shape[0]
    with cmd.Server(engine, max_batch=256, slots=3, max_wait_us=100, fused_threshold=0) as srv:
        ids = np.array([srv.add_key(s, sk) for s, sk in ring], np.uint32)
        outs = np.zeros((n, 1024), np.uint8)
        for a in range(0, n, 300):
            b = min(n, a + 300)
            assert srv.submit_many(ids[key_of[a:b]], cts[a:b], outs[a:b], np.arange(a, b) + 7) == b - a
        srv.drain()
        comps = srv.poll(max_n=n + 10)
        assert sorted(c[0] for c in comps) == list(range(7, n + 7))
    for i in range(n):
        s, _ = ring[key_of[i]]
        nb = cmd.set_info(s).err_bytes
        assert np.array_equal(outs[i, :nb], expect[i]), i
    with cmd.Server(engine, max_batch=64, slots=1, max_wait_us=100000, queue_capacity=50,
                    fused_threshold=0) as srv:
        ids = np.array([srv.add_key(s, sk) for s, sk in ring], np.uint32)
        # a first request keeps the one slot busy so that the group waits in the queue
        assert srv.submit_many(ids[key_of[:1]], cts[:1], None) == 1
        got = srv.submit_many(ids[key_of[:200]], cts[:200], None)
        assert 0 < got <= 50
        srv.drain()
        assert srv.stats()["refused"] >= 200 - got


def test_server_lru_eviction_under_budget(workload):
    ring, key_of, cts, expect = workload
    with cmd.Engine(0) as probe:
        k = cmd.Key(probe, 8192128, golden_sk(8192128))
        per_key = k.device_bytes()
        k.free()
    # room for the server's buffers plus about three keys
    with cmd.Engine(0) as eng0:
        srv0 = cmd.Server(eng0, max_batch=64, slots=2, fused_threshold=0)
        server_bytes = eng0.memory()[0]
        srv0.close()
    eng = cmd.Engine(0, hbm_budget=server_bytes + 3 * per_key + (1 << 16))
    try:
        with cmd.Server(eng, max_batch=64, slots=2, max_wait_us=100, fused_threshold=0) as srv:
            ids = [srv.add_key(s, sk) for s, sk in ring]
            n = 300
            outs = np.zeros((n, 1024), np.uint8)
            for i in range(n):
                srv.submit(ids[key_of[i]], cts[i], outs[i], i)
                if i % 50 == 49:
                    srv.drain()
            srv.drain()
            st = srv.stats()
            # the budget holds only a few keys: some had to be evicted and re-expanded
            assert st["resident_keys"] < len(ring)
            assert eng.memory()[0] <= eng.memory()[1]
            for i in range(n):
                s, _ = ring[key_of[i]]
                nb = cmd.set_info(s).err_bytes
                assert np.array_equal(outs[i, :nb], expect[i]), i
    finally:
        eng.close()


def test_server_poisson_loadgen(engine, workload):
    ring, key_of, cts, expect = workload
    with cmd.Server(engine, max_batch=1024, slots=4, max_wait_us=200, fused_threshold=512,
                    record_completions=False) as srv:
        ids = np.array([srv.add_key(s, sk) for s, sk in ring], np.uint32)
        pool = 1000
        err_pool = np.zeros((pool, 1024), np.uint8)
        st = srv.loadgen(ids[key_of[:pool]], cts[:pool], err_pool, rate=40000, seconds=0.5)
        assert st["completed"] == st["submitted"] > 5000
        assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
        for i in range(pool):
            s, _ = ring[key_of[i]]
            nb = cmd.set_info(s).err_bytes
            assert np.array_equal(err_pool[i, :nb], expect[i]), i


@pytest.mark.parametrize("fused_threshold", [0, 1, 300])
def test_server_registered_rows(engine, workload, fused_threshold):
    """Results into registered memory: the tile path's root kernel stores each
    row there itself (at 4-byte and 2-byte aligned starts), fused batches and
    odd addresses take the staged copy, and no byte around a row changes."""
    ring, key_of, cts, expect = workload
    n = cts.shape[0]
    stride = 1030  # 2 mod 4: row starts alternate between 4-byte and 2-byte alignment
    flat = np.full(n * stride + 64, 0xA5, np.uint8)
    plain = np.full((n, 1024), 0x5A, np.uint8)  # not registered
    with cmd.Server(engine, max_batch=512, slots=3, max_wait_us=300, fused_threshold=fused_threshold) as srv:
        ids = [srv.add_key(s, sk) for s, sk in ring]
        srv.register_rows(flat)
        offs = []
        for i in range(n):
            nb = cmd.set_info(ring[key_of[i]][0]).err_bytes
            off = 2 + i * stride + (1 if i % 97 == 5 else 0)  # a few odd starts
            offs.append(off)
            out = plain[i, :nb] if i % 11 == 3 else flat[off:off + nb]
            assert srv.submit(ids[key_of[i]], cts[i], out, i) == cmd.CMD_OK
        srv.drain()
        comps = srv.poll(max_n=n + 10)
        assert len(comps) == n and all(c[1] == cmd.CMD_OK for c in comps)
    touched = np.zeros(flat.size, bool)
    for i in range(n):
        nb = cmd.set_info(ring[key_of[i]][0]).err_bytes
        if i % 11 == 3:
            assert np.array_equal(plain[i, :nb], expect[i]), i
            assert (plain[i, nb:] == 0x5A).all(), i
        else:
            assert np.array_equal(flat[offs[i]:offs[i] + nb], expect[i]), i
            touched[offs[i]:offs[i] + nb] = True
    assert (flat[~touched] == 0xA5).all()
