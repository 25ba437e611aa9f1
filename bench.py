#!/usr/bin/env python
"""Benchmark: batched Classic McEliece decryption on B200.

Workload (one step): one batch of 65,536 mceliece6960119 ciphertexts (194 B,
1547-bit syndromes), each an encryption of a uniformly random weight-119 error
vector under one seeded key (the reference kem/ key regenerated from its fixed
DRBG seed), decrypted by the fused syndrome -> Berlekamp-Massey -> root search
kernel.  Every step's output is checked bit-exact against the planted error
vectors before timing is reported.

  value   decaps/s with ciphertexts resident in HBM (all ranks; weak scaling)
  e2e     the same through the public host-buffer call cmd_decrypt_batch from
          pinned host memory (H2D of the ciphertexts, D2H of error vectors and
          weights inside the timed region)
  plain   the three-kernel per-stage path on the same batch (the comparison the
          metric names)
  roofline: int-ALU -- algorithmic lane-ops of the executed algorithm (W per
          decap: syndrome + Berlekamp-Massey + additive-FFT root search, see
          cm_decrypt__b200.roofline) / fused-kernel time vs the device's
          measured lop3 rate; the Horner-yardstick equivalent and HBM
          bytes/decap shown beside it
  cpu_baseline: the reference's own CPU decoder (oracle/_ref, built from its
          sources) on all host cores over a bounded sample

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

# Hardware work queues of this process, read when its CUDA context is created:
# the serving leg keeps up to 16 batches in flight on their own streams, and
# with CUDA's default of 8 queues, streams share queues and a batch's first
# copy waits behind another batch's kernels (p99 then rose from 0.94 to
# 1.1-1.5 ms at 7.3 M requests/s).  A deployment of the server sets the same.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

SET = 6960119
COUNT = 65536
L2_BYTES = 126 * 2 ** 20
KEM_SK = os.path.join(REPO, "tests", "golden", "kem", f"sk_{SET}.bin")
TRAFFIC_FILE = os.path.join(REPO, "profiles", "fused_6960119_traffic.json")


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--count", type=int, default=COUNT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only the decrypt-kernel steps of --path (profiling runs: no peak, e2e or CPU legs)")
    ap.add_argument("--path", choices=["fused", "plain", "tile"], default="fused",
                    help="decrypt path the --kernel-only steps launch")
    ap.add_argument("--wpb", type=int, default=0,
                    help="--kernel-only: fused-kernel warps per CTA (0: the tuner's cached choice or the default)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop leg")
    ap.add_argument("--serve-keys", type=int, default=1024)
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--no-keygen", action="store_true", help="skip the key-generation leg")
    ap.add_argument("--keygen-only", action="store_true",
                    help="run only the key-generation leg and print its JSON (for profiling)")
    ap.add_argument("--keygen-count", type=int, default=64, help="seeds in the key-generation batch")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU_Optimised decoder (oracle/_ref)")
    ap.add_argument("--no-reference-check", action="store_true",
                    help="skip comparing every mixed-batch and serving row with the reference CPU decoder")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the all-sets (2^20 each) and mixed-batch (2^18) measurements")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    FIELDS = ("clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict | None:
        rows = [r.split(", ") for r in self.out.strip().splitlines() if r.count(",") >= 7]
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = max(float(r[1]) for r in rows)
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for nm, v in zip(names, r[4:8]):
                if v.strip() == "Active":
                    reasons.add(nm)
        busy = [x for x in sm if x > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())}


def cpu_reference(sk: bytes, cts: np.ndarray, seconds_target: float = 15.0) -> dict:
    """The reference CPU decoder (oracle/_ref, else the oracle restatement) on
    all host cores over a bounded sample of the workload."""
    from oracle import oracle as o
    cores = os.cpu_count() or 1
    if o.RefLib.available(SET):
        dec, kind = o.RefLib(SET), "reference"
    else:
        dec, kind = o.Oracle(SET), "port"
    probe = cts[: max(cores, 8)]
    t0 = time.perf_counter()
    dec.decrypt(sk, probe, nthreads=cores)
    rate = probe.shape[0] / (time.perf_counter() - t0)
    n = int(min(cts.shape[0], max(cores, rate * seconds_target)))
    t0 = time.perf_counter()
    dec.decrypt(sk, cts[:n], nthreads=cores)
    dt = time.perf_counter() - t0
    # one thread, a sample of about 4 s
    n1 = int(max(8, min(cts.shape[0], 4.0 * rate / cores)))
    t1 = time.perf_counter()
    dec.decrypt(sk, cts[:n1], nthreads=1)
    dt1 = time.perf_counter() - t1
    return {"value": n / dt, "unit": "decaps/s", "cores": cores, "kind": kind,
            "sample": f"{n} of the {cts.shape[0]} mceliece6960119 ciphertexts, {cores} threads, {dt:.1f} s",
            "single_thread": {"value": n1 / dt1, "unit": "decaps/s", "cores": 1,
                              "sample": f"{n1} ciphertexts, 1 thread, {dt1:.1f} s"}}


SERVE_SETS = (348864, 460896, 6688128, 6960119, 8192128)
SERVE_WEIGHTS = (30, 15, 20, 20, 15)


SERVER_CONFIG = {"max_batch": 8192, "slots": 16, "max_wait_us": 60, "fused_threshold": 0}


def serving_leg(cmd, eng, nkeys: int, rates: list[float], seconds: float, pool: int = 16384,
                server_config: dict | None = None, reference_check: bool = True) -> dict:
    """Serving workload: Poisson arrivals over `nkeys` seeded keys drawn from
    the five sets weighted 30/15/20/20/15, 5% malformed ciphertexts, keys
    device-resident, continuous batching.  Returns per-rate p50/p99 latency and
    sustained decaps/s.  Every result row a rate wrote, valid and malformed,
    is compared with the reference's own CPU decoder (oracle/_ref, decoded
    once for the request pool), the valid ones also with their planted
    vectors."""
    import concurrent.futures as cf

    from oracle import oracle as o
    golden = {s: open(os.path.join(REPO, "tests", "golden", "kem", f"sk_{s}.bin"), "rb").read() for s in SERVE_SETS}
    counts = [round(nkeys * w / 100) for w in SERVE_WEIGHTS]
    counts[0] += nkeys - sum(counts)
    plan = [(s, j) for s, c in zip(SERVE_SETS, counts) for j in range(c)]
    t0 = time.perf_counter()

    def make(item):
        s, j = item
        sk = cmd.synth_key(s, golden[s], 0x5EED * 7919 + j)
        return s, sk, cmd.PubKey(s, sk)

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        keys = list(ex.map(make, plan))
    keygen_s = time.perf_counter() - t0
    g = np.random.default_rng(0x5EED)
    key_of = g.integers(0, len(keys), pool)
    cts = np.zeros((pool, 208), np.uint8)
    planted = np.zeros((pool, 1024), np.uint8)
    valid = np.zeros(pool, np.uint8)
    for k in np.unique(key_of):
        idx = np.nonzero(key_of == k)[0]
        s, sk, pk = keys[k]
        c, e, v = pk.ciphertexts(seed=int(k) * 1000003 + 17, count=idx.size, malformed_permille=50)
        cts[idx, : c.shape[1]] = c
        planted[idx, : e.shape[1]] = e
        valid[idx] = v
    out = {"keys": len(keys), "keygen_s": keygen_s, "malformed_fraction": float(1 - valid.mean()), "points": []}
    ref = None
    if reference_check:
        t0 = time.perf_counter()
        ref, kind = o.reference_decrypt_rows([(s, sk) for s, sk, _ in keys], key_of, cts)
        out["reference_check"] = {"checker": kind, "pool_rows": pool, "seconds": time.perf_counter() - t0}
    cfg = dict(SERVER_CONFIG, **(server_config or {}))
    out["server_config"] = cfg
    with cmd.Server(eng, record_completions=False, **cfg) as srv:
        ids = np.array([srv.add_key(s, sk) for s, sk, _ in keys], np.uint32)
        err_pool = np.zeros((pool, 1024), np.uint8)
        # the result rows are registered: the root kernel stores each row
        # straight into the pool, and completion copies nothing on the host
        srv.register_rows(err_pool)
        out["result_rows"] = "registered (cmd_server_register_rows): stored by the GPU into the pool"
        srv.loadgen(ids[key_of], cts, err_pool, rate=20000, seconds=0.5)  # warm: expands every key
        out["resident_keys"] = srv.stats()["resident_keys"]
        for rate in rates:
            err_pool[:] = 0
            st = srv.loadgen(ids[key_of], cts, err_pool, rate=rate, seconds=seconds)
            # loadgen request i writes row i % pool
            written = min(int(st["completed"]), pool)
            vrows = np.nonzero(valid[:written])[0]
            ok = bool(vrows.size > 0 and np.array_equal(err_pool[vrows], planted[vrows]))
            pt = {"offered_per_s": st["offered_per_s"], "decaps_per_s": st["decaps_per_s"],
                  "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3,
                  "max_ms": st["max_us"] / 1e3, "mean_batch": st["mean_batch"],
                  "batches": st["batches"], "fused_batches": st["fused_batches"],
                  "refused": st["refused"], "results_match_planted": ok,
                  "gpu_batch_p50_ms": st["gpu_p50_us"] / 1e3,
                  "gpu_batch_p99_ms": st["gpu_p99_us"] / 1e3,
                  "wait_p50_ms": st["wait_p50_us"] / 1e3, "wait_p99_ms": st["wait_p99_us"] / 1e3,
                  "dispatch_busy": st["dispatch_busy"], "complete_busy": st["complete_busy"],
                  "mean_inflight": st["mean_inflight"]}
            if ref is not None:
                same = (err_pool[:written] == ref[:written]).all(axis=1)
                pt["rows_checked_vs_reference"] = written
                pt["malformed_rows_checked"] = int((valid[:written] == 0).sum())
                pt["bit_exact_vs_reference"] = bool(same.all() and st["refused"] == 0)
            out["points"].append(pt)
    under = [p for p in out["points"] if p["p99_ms"] < 1.0]
    out["max_decaps_per_s_p99_under_1ms"] = max((p["decaps_per_s"] for p in under), default=None)
    return out


def reference_gpu_leg(cmd, eng, key, stream) -> dict:
    """The reference's own GPU_Optimised decoder (its sources built for sm_100a
    by oracle/Makefile, run by oracle/run_gpu_optimised.py) on 50,000
    mceliece6960119 ciphertexts, its per-stage times beside this engine's
    per-stage kernels and fused kernel on a batch of the same size and key."""
    import torch
    from oracle import run_gpu_optimised as rgo
    if not rgo.available():
        return {"unavailable": "oracle/_ref GPU_Optimised build missing (make -C oracle gpu_optimised)"}
    ref = rgo.run(env={"CUDA_MODULE_LOADING": "EAGER"})  # no module load inside its first stage's timing
    out = {"reference": {k: ref.get(k) for k in ("synd_ms", "bm_ms", "chien_ms", "kernel_ms", "kernel_decaps_per_s",
                                                 "h2d_ms", "d2h_ms", "errorstream_matches", "rc")},
           "ciphertexts": rgo.COUNT,
           "timing": "reference: its own wall-clock stage times (kernel + synchronise, CUDA_MODULE_LOADING=EAGER); "
                     "ours: CUDA events per kernel on the same batch size"}
    _, cts, errs = rgo.make_inputs(rgo.COUNT)
    n, info = rgo.COUNT, key.info
    d_ct = torch.from_numpy(cts).cuda()
    d_s = torch.zeros((n, 2 * info.t), dtype=torch.int16, device="cuda")
    d_l = torch.zeros((n, info.t + 1), dtype=torch.int16, device="cuda")
    d_e = torch.zeros((n, info.err_words), dtype=torch.int32, device="cuda")
    d_w = torch.zeros(n, dtype=torch.int16, device="cuda")
    sp = stream.cuda_stream
    ours = {"synd_ms": _time_stream(lambda: cmd.synd(eng, key, d_ct.data_ptr(), n, d_s.data_ptr(), sp), stream, 3, 1),
            "bm_ms": _time_stream(lambda: cmd.bm(eng, SET, d_s.data_ptr(), n, d_l.data_ptr(), sp), stream, 3, 1),
            "root_ms": _time_stream(lambda: cmd.root(eng, key, d_l.data_ptr(), n, d_e.data_ptr(), d_w.data_ptr(), sp),
                                    stream, 3, 1)}
    plain_ok = bool(np.array_equal(d_e.cpu().numpy().astype("<u4").view(np.uint8).reshape(n, -1)[:, :info.err_bytes],
                                   errs))
    ours["fused_ms"] = _time_stream(lambda: cmd.decrypt_device(eng, key, d_ct.data_ptr(), n, d_e.data_ptr(),
                                                               d_w.data_ptr(), sp, "fused"), stream, 3, 1)
    fused_ok = bool(np.array_equal(d_e.cpu().numpy().astype("<u4").view(np.uint8).reshape(n, -1)[:, :info.err_bytes],
                                   errs))
    ours["results_match_planted"] = plain_ok and fused_ok
    out["ours"] = ours
    r = out["reference"]
    if r.get("synd_ms"):
        out["speedup"] = {"synd": r["synd_ms"] / ours["synd_ms"], "bm": r["bm_ms"] / ours["bm_ms"],
                          "root": r["chien_ms"] / ours["root_ms"], "fused_vs_reference_kernels": r["kernel_ms"] /
                          ours["fused_ms"]}
    return out


def plain_roofline(cmd, eng, key, d_ct, count: int, stream, int_peak: float) -> dict:
    """Each plain per-stage kernel timed alone (CUDA events on `stream`,
    3 calls after 1 warm-up) over the bench batch, against the work of the
    reference's own algorithm for that stage (roofline.plain_stage_work)."""
    import torch
    from cm_decrypt__b200.roofline import plain_stage_work
    info = key.info
    d_s = torch.zeros((count, 2 * info.t), dtype=torch.int16, device="cuda")
    d_l = torch.zeros((count, info.t + 1), dtype=torch.int16, device="cuda")
    d_e = torch.zeros((count, info.err_words), dtype=torch.int32, device="cuda")
    d_w = torch.zeros(count, dtype=torch.int16, device="cuda")
    sp = stream.cuda_stream
    ms = {"synd": _time_stream(lambda: cmd.synd(eng, key, d_ct.data_ptr(), count, d_s.data_ptr(), sp), stream, 3, 1),
          "bm": _time_stream(lambda: cmd.bm(eng, SET, d_s.data_ptr(), count, d_l.data_ptr(), sp), stream, 3, 1),
          "root": _time_stream(lambda: cmd.root(eng, key, d_l.data_ptr(), count, d_e.data_ptr(), d_w.data_ptr(), sp),
                               stream, 3, 1)}
    work = plain_stage_work(SET)
    out = {"bound": "int_alu", "unit": "Tlane-ops/s (lop3)", "peak": int_peak / 1e12,
           "work": "the reference's algorithm per stage: table-row sums, bm()'s multiplies, Horner at every "
                   "support point (cm_decrypt__b200/roofline.py)", "stages": {}}
    for k in ("synd", "bm", "root"):
        a = count / (ms[k] * 1e-3) * work[k]
        out["stages"][k] = {"ms": ms[k], "lane_ops_per_decap": work[k], "achieved": a / 1e12, "frac": a / int_peak}
    return out


def rank_seed(rank: int) -> int:
    """Seed of a replica's workload: every rank decrypts its own batch."""
    return 1000 + rank


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's figure: a multi-GPU step takes as long as its slowest
    replica (NCCL on the GPUs; any backend the process group runs)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput: the units all replicas processed / the slowest time."""
    return world * units_per_rank / seconds


def _time_stream(fn, stream, reps: int, warmup: int) -> float:
    """ms per call of fn(), CUDA events on `stream` after `warmup` untimed calls."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def config_all_sets(cmd, eng, stream, count: int = 1 << 20, reps: int = 3, int_peak: float = 0.0) -> dict:
    """All five parameter sets in turn, `count` ciphertexts of one
    seeded key (the reference kem/ key of the set), autotuned fused kernel
    replayed as a CUDA graph; every output checked against its planted error
    vector and weight t.  Inputs (>= 100 MB per set) exceed L2.  The plain
    path is timed beside it for 6960119."""
    import torch
    out = {}
    sp = stream.cuda_stream
    for s in SERVE_SETS:
        sk = open(os.path.join(REPO, "tests", "golden", "kem", f"sk_{s}.bin"), "rb").read()
        key = cmd.Key(eng, s, sk)
        info = key.info
        cts, planted, _ = cmd.PubKey(s, sk).ciphertexts(seed=77, count=count)
        d_ct = torch.from_numpy(cts).cuda()
        d_err = torch.zeros((count, info.err_words), dtype=torch.int32, device="cuda")
        d_w = torch.zeros(count, dtype=torch.int16, device="cuda")
        tuned = cmd.tune(eng, key)
        g = cmd.Graph(eng, key, d_ct.data_ptr(), count, d_err.data_ptr(), d_w.data_ptr(), path="fused")
        ms = _time_stream(lambda: g.launch(sp), stream, reps, 2)
        g.close()
        ok = bool(np.array_equal(d_err.cpu().numpy().astype("<u4").view(np.uint8).reshape(count, -1)
                                 [:, : info.err_bytes], planted)
                  and (d_w.cpu().numpy().view(np.uint16) == info.t).all())
        row = {"ciphertexts": count, "fused_ms": ms, "fused_decaps_per_s": count / (ms * 1e-3),
               "tuned": tuned, "results_match_planted": ok}
        if int_peak:
            # the executed algorithm's lane-ops at this rate against the measured lop3 rate
            from cm_decrypt__b200.roofline import work_per_decap
            row["roofline_frac"] = count / (ms * 1e-3) * work_per_decap(s, 32 * tuned["wpb"])["total"] / int_peak
        if s == SET:
            msp = _time_stream(lambda: cmd.decrypt_device(eng, key, d_ct.data_ptr(), count, d_err.data_ptr(),
                                                          d_w.data_ptr(), sp, "plain"), stream, 1, 1)
            row["plain_ms"] = msp
            row["plain_decaps_per_s"] = count / (msp * 1e-3)
            row["fused_speedup"] = msp / ms
        out[str(s)] = row
        del d_ct, d_err, d_w
        key.free()
    return out


def keygen_leg(cmd, eng, set_id: int = 6960119, count: int = 64, cpu_seconds: float = 12.0) -> dict:
    """Key generation (crypto_kem_keypair, kem/common/core/operations.c:36-107)
    for `count` seeds in one batched call, host seeds in and host key pairs
    out (pinned buffers), after a warm-up batch of the same size, against the
    reference's own key generation (oracle/_ref
    libkeygen_<set>, its SHAKE256 seed expansion done with hashlib) on all
    host cores over a bounded sample of seeds.  Rates count whole key pairs,
    rejected attempts included (about 3.5 attempts per key on average)."""
    import concurrent.futures as cf
    import threading

    import torch

    from oracle import oracle as o
    g = np.random.default_rng(0xC0FFEE)
    seeds = np.frombuffer(g.bytes(32 * count), np.uint8).reshape(count, 32)
    # warm-up: a batch of other seeds of the same size (the engine keeps the
    # workspace it grows to)
    cmd.kem_keypair_batch(eng, set_id, np.frombuffer(g.bytes(32 * count), np.uint8).reshape(count, 32))
    t0 = time.perf_counter()
    one = cmd.kem_keypair(eng, set_id, seeds[0].tobytes())
    single_s = time.perf_counter() - t0
    # pinned host buffers for the key pairs, as a service would keep them
    info = cmd.set_info(set_id)
    pk_pin = torch.empty((count, cmd.pk_bytes(set_id)), dtype=torch.uint8).pin_memory().numpy()
    sk_pin = torch.empty((count, info.sk_bytes), dtype=torch.uint8).pin_memory().numpy()
    l0 = eng.launch_count()
    t0 = time.perf_counter()
    pks, sks, att = cmd.kem_keypair_batch(eng, set_id, seeds, pk_out=pk_pin, sk_out=sk_pin)
    dt = time.perf_counter() - t0
    launches = eng.launch_count() - l0
    checker = o.RefKeygen(set_id) if o.RefKeygen.available(set_id) else o.Oracle(set_id)
    ok = all(checker.keypair(seeds[i].tobytes()) == (pks[i].tobytes(), sks[i].tobytes(), int(att[i]))
             for i in range(2)) and (one[0], one[1]) == (pks[0].tobytes(), sks[0].tobytes())
    out = {"set": set_id, "keys": count, "attempts": int(att.sum()), "seconds": dt,
           "keypairs_per_s": count / dt, "attempts_per_s": float(att.sum()) / dt, "gpu_launches": launches,
           "single_key_ms": single_s * 1e3, "single_key_attempts": one[2], "matches_reference": bool(ok)}
    if cpu_seconds <= 0:
        return out
    # CPU: the reference's keygen, one key per thread (ctypes drops the GIL)
    cores = os.cpu_count() or 1
    threading.stack_size(64 << 20)  # pk_gen keeps its matrix on the stack
    cpu_seeds = [np.random.default_rng(1000 + i).bytes(32) for i in range(4 * cores)]
    done, attempts = 0, 0
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        futs = [ex.submit(checker.keypair, sd) for sd in cpu_seeds]
        for f in futs:
            _, _, a = f.result()
            done += 1
            attempts += a
            if time.perf_counter() - t0 > cpu_seconds and done >= cores:
                break
        for f in futs:
            f.cancel()
    cpu_dt = time.perf_counter() - t0
    threading.stack_size(0)
    out["cpu_baseline"] = {"keypairs_per_s": done / cpu_dt, "attempts": attempts, "keys": done, "cores": cores,
                           "kind": "reference" if isinstance(checker, o.RefKeygen) else "port",
                           "sample": f"{done} seeds on {cores} threads, {cpu_dt:.1f} s"}
    return out


def config_mixed(cmd, eng, stream, nkeys: int = 64, count: int = 1 << 18, reps: int = 3,
                 reference_check: bool = True) -> dict:
    """Mixed batch: 64 seeded keys spread 13/13/13/13/12 over the five
    sets, `count` ciphertexts with the set drawn uniformly per ciphertext (key
    uniform within the set), 10% uniformly random mt-bit strings, all in one
    cmd_decrypt_mixed_device launch.  Every row, valid and malformed, is
    compared with the reference's own CPU decoder (oracle/_ref, all host
    threads), and the valid ones also with their planted vectors."""
    import torch
    from oracle import oracle as o
    golden = {s: open(os.path.join(REPO, "tests", "golden", "kem", f"sk_{s}.bin"), "rb").read() for s in SERVE_SETS}
    per_set = [nkeys // 5 + (1 if i < nkeys % 5 else 0) for i in range(5)]
    ring = [(s, cmd.synth_key(s, golden[s], 0xC0FFEE + 97 * i + j)) for i, s in enumerate(SERVE_SETS)
            for j in range(per_set[i])]
    keys = [cmd.Key(eng, s, sk) for s, sk in ring]
    g = np.random.default_rng(0x5EED4)
    set_of = g.integers(0, 5, count)
    first = np.cumsum([0] + per_set[:-1])
    key_idx = (first[set_of] + (g.random(count) * np.array(per_set)[set_of]).astype(np.int64)).astype(np.uint32)
    CT, EW = 208, 256
    buf = np.zeros((count, CT), np.uint8)
    planted = np.zeros((count, 1024), np.uint8)
    valid = np.zeros(count, np.uint8)
    for k in range(len(keys)):
        idx = np.nonzero(key_idx == k)[0]
        if idx.size == 0:
            continue
        c, e, v = cmd.PubKey(*ring[k]).ciphertexts(seed=1000 + k, count=idx.size, malformed_permille=100)
        buf[idx, : c.shape[1]] = c
        planted[idx, : e.shape[1]] = e
        valid[idx] = v
    ct_off = np.arange(count, dtype=np.uint64) * CT
    err_off = np.arange(count, dtype=np.uint64) * EW
    d_ct = torch.from_numpy(buf.reshape(-1)).cuda()
    d_err = torch.zeros(count * EW, dtype=torch.int32, device="cuda")
    d_w = torch.zeros(count, dtype=torch.int16, device="cuda")
    sp = stream.cuda_stream
    ms = _time_stream(lambda: cmd.decrypt_mixed_device(eng, keys, key_idx, d_ct.data_ptr(), ct_off, d_err.data_ptr(),
                                                       err_off, d_w.data_ptr(), sp), stream, reps, 2)
    E = d_err.cpu().numpy().astype("<u4").view(np.uint8).reshape(count, 1024)
    W = d_w.cpu().numpy().view(np.uint16)
    for k in keys:
        k.free()
    ok = True
    t_of = np.array([cmd.set_info(s).t for s, _ in ring])[key_idx]
    for i, s in enumerate(SERVE_SETS):
        rows = np.nonzero((valid == 1) & (set_of == i))[0]
        nb = cmd.set_info(s).err_bytes
        ok = ok and bool(np.array_equal(E[rows, :nb], planted[rows, :nb]) and (W[rows] == t_of[rows]).all())
    out = {"keys": len(keys), "ciphertexts": count, "malformed_fraction": float(1 - valid.mean()),
           "ms_per_launch": ms, "decaps_per_s": count / (ms * 1e-3), "valid_match_planted": ok,
           "timed": "whole cmd_decrypt_mixed_device call: host round planning, plan upload and the fused kernel"}
    if reference_check:
        t0 = time.perf_counter()
        ref, kind = o.reference_decrypt_rows(ring, key_idx, buf)
        weights = np.unpackbits(ref, axis=1).sum(axis=1)
        same = (E == ref).all(axis=1) & (W == weights)
        out["reference_check"] = {
            "checker": kind, "rows": int(count), "rows_equal": int(same.sum()),
            "malformed_rows_equal": int(same[valid == 0].sum()), "malformed_rows": int((valid == 0).sum()),
            "seconds": time.perf_counter() - t0, "threads": os.cpu_count() or 1}
        out["bit_exact_vs_reference"] = bool(same.all())
    return out


ERR_WORDS = 218  # u32 words of a mceliece6960119 error row (n = 6960 bits)
CT_BYTES = 194


def rotating_buffers(count: int) -> tuple[int, int]:
    """Device buffer sets the GPU arm rotates through so that no step finds
    its inputs or outputs in L2: (sets, bytes per set)."""
    per_set = count * (CT_BYTES + 4 * ERR_WORDS + 2)
    return max(2, math.ceil(2 * L2_BYTES / per_set)), per_set


def workload_config(count: int, world: int) -> dict:
    """The workload both arms name (the reference arm times a bounded sample
    of the same batch on the host cores)."""
    nbuf, per_set = rotating_buffers(count)
    return {"workload": "mceliece6960119 decrypt, 1 seeded key (reference kem/ key), "
                        f"{count} ciphertexts/step/GPU, uniform weight-119 errors",
            "set": SET, "ciphertexts_per_step": count, "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2: the GPU arm rotates {nbuf} device-resident buffer sets "
                  f"({nbuf * per_set / 2**20:.0f} MiB > 2x L2)"}


def run_reference(args) -> None:
    """The reference's own CPU decoder (CPU/ sources compiled unmodified into
    oracle/_ref by oracle/Makefile; the oracle restatement if that build is
    absent) on all host cores.  Its inputs come from the oracle alone: the
    public key of the kem/ key regenerated from the seed stored in it
    (crypto_kem_keypair), weight-119 error vectors and their encryptions
    (encrypt.c's syndrome rule).  Each step decodes a bounded sample of the
    workload's batch, sized so that the whole run stays within minutes, and
    every decoded vector is checked against the one encrypted."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import oracle as o
    sk = open(KEM_SK, "rb").read()
    orc = o.Oracle(SET)
    pk, sk_again, _ = orc.keypair(sk[:32])
    if sk_again != sk:
        raise SystemExit("reference arm: the kem/ key does not regenerate from its seed")
    cores = os.cpu_count() or 1
    kind = "reference" if o.RefLib.available(SET) else "port"
    dec = o.RefLib(SET) if kind == "reference" else orc
    probe_e = orc.random_errors(seed=rank_seed(0) + 7, count=2 * cores)
    probe = orc.encrypt(pk, probe_e)
    t0 = time.perf_counter()
    dec.decrypt(sk, probe, nthreads=cores)
    rate = probe.shape[0] / (time.perf_counter() - t0)
    # about 1.5 s of decoding per step, whole rounds of `cores` ciphertexts
    per_step = int(min(args.count, max(cores, round(1.5 * rate / cores) * cores)))
    planted = orc.random_errors(seed=rank_seed(0), count=per_step)
    cts = orc.encrypt(pk, planted)
    for _ in range(args.warmup):
        dec.decrypt(sk, cts, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        got = dec.decrypt(sk, cts, nthreads=cores)
    dt = time.perf_counter() - t0
    if not np.array_equal(got, planted):
        raise SystemExit("reference arm: decoded vectors differ from the encrypted ones")
    v = per_step * args.steps / dt
    sample = (f"{per_step} of the {args.count} mceliece6960119 ciphertexts of a step, decoded on {cores} "
              f"host threads, every step")
    line = {
        "impl": "reference", "metric": "decaps/s", "value": v, "unit": "decaps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16 GF(2^13)",
        "data": "synthetic",
        "config": workload_config(args.count, world),
        "sample": sample,
        "cpu_baseline": {"value": v, "unit": "decaps/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "decaps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "results_match_planted": True,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    import cm_decrypt__b200 as cmd
    from cm_decrypt__b200.roofline import hbm_bytes_per_decap, work_per_decap

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.keygen_only:
        eng = cmd.Engine(local)
        print(json.dumps(keygen_leg(cmd, eng, count=args.keygen_count,
                                    cpu_seconds=0.0 if args.no_cpu_baseline else 12.0)), flush=True)
        eng.close()
        return
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    count = args.count

    eng = cmd.Engine(local)
    sk = open(KEM_SK, "rb").read()
    key = cmd.Key(eng, SET, sk)
    info = key.info
    pk = cmd.PubKey(SET, sk)
    cts, planted, valid = pk.ciphertexts(seed=rank_seed(rank), count=count)

    # Rotating device buffer sets, together larger than 2x L2, so no step
    # reads inputs or writes outputs the previous step left in L2.
    assert info.ct_bytes == CT_BYTES and info.err_words == ERR_WORDS
    nbuf, per_set = rotating_buffers(count)
    d_cts = [torch.from_numpy(cts).cuda() for _ in range(nbuf)]
    d_err = [torch.zeros((count, info.err_words), dtype=torch.int32, device="cuda") for _ in range(nbuf)]
    d_w = [torch.zeros(count, dtype=torch.int16, device="cuda") for _ in range(nbuf)]
    # A dedicated stream: the engine launches on it and the CUDA events are
    # recorded on it (stream 0 would select the engine's own stream).
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    assert sp != 0

    # Launch configuration chosen by the autotuner (cached per GPU and set),
    # then one captured CUDA graph per buffer set, replayed every step.
    if args.kernel_only and args.wpb:
        cmd.set_fused_config(eng, SET, args.wpb)
    # tuned for this batch size (the winner depends on how the batch fills
    # whole rounds of the resident warps)
    tuned = cmd.fused_config(eng, SET) if args.kernel_only else cmd.tune(eng, key, sample_count=count)
    graphs = [cmd.Graph(eng, key, d_cts[b].data_ptr(), count, d_err[b].data_ptr(), d_w[b].data_ptr(), path="fused")
              for b in range(nbuf)]

    def step(i: int, path: str) -> None:
        b = i % nbuf
        if path == "fused":
            graphs[b].launch(sp)
        else:
            cmd.decrypt_device(eng, key, d_cts[b].data_ptr(), count, d_err[b].data_ptr(), d_w[b].data_ptr(), sp,
                               path)

    def check(b: int) -> None:
        w = d_err[b].cpu().numpy().astype("<u4").view(np.uint8).reshape(count, -1)[:, : info.err_bytes]
        if not np.array_equal(w, planted):
            raise SystemExit("bench: decrypt output differs from the planted error vectors")
        if not (d_w[b].cpu().numpy().view(np.uint16) == info.t).all():
            raise SystemExit("bench: weight check failed")

    def timed(path: str, steps: int, warmup: int) -> tuple[float, int, dict | None]:
        for i in range(warmup):
            step(i, path)
        torch.cuda.synchronize()
        for b in range(min(nbuf, warmup)):
            check(b)
        for b in range(nbuf):
            d_err[b].zero_()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = eng.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            e0.record(stream)
            for i in range(steps):
                step(i, path)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        launches = eng.launch_count() - l0
        for b in range(min(nbuf, steps)):
            check(b)
        ms = max_over_ranks(ms, world)
        return ms, launches, clk.summary()

    if args.kernel_only:
        ms, launches, _ = timed(args.path, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"kernel_only": True, "path": args.path,
                              "decaps_per_s": job_rate(world, count * args.steps, ms * 1e-3),
                              "ms_per_step": ms / args.steps, "gpu_launches": launches}), flush=True)
        return
    int_peak = eng.int_peak()
    ms, launches, clocks = timed("fused", args.steps, args.warmup)
    ms_plain, roof_plain = None, None
    if not args.no_plain:
        ms_plain, _, _ = timed("plain", max(1, min(args.steps, 3)), 1)
        roof_plain = plain_roofline(cmd, eng, key, d_cts[0], count, stream, int_peak)

    # End to end through the public host-buffer call, pinned host memory.
    h_cts = torch.from_numpy(cts).pin_memory().numpy()
    h_err = torch.empty((count, info.err_bytes), dtype=torch.uint8).pin_memory().numpy()
    h_w = torch.empty(count, dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    for _ in range(max(1, args.warmup)):
        cmd.decrypt_into(eng, key, h_cts, h_err, h_w, path="fused")
    if not np.array_equal(h_err, planted):
        raise SystemExit("bench: e2e output differs from the planted error vectors")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cmd.decrypt_into(eng, key, h_cts, h_err, h_w, path="fused")
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)

    # The same through cmd_decrypt_positions (binary wire format: t+1 u16 per
    # ciphertext come back instead of n/8 bytes).
    h_pos = torch.empty((count, info.t + 1), dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    L = cmd.lib()
    pos_call = lambda: cmd._check(L.cmd_decrypt_positions(eng.handle, key.handle, h_cts.ctypes.data, count,
                                                          h_pos.ctypes.data), "cmd_decrypt_positions")
    pos_call()
    if not (h_pos[:, 0] == info.t).all():
        raise SystemExit("bench: positions weights differ from t")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pos_call()
    torch.cuda.synchronize()
    pos_s = max_over_ranks(time.perf_counter() - t0, world)
    pos_ok = bool(np.array_equal(h_pos[:512], cmd.positions_from_errors(SET, planted[:512])))

    # KEM decapsulation on the same device-resident batches: decrypt, the
    # re-encoding / weight / padding check and SHAKE256 session keys.
    d_keys = torch.zeros((count, 32), dtype=torch.uint8, device="cuda")
    d_acc = torch.zeros(count, dtype=torch.uint8, device="cuda")
    t0 = time.perf_counter()
    cmd.prepare_decap(eng, key)  # public-key columns, derived on the device once per key
    prep_ms = (time.perf_counter() - t0) * 1e3
    dec_ms = _time_stream(lambda: cmd.kem_decap_device(eng, key, d_cts[0].data_ptr(), count, d_keys.data_ptr(),
                                                       d_acc.data_ptr(), sp), stream, max(1, args.steps // 2), 2)
    dec_ms = max_over_ranks(dec_ms, world)
    dec_ok = bool(d_acc.cpu().numpy().all())

    value = job_rate(world, count * args.steps, ms * 1e-3)
    per_rank = count * args.steps / (ms * 1e-3)
    w = work_per_decap(SET, 32 * tuned["wpb"])
    achieved = per_rank * w["total"]
    hbm = per_rank * hbm_bytes_per_decap(SET)
    traffic, traffic_detail = None, None
    if os.path.exists(TRAFFIC_FILE):
        # dram__bytes_read.sum + dram__bytes_write.sum of one captured launch,
        # per launch of this batch, with how the capture was scaled
        tr = json.load(open(TRAFFIC_FILE))
        traffic = tr.get("dram_bytes_per_launch")
        traffic_detail = {k: tr[k] for k in ("dram_read_bytes_per_launch", "dram_write_bytes_per_launch",
                                             "algorithmic_bytes_per_launch", "captured_cts", "scaling",
                                             "source") if k in tr}
    peaks = {}
    pk_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    line = {
        "metric": "decaps/s", "value": value, "unit": "decaps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 bitsliced GF(2^13)", "data": "synthetic",
        "config": workload_config(count, world),
        "gpu_launches": launches,
        "plain": None if ms_plain is None else {
            "value": job_rate(world, count * min(args.steps, 3), ms_plain * 1e-3),
            "ms_per_step": ms_plain / max(1, min(args.steps, 3)),
            "fused_speedup": (ms_plain / max(1, min(args.steps, 3))) / (ms / args.steps)},
        "e2e": {"value": job_rate(world, count * args.steps, e2e_s), "unit": "decaps/s",
                "h2d_bytes_per_step": count * info.ct_bytes,
                "d2h_bytes_per_step": count * (info.err_bytes + 2)},
        "kem_decap": {"value": job_rate(world, count, dec_ms * 1e-3), "unit": "decaps/s", "ms_per_batch": dec_ms,
                      "call": "cmd_kem_decap_device (decrypt + re-encoding check + SHAKE256 keys), device buffers",
                      "all_valid_accepted": dec_ok, "key_prepare_ms": prep_ms},
        "e2e_positions": {"value": job_rate(world, count * args.steps, pos_s), "unit": "decaps/s",
                          "call": "cmd_decrypt_positions (error positions, binary errorstream rows)",
                          "h2d_bytes_per_step": count * info.ct_bytes,
                          "d2h_bytes_per_step": count * (info.t + 1) * 2, "results_match_planted": pos_ok},
        "roofline": {"bound": "int_alu", "achieved": achieved / 1e12, "peak": int_peak / 1e12,
                     "unit": "Tlane-ops/s (lop3)", "frac": achieved / int_peak,
                     "peak_source": "measured on this GPU: lop3.b32 chains (cmd_bench_int_peak)",
                     "work_per_decap": w,
                     "yardstick": {"what": "the reference's algorithm (masked table rows, bm(), Horner at every support point): "
                                           "equivalent lane-ops/s at this decap rate",
                                   "equivalent": per_rank * w["yardstick_total"] / 1e12,
                                   "x_peak": per_rank * w["yardstick_total"] / int_peak},
                     "traffic": traffic, "traffic_detail": traffic_detail,
                     "hbm": {"achieved_gbs": hbm / 1e9, "peak_gbs": hbm_peak, "frac": hbm / 1e9 / hbm_peak,
                             "bytes_per_decap": hbm_bytes_per_decap(SET)},
                     "plain": roof_plain},
        "clocks": clocks,
        "fused_config": {"tuned": tuned, "launch": "CUDA graph replay, one graph per buffer set"},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(sk, cts)
    if world == 1 and not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_leg(cmd, eng, key, stream)
    if world == 1 and not args.no_configs:
        line["configs"] = {"all_sets_2^20": config_all_sets(cmd, eng, stream, int_peak=int_peak),
                           "mixed_64keys_2^18": config_mixed(cmd, eng, stream,
                                                             reference_check=not args.no_reference_check)}
    for g_ in graphs:
        g_.close()
    if world == 1 and not args.no_keygen:
        line["keygen"] = keygen_leg(cmd, eng, count=args.keygen_count)
    if world == 1 and not args.no_serve:
        fused_rate = value
        rates = sorted({1e4, 1e5, 5e5, 1e6, 2e6, 3e6, 4e6, 5e6, 6e6, 7e6, 7.5e6, 8e6,
                        round(0.5 * fused_rate, -5), round(0.6 * fused_rate, -5)})
        line["serving"] = serving_leg(cmd, eng, args.serve_keys, rates, args.serve_seconds,
                                      reference_check=not args.no_reference_check)
        line["serving"]["fused_batch_decaps_per_s"] = fused_rate
        best = line["serving"]["max_decaps_per_s_p99_under_1ms"]
        line["serving"]["frac_of_fused_at_p99_under_1ms"] = None if best is None else best / fused_rate
        pts = line["serving"]["points"]
        line["p50_ms"] = min(pts, key=lambda p: abs(p["offered_per_s"] - 0.5 * fused_rate))["p50_ms"]
        line["p99_ms"] = min(pts, key=lambda p: abs(p["offered_per_s"] - 0.5 * fused_rate))["p99_ms"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    key.free()
    eng.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
