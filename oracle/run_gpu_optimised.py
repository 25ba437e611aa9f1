"""Runs the reference's own GPU_Optimised decoder for mceliece6960119
(GPU_Optimised/param/param6960119/src/cuda/decrypt.cu), built for sm_100a by
`make -C oracle gpu_optimised`, on 50,000 ciphertexts: the batch its published
profiles use.

TEST INFRASTRUCTURE ONLY: a baseline measurement, never part of the product.
The binary finds its inputs and writes its outputs relative to its own path
(GPU_Optimised/src/host/util.c: <root>/kem/test_vectors/Cipher_Sk/{sk,ct}_
6960119.bin; decrypt.cu: <root>/GPU_Optimised/results/profile/ and
results/output/), so each run copies it into a scratch tree of that shape.
The inputs come from the oracle alone: the reference's kem/ key (regenerated
from the seed stored in it) and 50,000 encryptions of weight-119 error
vectors.  The run reports the binary's own per-stage times (wall clock around
each kernel and its synchronisation, decrypt.cu:371-419) and checks its
errorstream against the encrypted vectors.

    python oracle/run_gpu_optimised.py [--count 50000] [--keep DIR]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile


HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
BIN = os.path.join(HERE, "_ref", "gpu_optimised", "GPU_Optimised", "bin", "decrypt_gpu_optimised_6960119")
SET = 6960119
COUNT = 50000  # KATNUM the binary is built with (oracle/Makefile)


def available() -> bool:
    return os.path.exists(BIN)


def make_inputs(count: int = COUNT, seed: int = 4242):
    """(sk bytes, ciphertexts [count, 194], error vectors [count, 870])."""
    sys.path.insert(0, REPO)
    from oracle import oracle as o
    orc = o.Oracle(SET)
    sk = open(os.path.join(REPO, "tests", "golden", "kem", f"sk_{SET}.bin"), "rb").read()
    pk, sk_again, _ = orc.keypair(sk[:32])
    if sk_again != sk:
        raise RuntimeError("the kem/ key does not regenerate from its seed")
    errs = orc.random_errors(seed=seed, count=count)
    return sk, orc.encrypt(pk, errs), errs


def run(count: int = COUNT, keep: str | None = None, env: dict | None = None, prefix: list[str] | None = None) -> dict:
    """One run of the binary in a scratch tree; returns its stage times and
    whether its errorstream equals the encrypted vectors.  `prefix` wraps the
    command (a profiler), `env` adds environment variables."""
    if count != COUNT:
        raise ValueError(f"the binary is built for {COUNT} ciphertexts")
    sys.path.insert(0, REPO)
    from oracle import oracle as o
    sk, cts, errs = make_inputs(count)
    root = keep or tempfile.mkdtemp(prefix="gpu_optimised_")
    try:
        vec = os.path.join(root, "kem", "test_vectors", "Cipher_Sk")
        os.makedirs(vec, exist_ok=True)
        open(os.path.join(vec, f"sk_{SET}.bin"), "wb").write(sk)
        open(os.path.join(vec, f"ct_{SET}.bin"), "wb").write(cts.tobytes())
        bindir = os.path.join(root, "GPU_Optimised", "bin")
        os.makedirs(bindir, exist_ok=True)
        for sub in ("profile", "output"):
            os.makedirs(os.path.join(root, "GPU_Optimised", "results", sub), exist_ok=True)
        exe = os.path.join(bindir, os.path.basename(BIN))
        shutil.copy2(BIN, exe)
        res = subprocess.run((prefix or []) + [exe], capture_output=True, text=True,
                             env=dict(os.environ, **(env or {})), timeout=600)
        out = {"rc": res.returncode, "stdout_tail": res.stdout[-400:], "stderr_tail": res.stderr[-400:]}
        prof = os.path.join(root, "GPU_Optimised", "results", "profile", f"Profile_GPU_optimised_{SET}.txt")
        if os.path.exists(prof):
            text = open(prof).read()
            for key, pat in (("h2d_ms", r"H2D\s*:\s*([\d.]+)"), ("synd_ms", r"syndrome\s*:\s*([\d.]+)"),
                             ("bm_ms", r"Berlekamp-Massey\s*:\s*([\d.]+)"), ("chien_ms", r"Chien search\s*:\s*([\d.]+)"),
                             ("d2h_ms", r"D2H\s*:\s*([\d.]+)"), ("wall_ms", r"wall\s*:\s*([\d.]+)"),
                             ("throughput_ct_per_s", r"throughput\s*:\s*([\d.]+)")):
                m = re.search(pat, text)
                out[key] = float(m.group(1)) if m else None
            if out.get("synd_ms") is not None:
                k_ms = out["synd_ms"] + out["bm_ms"] + out["chien_ms"]
                out["kernel_ms"] = k_ms
                out["kernel_decaps_per_s"] = count / (k_ms * 1e-3)
        stream = os.path.join(root, "GPU_Optimised", "results", "output", f"errorstream0_{SET}.bin")
        if os.path.exists(stream):
            out["errorstream_matches"] = open(stream, "rb").read() == o.Oracle(SET).errorstream(errs)
        out["ciphertexts"] = count
        return out
    finally:
        if not keep:
            shutil.rmtree(root, ignore_errors=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=COUNT)
    ap.add_argument("--keep", default=None, help="scratch tree to create and keep")
    ap.add_argument("--eager", action="store_true", help="CUDA_MODULE_LOADING=EAGER (no module load in the first stage)")
    args = ap.parse_args()
    if not available():
        print(json.dumps({"unavailable": "make -C oracle gpu_optimised has not been run"}))
        return 0
    r = run(args.count, args.keep, env={"CUDA_MODULE_LOADING": "EAGER"} if args.eager else None)
    print(json.dumps(r))
    return 0 if r["rc"] == 0 and r.get("errorstream_matches") else 1


if __name__ == "__main__":
    sys.exit(main())
