"""Builds the engine in-tree: cm_decrypt__b200/libcmd_b200.so (sm_100a) and the
cm_decrypt__b200/cmd_decrypt CLI.  Objects go to cm_decrypt__b200/_build/;
a source is recompiled when it or any header under csrc/ or include/ is newer
than its object.  nvcc cross-compiles, so this runs without a GPU.

    python -m cm_decrypt__b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libcmd_b200.so")
CLI = os.path.join(PKG, "cmd_decrypt")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++20", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
              "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, force: bool, hdr_mtime: float, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj):
        om = os.path.getmtime(obj)
        if om >= os.path.getmtime(src) and om >= hdr_mtime:
            return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_mtime()
    lib_srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    lib_srcs = [s for s in lib_srcs if os.path.basename(s) != "cli.cpp"]
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr, extra), lib_srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    cli_src = os.path.join(CSRC, "cli.cpp")
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB),
                                                                         os.path.getmtime(cli_src)):
        cmd = [nvcc(), "-O2", "-std=c++20", "-I" + INCLUDE, "-o", CLI, cli_src, "-L" + PKG, "-lcmd_b200",
               "-Xlinker", "-rpath,$ORIGIN"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"cli link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--ptxas-v", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, jobs=args.j, verbose_ptxas=args.ptxas_v))
    return 0


if __name__ == "__main__":
    sys.exit(main())
