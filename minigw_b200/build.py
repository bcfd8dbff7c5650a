"""Build libgwb200.so (sm_100a) and the `gw` command-line driver in-tree.

    python minigw_b200/build.py [--verbose] [--ptxas-info]

Outputs (git-ignored, shipped with the tree):
    minigw_b200/libgwb200.so   C ABI of include/gwb200.h
    minigw_b200/bin/gw         drop-in for the reference's `gw` executable
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgwb200.so"
GW_BIN = PKG / "bin" / "gw"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels_fp64.cu", "kernels_f32.cu", "kernels_tc.cu", "kernels_oz.cu", "kernels_c64.cu",
              "kernels_small.cu", "kernels_batch.cu", "kernels_refine.cu", "kernels_gram_oz.cu", "kernels_offdiag.cu", "gwb200_abi.cu", "noalloc.cu"]
CXX_SOURCES = ["host_grid.cpp", "host_h5.cpp", "server.cpp"]
CLI_SOURCES = ["gw_main.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgwb200")


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return res.stdout + res.stderr


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "gwb200.h"]
    objs = []
    for src in CU_SOURCES:
        obj = BUILD / (src + ".o")
        if _stale(obj, [CSRC / src] + headers) or ptxas_info:
            cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
                   str(CSRC / src), "-o", str(obj)]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            out = _run(cmd, verbose)
            if ptxas_info:
                print(out)
        objs.append(obj)
    for src in CXX_SOURCES:
        obj = BUILD / (src + ".o")
        if _stale(obj, [CSRC / src] + headers):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-pthread", "-ffp-contract=off", "-Wall", "-Wextra",
                  "-I/usr/local/cuda/include", "-c", str(CSRC / src), "-o", str(obj)], verbose)
        objs.append(obj)
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-Xcompiler", "-pthread", "-o", str(LIB), *map(str, objs)], verbose)
    GW_BIN.parent.mkdir(exist_ok=True)
    cli = [CSRC / s for s in CLI_SOURCES]
    if all(p.exists() for p in cli) and _stale(GW_BIN, cli + [LIB, ROOT / "include" / "gwb200.h"]):
        _run(["g++", "-std=c++20", "-O2", "-ffp-contract=off", "-Wall", "-Wextra", f"-I{ROOT / 'include'}",
              *map(str, cli), "-o", str(GW_BIN), f"-L{PKG}", "-lgwb200", f"-Wl,-rpath,{PKG}"], verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills/shared memory per kernel")
    args = ap.parse_args()
    print(build(verbose=args.verbose, ptxas_info=args.ptxas_info))


if __name__ == "__main__":
    main()
