"""Builds libcfgmm.so in-tree with nvcc for sm_100a (B200).

Usage: python cfgable-matmul_b200/build.py [--force]

Every .cu file under csrc/ is compiled separately (so a change rebuilds only
what changed) and linked into cfgable-matmul_b200/libcfgmm.so with the static
CUDA runtime, so the library loads without any LD_LIBRARY_PATH setup.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcfgmm.so")
PEAKS_LIB = os.path.join(HERE, "libcfgmm_peaks.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
    "-I", INCLUDE, "-I", CSRC,
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(src: str, dst: str, deps: list[str]) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(x) > t for x in [src] + deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Builds libcfgmm.so (the product) and libcfgmm_peaks.so (peak probes
    used by bench.py as roofline denominators)."""
    _build_lib(sorted(glob.glob(os.path.join(CSRC, "*.cu"))), LIB, force, verbose)
    _build_lib(sorted(glob.glob(os.path.join(CSRC, "peaks", "*.cu"))), PEAKS_LIB, force, verbose)
    return LIB


def _build_lib(sources: list[str], lib: str, force: bool, verbose: bool) -> None:
    os.makedirs(BUILD, exist_ok=True)
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
                     + glob.glob(os.path.join(INCLUDE, "*.h")))
    objs = []
    procs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.relpath(src, CSRC).replace(os.sep, "_")[:-3] + ".o")
        objs.append(obj)
        if force or _newer(src, obj, headers):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append(src)
            sys.stderr.write(text)
        elif verbose and text:
            sys.stdout.write(text)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    if force or procs or not os.path.exists(lib):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs + ["-lpthread"]
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
