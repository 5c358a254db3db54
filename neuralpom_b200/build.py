"""Build the sm_100a shared library ``neuralpom_b200/_lib/libnpom_b200.so``.

The library is plain CUDA C++ behind the C ABI of ``include/npom.h``; it is
compiled with nvcc directly (no torch extension machinery), in-tree, so the
built file travels with the repository to the GPU host.

    python -m neuralpom_b200.build          # or build() from Python
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIBNAME = "libnpom_b200.so"
SOURCES = ["npom_kernels.cu"]
HEADERS = ["npom_ctx.cuh", "npom_phases_a.cuh", "npom_phases_ext.cuh", "npom_phases_int.cuh", "npom_host.cuh",
           "npom_pcg_cluster.cuh", "npom_lanes.cuh", "npom_adjoint.cuh", "npom_adjoint_launch.cuh", "npom_mpdata.cuh",
           "npom_mpdata_adjoint.cuh",
           "npom_batch.cuh"]

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    # the reference evaluates every expression without fused multiply-adds
    # (torch CPU, and enable_fp_fusion=False in its Triton kernels); keep
    # IEEE division and square root as well
    "--fmad=false",
    "-prec-div=true",
    "-prec-sqrt=true",
    "-Xcompiler", "-fPIC",
    "-shared",
]


def nvcc_path():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build neuralpom_b200")
    return cand


def lib_path():
    return os.path.join(LIBDIR, LIBNAME)


def _stale(out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "npom.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra_flags=()):
    """Compile the library if any source is newer than it; returns its path."""
    out = lib_path()
    if not force and not _stale(out):
        return out
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = out + ".tmp"
    cmd = [nvcc_path(), *NVCC_FLAGS, *extra_flags, "-I", os.path.join(ROOT, "include"),
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True,
                extra_flags=("-Xptxas", "-v") if "--ptxas" in sys.argv else ()))
