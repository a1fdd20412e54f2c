"""Build recipe of the native library libdgrain.so (C host code + sm_100a CUDA kernels).

    python dg-rain_b200/build.py            # builds dg-rain_b200/dgrain/libdgrain.so
    python dg-rain_b200/build.py --checked  # ... libdgrain_checked.so (-DDGR_CHECKED)

The library is built in-tree so that it travels with the repository to the GPU host.

Flags: sm_100a only; --fmad=false keeps every multiply and add a separately rounded IEEE
operation so that the kernels reproduce the reference C step's arithmetic.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "dgrain")
LIB = os.path.join(OUT_DIR, "libdgrain.so")
BUILD = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]
CC_FLAGS = ["-std=c99", "-O2", "-ffp-contract=off", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter"]

CU_SOURCES = ["dgr_capi.cu", "dgr_noalloc.cu", "dgr_adjoint.cu", "dgr_output.cu", "dgr_ingest.cu", "dgr_coupling.cu"]
C_SOURCES = ["dgr_host.c"]
DEPS = ["dgr_kernels.cuh", "dgr_device.cuh", "dgr_forcing.h", "dgr_internal.cuh", "dgr_scheme.cuh",
        "dgr_dual.cuh", "dgr_reverse.cuh", "dgr_tlm.cuh", "dgr_p2.cuh", "dgr_p2_adjoint.cuh", "dgr_format.cuh", "dgr_ptr.h", os.path.join("..", "..", "include", "dgrain.h")]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdgrain.so")
    return cand


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def build(verbose: bool = False, ptxas_verbose: bool = False, force: bool = False, out: str | None = None,
          defines: list[str] | None = None, build_dir: str | None = None) -> str:
    """Build libdgrain.so (or `out`, with extra -D `defines`, for tuning sweeps)."""
    lib = out or LIB
    build_dir = build_dir or (BUILD if out is None else out + ".build")
    os.makedirs(build_dir, exist_ok=True)
    dflags = [f"-D{d}" for d in (defines or [])]
    nvcc = _nvcc()
    all_src = [os.path.join(CSRC, f) for f in CU_SOURCES + C_SOURCES + DEPS]
    if not force and not _newer(lib, all_src + [__file__]):
        return lib
    objs, jobs = [], []
    for f in C_SOURCES:
        o = os.path.join(build_dir, f + ".o")
        jobs.append((["gcc", *CC_FLAGS, "-c", os.path.join(CSRC, f), "-o", o], verbose))
        objs.append(o)
    for f in CU_SOURCES:
        o = os.path.join(build_dir, f + ".o")
        extra = ["-Xptxas", "-v"] if ptxas_verbose else []
        jobs.append(([nvcc, *NVCC_FLAGS, *dflags, *extra, "-c", os.path.join(CSRC, f), "-o", o],
                     verbose or ptxas_verbose))
        objs.append(o)
    # the translation units are independent: compiled side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for fut in [ex.submit(_run, cmd, v) for cmd, v in jobs]:
            fut.result()
    tmp = lib + ".tmp"
    _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs, "-lm"], verbose)
    os.replace(tmp, lib)
    return lib


CHECKED_LIB = os.path.join(OUT_DIR, "libdgrain_checked.so")


def build_checked(verbose: bool = False, force: bool = False) -> str:
    """The checked build: the same sources with -DDGR_CHECKED (every index a kernel gathers
    from the connectivity is tested; see dgr_kernels.cuh), loaded by the package when
    DGRAIN_LIBRARY=checked."""
    return build(verbose=verbose, force=force, out=CHECKED_LIB, defines=["DGR_CHECKED"],
                 build_dir=os.path.join(HERE, "_build_checked"))


if __name__ == "__main__":
    if "--checked" in sys.argv:
        print(build_checked(verbose=True, force="-f" in sys.argv))
    else:
        path = build(verbose=True, ptxas_verbose="-v" in sys.argv, force="-f" in sys.argv)
        print(path)
