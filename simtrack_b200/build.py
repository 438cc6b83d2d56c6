"""Builds the native library simtrack_b200/_lib/libsimtrack_b200.so with nvcc.

All CUDA code targets sm_100a only.  Device code is compiled with
-fmad=false: the tracking maps must round every FP64 add and multiply
separately, exactly as the reference's x86-64 build does (no fused
multiply-add), for the per-element parity the tests enforce.  Kernels that
intentionally use fused multiply-adds call fma() explicitly.  The one
exception is stb_track_fast.cu, the same tracking kernel built with
-fmad=true (the "fast" contraction policy, selected per table).

Usage: python -m simtrack_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libsimtrack_b200.so"

CUDA_SOURCES = ["stb_track.cu", "stb_track_fast.cu", "stb_scan.cu", "stb_track_static.cu", "stb_tune.cu", "stb_spin.cu", "stb_radial.cu", "stb_diag.cu", "stb_mlp.cu", "stb_mlp_ops.cu", "stb_ssbb.cu", "stb_pic.cu"]
CXX_SOURCES = ["stb_elements.cpp", "stb_srloss.cpp", "stb_flatten.cpp", "stb_capi.cpp", "stb_scan_host.cpp", "stb_mlp_host.cpp",
               "stb_tune_host.cpp", "stb_readers.cpp", "stb_da.cpp",
               "stb_orbit.cpp", "stb_tbt.cpp"]
HEADERS = ["stb_table.hpp", "stb_physics.cuh", "stb_crmath.cuh", "stb_sincos_table.cuh", "stb_rng.cuh", "stb_photon_spectrum.cuh", "stb_kernels.hpp", "stb_status.hpp", "stb_flatten.hpp",
           "stb_track_impl.cuh", "stb_track_launch.cuh", "stb_scan.hpp", "stb_runtime.hpp", "stb_mlp.hpp", "stb_tune.hpp"]

# Units compiled with FMA contraction: the fast tracking kernel only.
FMA_SOURCES = {"stb_track_fast.cu"}

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", str(ROOT / "include"), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    srcs = [CSRC / s for s in CUDA_SOURCES + CXX_SOURCES]
    deps = srcs + [CSRC / h for h in HEADERS] + [ROOT / "include" / "simtrack_b200.h",
                                               ROOT / "include" / "simtrack_b200.hpp", Path(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    common_deps = deps[len(srcs):]
    jobs = []
    for s in srcs:
        o = objdir / (s.name + ".o")
        fmad = "-fmad=true" if s.name in FMA_SOURCES else "-fmad=false"
        cmd = [nvcc(), *ARCH, *COMMON, fmad, "-x", "cu" if s.suffix == ".cu" else "c++",
               "-c", str(s), "-o", str(o)]
        if force or _stale(o, [s] + common_deps):
            jobs.append(cmd)
    objs = [str(objdir / (s.name + ".o")) for s in srcs]

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(run, c) for c in jobs]:
            f.result()
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
