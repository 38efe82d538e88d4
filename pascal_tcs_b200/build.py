"""Build libtcs.so (the CUDA library behind include/tcs.h) in-tree for sm_100a.

Usage: python -m pascal_tcs_b200.build [--force] [--verbose]
nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.9.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtcs.so")
# the bounds-check build (-DTCS_BOUNDS_CHECK): every index the kernels form is
# checked; used by the tests, never by the benchmark
LIB_BC = os.path.join(HERE, "libtcs_bc.so")
SOURCES = ["tcs_thermal.cu", "tcs_momentum.cu", "tcs_pressure.cu", "tcs_post.cu",
           "tcs_tdma.cu", "tcs_capi.cu", "tcs_peak.cu"]
HEADERS = ["tcs_device.cuh", "tcs_fields.cuh", "tcs_kernels.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_compiler() -> list[str]:
    # The image's default CC wrapper lacks some host headers; prefer the system g++.
    for c in ("/usr/bin/g++",):
        if os.path.exists(c):
            return ["-ccbin", c]
    return []


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None, bounds_check: bool = False) -> str:
    """Compile libtcs.so (or, with bounds_check, libtcs_bc.so) and return its path."""
    if bounds_check:
        return _build(os.path.join(BUILD, "bc"), LIB_BC, force, verbose, ["-DTCS_BOUNDS_CHECK"] + (extra or []))
    return _build(BUILD, LIB, force, verbose, extra)


def _build(BUILD: str, LIB: str, force: bool, verbose: bool, extra: list[str] | None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "tcs.h")]
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs + [__file__]):
            cmd = [nvcc()] + _host_compiler() + ARCH + FLAGS + (extra or []) + ["-c", s, "-o", o]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(6, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed: {' '.join(cmd)}")
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc()] + _host_compiler() + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--bounds-check", action="store_true", help="build libtcs_bc.so with index checks")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, bounds_check=a.bounds_check))
