"""Build recipe for the native library and the MultiQW binary.

    python -m multistageqw_b200.build        # or __graft_entry__.build()

Produces, in-tree (so the files travel with the source tree):
  multistageqw_b200/_lib/libmqw.so   the C ABI of include/mqw.h
  multistageqw_b200/_lib/MultiQW      the drop-in command
CUDA sources are compiled for sm_100a only
(nvcc -gencode arch=compute_100a,code=sm_100a); host C++ with
g++ -O2 -march=x86-64-v3 -ffp-contract=fast.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "_lib")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = os.environ.get("CXX", "g++")

CU_SOURCES = ["mqw_diag.cu", "mqw_coeffs.cu", "mqw_propagate.cu", "mqw_noalloc.cu",
              "mqw_mlp.cu", "mqw_peaks.cu", "mqw_stage2.cu", "mqw_stage2_tc.cu"]
CPP_SOURCES = ["mqw_host.cpp", "mqw_schedule.cpp"]
HEADERS = ["mqw_internal.h", "mqw_cheb.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-march=x86-64-v3", "-ffp-contract=fast",
             "-I" + os.path.join(CUDA_HOME, "include"), "-Wall", "-Wno-unused-function"]


def _deps_mtime() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "mqw.h")]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _stale(out: str, src: str, deps: float) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return t < os.path.getmtime(src) or t < deps


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile everything that is out of date; returns the library path."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    deps = _deps_mtime()
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append([NVCC, *NVCC_FLAGS, "-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append([CXX, *CXX_FLAGS, "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    so = os.path.join(LIB, "libmqw.so")
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(so) or os.path.getmtime(so) < newest:
        tmp = so + ".tmp"
        _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs],
             verbose)
        os.replace(tmp, so)
    cli_src = os.path.join(CSRC, "multiqw_cli.cpp")
    cli = os.path.join(LIB, "MultiQW")
    if force or not os.path.exists(cli) or os.path.getmtime(cli) < max(
            os.path.getmtime(so), os.path.getmtime(cli_src)):
        _run([CXX, "-O2", "-std=c++17", "-o", cli, cli_src, "-L" + LIB, "-lmqw",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return so


def clean() -> None:
    for d in (BUILD, LIB):
        if os.path.isdir(d):
            shutil.rmtree(d)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(os.path.join(LIB, "libmqw.so"))
