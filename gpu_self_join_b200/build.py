"""Builds the native library and CLI in-tree for sm_100a.

    python -m gpu_self_join_b200.build            # libgpuselfjoin.so + main
    python -m gpu_self_join_b200.build --clean

Outputs (next to this file): ``libgpuselfjoin.so`` (the C ABI of
include/gpuselfjoin.h) and ``main`` (the ``./main <file> <eps> <dim> 3`` CLI).
Object files go to ``_build/``.  The params.h switch names of the reference
(GPUNUMDIM, NUMINDEXEDDIM, REORDER, SHORTCIRCUIT, ILP, STAMP, QUERYREORDER and
GSJ_DTYPE_DOUBLE for DTYPE=double) may be given as ``-D`` options through the
GSJ_DEFINES environment variable; they only set the defaults of
gsj_default_config().
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shlex
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpuselfjoin.so")
CLI = os.path.join(HERE, "main")

CU_SOURCES = ["gsj_index.cu", "gsj_join.cu", "gsj_join_tpq.cu", "gsj_join_tile.cu", "gsj_join_screen.cu", "gsj_join_sort.cu", "gsj_bruteforce.cu", "gsj_scan.cu", "gsj_sort.cu", "gsj_place.cu", "gsj_model.cu", "gsj_api.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-Xptxas", "-v", "-ccbin", "g++"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else "nvcc"


def _defines() -> list[str]:
    return shlex.split(os.environ.get("GSJ_DEFINES", ""))


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "gpuselfjoin.h"))
    return hs


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    srcp = os.path.join(CSRC, src)
    if _newer(obj, [srcp] + _headers()) and not _defines():
        return obj
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *_defines(), "-c", srcp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(BUILD, src + ".log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed for {src}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), CU_SOURCES))
    if not _newer(LIB, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-ccbin", "g++", *objs, "-o", LIB,
               "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
        subprocess.run(cmd, check=True)
    cli_src = os.path.join(CSRC, "gsj_cli.cpp")
    if os.path.exists(cli_src) and not _newer(CLI, [cli_src, LIB]):
        cmd = ["g++", "-O2", "-std=c++17", cli_src, "-o", CLI, "-I", os.path.join(os.path.dirname(HERE), "include"),
               "-L", HERE, "-lgpuselfjoin", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    for p in (LIB, CLI):
        if os.path.exists(p):
            os.remove(p)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    if a.clean:
        clean()
    else:
        build(a.verbose)
