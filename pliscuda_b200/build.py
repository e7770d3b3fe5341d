"""Build libplis.so (the sm_100a CUDA step + C ABI) in-tree.

    python pliscuda_b200/build.py [--force] [-v]

Objects go to pliscuda_b200/_build/, the shared library to pliscuda_b200/libplis.so, the
`pliscuda <configuration file>` command to pliscuda_b200/pliscuda.  Every CUDA
translation unit is compiled for sm_100a only, with -fmad=false so device floating point matches
the host oracle bit for bit (explicit fma() calls are kept where the code wants them).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libplis.so")
CLI = os.path.join(HERE, "pliscuda")
ROOT = os.path.dirname(HERE)

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-fmad=false", "-lineinfo", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
              "-I" + os.path.join(ROOT, "include")] + ARCH
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-Wno-unused-parameter",
             "-I" + os.path.join(CUDA_HOME, "include"), "-I" + os.path.join(ROOT, "include")]

SOURCES = ["inst_f64.cu", "inst_f32.cu", "batch_f64.cu", "batch_f32.cu", "engine.cu", "batch.cu", "noalloc.cu",
           "learned.cu",
           "capi.cpp", "loader.cpp", "simulate.cpp", "plis_model.cpp"]
HEADERS = ["engine_kernels.cuh", "batch_kernels.cuh", "batch.h", "engine.cuh", "engine.h", "learned.h",
           "tc_mlp.cuh", "learned_dev.cuh", "plis_model.h", "plis_stream.h"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src: str, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(OUT_DIR, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "plis.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= _newest(deps):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
    else:
        cmd = [os.environ.get("CXX", "g++")] + CXX_FLAGS + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src} failed:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA/C++ source of the step and link libplis.so.  Returns the library path."""
    os.makedirs(OUT_DIR, exist_ok=True)
    if force:
        for f in os.listdir(OUT_DIR):
            if f.endswith(".o"):
                os.remove(os.path.join(OUT_DIR, f))
    with cf.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(objs) and not force:
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-cudart", "static", "-lpthread", "-ldl", "-lrt"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"linking libplis.so failed:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_cli(verbose: bool = False) -> str:
    """The `pliscuda <configuration file>` command (csrc/cli.cpp) linked to libplis.so beside it."""
    src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(CLI) and os.path.getmtime(CLI) >= _newest([src, LIB, os.path.join(ROOT, "include", "plis.h")]):
        return CLI
    cmd = [os.environ.get("CXX", "g++")] + [f for f in CXX_FLAGS if f != "-fPIC"] + [
        src, "-o", CLI + ".tmp", "-L" + HERE, "-lplis", "-Wl,-rpath,$ORIGIN",
        "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building pliscuda failed:\n{r.stdout}\n{r.stderr}")
    os.replace(CLI + ".tmp", CLI)
    return CLI


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    print(build_cli(verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
