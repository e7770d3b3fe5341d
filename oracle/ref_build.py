"""TEST INFRASTRUCTURE: compile pieces of the reference from its own sources into oracle/_ref/.

    python oracle/ref_build.py --reference <reference tree> [--cuda] [--dropin]

The tree comes from --reference or the PLIS_REFERENCE environment variable.

* refdump       the reference's header-only input parsers (PLISCuda/include/cpp/*.hpp) driven by
                oracle/ref/refdump.cpp: g++ on the reference headers where they lie.
* pliscuda_dropin the reference's main.cpp and parsers with pliscuda_b200/compat/run_simulation_shim.cpp
                linked to libplis.so in place of driver.cu and its kernels.
* pliscuda_test the reference's CUDA step (PLISCuda/src/*.cu + main.cpp) built with nvcc for sm_100a
  pliscuda      with -DTEST (fixed per-subvolume seeds, PLISCuda/src/init.cu:9-11) and without.
                The reference makefile cannot be used as shipped (its -arch=sm_30 is gone from nvcc
                12.9 and CCCL needs C++17).  The build below keeps its -rdc=true and its release -O3 and
                changes two flags: -arch=sm_100a for sm_30 and -std=c++17 for c++11; the TEST binary
                adds -DTEST at -O3 (the makefile's test target uses -O2 -Wall).
Outputs go only to oracle/_ref/ (git-ignored; it travels with the tree to the GPU box).
oracle/_ref/reference_root.txt records the tree it was built from, for the CPU tests that read the
reference's own input files (tests/helpers.reference_root); they skip where the tree is absent.
Nothing from the reference is copied into the repository.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(" ".join(cmd) + "\n" + r.stdout + r.stderr)


def _fresh(out, sources):
    """True when `out` exists and is newer than every source (the recipe then skips it)."""
    return os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in sources)


def build_refdump(ref: str) -> str:
    os.makedirs(OUT, exist_ok=True)
    out = os.path.join(OUT, "refdump")
    inc = os.path.join(ref, "PLISCuda", "include", "cpp")
    _run(["g++", "-std=c++17", "-O1", "-I", inc, "-I/usr/local/cuda/include",
          os.path.join(HERE, "ref", "refdump.cpp"), "-o", out])
    return out


def build_cuda(ref: str, test: bool) -> str:
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(ref, "PLISCuda", "src")
    name = "pliscuda_test" if test else "pliscuda"
    out = os.path.join(OUT, name)
    obj_dir = os.path.join(OUT, "obj_" + name)
    os.makedirs(obj_dir, exist_ok=True)
    srcs = [os.path.join(src, f) for f in os.listdir(src)]
    srcs += [os.path.join(ref, "PLISCuda", "include", d, f) for d in ("cuda", "cpp")
             for f in os.listdir(os.path.join(ref, "PLISCuda", "include", d))]
    if _fresh(out, srcs):
        return out
    flags = ["-std=c++17", "-O3", "-rdc=true", "-arch=sm_100a"] + (["-DTEST"] if test else [])
    objs = []
    for f in ["driver.cu", "init.cu", "leap.cu", "log.cu", "rates.cu", "ssa.cu", "tau.cu"]:
        o = os.path.join(obj_dir, f + ".o")
        _run(["nvcc"] + flags + ["-c", os.path.join(src, f), "-o", o])
        objs.append(o)
    o = os.path.join(obj_dir, "main.o")
    _run(["nvcc"] + flags + ["-x", "cu", "-c", os.path.join(src, "main.cpp"), "-o", o])
    objs.append(o)
    _run(["nvcc", "-arch=sm_100a", "-rdc=true"] + objs + ["-o", out])
    return out


def build_dropin(ref: str) -> str:
    """The reference's own main.cpp and parsers linked with pliscuda_b200/compat/run_simulation_shim.cpp
    and libplis.so instead of driver.cu and the reference kernels: the literal drop-in."""
    os.makedirs(OUT, exist_ok=True)
    root = os.path.dirname(HERE)
    out = os.path.join(OUT, "pliscuda_dropin")
    obj_dir = os.path.join(OUT, "obj_dropin")
    os.makedirs(obj_dir, exist_ok=True)
    inc_cpp = os.path.join(ref, "PLISCuda", "include", "cpp")
    shim = os.path.join(root, "pliscuda_b200", "compat", "run_simulation_shim.cpp")
    if _fresh(out, [shim, os.path.join(ref, "PLISCuda", "src", "main.cpp"), os.path.join(root, "include", "plis.h")]
              + [os.path.join(inc_cpp, f) for f in os.listdir(inc_cpp)]):
        return out
    main_o = os.path.join(obj_dir, "main.o")
    _run(["nvcc", "-std=c++17", "-O2", "-arch=sm_100a", "-x", "cu", "-c",
          os.path.join(ref, "PLISCuda", "src", "main.cpp"), "-o", main_o])
    shim_o = os.path.join(obj_dir, "shim.o")
    _run(["g++", "-std=c++17", "-O2", "-I", inc_cpp, "-I/usr/local/cuda/include", "-I", os.path.join(root, "include"),
          "-c", os.path.join(root, "pliscuda_b200", "compat", "run_simulation_shim.cpp"), "-o", shim_o])
    libdir = os.path.join(root, "pliscuda_b200")
    _run(["nvcc", "-arch=sm_100a", main_o, shim_o, "-L" + libdir, "-lplis", "-Xlinker", "-rpath=$ORIGIN/../../pliscuda_b200",
          "-o", out])
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PLIS_REFERENCE"))
    ap.add_argument("--cuda", action="store_true", help="also build the reference CUDA binaries")
    ap.add_argument("--dropin", action="store_true", help="also build main.cpp + the run_simulation shim")
    a = ap.parse_args(argv)
    if not a.reference or not os.path.isdir(a.reference):
        print("no reference tree given (--reference or PLIS_REFERENCE); nothing to build")
        return 0
    print(build_refdump(a.reference))
    with open(os.path.join(OUT, "reference_root.txt"), "w") as f:
        f.write(os.path.abspath(a.reference) + "\n")
    if a.cuda:
        print(build_cuda(a.reference, True))
        print(build_cuda(a.reference, False))
    if a.dropin:
        print(build_dropin(a.reference))
    return 0


if __name__ == "__main__":
    sys.exit(main())
