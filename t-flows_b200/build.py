"""Build the B200 Krylov library and the CPU oracle in-tree.

    python t-flows_b200/build.py            # both
    python t-flows_b200/build.py --lib      # libtfkrylov.so only
    python t-flows_b200/build.py --oracle   # oracle/libtforacle.so only

libtfkrylov.so is compiled for sm_100a only, with the CUDA runtime linked
statically, so it depends on nothing but the driver (no torch).
"""
import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libtfkrylov.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "libtforacle.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(ROOT, "include", "tf_krylov.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force=False, verbose=False):
    if not force and not _stale(LIB, _deps()):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src in _sources():
        obj = os.path.join(LIBDIR, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


def build_oracle(force=False):
    src = os.path.join(ORACLE_DIR, "tf_oracle.cpp")
    if not force and not _stale(ORACLE_LIB, [src]):
        return ORACLE_LIB
    subprocess.run(["make", "-C", ORACLE_DIR, "-s"], check=True)
    return ORACLE_LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", action="store_true")
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    both = not (a.lib or a.oracle)
    if a.lib or both:
        print(build_lib(force=a.force, verbose=a.verbose))
    if a.oracle or both:
        print(build_oracle(force=a.force))


if __name__ == "__main__":
    sys.exit(main())
