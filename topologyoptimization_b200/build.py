"""Build libtpo.so in-tree with nvcc for sm_100a.

    python -m topologyoptimization_b200.build [--force] [--debug]

Objects go to topologyoptimization_b200/_build/, the library to
topologyoptimization_b200/libtpo.so.  exact.cu is compiled with --fmad=false because
its kernels reproduce the reference's operation order (WebAssembly/JavaScript have
no fused multiply-add); every other file lets the compiler contract a*b+c.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtpo.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", CSRC, "-I", INCLUDE]
SOURCES = {
    "api.cu": [],
    "kernels.cu": [],
    "exact.cu": ["--fmad=false"],
}


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "tpo.h"))
    return max(os.path.getmtime(f) for f in files)


def build(force=False, debug=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    newest = _deps()
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    extra = ["-DTPO_CHECK"] if debug else []
    objs = []
    for src, flags in SOURCES.items():
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *flags, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, debug=a.debug, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
