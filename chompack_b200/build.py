"""Build the in-tree native library `chompack_b200/libchompack_b200.so`.

    python chompack_b200/build.py

Host C++ sources are compiled with g++, CUDA sources with nvcc for sm_100a
only (`-gencode arch=compute_100a,code=sm_100a`), and everything is linked
into one shared library next to this file, so that it travels with the
working tree.  Rebuilds only when a source or header is newer than the
library.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libchompack_b200.so")
BUILD = os.path.join(ROOT, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-function", "-I" + INCLUDE,
            "-I" + os.path.join(CUDA_HOME, "include")]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "--expt-relaxed-constexpr",
           "-Xptxas", "-O3"] + ARCH


def _sources():
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                 glob.glob(os.path.join(INCLUDE, "*.h")))
    return cpp, cu, hdr


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: %s" % " ".join(cmd))
    return r.stdout


def build(force=False, verbose=False):
    cpp, cu, hdr = _sources()
    srcs = cpp + cu
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= max(os.path.getmtime(f) for f in srcs + hdr + [__file__])):
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    newest_hdr = max([os.path.getmtime(f) for f in hdr + [__file__]])

    def stale(src, obj):
        # an object is rebuilt when its source, any header or this script is newer
        return force or verbose or not os.path.exists(obj) or \
            os.path.getmtime(obj) < max(os.path.getmtime(src), newest_hdr)
    objs = []
    for f in cpp:
        o = os.path.join(BUILD, os.path.basename(f) + ".o")
        if stale(f, o):
            _run(["g++"] + CXXFLAGS + ["-c", f, "-o", o])
        objs.append(o)
    for f in cu:
        o = os.path.join(BUILD, os.path.basename(f) + ".o")
        if stale(f, o):
            out = _run([NVCC] + NVFLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", f, "-o", o])
            if verbose:
                sys.stdout.write(out)
        objs.append(o)
    tmp = OUT + ".tmp"
    _run([NVCC, "-shared"] + ARCH + ["-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
