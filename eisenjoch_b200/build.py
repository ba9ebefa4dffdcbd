"""Builds libeplace.so (sm_100a) in-tree with nvcc.

    python -m eisenjoch_b200.build [--force]

The library is a plain C-ABI shared object (include/eplace.h); no Python
extension machinery is involved.  Sources are compiled only when newer than
the library unless --force is given.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libeplace.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC,-O3,-Wall",
    "-Xptxas",
    "-v",
    "--expt-relaxed-constexpr",
]


# Host-only sources compiled by the host C++ compiler: the legaliser uses x86
# intrinsics with per-function targets, which nvcc's front end does not take.
HOST_CXX = {"host.cpp"}
CXX = os.environ.get("CXX", "g++")
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-ffp-contract=off"]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def headers():
    hs = [os.path.join(ROOT, "include", "eplace.h")]
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".h", ".cuh")):
            hs.append(os.path.join(CSRC, name))
    return hs


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in sources() + headers() + [__file__])


def build(force=False, verbose=False):
    """Compiles every .cu/.cpp under csrc/ into libeplace.so."""
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if os.path.basename(src) in HOST_CXX:
            cmd = [CXX] + CXXFLAGS + ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        elif src.endswith(".cpp"):
            cmd = [NVCC, "-x", "cu"] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on %s" % src)
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
