"""Build the in-tree shared library ``libesp_b200.so`` for sm_100a.

Compiles every source in ``csrc/`` with nvcc (``-gencode
arch=compute_100a,code=sm_100a``) into one shared library next to this
file. Incremental: objects are rebuilt only when a source or header is newer.
Usage: ``python -m esp_hoomd_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libesp_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + INC]


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INC, "*.h"))
    return max(os.path.getmtime(h) for h in hs)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr = _newest_header()
    objs = []
    changed = force or not os.path.exists(LIB)
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            changed = True
    if changed:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


PYEXT = os.path.join(HERE, "pyext")


def build_pyext(force: bool = False) -> str:
    """The `_esp` pybind11 module (pyext/esp_module.cpp, host code over the C
    ABI), linked against libesp_b200.so next to it."""
    import sysconfig

    import pybind11
    out = os.path.join(HERE, "_esp" + sysconfig.get_config_var("EXT_SUFFIX"))
    srcs = [os.path.join(PYEXT, f) for f in os.listdir(PYEXT)] + [LIB, os.path.join(CSRC, "esp_tables.h"),
                                                                    os.path.join(INC, "esp_b200.h")]
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(f) for f in srcs):
        return out
    cuda = os.path.dirname(os.path.dirname(NVCC))
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"], "-I" + INC, "-I" + CSRC,
           "-I" + PYEXT, "-I" + os.path.join(cuda, "include"), os.path.join(PYEXT, "esp_module.cpp"), "-o", out,
           "-L" + HERE, "-lesp_b200", "-L" + os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    build_pyext(force="--force" in sys.argv)
    print(LIB)
