"""Build recipe of the tinyMD B200 library and its md driver.

Compiles every CUDA source for sm_100a (nvcc -gencode
arch=compute_100a,code=sm_100a) into molecular-dynamics_b200/lib/:

  libtinymd_b200.so   the md_* C ABI (include/tinymd_b200.h)
  md                  the tinyMD command-line driver linked against it

Objects are rebuilt only when a source or header is newer.  Run
``python molecular-dynamics_b200/build.py`` or call ``build()``.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INC = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(LIB, "obj")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INC, "-I" + CSRC, "-I" + HOST]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I" + INC, "-I" + HOST, "-I" + CSRC]

CU_SOURCES = ["api.cu", "k_neigh.cu", "k_step.cu", "k_halo.cu", "adjoint.cu", "noalloc.cu"]
CPP_LIB_SOURCES = [os.path.join(CSRC, "setup_api.cpp"), os.path.join(HOST, "setups.cpp"), os.path.join(CSRC, "comm.cpp")]
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "include")
HEADERS = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + \
          [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")] + \
          [os.path.join(INC, "tinymd_b200.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        if _stale(obj, [path] + HEADERS):
            out = _run([NVCC] + NVFLAGS + ["-c", "-o", obj, path])
            if verbose and out:
                print(out)
        objs.append(obj)
    for path in CPP_LIB_SOURCES:
        obj = os.path.join(OBJ, os.path.basename(path) + ".o")
        if _stale(obj, [path] + HEADERS):
            _run([CXX] + CXXFLAGS + ["-I" + CUDA_INC, "-c", "-o", obj, path])
        objs.append(obj)
    so = os.path.join(LIB, "libtinymd_b200.so")
    if _stale(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xlinker", "-Bsymbolic", "-o", so] + objs + ["-ldl"])
    md = os.path.join(LIB, "md")
    main = os.path.join(HOST, "main.cpp")
    if os.path.exists(main) and _stale(md, [so, main] + HEADERS):
        _run([CXX] + CXXFLAGS + ["-o", md, main, "-L" + LIB, "-ltinymd_b200", "-Wl,-rpath,$ORIGIN"])
    return so


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(os.path.join(LIB, "libtinymd_b200.so"))
