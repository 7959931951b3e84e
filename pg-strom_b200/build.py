"""
Builds libxpu_b200.so in-tree: the sm_100a kernels (xb_exec.cu) and the
host-side bytecode translator (xb_compile.cpp) behind the C ABI of
include/xpu_b200.h.  The CUDA runtime is linked statically so the library
loads on any box with the driver.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxpu_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCS = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

SOURCES = {
    "xb_exec.o": ("xb_exec.cu", "cuda"),
    "xb_compile.o": ("xb_compile.cpp", "cxx"),
}
HEADERS = ["xb_plan.h", "xb_device.cuh", "xb_ops.cuh", "xb_hash.h", "xb_compile.h"]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def _deps_mtime():
    m = max(_mtime(os.path.join(CSRC, h)) for h in HEADERS)
    for h in ("pgstrom_abi.h", "pgstrom_opcodes.h", "xpu_b200.h"):
        m = max(m, _mtime(os.path.join(ROOT, "include", h)))
    return m


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps_mtime()
    objs = []
    for obj, (src, kind) in SOURCES.items():
        o = os.path.join(BUILD, obj)
        s = os.path.join(CSRC, src)
        objs.append(o)
        if not force and _mtime(o) > max(_mtime(s), deps):
            continue
        if kind == "cuda":
            _run([NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
                  *INCS, "-c", s, "-o", o], verbose)
        else:
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", *INCS, "-c", s, "-o", o], verbose)
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
