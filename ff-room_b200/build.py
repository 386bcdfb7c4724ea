"""Builds the B200 extension in-tree.

  libffroom_cuda.so       sm_100a kernels + the C ABI (include/ffroom.h)
  _ffroom_core<ext>.so    the drop-in pybind11 module (host C++17 only),
                          linked to libffroom_cuda.so through $ORIGIN

Run ``python ff-room_b200/build.py`` (or __graft_entry__.build()).  nvcc
cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_SOURCES = ["room.cu", "projection.cu", "mgpcg.cu", "lbm.cu", "noalloc.cu", "server.cu"]
HEADERS = ["common.cuh", "projection.cuh", "mgpcg.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB = os.path.join(PKG, "libffroom_cuda.so")
EXT = os.path.join(PKG, "_ffroom_core" + sysconfig.get_config_var("EXT_SUFFIX"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.check_call(cmd)


OBJ_DIR = os.path.join(PKG, "_build")


def build_cuda(force: bool = False) -> str:
    """Each .cu compiles to its own object (in parallel), then one link."""
    from concurrent.futures import ThreadPoolExecutor
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    common = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INC, "ffroom.h"), __file__]
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs = [os.path.join(OBJ_DIR, os.path.basename(s)[:-3] + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, [s] + common)]

    def compile_one(so):
        src, obj = so
        _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
              "-Xptxas", "-v" if os.environ.get("FFR_PTXAS_VERBOSE") else "-O3",
              "-I", INC, "-I", CSRC, src, "-o", obj])

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        list(ex.map(compile_one, todo))
    if force or todo or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", *objs, "-o", LIB])
    return LIB


def build_module(force: bool = False) -> str:
    import pybind11
    src = os.path.join(CSRC, "module.cpp")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    if force or _stale(EXT, [src, os.path.join(INC, "ffroom.h"), LIB, __file__]):
        inc_py = sysconfig.get_paths()["include"]
        _run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
              "-I", inc_py, "-I", pybind11.get_include(), "-I", INC, src,
              "-L", PKG, "-lffroom_cuda", "-Wl,-rpath,$ORIGIN", "-o", EXT])
    return EXT


def build(force: bool = False) -> None:
    build_cuda(force)
    build_module(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
