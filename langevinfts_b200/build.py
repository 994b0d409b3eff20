"""Build the in-tree native libraries for sm_100a.

  liblfts_b200.so                 CUDA engine behind the C ABI (include/lfts_b200.h)
  langevinfts.<EXT_SUFFIX>        pybind11 module `langevinfts` (C++ host code:
                                  molecules, propagator analyzer, scheduler,
                                  computation classes) linked to the engine

Usage: python -m langevinfts_b200.build  (or __graft_entry__.build()).
Rebuilds a target only when one of its sources is newer.
"""
import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["lfts_engine.cu", "lfts_langevin.cu"]
HOST_SOURCES = ["lfts_host.cpp", "lfts_computation.cpp", "lfts_langevin_host.cpp", "lfts_scft_host.cpp", "lfts_pybind.cpp"]
HEADERS = ["lfts_fft.cuh", "lfts_step_kernels.cuh", "lfts_step_fast.cuh", "lfts_step_r8.cuh", "lfts_step_r12.cuh", "lfts_realspace.cuh", "lfts_unet.cuh", "lfts_bulk.cuh", "lfts_host.h", "lfts_computation.h", "lfts_langevin.h", "lfts_scft.h"]

ENGINE = os.path.join(HERE, "liblfts_b200.so")
MODULE = os.path.join(HERE, "langevinfts" + sysconfig.get_config_var("EXT_SUFFIX"))


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(s) and os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_engine(force=False):
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HEADERS] + [os.path.join(INCLUDE, "lfts_b200.h")]
    if not force and not _newer(ENGINE, deps):
        return ENGINE
    objs = []
    cmds = []
    for src in CUDA_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        cmds.append([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
                     "-c", os.path.join(CSRC, src), "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, len(cmds))) as ex:
        list(ex.map(_run, cmds))
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", ENGINE, *objs])
    return ENGINE


def build_module(force=False):
    srcs = [os.path.join(CSRC, f) for f in HOST_SOURCES]
    if not all(os.path.exists(s) for s in srcs):
        return None
    deps = srcs + [os.path.join(CSRC, f) for f in HEADERS] + [os.path.join(INCLUDE, "lfts_b200.h"), ENGINE]
    if not force and not _newer(MODULE, deps):
        return MODULE
    import pybind11
    py_inc = sysconfig.get_paths()["include"]
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
           "-I", py_inc, "-I", pybind11.get_include(), *srcs, "-o", MODULE,
           "-L", HERE, "-l:liblfts_b200.so", "-Wl,-rpath,$ORIGIN"]
    _run(cmd)
    return MODULE


def build(force=False):
    build_engine(force)
    build_module(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
