"""Build recipe for the engine's native libraries (in-tree, sm_100a).

Produces, next to this file:
  libmhcuda.so                           the C ABI of include/minhashcuda*.h
                                         (CUDA runtime linked statically,
                                         cuRAND from the toolkit)
  libMHCUDA<EXT_SUFFIX>                  the CPython module ``libMHCUDA``
                                         (python.cc's surface), linked to
                                         libmhcuda.so via $ORIGIN
  libmhsynth.so                          synthetic CSR generators used by the
                                         benchmark and the tests

Run ``python minhashcuda_b200/_build.py`` (by path: importing the package
needs the libraries this builds) or ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The image exports CC/CXX pointing at a compiler wrapper without OpenMP
# support files; the system compilers are used as nvcc's host compiler.
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# No fast-math: the hash must round exactly like the reference (IEEE divide,
# denormals kept, logf from CUDA's math library).  Contraction is pinned in
# the source with explicit intrinsics, so -fmad does not matter there.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
              "-I" + INCLUDE, "--expt-relaxed-constexpr"]

ENGINE_SOURCES = ["hash_kernels.cu", "param_kernels.cu", "engine.cu", "noalloc.cu", "server.cu",
                  "lsh.cu", "host_copy.cc"]
HEADERS = ["wmh_internal.h"]

EXT_SUFFIX = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
LIB_ENGINE = os.path.join(HERE, "libmhcuda.so")
LIB_PY = os.path.join(HERE, "libMHCUDA" + EXT_SUFFIX)
LIB_SYNTH = os.path.join(HERE, "libmhsynth.so")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _header_deps():
    deps = [os.path.join(CSRC, h) for h in HEADERS]
    deps += [os.path.join(INCLUDE, h) for h in os.listdir(INCLUDE) if h.endswith(".h")]
    return deps


def build(verbose: bool = False, force: bool = False) -> None:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _header_deps()
    objs = []
    for src in ENGINE_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + hdrs):
            _run([NVCC, *ARCH, *NVCC_FLAGS, "-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _stale(LIB_ENGINE, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, "-cudart", "static", *objs,
              "-o", LIB_ENGINE, "-L" + os.path.join(CUDA_HOME, "lib64"),
              "-lcurand", "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")], verbose)

    import numpy
    py_inc = sysconfig.get_paths()["include"]
    pysrc = os.path.join(CSRC, "pymodule.cc")
    if force or _stale(LIB_PY, [pysrc, LIB_ENGINE] + hdrs):
        _run([HOST_CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + INCLUDE, "-I" + py_inc,
              "-I" + numpy.get_include(), pysrc, "-o", LIB_PY, "-L" + HERE, "-lmhcuda",
              "-Wl,-rpath,$ORIGIN"], verbose)

    synth = os.path.join(CSRC, "synth.cu")
    if os.path.exists(synth) and (force or _stale(LIB_SYNTH, [synth] + hdrs)):
        o = os.path.join(OBJ, "synth.cu.o")
        _run([NVCC, *ARCH, *NVCC_FLAGS, "-c", synth, "-o", o], verbose)
        _run([NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, "-cudart", "static", o,
              "-o", LIB_SYNTH], verbose)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
