"""B200-native weighted MinHash (Ioffe), a drop-in for src-d/minhashcuda.

Two ways in, both over the same native library:

* ``minhashcuda_b200.libMHCUDA`` -- the CPython module with the reference's
  Python surface (``minhash_cuda_init``, ``minhash_cuda_calc``, ...).  After
  ``import minhashcuda_b200`` it is also importable as plain ``libMHCUDA``.
* ``minhashcuda_b200.capi()`` -- a ctypes binding of the C ABI declared in
  ``include/minhashcuda.h`` and ``include/minhashcuda_b200.h``.

There is no fallback: if the native libraries are missing the import fails.
Build them with ``python minhashcuda_b200/_build.py``.
"""
from __future__ import annotations

import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmhcuda.so")
SYNTH_PATH = os.path.join(HERE, "libmhsynth.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"minhashcuda_b200: native library {LIB_PATH} is missing; "
        "build it with `python minhashcuda_b200/_build.py`")

from . import libMHCUDA  # noqa: E402  (the CPython extension next to this file)

sys.modules.setdefault("libMHCUDA", libMHCUDA)

# MHCUDAElementType (include/minhashcuda_b200.h)
FLOAT32, FLOAT64, UINT32, INT32, INT64, UINT64 = range(6)

# MHCUDAResult (include/minhashcuda.h)
SUCCESS = 0
INVALID_ARGUMENTS = 1
NO_SUCH_DEVICE = 2
MEMORY_ALLOCATION_FAILURE = 3
RUNTIME_ERROR = 4
MEMORY_COPY_ERROR = 5
RESULT_NAMES = {
    0: "mhcudaSuccess", 1: "mhcudaInvalidArguments", 2: "mhcudaNoSuchDevice",
    3: "mhcudaMemoryAllocationFailure", 4: "mhcudaRuntimeError", 5: "mhcudaMemoryCopyError",
}


class GeneratorParameters(ctypes.Structure):
    """MinhashCudaGeneratorParameters (minhashcuda.h)."""
    _fields_ = [("dim", ctypes.c_uint32), ("samples", ctypes.c_uint16),
                ("verbosity", ctypes.c_int)]


# Every extern "C" entry point of include/*.h: name -> (restype, argtypes).
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_RES = ctypes.c_int
SIGNATURES = {
    "mhcuda_init": (_P, [_U32, ctypes.c_uint16, _U32, ctypes.c_int, _U32, ctypes.c_int,
                         ctypes.POINTER(ctypes.c_int)]),
    "mhcuda_get_parameters": (GeneratorParameters, [_P]),
    "mhcuda_retrieve_random_vars": (_RES, [_P, _P, _P, _P]),
    "mhcuda_assign_random_vars": (_RES, [_P, _P, _P, _P]),
    "mhcuda_calc": (_RES, [_P, _P, _P, _P, _U32, _P]),
    "mhcuda_fini": (_RES, [_P]),
    "mhcuda_calc_device": (_RES, [_P, _P, _P, _P, _U32, _U32, _P, _P]),
    "mhcuda_device_status": (_RES, [_P]),
    "mhcuda_autotune": (_RES, [_P, _P, _P, _P, _U32, _U32, _P, _P,
                               ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_double)]),
    "mhcuda_calc_device_noalloc": (_RES, [_P, _P, _P, _P, _U32, _U32, _P, _P]),
    "mhcuda_calc_typed": (_RES, [_P, _P, ctypes.c_int, _P, ctypes.c_int, _P, ctypes.c_int, _U32,
                                 _P]),
    "mhcuda_calc_batch": (_RES, [_P, _U32, _P, _P, _P, _P, _P]),
    "mhcuda_calc_batch_device": (_RES, [_P, _U32, _P, _P, _P, _P, _P, _P]),
    "mhcuda_debug_device_logf": (_RES, [_U32, _P, _P, ctypes.c_uint64]),
    "mhcuda_host_register": (_RES, [_U32, _P, ctypes.c_uint64]),
    "mhcuda_host_unregister": (_RES, [_U32, _P]),
    "mhcuda_lsh_bands": (_RES, [_P, _P, _U32, _U32, _P, _P]),
    "mhcuda_jaccard": (_RES, [_P, _P, _U32, _P, ctypes.c_uint64, _P, _P]),
    "mhcuda_server_start": (_P, [_U32, ctypes.c_uint64, _U32, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int)]),
    "mhcuda_server_submit": (_RES, [_P, _P, _P, _P, _P, _U32, _P,
                                    ctypes.POINTER(ctypes.c_uint64)]),
    "mhcuda_server_poll": (_RES, [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)]),
    "mhcuda_server_wait": (_RES, [_P, ctypes.c_uint64, ctypes.c_double,
                                  ctypes.POINTER(ctypes.c_double)]),
    "mhcuda_server_cancel": (_RES, [_P, ctypes.c_uint64]),
    "mhcuda_server_stats": (_RES, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "mhcuda_server_stop": (_RES, [_P]),
    "mhcuda_profile": (_RES, [_P, ctypes.c_int]),
    "mhcuda_profile_read": (_RES, [_P, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_uint64)]),
}

_capi = None


def capi() -> ctypes.CDLL:
    """The C ABI (libmhcuda.so) with argument and result types set."""
    global _capi
    if _capi is None:
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _capi = lib
    return _capi


class MHCUDAError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed: {RESULT_NAMES.get(code, code)}")
        self.code = code


def check(fn: str, code: int) -> None:
    if code != SUCCESS:
        raise MHCUDAError(fn, code)


__all__ = ["libMHCUDA", "capi", "check", "MHCUDAError", "GeneratorParameters", "SIGNATURES",
           "LIB_PATH", "SYNTH_PATH"]
