"""CPU checks of the native boundary (no GPU needed, no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

import minhashcuda_b200 as mb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("minhashcuda.h", "minhashcuda_b200.h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(mhcuda_\w+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    syms = declared_symbols()
    assert "mhcuda_calc" in syms and "mhcuda_init" in syms
    lib = ctypes.CDLL(mb.LIB_PATH)
    for s in syms:
        assert hasattr(lib, s), s
    # and the Python binding covers them all
    assert set(syms) <= set(mb.SIGNATURES), set(syms) - set(mb.SIGNATURES)


def test_reference_symbols_present():
    """The six entry points of the reference header (minhashcuda.h:74-124)."""
    lib = mb.capi()
    for s in ("mhcuda_init", "mhcuda_get_parameters", "mhcuda_retrieve_random_vars",
              "mhcuda_assign_random_vars", "mhcuda_calc", "mhcuda_fini"):
        assert hasattr(lib, s)


def test_struct_and_enum_layout():
    assert ctypes.sizeof(mb.GeneratorParameters) == 12
    assert mb.GeneratorParameters.samples.offset == 4
    assert mb.GeneratorParameters.verbosity.offset == 8
    assert (mb.SUCCESS, mb.INVALID_ARGUMENTS, mb.NO_SUCH_DEVICE, mb.MEMORY_ALLOCATION_FAILURE,
            mb.RUNTIME_ERROR, mb.MEMORY_COPY_ERROR) == (0, 1, 2, 3, 4, 5)


def test_host_side_validation_without_gpu():
    lib = mb.capi()
    status = ctypes.c_int(-1)
    assert not lib.mhcuda_init(0, 128, 1, 0, 0, 0, ctypes.byref(status))
    assert status.value == mb.INVALID_ARGUMENTS
    assert not lib.mhcuda_init(10, 0, 1, 0, 0, 0, None)
    p = lib.mhcuda_get_parameters(None)
    assert (p.dim, p.samples, p.verbosity) == (0, 0, 0)
    one = np.ones(4, np.uint32)
    assert lib.mhcuda_calc(None, one.ctypes.data, one.ctypes.data, one.ctypes.data, 1,
                           one.ctypes.data) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_retrieve_random_vars(None, None, None, None) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_assign_random_vars(None, None, None, None) == mb.INVALID_ARGUMENTS
    # Added entry points refuse null arguments before touching a device.
    assert lib.mhcuda_calc_batch_device(None, 1, None, None, None, None, None,
                                        None) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_host_register(0, None, 16) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_host_register(0, one.ctypes.data, 0) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_host_unregister(0, None) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_calc_batch(None, 0, None, None, None, None, None) == mb.INVALID_ARGUMENTS
    assert lib.mhcuda_calc_typed(None, one.ctypes.data, mb.FLOAT64, one.ctypes.data, mb.INT64,
                                 one.ctypes.data, mb.INT64, 1, one.ctypes.data) == \
        mb.INVALID_ARGUMENTS
    assert lib.mhcuda_fini(None) == mb.SUCCESS


def test_typed_calc_rejects_bad_types_and_offsets_before_device_work():
    """Element types and 64-bit offsets are checked on the host before the
    generator is touched, so a dummy non-null handle is never dereferenced."""
    lib = mb.capi()
    w = np.ones(4, np.float64)
    c = np.zeros(4, np.int64)
    out = np.zeros(64, np.uint32)
    dummy = ctypes.c_void_p(1)

    def calc(wt, ct, rows, rt):
        return lib.mhcuda_calc_typed(dummy, w.ctypes.data, wt, c.ctypes.data, ct,
                                     rows.ctypes.data, rt, len(rows) - 1, out.ctypes.data)

    ok_rows = np.array([0, 2, 4], np.int64)
    assert calc(mb.UINT32, mb.INT64, ok_rows, mb.INT64) == mb.INVALID_ARGUMENTS  # int weights
    assert calc(mb.FLOAT64, mb.FLOAT32, ok_rows, mb.INT64) == mb.INVALID_ARGUMENTS  # float cols
    assert calc(mb.FLOAT64, mb.INT64, ok_rows, 17) == mb.INVALID_ARGUMENTS
    assert calc(mb.FLOAT64, mb.INT64, np.array([0, 3, 2], np.int64),
                mb.INT64) == mb.INVALID_ARGUMENTS  # decreasing
    assert calc(mb.FLOAT64, mb.INT64, np.array([-1, 2, 4], np.int64),
                mb.INT64) == mb.INVALID_ARGUMENTS  # negative
    assert calc(mb.FLOAT64, mb.INT64, np.array([0, 2, 1 << 32], np.int64),
                mb.INT64) == mb.INVALID_ARGUMENTS  # spans 2^32
    assert calc(mb.FLOAT64, mb.INT64, np.array([0, 2, 1 << 32], np.uint64),
                mb.UINT64) == mb.INVALID_ARGUMENTS


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_device_maps_to_no_such_device():
    lib = mb.capi()
    status = ctypes.c_int(-1)
    assert not lib.mhcuda_init(100, 128, 1, 0, 0, 0, ctypes.byref(status))
    assert status.value == mb.NO_SUCH_DEVICE
    with pytest.raises(ValueError, match="No such CUDA device exists"):
        mb.libMHCUDA.minhash_cuda_init(100, 128)


def test_python_surface():
    L = mb.libMHCUDA
    for name in ("minhash_cuda_init", "minhash_cuda_retrieve_vars", "minhash_cuda_assign_vars",
                 "minhash_cuda_assign_random_vars", "minhash_cuda_calc", "minhash_cuda_calc_batch",
                 "minhash_cuda_fini"):
        assert callable(getattr(L, name)), name
    import libMHCUDA
    assert libMHCUDA is L


def test_python_argument_checks_before_device_work():
    """Type and slice checks happen before the generator is touched
    (python.cc:305-347), so a dummy non-null handle is never dereferenced."""
    L = mb.libMHCUDA
    with pytest.raises(ValueError, match="null"):
        L.minhash_cuda_calc(0, sp.csr_matrix(np.ones((2, 2), np.float32)))
    with pytest.raises(TypeError):
        L.minhash_cuda_calc(1, np.ones((2, 2), np.float32))
    with pytest.raises(TypeError):
        L.minhash_cuda_calc(1, sp.coo_matrix(np.ones((2, 2), np.float32)))
    m = sp.csr_matrix(np.ones((3, 2), np.float32))
    with pytest.raises(ValueError, match="row_start"):
        L.minhash_cuda_calc(1, m, row_start=3)
    with pytest.raises(ValueError, match="row_finish"):
        L.minhash_cuda_calc(1, m, row_start=2, row_finish=1)
    with pytest.raises(TypeError):
        L.minhash_cuda_init("a", 128)
    L.minhash_cuda_fini(0)
