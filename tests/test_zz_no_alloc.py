"""The allocation-free entry point, mhcuda_calc_device_noalloc, through the C
ABI on a B200.

It exists for callers that must not allocate device memory (a process whose
device memory another allocator already holds, or a latency-critical loop
that cannot take the synchronisation of a cudaMalloc); its scratch is a fixed
8 MiB array in the library's device image.  These tests check that it gives
exactly what the ordinary device entry point (mhcuda_calc_device) gives, on
two calls in a row with different inputs (the shared array keeps the previous
call's contents), and that an input too large for the array is refused.

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_csr(m):
    import torch
    ip = torch.from_numpy(m.indptr.astype(np.int64).astype(np.uint32).view(np.int32)).cuda()
    cols = torch.from_numpy(m.indices.astype(np.uint32).view(np.int32)).cuda()
    w = torch.from_numpy(m.data.astype(np.float32)).cuda()
    return ip, cols, w


def _run(lib, entry, gen, m, samples):
    import torch
    ip, cols, w = _device_csr(m)
    out = torch.full((m.shape[0], samples, 2), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # the library works on its own stream
    rc = getattr(lib, entry)(gen, w.data_ptr(), cols.data_ptr(), ip.data_ptr(), m.shape[0],
                             m.nnz, out.data_ptr(), None)
    assert rc == 0, f"{entry} returned {rc}"
    if entry == "mhcuda_calc_device":
        assert lib.mhcuda_device_status(gen) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_device_entry_point_on_two_calls():
    import minhashcuda_b200 as mb
    from wmh_testlib import random_csr
    lib = mb.capi()
    rng = np.random.default_rng(31)
    dim, samples = 20000, 128
    status = ctypes.c_int(-1)
    gen = lib.mhcuda_init(dim, samples, 5, 0, 1, 0, ctypes.byref(status))
    assert gen, status.value
    try:
        first = random_csr(rng, 4000, dim, 300, long_rows=[(10, 15000)], empty_frac=0.02)
        second = random_csr(rng, 700, dim, 40)
        for m in (first, second):
            want = _run(lib, "mhcuda_calc_device", gen, m, samples)
            got = _run(lib, "mhcuda_calc_device_noalloc", gen, m, samples)
            np.testing.assert_array_equal(got, want)
    finally:
        lib.mhcuda_fini(gen)


def test_noalloc_refuses_inputs_beyond_its_scratch():
    import torch
    import minhashcuda_b200 as mb
    lib = mb.capi()
    dim, samples = 64, 65535
    gen = lib.mhcuda_init(dim, samples, 1, 1, 1, 0, None)
    assert gen
    try:
        nnz = 6 << 20  # > 5 chunks of 2^20 at 65535 samples
        rows = 64
        ip = torch.linspace(0, nnz, rows + 1, device="cuda").to(torch.int64).to(torch.int32)
        cols = torch.zeros(nnz, dtype=torch.int32, device="cuda")
        w = torch.ones(nnz, dtype=torch.float32, device="cuda")
        out = torch.empty((rows, 1, 2), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = lib.mhcuda_calc_device_noalloc(gen, w.data_ptr(), cols.data_ptr(), ip.data_ptr(),
                                            rows, nnz, out.data_ptr(), None)
        assert rc == mb.INVALID_ARGUMENTS
    finally:
        lib.mhcuda_fini(gen)
