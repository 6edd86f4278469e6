"""The allocation-free entry point, mhcuda_calc_device_noalloc, through the C
ABI on a B200.

It exists for callers that must not allocate device memory: a process whose
device memory another allocator (a framework's caching allocator, say)
already holds, where a cudaMalloc would fail, or a latency-critical loop that
cannot take the device-wide synchronisation a cudaMalloc or cudaFree may
cause.  Its scratch is a fixed 8 MiB array in the library's device image.
These tests check that:
 - it allocates no device memory on a generator that has never run a hash
   (the ordinary entry point would grow the generator's workspace there);
 - it gives the CPU oracle's hashes and exactly what the ordinary device entry
   point (mhcuda_calc_device) gives, on two calls in a row with different
   inputs (the shared array keeps the previous call's contents);
 - an input too large for the array is refused before anything runs.

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from wmh_testlib import device_logf, gamma_params, random_csr

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
    return out.cpu().numpy().view(np.uint32)


def _gen(lib, dim, samples, params):
    gen = lib.mhcuda_init(dim, samples, 1, 1, 1, 0, None)
    assert gen
    arrs = [np.ascontiguousarray(p, np.float32) for p in params]
    assert lib.mhcuda_assign_random_vars(gen, *[a.ctypes.data for a in arrs]) == 0
    return gen


def test_noalloc_matches_oracle_and_device_entry_point_on_two_calls():
    import torch
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(31)
    dim, samples = 20000, 128
    params = gamma_params(rng, dim, samples)
    co = O.COracle(*params)
    # ~1.2M nnz: the ordinary entry point's workspace for this input is tens
    # of MiB of partial minima, far above the driver's allocation granularity.
    first = random_csr(rng, 4000, dim, 300, long_rows=[(10, 15000)], empty_frac=0.02)
    second = random_csr(rng, 700, dim, 40)

    # Load every module the call uses (the library's static array is placed
    # on the device when its module loads) before memory is measured.
    warm = _gen(lib, dim, samples, params)
    try:
        _run(lib, "mhcuda_calc_device_noalloc", warm, second, samples)
    finally:
        lib.mhcuda_fini(warm)

    gen = _gen(lib, dim, samples, params)
    try:
        ip, cols, w = _device_csr(first)
        out = torch.full((first.shape[0], samples, 2), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.mhcuda_calc_device_noalloc(gen, w.data_ptr(), cols.data_ptr(), ip.data_ptr(),
                                            first.shape[0], first.nnz, out.data_ptr(), None)
        free_after = torch.cuda.mem_get_info()[0]
        assert rc == 0, rc
        assert free_before - free_after < (2 << 20), \
            f"the call took {free_before - free_after} bytes of device memory"
        got_first = out.cpu().numpy().view(np.uint32)
        del ip, cols, w, out

        for m, got in ((first, got_first),
                       (second, _run(lib, "mhcuda_calc_device_noalloc", gen, second, samples))):
            np.testing.assert_array_equal(got, co.hash_csr(m, lnw=device_logf(m.data)))
            np.testing.assert_array_equal(got, _run(lib, "mhcuda_calc_device", gen, m, samples))
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
        # Full-size output: were the size check ever to let this input
        # through, the hashes would land in a buffer that holds them.
        out = torch.empty((rows, samples, 2), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = lib.mhcuda_calc_device_noalloc(gen, w.data_ptr(), cols.data_ptr(), ip.data_ptr(),
                                            rows, nnz, out.data_ptr(), None)
        assert rc == mb.INVALID_ARGUMENTS
    finally:
        lib.mhcuda_fini(gen)
