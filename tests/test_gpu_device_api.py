"""Device-resident entry points on a B200: mhcuda_calc_device (with its CUDA
graph replay of repeated calls) and the autotuner.  Every variant and every
replay must give the oracle's hashes bit for bit."""
import ctypes

import numpy as np
import pytest

import oracle as O
from wmh_testlib import device_logf, gamma_params, random_csr

pytestmark = pytest.mark.gpu


def _dev(m):
    import torch
    ip = torch.from_numpy(m.indptr.astype(np.int64).astype(np.uint32).view(np.int32)).cuda()
    cols = torch.from_numpy(m.indices.astype(np.uint32).view(np.int32)).cuda()
    w = torch.from_numpy(m.data.astype(np.float32)).cuda()
    return ip, cols, w


def _gen(lib, dim, samples, params):
    g = lib.mhcuda_init(dim, samples, 1, 1, 1, 0, None)
    assert g
    arrs = [np.ascontiguousarray(p, np.float32) for p in params]
    assert lib.mhcuda_assign_random_vars(g, *[a.ctypes.data for a in arrs]) == 0
    return g


def test_repeated_device_calls_replay_graphs():
    import torch
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(40)
    dim, samples = 5000, 128
    params = gamma_params(rng, dim, samples)
    co = O.COracle(*params)
    g = _gen(lib, dim, samples, params)
    try:
        mats = [random_csr(rng, 800, dim, 60), random_csr(rng, 300, dim, 200)]
        for m in mats + mats:  # second pass replays the captured graphs
            ip, cols, w = _dev(m)
            out = torch.full((m.shape[0], samples, 2), -1, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            for _ in range(3):
                out.fill_(-1)
                torch.cuda.synchronize()
                assert lib.mhcuda_calc_device(g, w.data_ptr(), cols.data_ptr(), ip.data_ptr(),
                                              m.shape[0], m.nnz, out.data_ptr(), None) == 0
                assert lib.mhcuda_device_status(g) == 0
                np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32),
                                              co.hash_csr(m, lnw=device_logf(m.data)))
    finally:
        lib.mhcuda_fini(g)


def test_autotune_choice_is_used_and_exact():
    import torch
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(41)
    dim, samples = 8000, 256
    params = gamma_params(rng, dim, samples)
    g = _gen(lib, dim, samples, params)
    try:
        m = random_csr(rng, 3000, dim, 150)
        ip, cols, w = _dev(m)
        out = torch.zeros((m.shape[0], samples, 2), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        choice = (ctypes.c_uint32 * 3)()
        ms = ctypes.c_double(0)
        assert lib.mhcuda_autotune(g, w.data_ptr(), cols.data_ptr(), ip.data_ptr(), m.shape[0],
                                   m.nnz, out.data_ptr(), None, choice, ctypes.byref(ms)) == 0
        assert choice[0] in (1, 2, 4) and choice[1] in (2, 3, 4) and choice[2] in (8, 32, 128)
        assert ms.value > 0
        want = O.COracle(*params).hash_csr(m, lnw=device_logf(m.data))
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)
        out.zero_()
        torch.cuda.synchronize()
        assert lib.mhcuda_calc_device(g, w.data_ptr(), cols.data_ptr(), ip.data_ptr(),
                                      m.shape[0], m.nnz, out.data_ptr(), None) == 0
        assert lib.mhcuda_device_status(g) == 0
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)
        # Host buffers: the copy pipeline applies the choice made for
        # launches beside copies.
        hw = np.ascontiguousarray(m.data, np.float32)
        hc = np.ascontiguousarray(m.indices, np.uint32)
        hr = np.ascontiguousarray(m.indptr, np.uint32)
        hout = np.zeros((m.shape[0], samples, 2), np.uint32)
        assert lib.mhcuda_calc(g, hw.ctypes.data, hc.ctypes.data, hr.ctypes.data, m.shape[0],
                               hout.ctypes.data) == 0
        np.testing.assert_array_equal(hout, want)
    finally:
        lib.mhcuda_fini(g)


@pytest.mark.parametrize("samples", [128, 256, 100, 64])
def test_every_kernel_variant_is_exact(monkeypatch, samples):
    """Each instantiated hash kernel -- samples per lane 1/2/4, register budget
    of 4/3/2 blocks per SM, s_pad compiled in (64, 128, 256) or read at run
    time (100 samples) -- gives the oracle's hashes."""
    import torch
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(samples)
    dim = 3000
    params = gamma_params(rng, dim, samples)
    want_m = random_csr(rng, 700, dim, 90, long_rows=[(2, 2500)], empty_frac=0.02)
    want = O.COracle(*params).hash_csr(want_m, lnw=device_logf(want_m.data))
    g = _gen(lib, dim, samples, params)
    try:
        ip, cols, w = _dev(want_m)
        out = torch.zeros((want_m.shape[0], samples, 2), dtype=torch.int32, device="cuda")
        for spl, minbs in ((4, (4, 3, 2)), (2, (4,)), (1, (4,))):
            for minb in minbs:
                monkeypatch.setenv("MHCUDA_B200_SPL", str(spl))
                monkeypatch.setenv("MHCUDA_B200_MINB", str(minb))
                out.zero_()
                torch.cuda.synchronize()
                assert lib.mhcuda_calc_device(g, w.data_ptr(), cols.data_ptr(), ip.data_ptr(),
                                              want_m.shape[0], want_m.nnz, out.data_ptr(),
                                              None) == 0
                assert lib.mhcuda_device_status(g) == 0
                np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want,
                                              err_msg=f"spl {spl} minb {minb}")
    finally:
        lib.mhcuda_fini(g)
