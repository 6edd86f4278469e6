"""Ingestion of CSR arrays in the element types scipy produces (float64 data,
int64 indices and offsets) through mhcuda_calc_typed and the Python module:
the result must equal mhcuda_calc on the arrays cast as python.cc:310-327
casts them (float32 data, uint32 indices), bit for bit; values a uint32 cast
would wrap are rejected instead."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import minhashcuda_b200 as mb
from wmh_testlib import engine_gen, random_csr

L = mb.libMHCUDA


def _wide(m, data=np.float64, index=np.int64):
    """The same matrix with data/indices/indptr of the given dtypes (set
    after construction: scipy would narrow index arrays that fit)."""
    w = sp.csr_matrix(m, copy=True)
    w.data = m.data.astype(data)
    w.indices = m.indices.astype(index)
    w.indptr = m.indptr.astype(index)
    return w


def _typed(gen, weights, wt, cols, ct, rows, rt, length, samples, *, w_addr=None, c_addr=None):
    out = np.full((length, samples, 2), 0xA5A5A5A5, np.uint32)
    rc = mb.capi().mhcuda_calc_typed(
        gen.h, weights.ctypes.data if w_addr is None else w_addr, wt,
        cols.ctypes.data if c_addr is None else c_addr, ct, rows.ctypes.data, rt, length,
        out.ctypes.data)
    return rc, out


@pytest.mark.gpu
@pytest.mark.parametrize("data,index", [(np.float64, np.int64), (np.float32, np.int64),
                                        (np.float64, np.int32), (np.float64, np.uint64)])
def test_python_calc_wide_types_equal_cast(data, index):
    rng = np.random.default_rng(31)
    m = random_csr(rng, 3000, 5000, 40, empty_frac=0.02, zero_frac=0.01)
    m.data = (m.data.astype(np.float64) * (1 + 1e-9 * rng.standard_normal(m.nnz)))
    w = _wide(m, data, index)
    want_m = sp.csr_matrix((w.data.astype(np.float32), m.indices, m.indptr), shape=m.shape)
    gen = L.minhash_cuda_init(m.shape[1], 64, seed=5)
    try:
        want = L.minhash_cuda_calc(gen, want_m)
        np.testing.assert_array_equal(L.minhash_cuda_calc(gen, w), want)
        # Row slices of wide offsets are pointer offsets too.
        np.testing.assert_array_equal(
            L.minhash_cuda_calc(gen, w, row_start=517, row_finish=2222), want[517:2222])
    finally:
        L.minhash_cuda_fini(gen)


@pytest.mark.gpu
def test_typed_many_blocks_equal_plain(monkeypatch):
    """Small staging blocks: every block is converted on host threads and
    pipelined; results equal the plain call."""
    rng = np.random.default_rng(32)
    m = random_csr(rng, 20000, 100000, 300, long_rows=[(7, 40000), (19999, 25000)])
    monkeypatch.setenv("MHCUDA_B200_BLOCK_NNZ", str(1 << 19))
    with engine_gen(m.shape[1], 128, seed=3) as gen:
        want = gen.calc_csr(m)
        d64 = m.data.astype(np.float64)
        c64 = m.indices.astype(np.int64)
        r64 = m.indptr.astype(np.int64)
        rc, got = _typed(gen, d64, mb.FLOAT64, c64, mb.INT64, r64, mb.INT64, m.shape[0], 128)
        assert rc == mb.SUCCESS
        np.testing.assert_array_equal(got, want)
        rc, got = _typed(gen, d64, mb.FLOAT64, m.indices, mb.UINT32,
                         m.indptr.astype(np.uint32), mb.UINT32, m.shape[0], 128)
        assert rc == mb.SUCCESS
        np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_typed_offsets_beyond_2_32_are_rebased():
    """64-bit offsets are taken relative to rows[0]: a row range that starts
    past 2^32 entries reads weights[rows[0]:] (the base pointers are moved
    back by 2^32 + 7 entries here and never read there)."""
    rng = np.random.default_rng(33)
    m = random_csr(rng, 500, 3000, 30)
    base = (1 << 32) + 7
    d64 = m.data.astype(np.float64)
    c64 = m.indices.astype(np.int64)
    rows = m.indptr.astype(np.int64) + base
    with engine_gen(m.shape[1], 32, seed=4) as gen:
        want = gen.calc_csr(m)
        rc, got = _typed(gen, d64, mb.FLOAT64, c64, mb.INT64, rows, mb.INT64, m.shape[0], 32,
                         w_addr=d64.ctypes.data - base * 8, c_addr=c64.ctypes.data - base * 8)
        assert rc == mb.SUCCESS
        np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [-1, (1 << 32) + 5, 4000])
def test_wide_column_out_of_range_is_rejected(bad):
    """A uint32 cast would wrap (1<<32)+5 to column 5; the typed path rejects
    it, like a negative or >= dim column."""
    rng = np.random.default_rng(34)
    m = random_csr(rng, 200, 3000, 20)
    w = _wide(m)
    w.indices[len(w.indices) // 2] = bad
    gen = L.minhash_cuda_init(m.shape[1], 32, seed=6)
    try:
        with pytest.raises(ValueError):
            L.minhash_cuda_calc(gen, w)
        # The generator stays usable.
        np.testing.assert_array_equal(L.minhash_cuda_calc(gen, _wide(m)),
                                      L.minhash_cuda_calc(gen, m))
    finally:
        L.minhash_cuda_fini(gen)


@pytest.mark.gpu
def test_typed_rejects_decreasing_wide_offsets():
    rng = np.random.default_rng(35)
    m = random_csr(rng, 100, 1000, 10)
    rows = m.indptr.astype(np.int64)
    rows[50] = rows[49] - 1
    with engine_gen(m.shape[1], 32, seed=4) as gen:
        rc, _ = _typed(gen, m.data.astype(np.float64), mb.FLOAT64, m.indices.astype(np.int64),
                       mb.INT64, rows, mb.INT64, m.shape[0], 32)
        assert rc == mb.INVALID_ARGUMENTS


@pytest.mark.gpu
def test_pinned_matrix_streams_row_blocks(monkeypatch):
    """minhash_cuda_pin page-locks a matrix's own arrays; row_start/row_finish
    blocks of it then go to the device straight from them (the pipeline sees
    page-locked input) and equal the unpinned calls and the oracle."""
    import oracle as O
    from wmh_testlib import device_logf, gamma_params
    rng = np.random.default_rng(57)
    dim, samples = 4000, 128
    m = random_csr(rng, 3000, dim, 60, empty_frac=0.02, long_rows=[(11, 3000)])
    m.indices = m.indices.astype(np.int32)
    m.indptr = m.indptr.astype(np.int32)
    params = gamma_params(rng, dim, samples)
    want = O.COracle(*params).hash_csr(m, lnw=device_logf(m.data))
    gen = L.minhash_cuda_init(dim, samples, deferred=True)
    try:
        L.minhash_cuda_assign_vars(gen, *params)
        monkeypatch.setenv("MHCUDA_B200_PIPELINE_MIN_NNZ", "1")
        monkeypatch.setenv("MHCUDA_B200_BLOCK_NNZ", "5000")
        h = L.minhash_cuda_pin(m)
        try:
            assert mb.capi().mhcuda_host_register(0, m.data.ctypes.data, m.data.nbytes) == \
                mb.INVALID_ARGUMENTS  # already registered
            for r0, r1 in ((0, 700), (700, 2500), (2500, 3000)):
                np.testing.assert_array_equal(
                    L.minhash_cuda_calc(gen, m, row_start=r0, row_finish=r1), want[r0:r1])
        finally:
            L.minhash_cuda_unpin(h)
        with pytest.raises(ValueError):
            L.minhash_cuda_unpin(h)
        np.testing.assert_array_equal(L.minhash_cuda_calc(gen, m), want)
        with pytest.raises(ValueError):
            L.minhash_cuda_pin(_wide(m))  # float64 / int64: would not be read in place
    finally:
        L.minhash_cuda_fini(gen)
