"""Engine vs oracle through the C ABI on a B200: bit-exact hashes.

The oracle is fed the GPU's own logf of every weight (mhcuda_debug_device_logf)
so the comparison is exact by construction; every other operation is
correctly rounded on both sides.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from wmh_testlib import device_logf, engine_gen, gamma_params, random_csr

pytestmark = pytest.mark.gpu


def check(m, samples, params, **calc_kw):
    dim = m.shape[1]
    with engine_gen(dim, samples, deferred=True) as eng:
        eng.assign(*params)
        out = eng.calc_csr(m)
    want = O.COracle(*params).hash_csr(m, lnw=device_logf(m.data))
    np.testing.assert_array_equal(out, want)
    return out


@pytest.mark.parametrize("samples", [1, 2, 3, 5, 17, 31, 32, 33, 64, 100, 127, 128, 129, 200,
                                     256, 300, 512, 1000])
def test_samples_sweep(samples):
    rng = np.random.default_rng(samples)
    dim = 700
    m = random_csr(rng, 300, dim, 25, empty_frac=0.03)
    check(m, samples, gamma_params(rng, dim, samples))


@pytest.mark.parametrize("mean_nnz", [1, 3, 30, 200, 1500])
def test_row_length_sweep(mean_nnz):
    rng = np.random.default_rng(mean_nnz)
    dim = 4000
    m = random_csr(rng, 400, dim, mean_nnz)
    check(m, 128, gamma_params(rng, dim, 128))


def test_long_rows_cross_many_chunks():
    """Rows far longer than a chunk are merged across chunks in position order."""
    rng = np.random.default_rng(9)
    dim = 60000
    m = random_csr(rng, 50, dim, 10, long_rows=[(0, 50000), (7, 20000), (49, 33333)])
    check(m, 128, gamma_params(rng, dim, 128))
    check(m, 64, gamma_params(rng, dim, 64))


def test_empty_zero_negative_nan_rows():
    rng = np.random.default_rng(4)
    dim = 200
    m = random_csr(rng, 500, dim, 8, empty_frac=0.2, zero_frac=0.3)
    d = m.data.copy()
    d[rng.random(d.size) < 0.05] = -1.0
    d[rng.random(d.size) < 0.02] = np.nan
    d[rng.random(d.size) < 0.02] = np.inf
    m = sp.csr_matrix((d, m.indices, m.indptr), shape=m.shape)
    out = check(m, 128, gamma_params(rng, dim, 128))
    empty = np.diff(m.indptr) == 0
    assert (out[empty] == 0xFFFFFFFF).all()


def test_all_rows_empty_and_trailing_empty():
    rng = np.random.default_rng(1)
    dim = 50
    params = gamma_params(rng, dim, 32)
    m = sp.csr_matrix((5, dim), dtype=np.float32)
    out = check(m, 32, params)
    assert (out == 0xFFFFFFFF).all()
    m = random_csr(rng, 40, dim, 5)
    ip = np.concatenate([m.indptr, [m.indptr[-1]] * 7])
    m2 = sp.csr_matrix((m.data, m.indices, ip), shape=(47, dim))
    out = check(m2, 32, params)
    assert (out[40:] == 0xFFFFFFFF).all()


def test_duplicate_columns_and_ties():
    """Duplicate columns inside a row and identical parameters across columns:
    the first entry in storage order wins (strict '<', kernel.cu:106)."""
    dim, samples = 16, 64
    rng = np.random.default_rng(2)
    rs, lc, b = gamma_params(rng, dim, samples)
    rs[:, 5] = rs[:, 9]
    lc[:, 5] = lc[:, 9]
    b[:, 5] = b[:, 9]
    data = np.array([3.0, 3.0, 2.0, 2.0, 7.0, 7.0], np.float32)
    cols = np.array([9, 5, 4, 4, 1, 1], np.uint32)
    ip = np.array([0, 2, 4, 6])
    m = sp.csr_matrix((data, cols, ip), shape=(3, dim))
    out = check(m, samples, (rs, lc, b))
    assert (out[0, :, 0] == 9).all()


def test_unsorted_columns():
    rng = np.random.default_rng(8)
    dim = 900
    m = random_csr(rng, 300, dim, 40, sort_cols=False)
    check(m, 128, gamma_params(rng, dim, 128))


def test_invalid_column_is_rejected():
    rng = np.random.default_rng(0)
    dim = 10
    with engine_gen(dim, 16, seed=1) as eng:
        rc, _ = eng.calc_raw(np.ones(3, np.float32), np.array([1, 10, 2], np.uint32),
                             np.array([0, 3], np.uint32))
        assert rc == 1  # mhcudaInvalidArguments
        # The generator stays usable.
        out = eng.calc(np.ones(2, np.float32), np.array([1, 2], np.uint32),
                       np.array([0, 2], np.uint32))
        assert out.shape == (1, 16, 2)
    del rng


def test_decreasing_offsets_are_rejected():
    with engine_gen(10, 16, seed=1) as eng:
        rc, _ = eng.calc_raw(np.ones(4, np.float32), np.array([1, 2, 3, 4], np.uint32),
                             np.array([0, 3, 2, 4], np.uint32))
        assert rc == 1
        rc, _ = eng.calc_raw(np.ones(1, np.float32), np.array([1], np.uint32),
                             np.array([0, 1], np.uint32), length=0)
        assert rc == 1


def test_repeated_calls_reuse_buffers():
    """Grow-only workspace: a large call followed by smaller ones (and back)."""
    rng = np.random.default_rng(12)
    dim = 3000
    params = gamma_params(rng, dim, 128)
    co = O.COracle(*params)
    with engine_gen(dim, 128, deferred=True) as eng:
        eng.assign(*params)
        for rows, nnz in ((2000, 100), (3, 5), (500, 400), (1, 1), (2500, 50)):
            m = random_csr(rng, rows, dim, nnz)
            np.testing.assert_array_equal(eng.calc_csr(m),
                                          co.hash_csr(m, lnw=device_logf(m.data)))


def test_rows_offset_is_absolute():
    rng = np.random.default_rng(13)
    dim = 400
    params = gamma_params(rng, dim, 128)
    m = random_csr(rng, 100, dim, 30)
    with engine_gen(dim, 128, deferred=True) as eng:
        eng.assign(*params)
        full = eng.calc_csr(m)
        part = eng.calc(m.data, m.indices, m.indptr[20:61])
    np.testing.assert_array_equal(part, full[20:60])


def test_batch_equals_plain_calls():
    import minhashcuda_b200
    from minhashcuda_b200 import libMHCUDA as L
    rng = np.random.default_rng(14)
    dim = 2048
    params = gamma_params(rng, dim, 256)
    mats = [random_csr(rng, int(rng.integers(1, 300)), dim, float(rng.integers(1, 80)))
            for _ in range(40)]
    gen = L.minhash_cuda_init(dim, 256, deferred=True)
    try:
        L.minhash_cuda_assign_vars(gen, *params)
        batch = L.minhash_cuda_calc_batch(gen, mats)
        plain = [L.minhash_cuda_calc(gen, m) for m in mats]
    finally:
        L.minhash_cuda_fini(gen)
    assert len(batch) == len(mats)
    for b, p in zip(batch, plain):
        np.testing.assert_array_equal(b, p)
    del minhashcuda_b200


def _pinned(a):
    """A copy of numpy array `a` in page-locked host memory."""
    import torch
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    v = t.numpy().view(a.dtype)[:a.size].reshape(a.shape)
    v[...] = a
    return v, t


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("block_nnz", [1000, 7777, 100000])
def test_row_block_pipeline(monkeypatch, pinned, block_nnz):
    """mhcuda_calc's H2D/compute/D2H pipeline over row blocks equals the
    single-launch path and the oracle, for pageable and page-locked buffers
    and blocks smaller than a row."""
    rng = np.random.default_rng(block_nnz + int(pinned))
    dim = 6000
    params = gamma_params(rng, dim, 128)
    m = random_csr(rng, 900, dim, 120, long_rows=[(3, 5000), (450, 2500)], empty_frac=0.02)
    want = O.COracle(*params).hash_csr(m, lnw=device_logf(m.data))
    with engine_gen(dim, 128, deferred=True) as eng:
        eng.assign(*params)
        monkeypatch.setenv("MHCUDA_B200_PIPELINE_MIN_NNZ", "1")
        monkeypatch.setenv("MHCUDA_B200_BLOCK_NNZ", str(block_nnz))
        data, idx, ip = m.data, m.indices.astype(np.uint32), m.indptr.astype(np.uint32)
        keep = []
        out = np.full((m.shape[0], 128, 2), 7, np.uint32)
        if pinned:
            (data, t1), (idx, t2), (ip, t3), (out, t4) = (_pinned(data), _pinned(idx), _pinned(ip),
                                                          _pinned(out))
            keep = [t1, t2, t3, t4]
        rc = eng.lib.mhcuda_calc(eng.h, data.ctypes.data, idx.ctypes.data, ip.ctypes.data,
                                 m.shape[0], out.ctypes.data)
        assert rc == 0
        np.testing.assert_array_equal(out, want)
        # twice in a row (slot reuse), then the single-launch path
        rc = eng.lib.mhcuda_calc(eng.h, data.ctypes.data, idx.ctypes.data, ip.ctypes.data,
                                 m.shape[0], out.ctypes.data)
        assert rc == 0
        np.testing.assert_array_equal(out, want)
        monkeypatch.setenv("MHCUDA_B200_NO_PIPELINE", "1")
        np.testing.assert_array_equal(eng.calc_csr(m), want)
        del keep


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("dim,no_pack", [((1 << 20) + 123, "0"), (6000, "1")])
def test_row_block_pipeline_column_packing(monkeypatch, pinned, dim, no_pack):
    """The pipeline sends columns over the host link as 16 low bits plus 4
    (dim <= 2^20) or 8 (dim <= 2^24) high bits; byte-wide high parts (dim
    above 2^20) and the unpacked route (MHCUDA_B200_NO_PACK) give the
    oracle's hashes too."""
    rng = np.random.default_rng(dim % 1000 + int(pinned))
    samples = 32
    params = gamma_params(rng, dim, samples)
    m = random_csr(rng, 700, dim, 90, long_rows=[(5, 4000)], empty_frac=0.03)
    want = O.COracle(*params).hash_csr(m, lnw=device_logf(m.data))
    with engine_gen(dim, samples, deferred=True) as eng:
        eng.assign(*params)
        monkeypatch.setenv("MHCUDA_B200_PIPELINE_MIN_NNZ", "1")
        monkeypatch.setenv("MHCUDA_B200_BLOCK_NNZ", "7777")
        monkeypatch.setenv("MHCUDA_B200_NO_PACK", no_pack)
        data, idx, ip = m.data, m.indices.astype(np.uint32), m.indptr.astype(np.uint32)
        out = np.full((m.shape[0], samples, 2), 7, np.uint32)
        keep = []
        if pinned:
            (data, t1), (idx, t2), (ip, t3), (out, t4) = (_pinned(data), _pinned(idx), _pinned(ip),
                                                          _pinned(out))
            keep = [t1, t2, t3, t4]
        for _ in range(2):
            rc = eng.lib.mhcuda_calc(eng.h, data.ctypes.data, idx.ctypes.data, ip.ctypes.data,
                                     m.shape[0], out.ctypes.data)
            assert rc == 0
            np.testing.assert_array_equal(out, want)
        del keep


def test_row_block_pipeline_unpackable_column_is_rejected(monkeypatch):
    """A column too wide for the packed form (here 2^32 - 1 with dim 500)
    sends its block unpacked, where the device check rejects it."""
    rng = np.random.default_rng(78)
    dim = 500
    m = random_csr(rng, 400, dim, 30)
    idx = m.indices.astype(np.uint32).copy()
    idx[len(idx) // 2] = 0xFFFFFFFF
    with engine_gen(dim, 64, seed=3) as eng:
        monkeypatch.setenv("MHCUDA_B200_PIPELINE_MIN_NNZ", "1")
        monkeypatch.setenv("MHCUDA_B200_BLOCK_NNZ", "1000")
        rc, _ = eng.calc_raw(m.data, idx, m.indptr)
        assert rc == 1
        np.testing.assert_array_equal(eng.calc_csr(m), eng.calc_csr(m))


def test_row_block_pipeline_reports_bad_column_in_late_block(monkeypatch):
    rng = np.random.default_rng(77)
    dim = 500
    m = random_csr(rng, 400, dim, 30)
    idx = m.indices.astype(np.uint32).copy()
    idx[-3] = dim + 5
    with engine_gen(dim, 64, seed=3) as eng:
        monkeypatch.setenv("MHCUDA_B200_PIPELINE_MIN_NNZ", "1")
        monkeypatch.setenv("MHCUDA_B200_BLOCK_NNZ", "1000")
        rc, _ = eng.calc_raw(m.data, idx, m.indptr)
        assert rc == 1
        out = eng.calc_csr(m)  # still usable
        assert out.shape == (400, 64, 2)


@pytest.mark.parametrize("chunk,samples", [(64, 128), (96, 200), (64, 31)])
def test_rows_spanning_hundreds_of_chunks(monkeypatch, chunk, samples):
    """Rows of up to 50,000 nnz cut into 64/96-nnz chunks: every such row is
    merged from hundreds of partials by finalize (position order, earliest
    position on ties), and sample counts that are not a multiple of 32 leave
    a ragged last tile."""
    rng = np.random.default_rng(chunk + samples)
    dim = 60000
    m = random_csr(rng, 40, dim, 30, long_rows=[(0, 50000), (3, 20000), (4, 777), (39, 31000)])
    params = gamma_params(rng, dim, samples)
    monkeypatch.setenv("MHCUDA_B200_CHUNK", str(chunk))
    with engine_gen(dim, samples, deferred=True) as eng:
        eng.assign(*params)
        got = eng.calc_csr(m)
    want = O.COracle(*params).hash_csr(m, lnw=device_logf(m.data))
    np.testing.assert_array_equal(got, want)


def test_near_integer_quotients():
    """w/r + beta within 1e-9..1e-3 of an integer on either side: the fast
    reciprocal path must hand every such case to the exact IEEE quotient."""
    rng = np.random.default_rng(21)
    dim, samples = 3000, 128
    wt = np.exp(rng.uniform(-6, 6, dim)).astype(np.float32)
    w = np.log(wt.astype(np.float64))
    rs = rng.uniform(0.02, 6.0, (samples, dim))
    q = w[None, :] / rs
    delta = rng.choice([-1.0, 1.0], (samples, dim)) * 10.0 ** rng.uniform(-9, -3, (samples, dim))
    b = np.round(q) - q + delta
    lc = np.log(rng.gamma(2.0, 1.0, (samples, dim)))
    params = (rs.astype(np.float32), lc.astype(np.float32), b.astype(np.float32))
    # one row per column (the crafted weight alone), then rows mixing columns
    single = sp.csr_matrix((wt, np.arange(dim), np.arange(dim + 1)), shape=(dim, dim))
    mixed = random_csr(rng, 500, dim, 40)
    mixed = sp.csr_matrix((wt[mixed.indices], mixed.indices, mixed.indptr), shape=mixed.shape)
    check(sp.vstack([single, mixed]).tocsr(), samples, params)


@pytest.mark.parametrize("knob,group_nnz", [("MHCUDA_B200_BLOCK_NNZ", 1500),
                                            ("MHCUDA_B200_BLOCK_NNZ", 20000),
                                            ("MHCUDA_B200_BATCH_GROUP_NNZ", 20000),
                                            ("MHCUDA_B200_BATCH_GROUP_NNZ", 3000)])
def test_batch_groups_and_empty_matrices(monkeypatch, knob, group_nnz):
    """mhcuda_calc_batch cut into several pipelined groups (group size from
    either knob), including empty matrices and matrices larger than a group,
    equals one calc per matrix."""
    import ctypes
    rng = np.random.default_rng(group_nnz)
    dim, samples = 3000, 64
    params = gamma_params(rng, dim, samples)
    mats = []
    for i in range(60):
        rows = int(rng.integers(0, 120)) if i % 7 else 0
        mats.append(random_csr(rng, rows, dim, float(rng.integers(1, 90)),
                               long_rows=[(0, 2500)] if rows and i % 11 == 0 else ()))
    co = O.COracle(*params)
    with engine_gen(dim, samples, deferred=True) as eng:
        eng.assign(*params)
        monkeypatch.setenv(knob, str(group_nnz))
        arrs = [(m.data.astype(np.float32), m.indices.astype(np.uint32),
                 m.indptr.astype(np.uint32)) for m in mats]
        outs = [np.full((m.shape[0], samples, 2), 3, np.uint32) for m in mats]
        P = ctypes.c_void_p
        W = (P * len(mats))(*[a[0].ctypes.data for a in arrs])
        C = (P * len(mats))(*[a[1].ctypes.data for a in arrs])
        R = (P * len(mats))(*[a[2].ctypes.data for a in arrs])
        L = (ctypes.c_uint32 * len(mats))(*[m.shape[0] for m in mats])
        OUT = (P * len(mats))(*[o.ctypes.data for o in outs])
        for _ in range(2):  # twice: slots and staging are reused
            rc = eng.lib.mhcuda_calc_batch(eng.h, len(mats), W, C, R, L, OUT)
            assert rc == 0
            for m, o in zip(mats, outs):
                if m.shape[0]:
                    np.testing.assert_array_equal(o, co.hash_csr(m, lnw=device_logf(m.data)))
