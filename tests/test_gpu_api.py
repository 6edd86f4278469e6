"""The reference's own test suite (test.py of src-d/minhashcuda), case by
case, against the drop-in Python module.  datasketch is absent here, so its
role is taken by oracle.datasketch_f64 (a float64 restatement of the same
published algorithm) and by the C oracle.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.stats import gamma, uniform

import oracle as O
from minhashcuda_b200 import libMHCUDA
from wmh_testlib import device_logf

pytestmark = pytest.mark.gpu


def _ds_hashes(rs, lc, b, vectors):
    return np.array([O.datasketch_f64(rs, lc, b, v) for v in vectors])


def test_calc_tiny():
    """test.py:12-32."""
    v1, v2 = O.TINY_V1, O.TINY_V2
    rs, lc, b = O.datasketch_params(len(v1), 128, 1)
    gen = libMHCUDA.minhash_cuda_init(len(v1), 128, devices=1, verbosity=2)
    libMHCUDA.minhash_cuda_assign_vars(gen, rs, lc, b)
    m = sp.csr_matrix(np.array([v1, v2], dtype=np.float32))
    hashes = libMHCUDA.minhash_cuda_calc(gen, m)
    libMHCUDA.minhash_cuda_fini(gen)
    assert hashes.shape == (2, 128, 2)
    true_hashes = _ds_hashes(rs, lc, b, [v1, v2]).astype(np.uint32)
    np.testing.assert_array_equal(hashes, true_hashes)


@pytest.mark.parametrize("devices", [1, 3])
def test_calc_big(devices):
    """test.py:34-70 (devices 1 and 3; a mask naming two devices selects the
    first present one)."""
    data, m = O.reference_small_matrix(0)
    rs, lc, b = O.datasketch_params(data.shape[-1], 128, 1)
    gen = libMHCUDA.minhash_cuda_init(data.shape[-1], 128, devices=devices, verbosity=2)
    libMHCUDA.minhash_cuda_assign_vars(gen, rs, lc, b)
    hashes = libMHCUDA.minhash_cuda_calc(gen, m)
    libMHCUDA.minhash_cuda_fini(gen)
    assert hashes.shape == (len(data), 128, 2)
    true_hashes = _ds_hashes(rs, lc, b, data).astype(np.uint32)
    np.testing.assert_array_equal(hashes, true_hashes)
    # and bit-exact against the float32 oracle with the GPU's logf
    co = O.COracle(rs.astype(np.float32), lc.astype(np.float32), b.astype(np.float32))
    np.testing.assert_array_equal(hashes, co.hash_csr(m, lnw=device_logf(m.data)))


def test_random_vars():
    """test.py:72-90: Gamma(2,1) rs and cs, U(0,1) betas."""
    gen = libMHCUDA.minhash_cuda_init(1000, 128, devices=1, verbosity=2)
    rs, ln_cs, betas = libMHCUDA.minhash_cuda_retrieve_vars(gen)
    libMHCUDA.minhash_cuda_fini(gen)
    assert rs.shape == (128, 1000) and ln_cs.shape == (128, 1000) and betas.shape == (128, 1000)
    cs = np.exp(ln_cs)
    a, loc, scale = gamma.fit(rs)
    assert 1.97 < a < 2.03 and -0.01 < loc < 0.01 and 0.98 < scale < 1.02
    a, loc, scale = gamma.fit(cs)
    assert 1.97 < a < 2.03 and -0.01 < loc < 0.01 and 0.98 < scale < 1.02
    bmin, bmax = uniform.fit(betas)
    assert 0 <= bmin < 0.001 and 0.999 <= bmax <= 1


def _ds_jaccard(h1, h2):
    return float(np.count_nonzero(np.all(h1 == h2, axis=1))) / h1.shape[0]


def test_integration():
    """test.py:92-110: estimated weighted Jaccard within 0.005 of the truth."""
    data, m = O.reference_small_matrix(1)
    gen = libMHCUDA.minhash_cuda_init(data.shape[-1], 128, seed=1, verbosity=1)
    hashes = libMHCUDA.minhash_cuda_calc(gen, m)
    libMHCUDA.minhash_cuda_fini(gen)
    assert hashes.shape == (len(data), 128, 2)
    cudamh = _ds_jaccard(hashes[0], hashes[1])
    truemh = np.amin(data[:2], axis=0).sum() / np.amax(data[:2], axis=0).sum()
    assert abs(truemh - cudamh) < 0.005


def test_slice():
    """test.py:112-124."""
    data, m = O.reference_small_matrix(0)
    gen = libMHCUDA.minhash_cuda_init(data.shape[-1], 128, verbosity=2)
    hashes = libMHCUDA.minhash_cuda_calc(gen, m)
    hashes2 = libMHCUDA.minhash_cuda_calc(gen, m, row_start=3200, row_finish=4800)
    libMHCUDA.minhash_cuda_fini(gen)
    np.testing.assert_array_equal(hashes[3200:4800], hashes2)


def test_backwards():
    """test.py:126-152: GPU parameters fed to the datasketch restatement."""
    v1, v2 = O.TINY_V1, O.TINY_V2
    gen = libMHCUDA.minhash_cuda_init(len(v1), 128, devices=1, verbosity=2)
    rs, ln_cs, betas = libMHCUDA.minhash_cuda_retrieve_vars(gen)
    m = sp.csr_matrix(np.array([v1, v2], dtype=np.float32))
    hashes = libMHCUDA.minhash_cuda_calc(gen, m)
    libMHCUDA.minhash_cuda_fini(gen)
    assert hashes.shape == (2, 128, 2)
    true_hashes = _ds_hashes(rs, ln_cs, betas, [v1, v2]).astype(np.uint32)
    np.testing.assert_array_equal(hashes, true_hashes)


def test_deferred():
    """test.py:154-182."""
    v1, v2 = O.TINY_V1, O.TINY_V2
    gen = libMHCUDA.minhash_cuda_init(len(v1), 128, devices=1, verbosity=2)
    vars_ = libMHCUDA.minhash_cuda_retrieve_vars(gen)
    libMHCUDA.minhash_cuda_fini(gen)
    gen = libMHCUDA.minhash_cuda_init(len(v1), 128, devices=1, deferred=True, verbosity=2)
    libMHCUDA.minhash_cuda_assign_vars(gen, *vars_)
    m = sp.csr_matrix(np.array([v1, v2], dtype=np.float32))
    hashes = libMHCUDA.minhash_cuda_calc(gen, m)
    libMHCUDA.minhash_cuda_fini(gen)
    true_hashes = _ds_hashes(*vars_, [v1, v2]).astype(np.uint32)
    np.testing.assert_array_equal(hashes, true_hashes)


def test_float():
    """test.py:184-210: real-valued weights, negative t compared as int32."""
    v1 = O.FLOAT_V
    gen = libMHCUDA.minhash_cuda_init(len(v1), 128, devices=1, seed=7, verbosity=2)
    vars_ = libMHCUDA.minhash_cuda_retrieve_vars(gen)
    m = sp.csr_matrix(np.array(v1, dtype=np.float32))
    hashes = libMHCUDA.minhash_cuda_calc(gen, m).astype(np.int32)
    libMHCUDA.minhash_cuda_fini(gen)
    assert hashes.shape == (1, 128, 2)
    v32 = np.array(v1, np.float32).astype(np.float64)
    true_hashes = _ds_hashes(*vars_, [v32]).astype(np.int32)
    np.testing.assert_array_equal(hashes, true_hashes)


def test_split_shapes():
    """test.py:212-232 as intended (its loop is broken as written): unbalanced
    row lengths, one row each.  The reference uses mask 4 (device #2 only);
    like the reference, a mask that names no present device is refused."""
    import torch
    mask = 4
    if torch.cuda.device_count() < 3:
        with pytest.raises(ValueError, match="No such CUDA device"):
            libMHCUDA.minhash_cuda_init(10, 128, devices=4)
        mask = 1
    for v in ([[2], [1], [1], [1]], [[1] * 50, [1], [1], [1]], [[1], [1] * 50, [1], [1]],
              [[1], [1], [1] * 50, [1]], [[1], [1], [1], [1] * 50],
              [[1] * 3, [1] * 10, [1] * 5, [1] * 2]):
        flat = np.array(sum(v, []), dtype=np.float32)
        k = len(flat)
        gen = libMHCUDA.minhash_cuda_init(k, 128, devices=mask, verbosity=2)
        m = sp.csr_matrix(flat[None, :])
        hashes = libMHCUDA.minhash_cuda_calc(gen, m)
        libMHCUDA.minhash_cuda_fini(gen)
        assert hashes.shape == (1, 128, 2)


def test_error_mapping():
    """python.cc:119-142 / 375-398 exception map."""
    with pytest.raises(ValueError):
        libMHCUDA.minhash_cuda_init(0, 128)
    gen = libMHCUDA.minhash_cuda_init(10, 16, seed=1)
    try:
        m = sp.csr_matrix(np.ones((2, 10), np.float32))
        with pytest.raises(TypeError):
            libMHCUDA.minhash_cuda_calc(gen, m.toarray())
        with pytest.raises(ValueError):
            libMHCUDA.minhash_cuda_calc(gen, m, row_start=2)
        with pytest.raises(ValueError):
            libMHCUDA.minhash_cuda_calc(gen, m, row_start=1, row_finish=1)
        with pytest.raises(ValueError):
            libMHCUDA.minhash_cuda_assign_vars(gen, np.ones(3), np.ones(3), np.ones(3))
        bad = sp.csr_matrix((np.ones(1, np.float32), np.array([12]), np.array([0, 1])),
                            shape=(1, 20))
        with pytest.raises(ValueError):
            libMHCUDA.minhash_cuda_calc(gen, bad)
        assert libMHCUDA.minhash_cuda_calc(gen, m).shape == (2, 16, 2)
    finally:
        libMHCUDA.minhash_cuda_fini(gen)
