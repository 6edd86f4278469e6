"""CPU oracle for the weighted-minhash hash path -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.  The product package
never imports it.

Three restatements of the reference's arithmetic live here:

* ``hash_numpy`` -- a float32 numpy restatement of ``weighted_minhash_cuda``
  (kernel.cu:95-110 of src-d/minhashcuda), vectorised over samples x row nnz.
  Both FMA forms are exact: the fused form rounds ``ln_c - (t - beta) * r``
  once, through round-to-odd in float64 (Boldo & Melquiond, "Emulation of FMA
  and correctly rounded sums: proved algorithms using rounding to odd", IEEE
  TC 2008), because numpy has no fma.
* ``COracle`` -- ctypes wrapper of ``oracle/wmh_oracle.c`` (same arithmetic in
  C with OpenMP; the fast checker and the CPU baseline).
* ``datasketch_f64`` -- a float64 restatement of the published Ioffe weighted
  minhash as the reference's tests use it through the third-party package
  ``datasketch`` (test.py:4,22-23; unpinned there, absent here).  The
  reference's tests expect exact equality with it on their fixtures
  (test.py:26,56,146); that is a property of those fixtures, not a theorem.

Parameter layout everywhere in this module is the C-ABI one, row-major
``[samples][dim]`` float32 (minhashcuda.h:84-103, python.cc:157).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

NONE = np.uint32(0xFFFFFFFF)
FLT_MAX = np.float32(np.finfo(np.float32).max)
HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libwmh_oracle.so")
REF_LIB_DIR = os.path.join(HERE, "_ref")

FORM_UNFUSED = 0
FORM_FUSED = 1
# The form the reference build evaluates kernel.cu:104-105 in.  Pinned by
# tests/test_gpu_reference.py (the reference built for sm_100a, run on a
# B200, against both forms on inputs where they differ).
REFERENCE_FORM = FORM_FUSED


def gpu_f2i(t: np.ndarray) -> np.ndarray:
    """GPU float->int32 conversion: truncate toward zero, saturate, NaN->0."""
    t = np.asarray(t, dtype=np.float32)
    out = np.zeros(t.shape, dtype=np.int64)
    finite = ~np.isnan(t)
    out[finite] = np.clip(np.trunc(t[finite].astype(np.float64)), -2**31, 2**31 - 1)
    return out.astype(np.int32)


def _round_odd_sub_to_f32(a64: np.ndarray, b64: np.ndarray) -> np.ndarray:
    """float32(a - b) rounded once, for float64 inputs whose exact difference
    float64 may not hold: float64 round-to-odd, then round-to-nearest f32."""
    s = a64 - b64
    # TwoSum: e is the exact rounding error of s (a, b are float64 values).
    bb = s - a64
    e = (a64 - (s - bb)) + (-b64 - bb)
    bits = s.view(np.int64)
    need = (e != 0) & ((bits & 1) == 0) & np.isfinite(s)
    if need.any():
        towards = np.where(e > 0, np.inf, -np.inf)
        s = s.copy()
        s[need] = np.nextafter(s[need], towards[need])
    return s.astype(np.float32)


def hash_numpy(rs, ln_cs, betas, weights, cols, rows, form=REFERENCE_FORM, lnw=None):
    """float32 numpy restatement of kernel.cu:95-110.

    ``rows`` holds absolute offsets into ``weights``/``cols`` (rows[0] may be
    non-zero).  Returns uint32 ``[len(rows)-1, samples, 2]``; a (row, sample)
    with no entry below FLT_MAX gets (0xFFFFFFFF, 0xFFFFFFFF).
    """
    rs = np.asarray(rs, np.float32)
    ln_cs = np.asarray(ln_cs, np.float32)
    betas = np.asarray(betas, np.float32)
    weights = np.asarray(weights, np.float32)
    cols = np.asarray(cols, np.uint32)
    rows = np.asarray(rows, np.int64)
    samples, dim = rs.shape
    length = len(rows) - 1
    out = np.full((length, samples, 2), NONE, dtype=np.uint32)
    if lnw is None:
        with np.errstate(divide="ignore", invalid="ignore"):
            lnw = np.log(weights)
    lnw = np.asarray(lnw, np.float32)
    for row in range(length):
        a, b = int(rows[row]), int(rows[row + 1])
        if a == b:
            continue
        c = cols[a:b]
        keep = c < dim
        c = c[keep]
        w = lnw[a:b][keep]
        if c.size == 0:
            continue
        r = rs[:, c]
        beta = betas[:, c]
        lc = ln_cs[:, c]
        with np.errstate(all="ignore"):
            t = np.floor(w[None, :] / r + beta)
            tb = t - beta
            if form == FORM_FUSED:
                prod = tb.astype(np.float64) * r.astype(np.float64)  # exact
                ln_a = _round_odd_sub_to_f32(lc.astype(np.float64), prod) - r
            else:
                ln_a = (lc - tb * r) - r
        valid = ln_a < FLT_MAX  # NaN compares false
        masked = np.where(valid, ln_a, np.inf)
        j = np.argmin(masked, axis=1)  # first index wins ties, as strict '<'
        rows_any = valid.any(axis=1)
        s_idx = np.arange(samples)
        k = c[j].astype(np.uint32)
        tv = gpu_f2i(t[s_idx, j]).view(np.uint32)
        out[row, rows_any, 0] = k[rows_any]
        out[row, rows_any, 1] = tv[rows_any]
    return out


def params_from_uniforms(u1, u2, u3, u4, u5):
    """Parameter arithmetic of kernel.cu:18-36 in the draw order of
    minhashcuda.cc:186-200 (host logf; equal to the GPU up to logf rounding)."""
    with np.errstate(divide="ignore"):
        rs = -np.log(np.float32(u2) * np.float32(u1))
        ln_cs = np.log(-np.log(np.float32(u3) * np.float32(u4)))
    return rs.astype(np.float32), ln_cs.astype(np.float32), np.asarray(u5, np.float32)


def datasketch_params(dim, samples, seed=1):
    """float64 parameters drawn the way datasketch's WeightedMinHashGenerator
    is documented to draw them: Gamma(2,1) rs, log of Gamma(2,1) cs,
    Uniform(0,1) betas, each of shape (samples, dim), in that order, from
    ``numpy.random.RandomState(seed)``."""
    g = np.random.RandomState(seed)
    rs = g.gamma(2, 1, (samples, dim))
    ln_cs = np.log(g.gamma(2, 1, (samples, dim)))
    betas = g.uniform(0, 1, (samples, dim))
    return rs, ln_cs, betas


def datasketch_f64(rs, ln_cs, betas, v):
    """float64 Ioffe weighted minhash of one dense vector ``v`` as datasketch
    computes it: per sample, t = floor(log v / r + beta), ln_y = (t - beta) r,
    ln_a = ln_c - ln_y - r over the non-zero entries, k = argmin ln_a,
    hash = (k, int(t_k)).  Returns int64 [samples, 2]."""
    v = np.asarray(v, dtype=np.float64)
    nz = np.nonzero(v)[0]
    rs = np.asarray(rs, np.float64)[:, nz]
    ln_cs = np.asarray(ln_cs, np.float64)[:, nz]
    betas = np.asarray(betas, np.float64)[:, nz]
    t = np.floor(np.log(v[nz])[None, :] / rs + betas)
    ln_y = (t - betas) * rs
    ln_a = ln_cs - ln_y - rs
    k = np.argmin(ln_a, axis=1)
    s = np.arange(rs.shape[0])
    return np.stack([nz[k], t[s, k].astype(np.int64)], axis=1)


def build_c_oracle() -> str:
    """Compile oracle/wmh_oracle.c (oracle/Makefile) if needed."""
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "wmh_oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    return LIB_PATH


class COracle:
    """ctypes wrapper of the C restatement (oracle/wmh_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(build_c_oracle())
            P = ctypes.c_void_p
            lib.wmh_oracle_prepare.restype = P
            lib.wmh_oracle_prepare.argtypes = [P, P, P, ctypes.c_uint32, ctypes.c_uint32]
            lib.wmh_oracle_release.argtypes = [P]
            lib.wmh_oracle_hash.restype = ctypes.c_int
            lib.wmh_oracle_hash.argtypes = [P, P, P, P, P, ctypes.c_uint32, ctypes.c_int,
                                            ctypes.c_int, P]
            lib.wmh_oracle_params_from_uniforms.argtypes = [P] * 5 + [ctypes.c_uint64] + [P] * 3
            lib.wmh_oracle_logf.argtypes = [P, P, ctypes.c_uint64]
            cls._lib = lib
        return cls._lib

    def __init__(self, rs, ln_cs, betas):
        rs = np.ascontiguousarray(rs, np.float32)
        ln_cs = np.ascontiguousarray(ln_cs, np.float32)
        betas = np.ascontiguousarray(betas, np.float32)
        self.samples, self.dim = rs.shape
        self._h = self.lib().wmh_oracle_prepare(rs.ctypes.data, ln_cs.ctypes.data,
                                                betas.ctypes.data, self.dim, self.samples)
        if not self._h:
            raise MemoryError("oracle: cannot allocate the parameter table")

    def close(self):
        if self._h:
            self.lib().wmh_oracle_release(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def hash(self, weights, cols, rows, form=REFERENCE_FORM, lnw=None, threads=0, out=None):
        weights = np.ascontiguousarray(weights, np.float32)
        cols = np.ascontiguousarray(cols, np.uint32)
        rows = np.ascontiguousarray(rows, np.uint32)
        length = len(rows) - 1
        if out is None:
            out = np.empty((length, self.samples, 2), dtype=np.uint32)
        lnw_ptr = None
        if lnw is not None:
            lnw = np.ascontiguousarray(lnw, np.float32)
            assert lnw.shape == weights.shape
            lnw_ptr = lnw.ctypes.data
        rc = self.lib().wmh_oracle_hash(self._h, weights.ctypes.data, lnw_ptr, cols.ctypes.data,
                                        rows.ctypes.data, length, int(form), int(threads),
                                        out.ctypes.data)
        if rc != 0:
            raise ValueError("oracle: invalid arguments")
        return out

    def hash_csr(self, m, **kw):
        """Hash a scipy CSR matrix (indices/indptr cast to uint32)."""
        return self.hash(m.data, m.indices, m.indptr, **kw)


def host_logf(x):
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    COracle.lib().wmh_oracle_logf(x.ctypes.data, y.ctypes.data, x.size)
    return y


def reference_small_matrix(seed):
    """The 6400x130 test matrix of the reference's tests (test.py:35-39,
    93-97; README.md:85-89): randint(0,100) kept where randint(0,5) >= 4."""
    from scipy.sparse import csr_matrix
    rng = np.random.RandomState(seed)
    data = rng.randint(0, 100, (6400, 130))
    mask = rng.randint(0, 5, data.shape)
    data *= (mask >= 4)
    return data, csr_matrix(data, dtype=np.float32)


# The two 23-dimensional integer vectors of the reference's tiny tests
# (test.py:13-14) and its 20-dimensional real-valued vector (test.py:185-189).
TINY_V1 = [1, 0, 0, 0, 3, 4, 5, 0, 0, 0, 0, 6, 7, 8, 0, 0, 0, 0, 0, 0, 9, 10, 4]
TINY_V2 = [2, 0, 0, 0, 4, 3, 8, 0, 0, 0, 0, 4, 7, 10, 0, 0, 0, 0, 0, 0, 9, 0, 0]
FLOAT_V = [0, 1.0497366, 0.8494359, 0.66231006, 0.66231006, 0.8494359,
           0, 0.66231006, 0.33652836, 0, 0, 0.5359344,
           0.8494359, 0.66231006, 1.0497366, 0.33652836, 0.66231006, 0.8494359,
           0.6800841, 0.33652836]


def _splitmix64(x):
    """splitmix64 finaliser on uint64 numpy arrays (wrapping arithmetic)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def lsh_band_keys(hashes, band_width):
    """Band keys of [rows][samples][2] uint32 hashes as the engine defines them:
    h = 0x6A09E667F3BCC909 ^ b, then h = splitmix64(h ^ (k << 32 | t)) per
    sample of band b.  Returns uint64 [rows][samples // band_width]."""
    h = np.asarray(hashes, np.uint32)
    rows, samples, _ = h.shape
    bands = samples // band_width
    kt = (h[..., 0].astype(np.uint64) << np.uint64(32)) | h[..., 1].astype(np.uint64)
    out = np.empty((rows, bands), np.uint64)
    with np.errstate(over="ignore"):
        for b in range(bands):
            key = np.full(rows, np.uint64(0x6A09E667F3BCC909) ^ np.uint64(b), np.uint64)
            for s in range(b * band_width, (b + 1) * band_width):
                key = _splitmix64(key ^ kt[:, s])
            out[:, b] = key
    return out


def jaccard_estimate(hashes, pairs):
    """Fraction of samples whose (k, t) pairs agree, per row pair (the
    estimator of datasketch's WeightedMinHash.jaccard used by test.py:104-106)."""
    h = np.asarray(hashes, np.uint32)
    p = np.asarray(pairs, np.int64).reshape(-1, 2)
    same = np.all(h[p[:, 0]] == h[p[:, 1]], axis=2)
    return same.mean(axis=1).astype(np.float32)
