"""Helpers shared by the tests: C-ABI wrappers for the engine and for the
reference build, and seeded CSR generators."""
from __future__ import annotations

import ctypes
import os

import numpy as np
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libMHCUDA.so")


def _ptr(a):
    return a.ctypes.data if a is not None else None


class CGen:
    """A generator driven through the C ABI of include/minhashcuda.h."""

    def __init__(self, lib, dim, samples, seed=1, deferred=False, devices=0, verbosity=0):
        self.lib = lib
        status = ctypes.c_int(-1)
        self.h = lib.mhcuda_init(dim, samples, seed, int(deferred), devices, verbosity,
                                 ctypes.byref(status))
        if not self.h:
            raise RuntimeError(f"mhcuda_init failed with status {status.value}")
        self.dim, self.samples = dim, samples

    def close(self):
        if self.h:
            self.lib.mhcuda_fini(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def assign(self, rs, ln_cs, betas):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (rs, ln_cs, betas)]
        rc = self.lib.mhcuda_assign_random_vars(self.h, *[a.ctypes.data for a in arrs])
        assert rc == 0, rc

    def retrieve(self):
        out = [np.empty((self.samples, self.dim), np.float32) for _ in range(3)]
        rc = self.lib.mhcuda_retrieve_random_vars(self.h, *[a.ctypes.data for a in out])
        assert rc == 0, rc
        return tuple(out)

    def calc_raw(self, weights, cols, rows, length=None):
        weights = np.ascontiguousarray(weights, np.float32)
        cols = np.ascontiguousarray(cols, np.uint32)
        rows = np.ascontiguousarray(rows, np.uint32)
        length = len(rows) - 1 if length is None else length
        out = np.full((length, self.samples, 2), 0xA5A5A5A5, np.uint32)
        rc = self.lib.mhcuda_calc(self.h, weights.ctypes.data, cols.ctypes.data,
                                  rows.ctypes.data, length, out.ctypes.data)
        return rc, out

    def calc(self, weights, cols, rows):
        rc, out = self.calc_raw(weights, cols, rows)
        assert rc == 0, f"mhcuda_calc returned {rc}"
        return out

    def calc_csr(self, m):
        return self.calc(m.data, m.indices, m.indptr)


def engine_gen(dim, samples, **kw):
    import minhashcuda_b200
    return CGen(minhashcuda_b200.capi(), dim, samples, **kw)


_ref = None


def reference_lib():
    """The reference built from its own sources (oracle/Makefile `ref`)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        lib = ctypes.CDLL(REF_LIB)
        P, U32 = ctypes.c_void_p, ctypes.c_uint32
        lib.mhcuda_init.restype = P
        lib.mhcuda_init.argtypes = [U32, ctypes.c_uint16, U32, ctypes.c_int, U32, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int)]
        for name, args in (("mhcuda_retrieve_random_vars", [P, P, P, P]),
                           ("mhcuda_assign_random_vars", [P, P, P, P]),
                           ("mhcuda_calc", [P, P, P, P, U32, P]),
                           ("mhcuda_fini", [P])):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = args
        _ref = lib
    return _ref


def device_logf(x):
    import minhashcuda_b200
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    rc = minhashcuda_b200.capi().mhcuda_debug_device_logf(0, x.ctypes.data, y.ctypes.data, x.size)
    assert rc == 0, rc
    return y


def random_csr(rng, rows, dim, mean_nnz, *, values="lognormal", empty_frac=0.0,
               zero_frac=0.0, long_rows=(), sort_cols=True):
    """Seeded CSR with Poisson row lengths (plus chosen long rows), distinct
    columns per row, optional empty rows and explicit zero entries."""
    lengths = rng.poisson(mean_nnz, rows).astype(np.int64)
    lengths = np.minimum(lengths, dim)
    if empty_frac:
        lengths[rng.random(rows) < empty_frac] = 0
    for r, n in long_rows:
        lengths[r] = min(n, dim)
    indptr = np.zeros(rows + 1, np.int64)
    np.cumsum(lengths, out=indptr[1:])
    nnz = int(indptr[-1])
    cols = np.empty(nnz, np.uint32)
    for r in range(rows):
        n = int(lengths[r])
        if n:
            c = rng.choice(dim, n, replace=False)
            cols[indptr[r]:indptr[r + 1]] = np.sort(c) if sort_cols else c
    if values == "lognormal":
        data = rng.lognormal(0.0, 1.0, nnz).astype(np.float32)
    elif values == "int":
        data = rng.integers(1, 100, nnz).astype(np.float32)
    else:
        data = rng.random(nnz).astype(np.float32) + np.float32(1e-3)
    if zero_frac:
        data[rng.random(nnz) < zero_frac] = 0.0
    return sp.csr_matrix((data, cols, indptr), shape=(rows, dim))


def gamma_params(rng, dim, samples):
    """float32 parameters with the reference's distributions."""
    rs = rng.gamma(2.0, 1.0, (samples, dim)).astype(np.float32)
    ln_cs = np.log(rng.gamma(2.0, 1.0, (samples, dim))).astype(np.float32)
    betas = rng.uniform(0.0, 1.0, (samples, dim)).astype(np.float32)
    return rs, ln_cs, betas


def selected(out):
    """Mask of (row, sample) cells that hold a selection (not the sentinel)."""
    return ~((out[..., 0] == 0xFFFFFFFF) & (out[..., 1] == 0xFFFFFFFF))
