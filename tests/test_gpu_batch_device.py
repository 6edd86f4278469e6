"""mhcuda_calc_batch_device on a B200: many device-resident CSR matrices in
one persistent launch driven by a device-side (matrix, chunk) table.

Every matrix's hashes must equal the CPU oracle's (fed the device's logf) bit
for bit, on ragged batches that include matrices without rows, matrices whose
rows are all empty, long rows that cross chunks, misaligned CSR starts, and
repeated calls (the second call captures a CUDA graph, later ones replay it).
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from wmh_testlib import device_logf, gamma_params, random_csr

pytestmark = pytest.mark.gpu

P = ctypes.c_void_p


def _gen(lib, dim, samples, params):
    g = lib.mhcuda_init(dim, samples, 1, 1, 1, 0, None)
    assert g
    arrs = [np.ascontiguousarray(p, np.float32) for p in params]
    assert lib.mhcuda_assign_random_vars(g, *[a.ctypes.data for a in arrs]) == 0
    return g


class DeviceBatch:
    """Device copies of a list of scipy CSR matrices (None = no rows), each
    in its own allocations, optionally entered `skew` entries into them."""

    def __init__(self, mats, samples, skew=0):
        import torch
        self.mats, self.samples = mats, samples
        self.keep, w, c, r, lens, outs = [], [], [], [], [], []
        for m in mats:
            if m is None or m.shape[0] == 0:
                w.append(None), c.append(None), r.append(None), outs.append(None)
                lens.append(0)
                continue
            ip = (m.indptr.astype(np.int64) + skew).astype(np.uint32)
            dw = torch.zeros(m.nnz + skew + 1, dtype=torch.float32, device="cuda")
            dc = torch.zeros(m.nnz + skew + 1, dtype=torch.int32, device="cuda")
            if m.nnz:
                dw[skew:skew + m.nnz] = torch.from_numpy(m.data.astype(np.float32))
                dc[skew:skew + m.nnz] = torch.from_numpy(m.indices.astype(np.uint32).view(np.int32))
            dr = torch.from_numpy(ip.view(np.int32)).cuda()
            do = torch.full((m.shape[0], samples, 2), -1, dtype=torch.int32, device="cuda")
            self.keep += [dw, dc, dr, do]
            # d_rows[0] is the offset of d_weights[0]: point at entry `skew`.
            w.append(dw.data_ptr() + 4 * skew), c.append(dc.data_ptr() + 4 * skew)
            r.append(dr.data_ptr()), outs.append(do)
            lens.append(m.shape[0])
        n = len(mats)
        self.W = (P * n)(*w)
        self.C = (P * n)(*c)
        self.R = (P * n)(*r)
        self.L = (ctypes.c_uint32 * n)(*lens)
        self.outs = outs
        self.O = (P * n)(*[o.data_ptr() if o is not None else None for o in outs])

    def run(self, lib, gen, stream=None):
        import torch
        for o in self.outs:
            if o is not None:
                o.fill_(-1)
        torch.cuda.synchronize()
        rc = lib.mhcuda_calc_batch_device(gen, len(self.mats), self.W, self.C, self.R, self.L,
                                          self.O, stream)
        assert rc == 0, rc
        return lib.mhcuda_device_status(gen)

    def results(self):
        return [None if o is None else o.cpu().numpy().view(np.uint32) for o in self.outs]


def _check(co, mats, results):
    for i, (m, got) in enumerate(zip(mats, results)):
        if m is None or m.shape[0] == 0:
            continue
        want = co.hash_csr(m, lnw=device_logf(m.data))
        np.testing.assert_array_equal(got, want, err_msg=f"matrix {i}")


def _ragged(rng, dim, count):
    import scipy.sparse as sp
    mats = []
    for i in range(count):
        kind = i % 7
        if kind == 0:
            mats.append(None)  # no rows
        elif kind == 1:
            rows = int(rng.integers(1, 20))
            mats.append(sp.csr_matrix((rows, dim), dtype=np.float32))  # rows, no entries
        elif kind == 2:
            mats.append(random_csr(rng, int(rng.integers(1, 40)), dim, 30,
                                   long_rows=[(0, min(dim, 3000))]))
        else:
            mats.append(random_csr(rng, int(rng.integers(1, 300)), dim,
                                   float(rng.integers(1, 120)), empty_frac=0.05))
    return mats


@pytest.mark.parametrize("samples", [128, 256, 64, 37])
def test_ragged_batch_matches_oracle(samples):
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(100 + samples)
    dim = 5000
    params = gamma_params(rng, dim, samples)
    co = O.COracle(*params)
    g = _gen(lib, dim, samples, params)
    try:
        mats = _ragged(rng, dim, 60)
        batch = DeviceBatch(mats, samples)
        assert batch.run(lib, g) == 0
        _check(co, mats, batch.results())
    finally:
        lib.mhcuda_fini(g)


def test_repeated_batches_replay_and_misaligned_starts():
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(7)
    dim, samples = 3000, 128
    params = gamma_params(rng, dim, samples)
    co = O.COracle(*params)
    g = _gen(lib, dim, samples, params)
    try:
        mats = _ragged(rng, dim, 25)
        for skew in (0, 1, 3):  # 1 and 3: CSR starts off the 16-byte grid
            batch = DeviceBatch(mats, samples, skew=skew)
            for _ in range(3):  # eager, captured, replayed
                assert batch.run(lib, g) == 0
                _check(co, mats, batch.results())
    finally:
        lib.mhcuda_fini(g)


def test_batch_equals_one_device_call_per_matrix():
    """512 matrices of the uneven-batch shape (rows log-uniform 1..4096,
    lognormal row nnz) against one mhcuda_calc_device per matrix."""
    import torch
    import minhashcuda_b200 as mb
    import scipy.sparse as sp
    from minhashcuda_b200 import synth
    lib = mb.capi()
    w = synth.WORKLOADS["batched"]
    shapes = synth.batched_shapes(w)[:512]
    ip, cols, wts = synth.host_csr(w, 0, int(shapes.sum()))
    base = np.concatenate([[0], np.cumsum(shapes)])
    mats = []
    for i in range(len(shapes)):
        a, b = int(ip[base[i]]), int(ip[base[i + 1]])
        mats.append(sp.csr_matrix((wts[a:b], cols[a:b], ip[base[i]:base[i + 1] + 1] - a),
                                  shape=(int(shapes[i]), w.dim)))
    st = ctypes.c_int(-1)
    g = lib.mhcuda_init(w.dim, w.samples, w.seed, 0, 1, 0, ctypes.byref(st))
    assert g, st.value
    try:
        batch = DeviceBatch(mats, w.samples)
        assert batch.run(lib, g) == 0
        got = batch.results()
        for i in range(0, len(mats), 7):
            m = mats[i]
            d = DeviceBatch([m], w.samples)
            torch.cuda.synchronize()
            assert lib.mhcuda_calc_device(g, d.W[0], d.C[0], d.R[0], m.shape[0], m.nnz,
                                          d.O[0], None) == 0
            assert lib.mhcuda_device_status(g) == 0
            np.testing.assert_array_equal(got[i], d.results()[0], err_msg=f"matrix {i}")
    finally:
        lib.mhcuda_fini(g)


def test_invalid_column_fails_the_batch():
    import minhashcuda_b200 as mb
    lib = mb.capi()
    rng = np.random.default_rng(9)
    dim, samples = 1000, 64
    params = gamma_params(rng, dim, samples)
    g = _gen(lib, dim, samples, params)
    try:
        mats = [random_csr(rng, 50, dim, 20) for _ in range(6)]
        bad = mats[3].copy()
        bad.indices[5] = dim + 7
        mats[3] = bad
        batch = DeviceBatch(mats, samples)
        assert batch.run(lib, g) == mb.INVALID_ARGUMENTS
        # The generator stays usable.
        mats[3] = random_csr(rng, 50, dim, 20)
        co = O.COracle(*params)
        batch = DeviceBatch(mats, samples)
        assert batch.run(lib, g) == 0
        _check(co, mats, batch.results())
    finally:
        lib.mhcuda_fini(g)


def test_empty_and_rowless_batches():
    import minhashcuda_b200 as mb
    lib = mb.capi()
    g = lib.mhcuda_init(100, 32, 1, 0, 1, 0, None)
    assert g
    try:
        n = 3
        z = (P * n)()
        lens = (ctypes.c_uint32 * n)(0, 0, 0)
        assert lib.mhcuda_calc_batch_device(g, n, z, z, z, lens, z, None) == 0
        assert lib.mhcuda_calc_batch_device(g, 0, None, None, None, None, None, None) == 0
        lens[1] = 4  # rows but null pointers
        assert lib.mhcuda_calc_batch_device(g, n, z, z, z, lens, z, None) == mb.INVALID_ARGUMENTS
    finally:
        lib.mhcuda_fini(g)
