"""mhcuda_calc's row-block pipeline at its default block shape, on a B200.

The other pipeline tests force constant blocks (MHCUDA_B200_BLOCK_NNZ) on
small matrices.  Here a 150M-nnz matrix of page-locked host buffers takes the
default shape: a first block of at most 16M nnz, blocks doubling to the
steady size (an eighth of the input, 8M to 48M nnz), a small last block,
three blocks in flight.  The test checks that
 - the hashes equal mhcuda_calc_device's on the same CSR, and the oracle's on
   the first rows;
 - the per-block timeline written under MHCUDA_B200_PIPE_TRACE has that shape
   and its events in stream order: a block's hashing starts after its copy-in
   ends, its copy-out after its hashing, and a block's copy-in after the
   copy-out of the block that last used its slot (three before it).
"""
import csv
import ctypes

import numpy as np
import pytest

import oracle as O
from wmh_testlib import device_logf

pytestmark = pytest.mark.gpu

EPS_MS = 0.05  # event timestamps have ~0.5 us resolution; allow for rounding


def test_default_block_shape_and_trace(tmp_path, monkeypatch):
    import torch
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import synth
    lib = mb.capi()
    base = synth.WORKLOADS["large"]
    w = synth.Workload(**{**base.__dict__, "rows": 110_000, "dim": 100_000})
    st = ctypes.c_int(-1)
    gen = lib.mhcuda_init(w.dim, w.samples, w.seed, 0, 1, 0, ctypes.byref(st))
    assert gen, st.value
    try:
        ip, cols, wts, nnz = synth.device_csr(w, 0, w.rows)
        assert nnz > 140 << 20
        R, S = w.rows, w.samples
        out = torch.zeros((R, S, 2), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert lib.mhcuda_calc_device(gen, wts.data_ptr(), cols.data_ptr(), ip.data_ptr(), R,
                                      nnz, out.data_ptr(), None) == 0
        assert lib.mhcuda_device_status(gen) == 0
        want = out.cpu().numpy().view(np.uint32)

        h_w = torch.empty(nnz, dtype=torch.float32, pin_memory=True)
        h_c = torch.empty(nnz, dtype=torch.int32, pin_memory=True)
        h_i = torch.empty(R + 1, dtype=torch.int32, pin_memory=True)
        h_o = torch.full((R, S, 2), 7, dtype=torch.int32, pin_memory=True)
        h_w.copy_(wts[:nnz])
        h_c.copy_(cols[:nnz])
        h_i.copy_(ip)
        del out, wts, cols, ip
        torch.cuda.empty_cache()

        trace = tmp_path / "pipe.csv"
        monkeypatch.setenv("MHCUDA_B200_PIPE_TRACE", str(trace))
        assert lib.mhcuda_calc(gen, h_w.data_ptr(), h_c.data_ptr(), h_i.data_ptr(), R,
                               h_o.data_ptr()) == 0
        got = h_o.numpy().view(np.uint32)
        np.testing.assert_array_equal(got, want)

        # The oracle on the first rows.
        params = [np.empty((S, w.dim), np.float32) for _ in range(3)]
        assert lib.mhcuda_retrieve_random_vars(gen, *[p.ctypes.data for p in params]) == 0
        n0 = 1500
        ipn = h_i.numpy().view(np.uint32)[:n0 + 1].copy()
        e = int(ipn[-1])
        wt = h_w.numpy()[:e].copy()
        cl = h_c.numpy().view(np.uint32)[:e].copy()
        oracle_out = O.COracle(*params).hash(wt, cl, ipn, lnw=device_logf(wt))
        np.testing.assert_array_equal(got[:n0], oracle_out)

        rows = list(csv.DictReader(open(trace)))
        assert rows and all(r["call"] == rows[0]["call"] for r in rows)
        sizes = [int(r["nnz"]) for r in rows]
        assert sum(sizes) == nnz
        longest_row = int(np.diff(h_i.numpy().view(np.uint32).astype(np.int64)).max())
        # steady size: an eighth of the input, between 8M and 48M nnz; the
        # first block is 16M at most, later ones double up to the steady size
        # (blocks hold whole rows)
        cap = min(max(nnz // 8, 8 << 20), 48 << 20)
        assert sizes[0] <= min(cap, 16 << 20) + longest_row
        assert max(sizes) <= cap + longest_row
        for a, b in zip(sizes[:-3], sizes[1:-2]):
            assert b <= 2 * a + longest_row
        assert sizes[-1] < sizes[-2]  # the small last block
        assert any(s > cap - longest_row for s in sizes[:-2])
        t = [{k: float(r[k]) for k in r if k not in ("call", "block", "nnz")} for r in rows]
        for i, b in enumerate(t):
            assert b["h2d_start"] <= b["h2d_end"] + EPS_MS
            assert b["h2d_end"] <= b["hash_start"] + EPS_MS
            assert b["hash_start"] <= b["hash_end"] + EPS_MS
            assert b["hash_end"] <= b["d2h_start"] + EPS_MS
            assert b["d2h_start"] <= b["d2h_end"] + EPS_MS
            if i >= 1:
                assert t[i - 1]["hash_end"] <= b["hash_start"] + EPS_MS  # one generator stream
                assert t[i - 1]["h2d_end"] <= b["h2d_start"] + EPS_MS
            if i >= 3:
                assert t[i - 3]["d2h_end"] <= b["h2d_start"] + EPS_MS  # slot reuse
    finally:
        lib.mhcuda_fini(gen)
