"""The continuous-batching server (mhcuda_server_*) on a B200.

Every result must equal the same request hashed alone by mhcuda_calc, bit for
bit, whatever else shares its batch or runs beside it.  Failures are made on
the host: invalid CSR in one request, cancellation, requests too large for a
lane.  Nothing here faults or hangs the GPU.
"""
import numpy as np
import pytest

import oracle as O
from wmh_testlib import device_logf, gamma_params, random_csr

pytestmark = pytest.mark.gpu


def _gens(specs, rng):
    from minhashcuda_b200 import libMHCUDA as L
    gens = []
    for dim, samples in specs:
        g = L.minhash_cuda_init(dim, samples, deferred=True)
        params = gamma_params(rng, dim, samples)
        L.minhash_cuda_assign_vars(g, *params)
        gens.append((g, dim, samples, params))
    return gens


def _fini(gens):
    from minhashcuda_b200 import libMHCUDA as L
    for g in gens:
        L.minhash_cuda_fini(g[0])


def test_mixed_requests_equal_requests_alone():
    from minhashcuda_b200 import libMHCUDA as L
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(5)
    gens = _gens([(3000, 128), (5000, 64), (2000, 256)], rng)
    try:
        reqs = []
        for i in range(90):
            g = gens[int(rng.integers(0, 3))]
            rows = int(np.exp(rng.uniform(0, np.log(3000))))
            reqs.append((g, random_csr(rng, rows, g[1], float(rng.integers(1, 200)))))
        with Server(hbm_budget=1 << 30, lanes=3) as srv:
            tickets = [srv.submit(g[0], m) for g, m in reqs]
            got = [srv.wait(t) for t in tickets]
            st = srv.stats()
        assert st["completed"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
        for (g, m), out in zip(reqs, got):
            np.testing.assert_array_equal(out, L.minhash_cuda_calc(g[0], m))
    finally:
        _fini(gens)


def test_oversized_requests_are_streamed_in_row_blocks():
    """A 64 MiB budget over 2 lanes leaves ~12.8 MB of CSR per lane; a request
    of ~6M nnz is cut into row blocks that run one after another and in
    parallel on both lanes."""
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(6)
    gens = _gens([(4000, 128)], rng)
    g, dim, samples, params = gens[0]
    try:
        big = random_csr(rng, 6000, dim, 1000)
        small = random_csr(rng, 50, dim, 30)
        with Server(hbm_budget=64 << 20, lanes=2) as srv:
            t1 = srv.submit(g, big)
            t2 = srv.submit(g, small)
            out_big, out_small = srv.wait(t1), srv.wait(t2)
        co = O.COracle(*params)
        np.testing.assert_array_equal(out_big, co.hash_csr(big, lnw=device_logf(big.data)))
        np.testing.assert_array_equal(out_small, co.hash_csr(small, lnw=device_logf(small.data)))
    finally:
        _fini(gens)


def test_invalid_request_fails_alone():
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import libMHCUDA as L
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(7)
    gens = _gens([(1000, 64)], rng)
    g, dim = gens[0][0], gens[0][1]
    try:
        good = [random_csr(rng, 40, dim, 20) for _ in range(12)]
        bad = random_csr(rng, 40, dim, 20)
        idx = bad.indices.copy()
        idx[5] = dim + 3
        import scipy.sparse as sp
        bad = sp.csr_matrix((bad.data, idx, bad.indptr), shape=(40, dim + 10))
        with Server(hbm_budget=256 << 20, lanes=1) as srv:
            tickets = [srv.submit(g, m) for m in good[:6]] + [srv.submit(g, bad)] + \
                      [srv.submit(g, m) for m in good[6:]]
            results = []
            for t in tickets:
                try:
                    results.append(srv.wait(t))
                except mb.MHCUDAError as e:
                    results.append(e.code)
        assert results[6] == mb.INVALID_ARGUMENTS
        for m, out in zip(good, results[:6] + results[7:]):
            np.testing.assert_array_equal(out, L.minhash_cuda_calc(g, m))
    finally:
        _fini(gens)


def test_cancel_and_refusals():
    import minhashcuda_b200 as mb
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(8)
    gens = _gens([(20000, 256)], rng)
    g = gens[0][0]
    try:
        with Server(hbm_budget=64 << 20, lanes=16) as srv:
            # a single row larger than a lane's CSR capacity is refused
            huge = random_csr(rng, 1, 20000, 1, long_rows=[(0, 19999)])
            import scipy.sparse as sp
            wide = sp.csr_matrix(np.ones((1, 300000), np.float32))
            with pytest.raises(mb.MHCUDAError) as e:
                srv.submit(g, wide)
            assert e.value.code == mb.MEMORY_ALLOCATION_FAILURE
            # cancel requests while the lanes are busy with earlier ones; a
            # request that already finished reports that and keeps its result
            many = [random_csr(rng, 300, 20000, 200) for _ in range(40)]
            tickets = [srv.submit(g, m) for m in many]
            cancelled = [t for t in tickets[-10:] if srv.cancel(t)]
            ok = 0
            for t in tickets:
                try:
                    srv.wait(t)
                    ok += 1
                    assert t not in cancelled
                except mb.MHCUDAError as err:
                    assert t in cancelled and err.code == mb.RUNTIME_ERROR
            assert ok == len(tickets) - len(cancelled)
            assert srv.wait(srv.submit(g, huge)).shape == (1, 256, 2)
    finally:
        _fini(gens)


def test_cancel_pending_request():
    """With one lane busy on large requests, the last ones are still waiting
    and are cancelled before any of their rows run."""
    import minhashcuda_b200 as mb
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(10)
    gens = _gens([(20000, 256)], rng)
    g = gens[0][0]
    try:
        with Server(hbm_budget=256 << 20, lanes=1) as srv:
            big = [random_csr(rng, 3000, 20000, 1500) for _ in range(6)]
            tickets = [srv.submit(g, m) for m in big]
            assert srv.cancel(tickets[-1])
            with pytest.raises(mb.MHCUDAError) as e:
                srv.wait(tickets[-1])
            assert e.value.code == mb.RUNTIME_ERROR
            for t in tickets[:-1]:
                assert srv.wait(t).shape == (3000, 256, 2)
    finally:
        _fini(gens)


def test_page_locked_requests_copy_directly():
    """Large requests in page-locked memory bypass the lane staging; results
    still equal mhcuda_calc alone."""
    import torch
    from minhashcuda_b200 import libMHCUDA as L
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(9)
    gens = _gens([(50000, 128)], rng)
    g = gens[0][0]

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype)[:a.size].reshape(a.shape)
        v[...] = a
        return v, t

    try:
        mats = [random_csr(rng, int(rng.integers(1000, 4000)), 50000, 400) for _ in range(6)]
        keep = []
        with Server(hbm_budget=2 << 30, lanes=2) as srv:
            tickets = []
            for m in mats:
                d, t1 = pinned(m.data.astype(np.float32))
                i, t2 = pinned(m.indices.astype(np.uint32))
                p, t3 = pinned(m.indptr.astype(np.uint32))
                o, t4 = pinned(np.zeros((m.shape[0], 128, 2), np.uint32))
                keep += [t1, t2, t3, t4]
                tickets.append(srv.submit_raw(g, d, i, p, m.shape[0], o))
            outs = [srv.wait(t) for t in tickets]
        for m, out in zip(mats, outs):
            np.testing.assert_array_equal(out, L.minhash_cuda_calc(g, m))
        del keep
    finally:
        _fini(gens)


def test_stage_trace_has_one_row_per_request(monkeypatch, tmp_path):
    """MHCUDA_B200_SERVER_TRACE: when the server stops, every completed request
    has a CSV row whose stage times add up to its total latency."""
    import csv
    from minhashcuda_b200.server import Server
    rng = np.random.default_rng(8)
    gens = _gens([(2000, 128)], rng)
    trace = tmp_path / "trace.csv"
    monkeypatch.setenv("MHCUDA_B200_SERVER_TRACE", str(trace))
    try:
        g = gens[0]
        reqs = [random_csr(rng, int(rng.integers(1, 400)), g[1], 40) for _ in range(25)]
        with Server(hbm_budget=256 << 20, lanes=2) as srv:
            for t in [srv.submit(g[0], m) for m in reqs]:
                srv.wait(t)
        rows = list(csv.DictReader(open(trace)))
        assert len(rows) == len(reqs)
        assert sorted(int(r["rows"]) for r in rows) == sorted(m.shape[0] for m in reqs)
        for r in rows:
            parts = sum(float(r[k]) for k in ("queued_ms", "gather_launch_ms", "device_ms",
                                              "complete_ms"))
            assert abs(parts - float(r["total_ms"])) < 0.01 and float(r["total_ms"]) > 0
    finally:
        _fini(gens)
