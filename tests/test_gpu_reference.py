"""The reference itself, built from its own sources for sm_100a
(oracle/Makefile `ref` -> oracle/_ref/libMHCUDA.so), run on the same B200 as
the engine.  These tests pin the oracle and the engine to the reference:

  * which float form the reference build evaluates kernel.cu:104-105 in
    (crafted near-tie inputs where the fused and unfused forms pick different
    columns),
  * the cuRAND parameter stream: equal seeds give bit-equal rs/ln_cs/betas,
  * hash outputs: bit-equal on every (row, sample) the reference defines.

Cells without any selectable entry are undefined in the reference (it writes
stale memory, kernel.cu:81-87) and are excluded.
"""
import numpy as np
import pytest

import oracle as O
from wmh_testlib import (CGen, device_logf, engine_gen, gamma_params, random_csr, reference_lib,
                         selected)


def crafted_form_case(rng, rows=16, samples=64):
    """Rows of two entries (columns 2i, 2i+1, equal weights) whose params make
    the fused and unfused evaluation of ln_a order the two entries
    differently, in (almost) every sample."""
    import scipy.sparse as sp
    dim = 2 * rows
    rs = np.ones((samples, dim), np.float32)
    lc = np.zeros((samples, dim), np.float32)
    b = np.zeros((samples, dim), np.float32)
    w = rng.uniform(-4, 4, rows).astype(np.float32)
    weights = np.exp(w.astype(np.float64)).astype(np.float32)
    lnw = np.log(weights)  # host log; the GPU's may differ by an ulp -> recomputed below
    M = 256
    for i in range(rows):
        for s in range(samples):
            r = rng.uniform(0.05, 6, M).astype(np.float32)
            beta = rng.uniform(0, 1, M).astype(np.float32)
            ca = rng.uniform(-3, 3, M).astype(np.float32)
            k = rng.integers(-3, 4, M)
            cb = (ca.view(np.int32) + k.astype(np.int32)).view(np.float32)
            with np.errstate(all="ignore"):
                t = np.floor(lnw[i] / r + beta)
                tb = t - beta
                prod = tb.astype(np.float64) * r.astype(np.float64)
                fa = O._round_odd_sub_to_f32(ca.astype(np.float64), prod) - r
                fb = O._round_odd_sub_to_f32(cb.astype(np.float64), prod) - r
                ua = (ca - tb * r) - r
                ub = (cb - tb * r) - r
            differ = (fb < fa) != (ub < ua)
            j = int(np.argmax(differ)) if differ.any() else 0
            rs[s, 2 * i] = rs[s, 2 * i + 1] = r[j]
            b[s, 2 * i] = b[s, 2 * i + 1] = beta[j]
            lc[s, 2 * i], lc[s, 2 * i + 1] = ca[j], cb[j]
    cols = np.arange(dim, dtype=np.uint32)
    indptr = np.arange(0, dim + 1, 2, dtype=np.int64)
    data = np.repeat(weights, 2)
    return rs, lc, b, sp.csr_matrix((data, cols, indptr), shape=(rows, dim))


def _ref_gen(dim, samples, seed=1, deferred=False):
    lib = reference_lib()
    if lib is None:
        pytest.skip("reference build oracle/_ref/libMHCUDA.so not present")
    return CGen(lib, dim, samples, seed=seed, deferred=deferred, devices=1)


@pytest.mark.gpu
def test_reference_fma_form():
    """The reference build contracts ln_c - (t-beta)*r into one FMA, and the
    engine and the oracle's REFERENCE_FORM do the same."""
    rng = np.random.default_rng(11)
    rs, lc, b, m = crafted_form_case(rng, rows=16, samples=64)
    lnw = device_logf(m.data)
    co = O.COracle(rs, lc, b)
    fused = co.hash_csr(m, form=O.FORM_FUSED, lnw=lnw)
    unfused = co.hash_csr(m, form=O.FORM_UNFUSED, lnw=lnw)
    differ = (fused != unfused).any(axis=2)
    assert differ.mean() > 0.9
    with _ref_gen(m.shape[1], 64, deferred=True) as ref:
        ref.assign(rs, lc, b)
        rout = ref.calc_csr(m)
    match_fused = (rout == fused).all(axis=2)[differ].mean()
    match_unfused = (rout == unfused).all(axis=2)[differ].mean()
    print(f"reference matches fused on {match_fused:.4f}, unfused on {match_unfused:.4f} "
          f"of {differ.sum()} separating cells")
    expected = fused if O.REFERENCE_FORM == O.FORM_FUSED else unfused
    np.testing.assert_array_equal(rout, expected)
    with engine_gen(m.shape[1], 64, deferred=True) as eng:
        eng.assign(rs, lc, b)
        np.testing.assert_array_equal(eng.calc_csr(m), expected)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,samples,seed", [(130, 128, 1), (1000, 128, 7), (23, 128, 0),
                                              (4096, 64, 3), (777, 256, 42)])
def test_curand_parameter_parity(dim, samples, seed):
    """Same seed -> the same cuRAND draws and the same float ops as
    minhashcuda.cc:179-200 / kernel.cu:18-36: bit-equal parameters."""
    with _ref_gen(dim, samples, seed=seed) as ref:
        want = ref.retrieve()
    with engine_gen(dim, samples, seed=seed) as eng:
        got = eng.retrieve()
    for name, g, w in zip(("rs", "ln_cs", "betas"), got, want):
        np.testing.assert_array_equal(g.view(np.uint32), w.view(np.uint32), err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("chunk_rows", [1, 3, 8, 37])
@pytest.mark.parametrize("dim,samples,seed", [(777, 256, 42), (130, 128, 1)])
def test_curand_parameter_parity_chunked(dim, samples, seed, chunk_rows, monkeypatch):
    """The table is built a block of sample rows at a time from two
    generators positioned at absolute offsets; any block size (ragged last
    blocks, odd dims) gives the reference's single-call draws bit for bit,
    and retrieve/assign in blocks round-trip."""
    with _ref_gen(dim, samples, seed=seed) as ref:
        want = ref.retrieve()
    monkeypatch.setenv("MHCUDA_B200_PARAM_CHUNK_ROWS", str(chunk_rows))
    with engine_gen(dim, samples, seed=seed) as eng:
        got = eng.retrieve()
    for name, g, w in zip(("rs", "ln_cs", "betas"), got, want):
        np.testing.assert_array_equal(g.view(np.uint32), w.view(np.uint32), err_msg=name)
    rng = np.random.default_rng(chunk_rows)
    mine = [rng.standard_normal((samples, dim)).astype(np.float32) for _ in range(3)]
    with engine_gen(dim, samples, deferred=True) as eng:
        eng.assign(*mine)
        monkeypatch.setenv("MHCUDA_B200_PARAM_CHUNK_ROWS", str(chunk_rows + 5))
        back = eng.retrieve()
    for g, w in zip(back, mine):
        np.testing.assert_array_equal(g, w)


@pytest.mark.gpu
def test_curand_parameter_parity_default_blocks():
    """3*2^20 dims x 128 samples: 12 MiB per sample row, so the default
    1 GiB blocks split every run into blocks of 80 and 48 sample rows."""
    dim, samples, seed = 3 << 20, 128, 9
    with _ref_gen(dim, samples, seed=seed) as ref:
        want = ref.retrieve()
    with engine_gen(dim, samples, seed=seed) as eng:
        got = eng.retrieve()
    for name, g, w in zip(("rs", "ln_cs", "betas"), got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32)), name


def _init_peak(dim, samples, seed, make):
    """Wall time of one generator init (after a warm-up init of the same
    shape) and the most device memory in use above the starting level while
    it ran, sampled from a second thread."""
    import threading
    import time
    import torch
    make(dim, samples, seed).__exit__(None, None, None)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    low = [free0]
    stop = threading.Event()

    def poll():
        while not stop.is_set():
            low[0] = min(low[0], torch.cuda.mem_get_info()[0])
            time.sleep(0.0005)

    th = threading.Thread(target=poll)
    th.start()
    t0 = time.perf_counter()
    g = make(dim, samples, seed)
    t = time.perf_counter() - t0
    stop.set()
    th.join()
    g.__exit__(None, None, None)
    return t, free0 - low[0]


@pytest.mark.gpu
def test_param_init_scratch_and_time():
    """Init builds the table a block of sample rows at a time: device memory
    above the table stays near two 1 GiB blocks (plus cuRAND state) even for
    2^24 x 256 (a 51.5 GB table, dim*samples = 2^32, which the reference
    cannot hold), where whole runs would take 2 x 17 GB.  12M x 128 is also
    timed on the reference build (three full [samples][dim] arrays)."""
    rec = {"test": "param_init"}
    eng = lambda d, s, seed: engine_gen(d, s, seed=seed)  # noqa: E731
    for dim, samples in [(12_000_000, 128), (1 << 24, 256)]:
        table = dim * 3 * ((samples + 3) // 4 * 4) * 4
        t, peak = _init_peak(dim, samples, 5, eng)
        rec[f"engine_{dim}x{samples}"] = {"s": t, "peak_bytes": peak, "table_bytes": table,
                                          "above_table_bytes": peak - table}
        assert peak - table < (4 << 30), (peak, table)
    ref = lambda d, s, seed: _ref_gen(d, s, seed=seed)  # noqa: E731
    t, peak = _init_peak(12_000_000, 128, 5, ref)
    rec["reference_12000000x128"] = {"s": t, "peak_bytes": peak}
    _record(rec)


def _compare_with_reference(m, samples, params=None, seed=1):
    dim = m.shape[1]
    with _ref_gen(dim, samples, seed=seed, deferred=params is not None) as ref:
        if params is not None:
            ref.assign(*params)
        rout = ref.calc_csr(m)
        rparams = ref.retrieve()
    with engine_gen(dim, samples, deferred=True) as eng:
        eng.assign(*rparams)
        eout = eng.calc_csr(m)
    mask = selected(eout)
    np.testing.assert_array_equal(eout[mask], rout[mask])
    # The engine's undefined cells hold the sentinel; the oracle agrees.
    co = O.COracle(*rparams)
    np.testing.assert_array_equal(co.hash_csr(m, lnw=device_logf(m.data)), eout)
    return mask.mean()


@pytest.mark.gpu
def test_reference_small_config_seeded():
    """6400x130, seed 1 (test.py:92-101 / README.md:85-98)."""
    _, m = O.reference_small_matrix(1)
    frac = _compare_with_reference(m, 128, seed=1)
    assert frac > 0.99


@pytest.mark.gpu
@pytest.mark.parametrize("samples", [2, 64, 128, 256])
def test_reference_random_lognormal(samples):
    rng = np.random.default_rng(samples)
    m = random_csr(rng, 3000, 5000, 60, long_rows=[(5, 4000), (1700, 2500)])
    params = gamma_params(rng, 5000, samples)
    _compare_with_reference(m, samples, params=params)


@pytest.mark.gpu
def test_reference_integer_weights_with_zeros():
    rng = np.random.default_rng(3)
    m = random_csr(rng, 2000, 300, 40, values="int", zero_frac=0.1)
    _compare_with_reference(m, 128, params=gamma_params(rng, 300, 128))


@pytest.mark.gpu
def test_large_workload_slice_vs_reference_build():
    """200,000 rows of the benchmark workload (Poisson(1400) nnz, Zipf(1.1)
    columns over 1M dims, 128 samples, seed 2): the reference build and the
    engine produce the same hashes through their C ABIs on the same host
    buffers.  Both calls are timed end to end (host buffers in, hashes out);
    with MHB_PERF_OUT set the timings are appended there as JSON."""
    import json
    import os
    import time
    from minhashcuda_b200 import synth
    w = synth.WORKLOADS["large"]
    rows = int(os.environ.get("MHB_REF_ROWS", "200000"))
    ip, cols, wts = synth.host_csr(w, 0, rows)
    with _ref_gen(w.dim, w.samples, seed=w.seed) as ref:
        ref.calc(wts, cols, ip)  # warm-up with the same call
        t0 = time.perf_counter()
        rout = ref.calc(wts, cols, ip)
        t_ref = time.perf_counter() - t0
        params = ref.retrieve()
    with engine_gen(w.dim, w.samples, seed=w.seed) as eng:
        got = eng.retrieve()
        for g, p in zip(got, params):
            np.testing.assert_array_equal(g.view(np.uint32), p.view(np.uint32))
        eng.calc(wts, cols, ip)  # warm-up with the same call
        t0 = time.perf_counter()
        eout = eng.calc(wts, cols, ip)
        t_eng = time.perf_counter() - t0
    mask = selected(eout)
    assert mask.all()
    np.testing.assert_array_equal(eout, rout)
    evals = int(ip[-1]) * w.samples
    rec = {"test": "large_workload_slice", "rows": rows, "nnz": int(ip[-1]),
           "samples": w.samples, "reference_s": t_ref, "engine_s": t_eng,
           "reference_evals_per_s": evals / t_ref, "engine_evals_per_s": evals / t_eng,
           "host_buffers": "pageable numpy"}
    print(json.dumps(rec))
    out = os.environ.get("MHB_PERF_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(rec) + "\n")


def _record(rec):
    import json
    import os
    print(json.dumps(rec))
    out = os.environ.get("MHB_PERF_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(rec) + "\n")


def _timed(fn, reps):
    import time
    fn()
    t = time.perf_counter()
    for _ in range(reps):
        r = fn()
    return (time.perf_counter() - t) / reps, r


@pytest.mark.gpu
def test_small_config_timing_vs_reference_build():
    """6400x130, 128 samples, seed 1 (test.py:92-101): one calc, host buffers."""
    _, m = O.reference_small_matrix(1)
    with _ref_gen(130, 128, seed=1) as ref, engine_gen(130, 128, seed=1) as eng:
        t_ref, rout = _timed(lambda: ref.calc_csr(m), 20)
        t_eng, eout = _timed(lambda: eng.calc_csr(m), 20)
    mask = selected(eout)
    np.testing.assert_array_equal(eout[mask], rout[mask])
    _record({"test": "small_config", "rows": 6400, "nnz": int(m.nnz), "samples": 128,
             "reference_s": t_ref, "engine_s": t_eng,
             "reference_evals_per_s": m.nnz * 128 / t_ref, "engine_evals_per_s": m.nnz * 128 / t_eng})


@pytest.mark.gpu
def test_batched_subset_timing_vs_reference_build():
    """The first 512 matrices of the uneven batch (2^20 dims, 256 samples):
    the reference makes one calc per matrix; the engine both that way and
    as one mhcuda_calc_batch."""
    import ctypes
    from minhashcuda_b200 import synth
    w = synth.WORKLOADS["batched"]
    shapes = synth.batched_shapes(w)[:512]
    total = int(shapes.sum())
    ip, cols, wts = synth.host_csr(w, 0, total)
    base = np.concatenate([[0], np.cumsum(shapes)])
    S = w.samples
    with _ref_gen(w.dim, S, seed=w.seed) as ref, engine_gen(w.dim, S, seed=w.seed) as eng:
        def plain(g):
            outs = []
            for i in range(len(shapes)):
                outs.append(g.calc(wts, cols, ip[base[i]:base[i + 1] + 1]))
            return outs
        t_ref, rout = _timed(lambda: plain(ref), 1)
        t_eng, eout = _timed(lambda: plain(eng), 1)
        n = len(shapes)
        P = ctypes.c_void_p
        out_b = np.empty((total, S, 2), np.uint32)
        rb = S * 8
        W = (P * n)(*([wts.ctypes.data] * n))
        C = (P * n)(*([cols.ctypes.data] * n))
        R = (P * n)(*[ip.ctypes.data + 4 * int(b) for b in base[:-1]])
        L = (ctypes.c_uint32 * n)(*[int(x) for x in shapes])
        Ob = (P * n)(*[out_b.ctypes.data + rb * int(b) for b in base[:-1]])
        t_bat, _ = _timed(lambda: eng.lib.mhcuda_calc_batch(eng.h, n, W, C, R, L, Ob), 3)
    for r_, e_ in zip(rout, eout):
        mask = selected(e_)
        np.testing.assert_array_equal(e_[mask], r_[mask])
    np.testing.assert_array_equal(np.concatenate(eout), out_b)
    evals = int(ip[-1]) * S
    _record({"test": "batched_subset", "matrices": n, "rows": total, "nnz": int(ip[-1]),
             "samples": S, "reference_plain_s": t_ref, "engine_plain_s": t_eng,
             "engine_batch_s": t_bat, "reference_plain_evals_per_s": evals / t_ref,
             "engine_plain_evals_per_s": evals / t_eng, "engine_batch_evals_per_s": evals / t_bat})


@pytest.mark.gpu
def test_streamed_block_timing_vs_reference_build():
    """One 524,288-row block of the row-streamed workload (12M dims, 128
    samples, 18.4 GB of parameters): one calc each, host buffers."""
    from minhashcuda_b200 import synth
    w = synth.WORKLOADS["streamed"]
    rows = w.extra["block_rows"]
    ip, cols, wts = synth.host_csr(w, 0, rows)
    with _ref_gen(w.dim, w.samples, seed=w.seed) as ref:
        t_ref, rout = _timed(lambda: ref.calc(wts, cols, ip), 1)
    with engine_gen(w.dim, w.samples, seed=w.seed) as eng:
        t_eng, eout = _timed(lambda: eng.calc(wts, cols, ip), 3)
    np.testing.assert_array_equal(eout, rout)
    evals = int(ip[-1]) * w.samples
    _record({"test": "streamed_block", "rows": rows, "nnz": int(ip[-1]), "samples": w.samples,
             "dim": w.dim, "reference_s": t_ref, "engine_s": t_eng,
             "reference_evals_per_s": evals / t_ref, "engine_evals_per_s": evals / t_eng})
