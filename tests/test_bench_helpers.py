"""CPU checks of bench.py's helpers (no GPU): the ideal shortest-remaining-
work-first bound printed beside the serving latencies."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_srpt_ideal_light_load_is_service_time():
    """Far apart arrivals never queue: every response is its own service
    time, size / rate."""
    b = _bench()
    sizes = np.full(2000, 1e9)
    r = b.srpt_ideal(sizes, rate=1e12, load=1e-4, seed=0)
    assert abs(r["p50_ms"] - 1.0) < 1e-6 and abs(r["p99_ms"] - 1.0) < 1e-6


def test_srpt_ideal_small_jobs_preempt_large_ones():
    """Mixed sizes at moderate load: the small requests' median stays at
    their service time (they preempt), the tail grows with load."""
    b = _bench()
    rng = np.random.default_rng(1)
    sizes = np.where(rng.random(20000) < 0.9, 1e6, 1e9)
    lo = b.srpt_ideal(sizes, rate=1e12, load=0.3, seed=2)
    hi = b.srpt_ideal(sizes, rate=1e12, load=0.8, seed=2)
    assert abs(lo["p50_ms"] - 1e-3) < 1e-6 and abs(hi["p50_ms"] - 1e-3) < 1e-6
    assert hi["p99_ms"] > lo["p99_ms"] >= 1.0 - 1e-9


def test_hash_roofline_picks_the_binding_resource():
    """The roofline reports DRAM, issue and the FP32 floor side by side and
    names the one closest to its peak; the algorithmic-byte rate is kept
    beside them."""
    b = _bench()
    prof = {"dram_bytes_per_eval": 4.0, "thread_inst_per_eval": 20.0, "captured_case": "x",
            "variant": "spl4_minb3"}
    nnz, R, S = 1_000_000_000, 1_000_000, 128
    evals = nnz * S
    t_ms = 200.0
    r = b.hash_roofline(nnz, R, S, t_ms, 1500.0, 6500.0, "measured", prof, True)
    dram = 4.0 * evals / (t_ms / 1e3) / 1e9 / 6500.0
    issue = 20.0 * evals / (t_ms / 1e3) / (148 * 128 * 1500e6)
    assert abs(r["dram"]["frac"] - dram) < 1e-9 and abs(r["issue"]["frac"] - issue) < 1e-9
    assert r["bound"] == ("issue" if issue > dram else "hbm")
    assert r["frac"] == max(dram, issue)
    assert abs(r["fp32_floor"]["frac"] - issue * 8 / 20) < 1e-9
    alg = 12 * nnz * S + 8 * nnz + 4 * (R + 1) + 8 * R * S
    assert abs(r["algorithmic_frac"] - alg / (t_ms / 1e3) / 1e9 / 6500.0) < 1e-9
    assert r["traffic"] == 4.0 * evals
    # Without counters only the algorithmic HBM bound is left.
    r2 = b.hash_roofline(nnz, R, S, t_ms, None, 6500.0, "measured", None, False)
    assert r2["bound"] == "hbm" and r2["traffic"] is None


def test_small_config_matrix_matches_the_oracle_restatement():
    """bench's small configuration matrix is the reference tests' 6400x130
    matrix."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from minhashcuda_b200 import synth
    ip, cols, w = synth.small_csr(1)
    _, m = O.reference_small_matrix(1)
    assert np.array_equal(ip, m.indptr) and np.array_equal(cols, m.indices)
    assert np.array_equal(w, m.data)


def test_kernel_profile_matches_the_built_source():
    """The committed ncu counters name the kernel source they were taken on;
    bench.py reports whether that is the source of this build."""
    b = _bench()
    import json
    d = json.load(open(b.PROFILE_JSON))
    assert set(d["variants"]) >= {"spl4_minb3", "spl4_minb4"}
    for v in d["variants"].values():
        assert v["dram_bytes_per_eval"] > 0 and v["thread_inst_per_eval"] > 0
    prof, current = b.kernel_profile("spl4_minb3")
    assert prof["variant"] == "spl4_minb3"
    assert current == (d["source_sha16"] == b.kernel_source_sha16())
