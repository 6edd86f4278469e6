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
