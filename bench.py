#!/usr/bin/env python
"""Benchmark: weighted-minhash throughput (nnz*samples evaluations/s) on B200.

Default workload ("large"): one 2,000,000 x 1,000,000 fp32 CSR matrix, row
nnz ~ Poisson(1400) (~2.8e9 nnz), Zipf(1.1) columns, lognormal values, 128
samples, generator seed 2.  Inputs (22.4 GB of CSR) and the parameter table
(1.5 GB) are far larger than the 126 MB L2, so no L2 flush is needed between
steps.

  value  device throughput: the CSR is resident in HBM, one step is one
         mhcuda_calc_device call (plan + hash + finalize kernels), timed with
         CUDA events on the launch stream.  Before warm-up, mhcuda_autotune
         picks the kernel variant for this data (samples per lane, register
         budget, chunk granularity; results never depend on it) and the line
         reports its choice under "autotuned" (--no-autotune: the planner's
         default).
  e2e    the same metric through the drop-in C ABI call mhcuda_calc with
         pinned host buffers: every step copies the CSR host->device and the
         hashes device->host inside the timed region.
  roofline  the hash kernel alone, timed with events the library records
         around each launch on its stream; algorithmic bytes per launch
         B = 12*N*S + 8*N + 4*(R+1) + 8*R*S over the measured HBM copy
         bandwidth.
  cpu_baseline  the C oracle (oracle/wmh_oracle.c, OpenMP on all host cores)
         on a bounded sample of the same rows, which is also checked bit for
         bit against the GPU's output for those rows.

--impl reference runs the reference arm: the reference has no CPU
implementation of the hash (kernel.cu is CUDA only), so it times the C oracle
port of the reference kernel on all host cores over a bounded sample of the
same workload per step.

Multi-GPU: the path has no exchange step; N ranks run N independent replicas,
rank r on rows [r*R, (r+1)*R) of the seeded workload (weak scaling, one
process per GPU, no data-path collective).  Timing is the max over ranks of
the per-rank device time; the job's evals are summed over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "WMH nnz*samples/s (plain calc, 1 B200, bit-exact)"
UNIT = "nnz*samples/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """Samples nvidia-smi clocks / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(float(r[2]) for r in rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()),
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


KERNEL_SOURCE = os.path.join(ROOT, "minhashcuda_b200", "csrc", "hash_kernels.cu")
PROFILE_JSON = os.path.join(ROOT, "profiles", "hash_kernel_traffic.json")
SMS = 148
ISSUE_PER_SM_CLK = 4 * 32  # four schedulers, one warp-instruction (32 threads) per clock each


def kernel_source_sha16():
    import hashlib
    with open(KERNEL_SOURCE, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()[:16]


def kernel_profile(variant):
    """Counters ncu measured for the hash kernel variant `variant` (e.g.
    "spl4_minb3") on a 20,000-row case of the large workload
    (profiles/hash_kernel_traffic.json), and whether they were taken on the
    kernel source this run built."""
    if not os.path.exists(PROFILE_JSON):
        return None, False
    d = json.load(open(PROFILE_JSON))
    v = d.get("variants", {}).get(variant)
    if v is None:
        return None, False
    v = dict(v, captured_case=d.get("captured_case"), variant=variant)
    return v, d.get("source_sha16") == kernel_source_sha16()


def digest(a):
    import hashlib
    return hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def hash_roofline(nnz, R, S, kernel_ms, sm_mhz, peak, peak_kind, profile, profile_current):
    """Roofline of one hash launch.  Three bounds are reported side by side:
    DRAM traffic (ncu bytes per eval of this workload, scaled to the launch)
    over the measured HBM bandwidth; issue (ncu thread-instructions per eval
    over 148 SMs x 128 thread-instructions per clock at the run's median SM
    clock); and the FP32 issue floor of 8 operations per eval.  `bound` is the
    one closest to its peak; the algorithmic bytes 12NS + 8N + 4(R+1) + 8RS
    are kept beside them (their rate exceeds HBM when hot columns hit L2)."""
    t = kernel_ms / 1e3
    evals = nnz * S
    alg = 12 * nnz * S + 8 * nnz + 4 * (R + 1) + 8 * R * S
    out = {"kernel": "hash_kernel", "kernel_ms": kernel_ms, "algorithmic_bytes": alg,
           "algorithmic_gbs": alg / t / 1e9, "algorithmic_frac": alg / t / 1e9 / peak,
           "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)", "sm_mhz": sm_mhz}
    cands = {}
    traffic = None
    if profile and profile.get("dram_bytes_per_eval"):
        traffic = profile["dram_bytes_per_eval"] * evals
        gbs = traffic / t / 1e9
        out["dram"] = {"achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                       "bytes_per_eval": profile["dram_bytes_per_eval"]}
        cands["hbm"] = out["dram"]
    if sm_mhz:
        issue_peak = SMS * ISSUE_PER_SM_CLK * sm_mhz * 1e6 / 1e12
        if profile and profile.get("thread_inst_per_eval"):
            ach = profile["thread_inst_per_eval"] * evals / t / 1e12
            out["issue"] = {"achieved": ach, "peak": issue_peak, "unit": "T thread-inst/s",
                            "frac": ach / issue_peak,
                            "inst_per_eval": profile["thread_inst_per_eval"]}
            cands["issue"] = out["issue"]
        fp = 8 * evals / t / 1e12
        out["fp32_floor"] = {"achieved": fp, "peak": issue_peak, "unit": "T ops/s",
                             "frac": fp / issue_peak, "ops_per_eval": 8}
    out["profile"] = {"source": os.path.relpath(PROFILE_JSON, ROOT),
                      "case": profile.get("captured_case") if profile else None,
                      "variant": profile.get("variant") if profile else None,
                      "matches_built_kernel": profile_current}
    if cands:
        bound = max(cands, key=lambda k: cands[k]["frac"])
        b = cands[bound]
        out.update({"bound": bound, "achieved": b["achieved"], "peak": b["peak"],
                    "unit": b["unit"], "frac": b["frac"]})
    else:
        out.update({"bound": "hbm", "achieved": alg / t / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": alg / t / 1e9 / peak})
    out["traffic"] = traffic
    return out


def cpu_oracle_sample(w, params_host, target_s=12.0, check=None, nthreads=0, max_rows=20000):
    """Times the C oracle on the first rows of the workload, growing the
    sample until it takes ~target_s.  Returns (evals/s, rows, nnz, seconds,
    bit_exact or None)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from minhashcuda_b200 import synth
    co = O.COracle(*params_host)
    rows = 64
    while True:
        ip, cols, wts = synth.host_csr(w, 0, rows)
        t0 = time.perf_counter()
        out = co.hash(wts, cols, ip, threads=nthreads)
        dt = time.perf_counter() - t0
        if dt >= target_s / 4 or rows >= max_rows:
            break
        rows = min(max_rows, int(rows * max(2.0, min(8.0, (target_s / 4) / max(dt, 1e-3)))))
    nnz = int(ip[-1])
    exact = None
    if check is not None:
        exact = check(rows, ip, cols, wts, co)
    return nnz * w.samples / dt, rows, nnz, dt, exact


def run_reference_arm(args, rank):
    """--impl reference: the C oracle port on all host cores, K timed steps of a
    bounded sample of the workload."""
    if rank != 0:
        return
    import torch
    from minhashcuda_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    w = synth.WORKLOADS[args.workload]
    torch.cuda.set_device(0)
    g = np.random.default_rng(w.seed)
    # The oracle only reads the parameter table; a seeded Gamma/uniform table
    # has the generator's distributions (its values do not change the work).
    rs = g.gamma(2.0, 1.0, (w.samples, w.dim)).astype(np.float32)
    lc = np.log(g.gamma(2.0, 1.0, (w.samples, w.dim))).astype(np.float32)
    bt = g.uniform(0, 1, (w.samples, w.dim)).astype(np.float32)
    co = O.COracle(rs, lc, bt)
    del rs, lc, bt
    rows = args.cpu_rows
    ip, cols, wts = synth.host_csr(w, 0, rows)
    nnz = int(ip[-1])
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        co.hash(wts, cols, ip, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        co.hash(wts, cols, ip, threads=threads)
        times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    value = nnz * w.samples / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(w, args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {rows} rows ({nnz} nnz) of the workload per step; the "
                                   "reference has no CPU hash path, so this is the C port of "
                                   "kernel.cu:95-110 (oracle/wmh_oracle.c)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "rows_per_s": rows / t,
    }
    del co
    if args.extras and args.gpus == 1:
        line["reference_cuda"] = reference_cuda_cases()
    print(json.dumps(line), flush=True)


def reference_cuda_cases():
    """The reference's own CUDA implementation, compiled from its sources for
    sm_100a (oracle/_ref/libMHCUDA.so, oracle/Makefile), timed through its C
    ABI on the inputs the default arm times this engine on
    (`same_inputs_as_reference_cuda`); equal digests mean bit-identical
    hashes."""
    path = os.path.join(ROOT, "oracle", "_ref", "libMHCUDA.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libMHCUDA.so was not built (no reference sources)"}
    lib = ctypes.CDLL(path)
    Pt, U32 = ctypes.c_void_p, ctypes.c_uint32
    lib.mhcuda_init.restype = Pt
    lib.mhcuda_init.argtypes = [U32, ctypes.c_uint16, U32, ctypes.c_int, U32, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_int)]
    lib.mhcuda_calc.restype = ctypes.c_int
    lib.mhcuda_calc.argtypes = [Pt, Pt, Pt, Pt, U32, Pt]
    lib.mhcuda_fini.restype = ctypes.c_int
    lib.mhcuda_fini.argtypes = [Pt]
    try:
        res = time_reference_cases(lib, 0)
    except Exception as e:  # recorded; the CPU arm's value stands
        return {"error": f"{type(e).__name__}: {e}"}
    res["build"] = "reference kernel.cu/minhashcuda.cc compiled for sm_100a (oracle/Makefile ref)"
    return res


def _free_cuda():
    import gc
    import torch
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def extra_uniform(lib, local, peak, peak_kind):
    """HBM roofline on uniform columns: one 524,288-row block of the streamed
    workload (12,000,000 dims x 128 samples, 18.4 GB of parameters, uniform
    columns, so the gathers find nothing in L2), device-resident, one
    mhcuda_calc_device per step, the hash kernel timed with the events the
    library records around it."""
    import torch
    from minhashcuda_b200 import synth
    w = synth.WORKLOADS["streamed"]
    rows, S = w.extra["block_rows"], w.samples
    st = ctypes.c_int(-1)
    gen = lib.mhcuda_init(w.dim, S, w.seed, 0, 1 << local, 0, ctypes.byref(st))
    assert gen, st.value
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ip, cols, wts, nnz = synth.device_csr(w, 0, rows, stream=stream)
    out = torch.empty((rows, S, 2), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step():
        assert lib.mhcuda_calc_device(gen, wts.data_ptr(), cols.data_ptr(), ip.data_ptr(), rows,
                                      nnz, out.data_ptr(), sp) == 0

    for _ in range(3):
        step()
    lib.mhcuda_profile(gen, 1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    hm, nl = ctypes.c_double(0), ctypes.c_uint64(0)
    assert lib.mhcuda_profile_read(gen, ctypes.byref(hm), ctypes.byref(nl)) == 0
    lib.mhcuda_profile(gen, 0)
    assert lib.mhcuda_device_status(gen) == 0
    lib.mhcuda_fini(gen)
    kernel_ms = hm.value / max(1, nl.value)
    alg = 12 * nnz * S + 8 * nnz + 4 * (rows + 1) + 8 * rows * S
    gbs = alg / (kernel_ms / 1e3) / 1e9
    del ip, cols, wts, out
    _free_cuda()
    return {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "traffic": None, "kernel": "hash_kernel", "kernel_ms": kernel_ms,
            "algorithmic_bytes": alg, "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
            "value": nnz * S / (e0.elapsed_time(e1) / 5 / 1e3), "unit_value": UNIT,
            "workload": f"streamed block: {rows} rows x {w.dim} dims, {S} samples, {nnz} nnz, "
                        "uniform columns, device-resident"}


def _time_host_calls(lib, gen, calls, S, reps, warmup=1):
    """Times `reps` passes over `calls` [(weights, cols, indptr)] through the
    C ABI mhcuda_calc with pageable numpy buffers (the reference's calling
    convention); returns (seconds per pass, outputs of the last pass)."""
    outs = [np.empty((len(ip) - 1, S, 2), np.uint32) for _, _, ip in calls]

    def one():
        for (wt, cl, ip), o in zip(calls, outs):
            rc = lib.mhcuda_calc(gen, wt.ctypes.data, cl.ctypes.data, ip.ctypes.data,
                                 len(ip) - 1, o.ctypes.data)
            assert rc == 0, rc

    for _ in range(warmup):
        one()
    t = time.perf_counter()
    for _ in range(reps):
        one()
    return (time.perf_counter() - t) / reps, outs


def reference_cases():
    """Inputs the reference CUDA build (in the reference arm) and this engine
    (in the default arm) both hash through their own C ABI, mhcuda_calc, with
    pageable numpy buffers, for a same-box comparison: name -> (dim, samples,
    seed, calls, reps)."""
    from minhashcuda_b200 import synth
    cases = {}
    ip, cl, wt = synth.small_csr(1)
    cases["small_6400x130"] = (130, 128, 1, [(wt, cl, ip)], 20)
    w = synth.WORKLOADS["large"]
    ip, cl, wt = synth.host_csr(w, 0, 200_000)
    cases["large_first_200000_rows"] = (w.dim, w.samples, w.seed, [(wt, cl, ip)], 2)
    w = synth.WORKLOADS["batched"]
    shapes = synth.batched_shapes(w)[:512]
    ip, cl, wt = synth.host_csr(w, 0, int(shapes.sum()))
    base = np.concatenate([[0], np.cumsum(shapes)])
    calls = [(wt, cl, ip[base[i]:base[i + 1] + 1]) for i in range(len(shapes))]
    cases["batched_first_512_matrices"] = (w.dim, w.samples, w.seed, calls, 1)
    return cases


def time_reference_cases(lib, local):
    """Times every reference case through `lib`'s mhcuda_calc; each entry
    carries evals/s and a digest of the hashes (equal digests in the two arms
    mean bit-identical output)."""
    res = {}
    for name, (dim, S, seed, calls, reps) in reference_cases().items():
        st = ctypes.c_int(-1)
        gen = lib.mhcuda_init(dim, S, seed, 0, 1 << local, 0, ctypes.byref(st))
        assert gen, f"mhcuda_init failed: {st.value}"
        t, outs = _time_host_calls(lib, gen, calls, S, reps)
        lib.mhcuda_fini(gen)
        nnz = sum(int(ip[-1]) - int(ip[0]) for _, _, ip in calls)
        rows = sum(len(ip) - 1 for _, _, ip in calls)
        res[name] = {"value": nnz * S / t, "unit": UNIT, "ms_per_pass": t * 1e3,
                     "calls_per_pass": len(calls), "rows": rows, "nnz": nnz, "samples": S,
                     "digest": digest(np.concatenate([o.reshape(-1) for o in outs]))}
    return res


def run_batched(args, rank, world, local, emit=True, steps=None, warmup=None):
    """The uneven-batch configuration: 4096 CSR matrices sharing one generator
    (2^20 dims, 256 samples), rows per matrix log-uniform in [1, 4096], row
    nnz lognormal(median 64, sigma 1.5) clipped to [1, 20000], uniform
    columns, lognormal values.  Three ways through the C ABI:
      plain    one mhcuda_calc per matrix, pageable host buffers in and out;
      batched  one mhcuda_calc_batch over all of them, same host buffers;
      device   one mhcuda_calc_batch_device with the matrices resident in
               device memory (each starting on a 16-byte boundary), outputs
               left there; repeated calls replay its CUDA graph."""
    import torch
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import synth
    steps = steps or args.steps
    warmup = warmup if warmup is not None else args.warmup
    torch.cuda.set_device(local)
    w = synth.WORKLOADS["batched"]
    shapes = synth.batched_shapes(w)
    total_rows = int(shapes.sum())
    t0 = time.perf_counter()
    ip, cols, wts = synth.host_csr(w, 0, total_rows)
    nnz = int(ip[-1])
    log(f"[rank {rank}] batched: {len(shapes)} matrices, {total_rows} rows, {nnz} nnz, "
        f"generated in {time.perf_counter() - t0:.1f}s")
    lib = mb.capi()
    S = w.samples
    gen = lib.mhcuda_init(w.dim, S, w.seed, 0, 1 << local, 0, None)
    assert gen
    base = np.zeros(len(shapes) + 1, np.int64)
    np.cumsum(shapes, out=base[1:])
    out_plain = np.empty((total_rows, S, 2), np.uint32)
    out_batch = np.empty((total_rows, S, 2), np.uint32)
    P = ctypes.c_void_p
    n = len(shapes)
    row_bytes = S * 2 * 4
    ipp = ip.ctypes.data
    Wp = (P * n)(*([wts.ctypes.data] * n))
    Cp = (P * n)(*([cols.ctypes.data] * n))
    Rp = (P * n)(*[ipp + 4 * int(b) for b in base[:-1]])
    Lp = (ctypes.c_uint32 * n)(*[int(x) for x in shapes])
    Op = (P * n)(*[out_batch.ctypes.data + row_bytes * int(b) for b in base[:-1]])
    Opl = [out_plain.ctypes.data + row_bytes * int(b) for b in base[:-1]]

    # Device-resident copy: matrix i's entries start on a 16-byte boundary of
    # one buffer; its offsets are the absolute ones of the host arrays.
    starts = ip[base[:-1]].astype(np.int64)
    counts = ip[base[1:]].astype(np.int64) - starts
    padded = np.zeros(n + 1, np.int64)
    np.cumsum((counts + 3) // 4 * 4, out=padded[1:])
    src_idx = np.concatenate([np.arange(a, a + c) for a, c in zip(starts, counts)])
    dst_idx = np.concatenate([np.arange(p, p + c) for p, c in zip(padded[:-1], counts)])
    d_w = torch.zeros(int(padded[-1]) + 4, dtype=torch.float32, device="cuda")
    d_c = torch.zeros(int(padded[-1]) + 4, dtype=torch.int32, device="cuda")
    d_w[torch.from_numpy(dst_idx).cuda()] = torch.from_numpy(wts[src_idx]).cuda()
    d_c[torch.from_numpy(dst_idx).cuda()] = torch.from_numpy(cols[src_idx].view(np.int32)).cuda()
    del src_idx, dst_idx
    d_ip = torch.from_numpy(ip.view(np.int32)).cuda()
    d_out = torch.empty((total_rows, S, 2), dtype=torch.int32, device="cuda")
    DW = (P * n)(*[d_w.data_ptr() + 4 * int(p) for p in padded[:-1]])
    DC = (P * n)(*[d_c.data_ptr() + 4 * int(p) for p in padded[:-1]])
    DR = (P * n)(*[d_ip.data_ptr() + 4 * int(b) for b in base[:-1]])
    DO = (P * n)(*[d_out.data_ptr() + row_bytes * int(b) for b in base[:-1]])
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    torch.cuda.synchronize()

    def plain():
        for i in range(n):
            rc = lib.mhcuda_calc(gen, wts.ctypes.data, cols.ctypes.data, Rp[i], int(shapes[i]),
                                 Opl[i])
            assert rc == 0, rc

    def batched():
        rc = lib.mhcuda_calc_batch(gen, n, Wp, Cp, Rp, Lp, Op)
        assert rc == 0, rc

    def device():
        rc = lib.mhcuda_calc_batch_device(gen, n, DW, DC, DR, Lp, DO, sp)
        assert rc == 0, rc

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t)
        return sum(ts) / len(ts)

    with Clocks(local) as clk:
        t_plain = timed(plain)
        t_batch = timed(batched)
        for _ in range(max(2, warmup)):  # eager, then captured
            device()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            device()
        e1.record(stream)
        torch.cuda.synchronize()
        t_dev = e0.elapsed_time(e1) / steps / 1e3
    assert lib.mhcuda_device_status(gen) == 0
    exact = bool(np.array_equal(out_plain, out_batch))
    exact_dev = bool(np.array_equal(out_plain, d_out.cpu().numpy().view(np.uint32)))
    lib.mhcuda_fini(gen)
    del d_w, d_c, d_ip, d_out
    _free_cuda()
    evals = nnz * S
    line = {
        "metric": "WMH nnz*samples/s (batched: 4096 uneven CSR, one call)",
        "value": evals / t_batch, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": t_batch * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded, generated on the device, copied to pageable host arrays)",
        "config": {"workload": f"batched: {n} matrices, {total_rows} rows, {nnz} nnz, "
                               f"{w.dim} dims, {S} samples", "matrices": n,
                   "rows": total_rows, "nnz": nnz, "dim": w.dim, "samples": S},
        "plain": {"value": evals / t_plain, "unit": UNIT, "ms_per_step": t_plain * 1e3,
                  "calls_per_step": n},
        "device_resident": {"value": evals / t_dev, "unit": UNIT, "ms_per_step": t_dev * 1e3,
                            "call": "mhcuda_calc_batch_device (CUDA graph replay)",
                            "over_plain": t_plain / t_dev},
        "batched_over_plain": t_plain / t_batch, "bit_exact_plain_vs_batched": exact,
        "bit_exact_plain_vs_device_batch": exact_dev,
        "rows_per_s": total_rows / t_batch, "clocks": clk.summary(),
        "e2e": {"value": evals / t_batch, "unit": UNIT,
                "h2d_bytes_per_step": 8 * nnz + 4 * total_rows,
                "d2h_bytes_per_step": total_rows * row_bytes},
    }
    if emit and rank == 0:
        print(json.dumps(line), flush=True)
    return line


def run_ingest(args, rank, world, local):
    """scipy ingestion through the Python module: the first rows of the large
    workload (default 200,000 rows, ~2.8e8 nnz; 1,000,000 dims, 128 samples)
    as a scipy csr_matrix with float64 data and int64 indices/offsets -- the
    types scipy gives a matrix with 2^31 nnz or more -- hashed by
    libMHCUDA.minhash_cuda_calc, which converts each block while staging it.
    Beside it: the same matrix as float32/int32 (used in place) and the
    reference module's route for wide types, a whole-array cast to
    float32/uint32 before the call (python.cc:310-327).  Pageable host arrays,
    hashes returned to a new numpy array, every step."""
    import scipy.sparse as sp
    import torch
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import synth
    torch.cuda.set_device(local)
    L = mb.libMHCUDA
    w = synth.WORKLOADS["large"]
    rows = args.rows or 200_000
    t0 = time.perf_counter()
    ip, cols, wts = synth.host_csr(w, 0, rows, device=f"cuda:{local}")
    nnz = int(ip[-1])
    m32 = sp.csr_matrix((wts, cols.view(np.int32), ip.view(np.int32)), shape=(rows, w.dim))
    m64 = sp.csr_matrix(m32, copy=True)
    m64.data = wts.astype(np.float64)
    m64.indices = cols.astype(np.int64)
    m64.indptr = ip.astype(np.int64)
    log(f"[rank {rank}] ingest: {rows} rows, {nnz} nnz, prepared in "
        f"{time.perf_counter() - t0:.1f}s")
    gen = L.minhash_cuda_init(w.dim, w.samples, seed=w.seed, devices=1 << local)

    def cast_then_calc():
        c = sp.csr_matrix(m64, copy=False)
        c.data = m64.data.astype(np.float32)
        c.indices = m64.indices.astype(np.uint32)
        c.indptr = m64.indptr.astype(np.uint32)
        return L.minhash_cuda_calc(gen, c)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ts = []
        for _ in range(args.steps):
            t = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t)
        return sum(ts) / len(ts)

    with Clocks(local) as clk:
        t_wide = timed(lambda: L.minhash_cuda_calc(gen, m64))
        t_native = timed(lambda: L.minhash_cuda_calc(gen, m32))
        t_cast = timed(cast_then_calc)
        # The same float32 matrix page-locked in place once (minhash_cuda_pin),
        # then hashed straight from its own arrays.
        t0 = time.perf_counter()
        pin = L.minhash_cuda_pin(m32, devices=1 << local)
        t_pin = time.perf_counter() - t0
        t_pinned = timed(lambda: L.minhash_cuda_calc(gen, m32))
        pinned_out = L.minhash_cuda_calc(gen, m32)
        L.minhash_cuda_unpin(pin)
    want = L.minhash_cuda_calc(gen, m32)
    exact = bool(np.array_equal(L.minhash_cuda_calc(gen, m64), want) and
                 np.array_equal(cast_then_calc(), want) and np.array_equal(pinned_out, want))
    L.minhash_cuda_fini(gen)
    evals = nnz * w.samples
    if rank == 0:
        line = {
            "metric": "WMH nnz*samples/s (scipy float64/int64 CSR through minhash_cuda_calc)",
            "value": evals / t_wide, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_wide * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded large-workload rows, generated on the device, copied to "
                    "pageable scipy arrays)",
            "config": {"workload": f"ingest: first {rows} rows of large ({nnz} nnz, {w.dim} "
                                   f"dims, {w.samples} samples), float64 data, int64 indices",
                       "rows": rows, "nnz": nnz, "dim": w.dim, "samples": w.samples},
            "float32_int32_in_place": {"value": evals / t_native, "unit": UNIT,
                                       "ms_per_step": t_native * 1e3},
            "whole_array_cast_then_calc": {"value": evals / t_cast, "unit": UNIT,
                                           "ms_per_step": t_cast * 1e3},
            "float32_pinned_in_place": {"value": evals / t_pinned, "unit": UNIT,
                                        "ms_per_step": t_pinned * 1e3,
                                        "pin_seconds_once": t_pin,
                                        "bytes_pinned": int(m32.data.nbytes + m32.indices.nbytes
                                                            + m32.indptr.nbytes)},
            "bit_exact": exact, "clocks": clk.summary(),
            "e2e": {"value": evals / t_wide, "unit": UNIT, "h2d_bytes_per_step": 8 * nnz + 4 * (rows + 1),
                    "d2h_bytes_per_step": rows * w.samples * 8},
        }
        print(json.dumps(line), flush=True)


def run_streamed(args, rank, world, local, emit=True, n_passes=None):
    """Row-streamed wide generator: 12,000,000 dims x 128 samples (18.4 GB of
    parameters resident), 10,000,000 rows hashed as 19 blocks of 524,288 rows
    plus one of 38,528, each block an mhcuda_calc call on page-locked host
    buffers (row nnz lognormal, median 200, capped at 50,000; uniform
    columns; lognormal values).  Three distinct blocks are generated and
    cycled, so host memory stays bounded; every block is copied in and its
    hashes copied out inside the timed region."""
    import torch
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import synth
    torch.cuda.set_device(local)
    w = synth.WORKLOADS["streamed"]
    block_rows = w.extra["block_rows"]
    lib = mb.capi()
    t0 = time.perf_counter()
    st = ctypes.c_int(-1)
    gen = lib.mhcuda_init(w.dim, w.samples, w.seed, 0, 1 << local, 0, ctypes.byref(st))
    assert gen, f"mhcuda_init failed: {st.value}"
    t_init = time.perf_counter() - t0

    def pin(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype)[:a.size]
        v[...] = a
        return v, t

    blocks = []
    for b in range(3):
        ip, cols, wts = synth.host_csr(w, b * block_rows, block_rows)
        (pi, t1), (pc, t2), (pw, t3) = pin(ip), pin(cols), pin(wts)
        blocks.append((pi, pc, pw, (t1, t2, t3)))
        del ip, cols, wts
    S = w.samples
    out_t = torch.empty((block_rows, S, 2), dtype=torch.int32, pin_memory=True)
    out = out_t.numpy().view(np.uint32)
    full = w.rows // block_rows
    tail = w.rows - full * block_rows
    schedule = [(k % 3, block_rows) for k in range(full)] + ([(full % 3, tail)] if tail else [])
    log(f"[rank {rank}] streamed: init {t_init:.1f}s, blocks ready in "
        f"{time.perf_counter() - t0:.1f}s; {len(schedule)} blocks")

    def run_block(k, rows):
        pi, pc, pw, _ = blocks[k]
        rc = lib.mhcuda_calc(gen, pw.ctypes.data, pc.ctypes.data, pi.ctypes.data, rows,
                             out.ctypes.data)
        assert rc == 0, rc
        return int(pi[rows]) * S

    run_block(0, block_rows)  # warm-up
    torch.cuda.synchronize()
    # `steps` passes over the 20 blocks; the median pass is reported (one pass
    # is ~1.4 s of host<->device traffic, exposed to other users of the host).
    passes = []
    with Clocks(local) as clk:
        for _ in range(max(1, n_passes or args.steps)):
            t = time.perf_counter()
            evals = sum(run_block(k, rows) for k, rows in schedule)
            passes.append(time.perf_counter() - t)
    elapsed = float(np.median(passes))
    # Device-resident rate for the same blocks (kernel only, no copies).
    pi, pc, pw, _ = blocks[0]
    nnz0 = int(pi[block_rows])
    d_ip = torch.from_numpy(pi.view(np.int32)).cuda()
    d_c = torch.from_numpy(pc.view(np.int32)).cuda()
    d_w = torch.from_numpy(pw).cuda()
    d_o = torch.empty((block_rows, S, 2), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    for _ in range(2):
        assert lib.mhcuda_calc_device(gen, d_w.data_ptr(), d_c.data_ptr(), d_ip.data_ptr(),
                                      block_rows, nnz0, d_o.data_ptr(), sptr) == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        assert lib.mhcuda_calc_device(gen, d_w.data_ptr(), d_c.data_ptr(), d_ip.data_ptr(),
                                      block_rows, nnz0, d_o.data_ptr(), sptr) == 0
    e1.record(stream)
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1) / 3
    run_block(0, block_rows)
    same = bool(np.array_equal(out, d_o.cpu().numpy().view(np.uint32)))
    lib.mhcuda_fini(gen)
    del d_ip, d_c, d_w, d_o, blocks, out_t, out
    _free_cuda()
    if True:
        nnz_total = evals // S
        line = {
            "metric": "WMH nnz*samples/s (row-streamed: 10M rows x 12M dims, 128 samples)",
            "value": evals / elapsed, "unit": UNIT, "n_gpus": world, "steps": len(schedule),
            "warmup": 1, "ms_per_step": elapsed / len(schedule) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, 3 distinct 524,288-row blocks cycled, page-locked)",
            "config": {"workload": f"streamed: {w.rows} rows in {len(schedule)} blocks of "
                                   f"{block_rows}, {w.dim} dims, {S} samples, {nnz_total} nnz",
                       "rows": w.rows, "dim": w.dim, "samples": S, "block_rows": block_rows},
            "rows_per_s": w.rows / elapsed, "seconds_total": elapsed,
            "pass_seconds": [round(x, 4) for x in passes], "generator_init_s": t_init,
            "params_gb": w.dim * 3 * S * 4 / 1e9,
            "device_resident": {"value": nnz0 * S / (dev_ms / 1e3), "unit": UNIT,
                                "ms_per_block": dev_ms},
            "streamed_equals_device_path": same, "clocks": clk.summary(),
            "e2e": {"value": evals / elapsed, "unit": UNIT,
                    "h2d_bytes_per_step": int(8 * nnz_total / len(schedule)),
                    "d2h_bytes_per_step": int(w.rows * S * 8 / len(schedule))},
        }
        if emit and rank == 0:
            print(json.dumps(line), flush=True)
        return line


def srpt_ideal(sizes, rate, load, seed):
    """Response-time percentiles (ms) of an ideal preemptive
    shortest-remaining-work-first server of `rate` evals/s, zero overheads,
    Poisson arrivals at `load` * rate, request sizes `sizes` (evals): a lower
    bound for any work-conserving scheduler of these requests at that rate."""
    import heapq
    rng = np.random.default_rng(seed)
    sizes = np.asarray(sizes, dtype=np.float64)
    n = len(sizes)
    lam = load * rate / sizes.mean()
    arr = np.cumsum(rng.exponential(1.0 / lam, n))
    t, heap, resp, i = 0.0, [], np.zeros(n), 0
    while i < n or heap:
        if not heap:
            t = max(t, arr[i])
            heapq.heappush(heap, (sizes[i] / rate, i))
            i += 1
            continue
        rem, j = heap[0]
        nxt = arr[i] if i < n else np.inf
        if t + rem <= nxt:
            t += rem
            heapq.heappop(heap)
            resp[j] = t - arr[j]
        else:
            heapq.heapreplace(heap, (rem - (nxt - t), j))
            t = nxt
            heapq.heappush(heap, (sizes[i] / rate, i))
            i += 1
    r = resp[n // 10:] * 1e3  # skip the warm-up tenth
    p50, p99, p999 = np.percentile(r, [50, 99, 99.9])
    return {"p50_ms": float(p50), "p99_ms": float(p99), "p999_ms": float(p999)}


def run_serving(args, rank, world, local, emit=True, seconds=None):
    """Serving: Poisson-arriving requests over three resident generators
    (2^20 dims / 128 samples, 2^22 / 64, 2^24 / 256; 1.6 + 3.2 + 51.5 GB of
    parameters), each request a CSR of log-uniform 1..50,000 rows with
    Zipf-tailed row nnz (median 100), through the continuous-batching server.
    First the saturated throughput ("batched peak"), then p50/p99/p99.9
    latency and throughput at fractions of it.  Request buffers are
    page-locked."""
    import threading
    import torch
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import synth
    from minhashcuda_b200.server import Server
    if rank != 0:
        return
    torch.cuda.set_device(local)
    lib = mb.capi()
    specs = [synth.WORKLOADS[k] for k in ("serving_g1", "serving_g2", "serving_g3")]
    gens, pools = [], []
    t0 = time.perf_counter()
    for w in specs:
        st = ctypes.c_int(-1)
        g = lib.mhcuda_init(w.dim, w.samples, w.seed, 0, 1 << local, 0, ctypes.byref(st))
        assert g, f"mhcuda_init({w.dim}, {w.samples}) failed: {st.value}"
        ip, cols, wts = synth.host_csr(w, 0, w.rows)

        def pin(a):
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            v = t.numpy().view(a.dtype)[:a.size]
            v[...] = a
            return v, t

        (pw, tw), (pc, tc), (pi, ti) = pin(wts), pin(cols), pin(ip)
        gens.append(g)
        pools.append({"w": pw, "c": pc, "ip": pi, "keep": (tw, tc, ti), "S": w.samples,
                      "rows": w.rows})
        del ip, cols, wts
    log(f"serving: generators and pools ready in {time.perf_counter() - t0:.1f}s")
    rng = np.random.default_rng(4)
    max_rows = 50000

    def make_req():
        gi = int(rng.integers(0, 3))
        p = pools[gi]
        rows = int(min(max_rows, max(1, np.floor(np.exp(rng.uniform(0, np.log(max_rows)))))))
        r0 = int(rng.integers(0, p["rows"] - rows + 1))
        nnz = int(p["ip"][r0 + rows]) - int(p["ip"][r0])
        return gi, r0, rows, nnz * p["S"]

    # Page-locked output rings per generator (recycled once a request is waited for).
    ring = 48
    outs = []
    for p in pools:
        t = torch.empty((ring, max_rows, p["S"], 2), dtype=torch.int32, pin_memory=True)
        outs.append((t, t.numpy().view(np.uint32)))
    free = [list(range(ring)) for _ in pools]
    free_cv = threading.Condition()

    srv = Server(hbm_budget=args.serving_budget << 30, lanes=args.serving_lanes,
                 devices=1 << local)

    def submit(req):
        gi, r0, rows, _ = req
        p = pools[gi]
        with free_cv:
            while not free[gi]:
                free_cv.wait()
            slot = free[gi].pop()
        out = outs[gi][1][slot][:rows]
        t = srv.submit_raw(gens[gi], p["w"], p["c"], p["ip"][r0:r0 + rows + 1], rows, out)
        return t, gi, slot

    def release(gi, slot):
        with free_cv:
            free[gi].append(slot)
            free_cv.notify()

    def run_closed(reqs):
        """Submits back to back; when a generator's output ring is empty the
        oldest outstanding request is waited for first (bounded window)."""
        import collections
        t = time.perf_counter()
        pend = collections.deque()
        for r in reqs:
            while not free[r[0]]:
                tk, g2, slot = pend.popleft()
                srv.wait(tk, timeout=120.0)
                release(g2, slot)
            pend.append(submit(r))
        while pend:
            tk, g2, slot = pend.popleft()
            srv.wait(tk, timeout=120.0)
            release(g2, slot)
        return time.perf_counter() - t

    run_closed([make_req() for _ in range(60)])  # warm-up
    peak_reqs = [make_req() for _ in range(400)]
    peak_t = run_closed(peak_reqs)
    peak = sum(r[3] for r in peak_reqs) / peak_t
    size_sample = [make_req()[3] for _ in range(40000)]
    mean_evals = float(np.mean(size_sample))
    log(f"serving: saturated throughput {peak:.3e} evals/s over 400 requests")

    levels = []
    for frac in args.serving_loads:
        lam = frac * peak / mean_evals
        duration = seconds or args.serving_seconds
        arrivals = np.cumsum(rng.exponential(1.0 / lam, int(lam * duration * 1.2) + 10))
        arrivals = arrivals[arrivals < duration]
        reqs = [make_req() for _ in arrivals]
        lat = []
        done_evals = [0]
        q = []
        qcv = threading.Condition()

        def waiter():
            n = 0
            while n < len(reqs):
                with qcv:
                    while not q:
                        qcv.wait()
                    tk, gi, slot, ev = q.pop(0)
                _, ms = srv.wait(tk, timeout=120.0, with_latency=True)
                release(gi, slot)
                lat.append(ms)
                done_evals[0] += ev
                n += 1

        th = threading.Thread(target=waiter)
        th.start()
        start = time.perf_counter()
        for at, r in zip(arrivals, reqs):
            delay = start + at - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tk, gi, slot = submit(r)
            with qcv:
                q.append((tk, gi, slot, r[3]))
                qcv.notify()
        th.join()
        elapsed = time.perf_counter() - start
        a = np.sort(np.array(lat))
        levels.append({"load": frac, "offered_evals_per_s": lam * mean_evals,
                       "requests": len(reqs), "evals_per_s": done_evals[0] / elapsed,
                       "p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)),
                       "p999_ms": float(np.percentile(a, 99.9)), "max_ms": float(a[-1]),
                       "srpt_ideal_at_saturated_rate": srpt_ideal(size_sample, peak, frac, 5)})
        log(f"serving: load {frac:.2f}: {levels[-1]}")

    # Each served result equals the same request hashed alone.
    exact = True
    for r in [make_req() for _ in range(12)]:
        gi, r0, rows, _ = r
        p = pools[gi]
        tk, g2, slot = submit(r)
        srv.wait(tk, timeout=120.0)
        served = outs[gi][1][slot][:rows].copy()
        release(g2, slot)
        alone = np.empty_like(served)
        assert lib.mhcuda_calc(gens[gi], p["w"].ctypes.data, p["c"].ctypes.data,
                               p["ip"][r0:].ctypes.data, rows, alone.ctypes.data) == 0
        exact &= bool(np.array_equal(served, alone))
    srv.stop()
    for g in gens:
        lib.mhcuda_fini(g)
    at80 = min(levels, key=lambda l: abs(l["load"] - 0.8))
    line = {
        "metric": "WMH serving p99 latency at 80% of saturated throughput (3 resident generators)",
        "value": at80["p99_ms"], "unit": "ms", "n_gpus": 1, "steps": len(levels), "warmup": 1,
        "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded, generated on the device, page-locked host pools)",
        "config": {"workload": "serving: generators 2^20/128, 2^22/64, 2^24/256; requests of "
                               "log-uniform 1..50000 rows, row nnz 50*(1+Zipf(2)), Poisson arrivals",
                   "lanes": args.serving_lanes, "hbm_budget_gib": args.serving_budget,
                   "seconds_per_level": seconds or args.serving_seconds},
        "saturated_evals_per_s": peak, "mean_evals_per_request": mean_evals,
        "request_evals_p50_p99": [float(x) for x in np.percentile(size_sample, [50, 99])],
        "levels": levels,
        "bit_exact_served_vs_alone": exact,
    }
    del outs, pools
    _free_cuda()
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_extras(args, rank, world, local, lib, peak, peak_kind):
    """The other configurations, measured after the large one on the same
    GPU, as sub-objects of the one JSON line (each bounded to a few seconds
    of timed work; an error in one is recorded in its place)."""
    def summary(line, keys):
        return {k: line[k] for k in keys if k in line}

    parts = {
        "roofline_uniform": lambda: extra_uniform(lib, local, peak, peak_kind),
        "same_inputs_as_reference_cuda": lambda: time_reference_cases(lib, local),
        "batched": lambda: summary(
            run_batched(args, rank, world, local, emit=False, steps=2, warmup=1),
            ["value", "unit", "ms_per_step", "config", "plain", "device_resident",
             "batched_over_plain", "bit_exact_plain_vs_batched",
             "bit_exact_plain_vs_device_batch", "rows_per_s", "e2e"]),
        "streamed": lambda: summary(
            run_streamed(args, rank, world, local, emit=False, n_passes=3),
            ["value", "unit", "config", "rows_per_s", "seconds_total", "pass_seconds",
             "device_resident", "streamed_equals_device_path", "e2e"]),
        "serving": lambda: summary(
            run_serving(args, rank, world, local, emit=False, seconds=5.0),
            ["metric", "value", "unit", "config", "saturated_evals_per_s", "levels",
             "bit_exact_served_vs_alone"]),
    }
    out = {}
    for name, fn in parts.items():
        t = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:  # recorded, the main line stands
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["bench_seconds"] = round(time.perf_counter() - t, 1)
        log(f"[rank {rank}] {name}: {time.perf_counter() - t:.1f}s")
    return out


def workload_config(w, args):
    return {"workload": f"{w.name}: {w.rows} rows x {w.dim} dims, samples {w.samples}, "
                        f"row nnz {['Poisson', 'lognormal', 'log-uniform', 'Zipf'][w.nnz_kind]}"
                        f"({w.nnz_p1:g}{', %g' % w.nnz_p2 if w.nnz_p2 else ''}), {w.cols} columns, "
                        "lognormal(0,1) values",
            "rows": w.rows, "dim": w.dim, "samples": w.samples, "seed": w.seed,
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas{args.gpus}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large",
                    choices=["large", "batched", "serving", "streamed", "ingest"])
    ap.add_argument("--serving-budget", type=int, default=24, help="server HBM budget, GiB")
    ap.add_argument("--serving-lanes", type=int, default=8)
    ap.add_argument("--serving-seconds", type=float, default=6.0)
    ap.add_argument("--serving-loads", type=float, nargs="+", default=[0.5, 0.8, 0.9])
    ap.add_argument("--rows", type=int, default=0, help="override the row count (smaller runs)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-rows", type=int, default=3000)
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="print only the large configuration (no uniform-column roofline, "
                         "batched, streamed, serving or same-input sub-objects)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="time the planner's default kernel variant instead of the one "
                         "mhcuda_autotune picks for this data before the timed region")
    args = ap.parse_args()

    rank, world, local = dist_setup()
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    if args.workload == "batched":
        return run_batched(args, rank, world, local)
    if args.workload == "serving":
        return run_serving(args, rank, world, local)
    if args.workload == "streamed":
        return run_streamed(args, rank, world, local)
    if args.workload == "ingest":
        return run_ingest(args, rank, world, local)

    import torch
    import minhashcuda_b200 as mb
    from minhashcuda_b200 import synth

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    w = synth.WORKLOADS[args.workload]
    if args.rows:
        w = synth.Workload(**{**w.__dict__, "rows": args.rows})
    lib = mb.capi()
    dev_mask = 1 << local

    # ---- generator (cuRAND, seed) and device-resident workload -------------
    status = ctypes.c_int(-1)
    t0 = time.perf_counter()
    gen = lib.mhcuda_init(w.dim, w.samples, w.seed, 0, dev_mask, 0, ctypes.byref(status))
    assert gen, f"mhcuda_init failed: {status.value}"
    stream = torch.cuda.Stream()
    # Each rank hashes its own shard: rows [rank*R, (rank+1)*R) of the seeded
    # workload (every draw is keyed by absolute row index), so N ranks hash N
    # distinct blocks of R rows (weak scaling, no data-path collective).
    row0 = rank * w.rows
    with torch.cuda.stream(stream):
        indptr, cols, weights, nnz = synth.device_csr(w, row0, w.rows, stream=stream)
    torch.cuda.synchronize()
    log(f"[rank {rank}] workload {w.name}: rows={w.rows} nnz={nnz} "
        f"generated in {time.perf_counter() - t0:.1f}s")
    R, S = w.rows, w.samples
    out = torch.empty((R, S, 2), dtype=torch.int32, device="cuda")
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def step():
        rc = lib.mhcuda_calc_device(gen, weights.data_ptr(), cols.data_ptr(), indptr.data_ptr(),
                                    R, nnz, out.data_ptr(), sptr)
        assert rc == 0, rc

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    def max_over_ranks(x):
        from minhashcuda_b200.replicas import max_over_ranks as reduce_max
        return reduce_max(x, pg, device="cuda")

    tuned = None
    if args.autotune:
        choice = (ctypes.c_uint32 * 3)()
        best = ctypes.c_double(0)
        t_tune = time.perf_counter()
        assert lib.mhcuda_autotune(gen, weights.data_ptr(), cols.data_ptr(), indptr.data_ptr(),
                                   R, nnz, out.data_ptr(), sptr, choice, ctypes.byref(best)) == 0
        tuned = {"samples_per_lane": choice[0], "min_blocks_per_sm": choice[1],
                 "items_per_resident_warp": choice[2], "best_ms": best.value,
                 "tuning_s": time.perf_counter() - t_tune}
        log(f"[rank {rank}] autotune: {tuned}")

    # ---- value: device-resident throughput ---------------------------------
    for _ in range(args.warmup):
        step()
    assert lib.mhcuda_device_status(gen) == 0, "device reported invalid CSR"
    barrier()
    lib.mhcuda_profile(gen, 1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms_total = ev0.elapsed_time(ev1)
    hash_ms = ctypes.c_double(0)
    launches = ctypes.c_uint64(0)
    assert lib.mhcuda_profile_read(gen, ctypes.byref(hash_ms), ctypes.byref(launches)) == 0
    lib.mhcuda_profile(gen, 0)
    clocks = clk.summary()
    barrier()
    ms_step = max_over_ranks(ms_total / args.steps)
    evals = nnz * S
    from minhashcuda_b200.replicas import sum_over_ranks
    job_evals = sum_over_ranks(evals, pg, device="cuda")
    value = job_evals / (ms_step / 1e3)

    hash_ms_launch = hash_ms.value / max(1, launches.value)
    peak, peak_kind = measured_peaks()
    if tuned:
        variant = f"spl{tuned['samples_per_lane']}_minb{tuned['min_blocks_per_sm']}"
    else:
        variant = f"spl{os.environ.get('MHCUDA_B200_SPL', '4')}_minb" \
                  f"{os.environ.get('MHCUDA_B200_MINB', '4')}"
    prof, prof_current = kernel_profile(variant) if w.name == "large" else (None, False)
    roofline = hash_roofline(nnz, R, S, hash_ms_launch, clocks.get("sm_mhz"), peak, peak_kind,
                             prof, prof_current)

    # ---- parity spot check + CPU baseline (rank 0) -----------------------------
    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu:
        params = [np.empty((S, w.dim), np.float32) for _ in range(3)]
        assert lib.mhcuda_retrieve_random_vars(gen, *[p.ctypes.data for p in params]) == 0
        gpu_out = out.cpu().numpy().view(np.uint32)

        def check(rows, ip, cl, wt, co):
            lnw = np.empty_like(wt)
            assert lib.mhcuda_debug_device_logf(dev_mask, wt.ctypes.data, lnw.ctypes.data,
                                                wt.size) == 0
            want = co.hash(wt, cl, ip, lnw=lnw)
            return bool(np.array_equal(want, gpu_out[:rows]))

        v, rows_s, nnz_s, dt, exact = cpu_oracle_sample(w, params, check=check)
        cores = os.cpu_count()
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"first {rows_s} rows ({nnz_s} nnz x {S} samples) of the workload, "
                         f"{dt:.2f}s on {cores} threads (C oracle, OpenMP)"}
        parity = {"rows_checked": rows_s, "bit_exact": exact}
        del params, gpu_out

    # ---- e2e through the drop-in C ABI with pinned host buffers ----------------
    e2e = None
    if not args.no_e2e:
        h_w = torch.empty(nnz, dtype=torch.float32, pin_memory=True)
        h_c = torch.empty(nnz, dtype=torch.int32, pin_memory=True)
        h_i = torch.empty(R + 1, dtype=torch.int32, pin_memory=True)
        h_o = torch.empty((R, S, 2), dtype=torch.int32, pin_memory=True)
        h_w.copy_(weights[:nnz])
        h_c.copy_(cols[:nnz])
        h_i.copy_(indptr)
        del weights, cols  # the e2e path stages its own device copy
        torch.cuda.empty_cache()

        def e2e_step():
            rc = lib.mhcuda_calc(gen, h_w.data_ptr(), h_c.data_ptr(), h_i.data_ptr(), R,
                                 h_o.data_ptr())
            assert rc == 0, rc

        for _ in range(min(args.warmup, 3)):
            e2e_step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for _ in range(args.steps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) / args.steps
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        same = bool(torch.equal(h_o.cuda(), out))
        e2e = {"value": job_evals / (e2e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 8 * nnz + 4 * (R + 1), "d2h_bytes_per_step": 8 * R * S,
               "ms_per_step": e2e_ms, "wall_ms_per_step": wall * 1e3,
               "matches_device_path": same}
        del h_w, h_c, h_i, h_o
    lib.mhcuda_fini(gen)
    weights = cols = indptr = out = None  # noqa: F841  (device memory back for the extras)
    _free_cuda()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, generated on the device)",
            "config": workload_config(w, args), "rows_per_s": R * world / (ms_step / 1e3),
            "nnz": nnz, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "parity": parity, "clocks": clocks,
            "gpu_launches": 3 * args.steps, "autotuned": tuned,
        }
        if world == 1 and args.extras:
            line.update(run_extras(args, rank, world, local, lib, peak, peak_kind))
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
