"""Seeded synthetic CSR workloads for the benchmark and the tests.

Each workload is generated on the GPU (libmhsynth.so) with every draw keyed
by the absolute row index, so any row range -- for instance the sample a CPU
baseline hashes -- can be regenerated on its own, bit for bit.

The shapes follow the benchmark configurations of the reference's workload
(synthetic stand-ins; no dataset is involved):

  small     6400 x 130, the reference's test matrix (uniform integers 0..99
            kept with probability 0.2), samples 128, generator seed 1
  large     2,000,000 x 1,000,000, row nnz ~ Poisson(1400), Zipf(1.1)
            columns without replacement, lognormal(0, 1) values, samples 128
  streamed  10,000,000 rows in blocks of 524,288 x 12,000,000 dims, row nnz
            lognormal(median 200, sigma 1.354) clipped to [1, 50000], uniform
            columns, lognormal values, samples 128
  batched   4096 matrices x 2^20 dims, rows log-uniform in [1, 4096], row nnz
            lognormal(median 64, sigma 1.5) clipped to [1, 20000], uniform
            columns, lognormal values, samples 256
  serving   three resident generators (2^20 dims / 128 samples, 2^22 / 64,
            2^24 / 256), each with a pool of 400,000 rows whose nnz is
            50 * (1 + K), P(K >= k) = 1/k (median 100, capped at 50,000);
            requests are row ranges of log-uniform length in [1, 50,000]
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import SYNTH_PATH

NNZ_POISSON, NNZ_LOGNORMAL, NNZ_LOGUNIFORM, NNZ_ZIPF = 0, 1, 2, 3


@dataclass
class Workload:
    name: str
    rows: int
    dim: int
    samples: int
    seed: int
    nnz_kind: int
    nnz_p1: float
    nnz_p2: float = 0.0
    nnz_lo: int = 0
    nnz_hi: int = 0xFFFFFFFF
    cols: str = "uniform"        # "uniform" or "zipf"
    zipf_s: float = 1.1
    extra: dict = field(default_factory=dict)


WORKLOADS = {
    "large": Workload("large", rows=2_000_000, dim=1_000_000, samples=128, seed=2,
                      nnz_kind=NNZ_POISSON, nnz_p1=1400.0, nnz_lo=0, nnz_hi=2048, cols="zipf",
                      zipf_s=1.1),
    "streamed": Workload("streamed", rows=10_000_000, dim=12_000_000, samples=128, seed=1000,
                         nnz_kind=NNZ_LOGNORMAL, nnz_p1=200.0, nnz_p2=1.354, nnz_lo=1,
                         nnz_hi=50000, extra={"block_rows": 524_288}),
    "serving_g1": Workload("serving_g1", rows=400_000, dim=1 << 20, samples=128, seed=41,
                           nnz_kind=NNZ_ZIPF, nnz_p1=50.0, nnz_p2=2.0, nnz_lo=1, nnz_hi=50000),
    "serving_g2": Workload("serving_g2", rows=400_000, dim=1 << 22, samples=64, seed=42,
                           nnz_kind=NNZ_ZIPF, nnz_p1=50.0, nnz_p2=2.0, nnz_lo=1, nnz_hi=50000),
    "serving_g3": Workload("serving_g3", rows=400_000, dim=1 << 24, samples=256, seed=43,
                           nnz_kind=NNZ_ZIPF, nnz_p1=50.0, nnz_p2=2.0, nnz_lo=1, nnz_hi=50000),
    "batched": Workload("batched", rows=0, dim=1 << 20, samples=256, seed=3,
                        nnz_kind=NNZ_LOGNORMAL, nnz_p1=64.0, nnz_p2=1.5, nnz_lo=1,
                        nnz_hi=20000, extra={"matrices": 4096, "max_rows": 4096}),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(SYNTH_PATH)
        P, U32, U64, D = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double
        L.mhs_row_nnz.argtypes = [U32, U64, ctypes.c_int, D, D, U32, U32, U64, P, P]
        L.mhs_lognormal_values.argtypes = [U32, U64, P, D, D, U64, P, P]
        L.mhs_zipf_cols.argtypes = [U32, U64, P, U32, D, U64, P, P]
        L.mhs_uniform_cols.argtypes = [U32, U64, P, U32, U64, P, P]
        for f in (L.mhs_row_nnz, L.mhs_lognormal_values, L.mhs_zipf_cols, L.mhs_uniform_cols):
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _u32(t):
    """int64 tensor of values < 2^32 -> int32 tensor holding the same bits."""
    import torch
    return torch.where(t >= 2**31, t - 2**32, t).to(torch.int32)


def device_csr(w: Workload, row0: int, rows: int, device="cuda", stream=None):
    """Rows [row0, row0+rows) of workload `w` on the device.

    Returns (indptr, cols, weights, nnz) with indptr/cols int32 tensors that
    hold uint32 bit patterns (indptr relative, starting at 0)."""
    import torch
    L = lib()
    st = ctypes.c_void_p(stream.cuda_stream if stream is not None
                         else torch.cuda.current_stream(device).cuda_stream)
    lens = torch.empty(rows, dtype=torch.int32, device=device)
    rc = L.mhs_row_nnz(rows, row0, w.nnz_kind, w.nnz_p1, w.nnz_p2, w.nnz_lo,
                       min(w.nnz_hi, w.dim), w.seed * 7 + 1, lens.data_ptr(), st)
    assert rc == 0, rc
    indptr64 = torch.zeros(rows + 1, dtype=torch.int64, device=device)
    torch.cumsum(lens.to(torch.int64), 0, out=indptr64[1:])
    nnz = int(indptr64[-1])
    assert nnz < 2**32, "one launch addresses fewer than 2^32 entries"
    indptr = _u32(indptr64)
    del lens, indptr64
    cols = torch.empty(max(nnz, 1), dtype=torch.int32, device=device)
    weights = torch.empty(max(nnz, 1), dtype=torch.float32, device=device)
    if w.cols == "zipf":
        rc = L.mhs_zipf_cols(rows, row0, indptr.data_ptr(), w.dim, w.zipf_s, w.seed * 7 + 2,
                             cols.data_ptr(), st)
    else:
        rc = L.mhs_uniform_cols(rows, row0, indptr.data_ptr(), w.dim, w.seed * 7 + 2,
                                cols.data_ptr(), st)
    assert rc == 0, f"column generator failed ({rc})"
    rc = L.mhs_lognormal_values(rows, row0, indptr.data_ptr(), 0.0, 1.0, w.seed * 7 + 3,
                                weights.data_ptr(), st)
    assert rc == 0, rc
    return indptr, cols, weights, nnz


def host_csr(w: Workload, row0: int, rows: int, device="cuda"):
    """The same rows as numpy arrays (indptr/cols uint32, weights float32)."""
    indptr, cols, weights, nnz = device_csr(w, row0, rows, device)
    return (indptr.cpu().numpy().view(np.uint32), cols[:nnz].cpu().numpy().view(np.uint32),
            weights[:nnz].cpu().numpy())


def small_csr(seed: int = 1):
    """The small configuration's 6400 x 130 float32 CSR: uniform integers
    0..99, each kept where a second uniform integer 0..4 is >= 4 (~80% zeros),
    drawn with numpy's legacy RandomState(seed) in that order (the reference
    tests' matrix, test.py:35-39 / 93-97).  Returns (indptr, cols, weights) as
    uint32 / uint32 / float32 numpy arrays."""
    rng = np.random.RandomState(seed)
    data = rng.randint(0, 100, (6400, 130))
    mask = rng.randint(0, 5, data.shape)
    data = (data * (mask >= 4)).astype(np.float32)
    nz = data != 0
    indptr = np.zeros(data.shape[0] + 1, np.uint32)
    np.cumsum(nz.sum(axis=1), out=indptr[1:])
    cols = np.nonzero(nz)[1].astype(np.uint32)
    return indptr, cols, data[nz].astype(np.float32)


def batched_shapes(w: Workload):
    """Row counts of the batched workload's matrices: floor(exp(U(0, ln 4096)))
    clipped to [1, 4096], seeded."""
    rng = np.random.default_rng(w.seed)
    m, mx = w.extra["matrices"], w.extra["max_rows"]
    r = np.floor(np.exp(rng.uniform(0.0, math.log(mx), m))).astype(np.int64)
    return np.clip(r, 1, mx)
