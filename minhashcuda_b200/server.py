"""Python handle on the continuous-batching server (mhcuda_server_* in
include/minhashcuda_b200.h).

    srv = Server(hbm_budget=8 << 30, lanes=8)
    t = srv.submit(gen, csr)          # gen: handle from libMHCUDA.minhash_cuda_init
    hashes = srv.wait(t)              # (rows, samples, 2) uint32, as minhash_cuda_calc
    srv.stop()

The server keeps the request's input arrays and its output array alive until
`wait` returns.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import MHCUDAError, RUNTIME_ERROR, capi, check


class Server:
    def __init__(self, hbm_budget: int = 8 << 30, lanes: int = 8, devices: int = 0,
                 verbosity: int = 0):
        """Starts a server on one device.  Two of the `lanes` are kept for small
        requests (at most lanes - 2 large batches are out at once); the device
        memory used is `hbm_budget` bytes, split between the lanes."""
        self._lib = capi()
        status = ctypes.c_int(-1)
        self._h = self._lib.mhcuda_server_start(devices, int(hbm_budget), lanes, verbosity,
                                                ctypes.byref(status))
        if not self._h:
            raise MHCUDAError("mhcuda_server_start", status.value)
        self._live = {}

    def submit(self, gen: int, matrix, out: np.ndarray | None = None) -> int:
        """Queues the hashing of a scipy CSR matrix against generator `gen`."""
        samples = self._lib.mhcuda_get_parameters(ctypes.c_void_p(gen)).samples
        data = np.ascontiguousarray(matrix.data, dtype=np.float32)
        idx = np.ascontiguousarray(matrix.indices, dtype=np.uint32)
        ptr = np.ascontiguousarray(matrix.indptr, dtype=np.uint32)
        rows = len(ptr) - 1
        if out is None:
            out = np.empty((rows, samples, 2), dtype=np.uint32)
        return self.submit_raw(gen, data, idx, ptr, rows, out)

    def submit_raw(self, gen: int, data, idx, ptr, rows: int, out: np.ndarray) -> int:
        ticket = ctypes.c_uint64(0)
        check("mhcuda_server_submit", self._lib.mhcuda_server_submit(
            self._h, ctypes.c_void_p(gen), data.ctypes.data, idx.ctypes.data, ptr.ctypes.data,
            rows, out.ctypes.data, ctypes.byref(ticket)))
        self._live[ticket.value] = (data, idx, ptr, out)
        return ticket.value

    def done(self, ticket: int) -> bool:
        flag = ctypes.c_int(0)
        check("mhcuda_server_poll", self._lib.mhcuda_server_poll(self._h, ticket,
                                                                ctypes.byref(flag)))
        return bool(flag.value)

    def wait(self, ticket: int, timeout: float = 600.0, with_latency: bool = False):
        lat = ctypes.c_double(0.0)
        rc = self._lib.mhcuda_server_wait(self._h, ticket, timeout, ctypes.byref(lat))
        keep = self._live.pop(ticket, None)
        check("mhcuda_server_wait", rc)
        out = keep[3] if keep else None
        return (out, lat.value) if with_latency else out

    def cancel(self, ticket: int) -> bool:
        """True if the request was cancelled (wait() then raises), False if it
        had already finished (wait() returns its hashes)."""
        return self._lib.mhcuda_server_cancel(self._h, ticket) == 0

    def stats(self, reset: bool = False) -> dict:
        n = ctypes.c_uint64(0)
        p50, p99, p999, eps = (ctypes.c_double(0) for _ in range(4))
        check("mhcuda_server_stats", self._lib.mhcuda_server_stats(
            self._h, int(reset), ctypes.byref(n), ctypes.byref(p50), ctypes.byref(p99),
            ctypes.byref(p999), ctypes.byref(eps)))
        return {"completed": n.value, "p50_ms": p50.value, "p99_ms": p99.value,
                "p999_ms": p999.value, "evals_per_s": eps.value}

    def stop(self) -> None:
        if self._h:
            self._lib.mhcuda_server_stop(self._h)
            self._h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


__all__ = ["Server", "RUNTIME_ERROR"]
