"""Request server (rs_server_*): continuous batching of encode and reconstruct requests.

A request is one stripe: k data + m parity rows of `row_len` bytes stored back to back
(data first), in host memory (staged through the server's device arena) or in device
memory (a CUDA tensor or device pointer the caller keeps alive until completion).
`submit` never blocks on the device; `poll` returns completions with host timestamps
(submit, admit, done) so a caller can compute queueing and service latency.
"""
import ctypes

import numpy as np

from . import _lib
from .coder import ENCODE, RECONSTRUCT, RECONSTRUCT_DATA, _check, _dev_ptr  # noqa: F401


class Request(ctypes.Structure):
    _fields_ = [("field", ctypes.c_int), ("op", ctypes.c_int), ("data_shards", ctypes.c_size_t),
                ("parity_shards", ctypes.c_size_t), ("row_len", ctypes.c_size_t), ("rows", ctypes.c_void_p),
                ("rows_on_host", ctypes.c_int), ("present", ctypes.POINTER(ctypes.c_uint8)),
                ("tag", ctypes.c_uint64)]


class Completion(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("status", ctypes.c_int), ("group_size", ctypes.c_uint32),
                ("submit_ns", ctypes.c_uint64), ("admit_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64),
                ("bytes", ctypes.c_uint64)]


class Config(ctypes.Structure):
    _fields_ = [("arena_bytes", ctypes.c_size_t), ("pinned_bytes", ctypes.c_size_t), ("slots", ctypes.c_int),
                ("streams", ctypes.c_int), ("max_batch", ctypes.c_int), ("lookahead", ctypes.c_int),
                ("model", ctypes.c_void_p)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "completed", "rejected", "groups", "launches",
                                               "merged", "bytes", "table_builds", "table_hits", "evictions")] + \
               [(n, ctypes.c_size_t) for n in ("arena_bytes", "arena_used", "arena_peak", "queued", "in_flight",
                                               "resident_tables")]


class Server:
    """rs_server_create with the given limits (0 = library default)."""

    def __init__(self, arena_bytes=1 << 30, slots=64, streams=4, max_batch=64, lookahead=0, pinned_bytes=0,
                 model=None):
        self._L = _lib.load()
        # model: a tuner.CostModel choosing FFT launch shapes (kept alive with the server).
        self._model = model
        cfg = Config(arena_bytes, pinned_bytes, slots, streams, max_batch, lookahead,
                     model._h.value if model is not None else None)
        h = ctypes.c_void_p()
        _check(self._L.rs_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}  # tag -> objects that must outlive the request

    def submit(self, requests):
        """requests: dicts with field, op, k, m, row_len, rows (numpy array for host
        memory, CUDA tensor / int pointer for device memory), present (reconstruct),
        tag. Returns the per-request statuses (0 = queued)."""
        n = len(requests)
        arr = (Request * max(n, 1))()
        for i, r in enumerate(requests):
            rows = r["rows"]
            on_host = isinstance(rows, np.ndarray)
            keep = [rows]
            arr[i].field = r.get("field", 8)
            arr[i].op = r.get("op", ENCODE)
            arr[i].data_shards = r["k"]
            arr[i].parity_shards = r["m"]
            arr[i].row_len = r["row_len"]
            arr[i].rows = rows.ctypes.data if on_host else _dev_ptr(rows)
            arr[i].rows_on_host = int(on_host)
            if r.get("present") is not None:
                f = np.ascontiguousarray(r["present"], dtype=np.uint8)
                keep.append(f)
                arr[i].present = f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
            arr[i].tag = r["tag"]
            self._keep[r["tag"]] = keep
        st = (ctypes.c_int * max(n, 1))()
        _check(self._L.rs_server_submit(self._h, arr, n, st))
        out = list(st)[:n]
        for r, s in zip(requests, out):
            if s:
                self._keep.pop(r["tag"], None)
        return out

    def poll(self, cap=1024, timeout_ms=0):
        arr = (Completion * cap)()
        n = ctypes.c_size_t()
        _check(self._L.rs_server_poll(self._h, arr, cap, ctypes.byref(n), timeout_ms))
        out = []
        for i in range(n.value):
            c = arr[i]
            self._keep.pop(c.tag, None)
            out.append({"tag": c.tag, "status": c.status, "group_size": c.group_size, "submit_ns": c.submit_ns,
                        "admit_ns": c.admit_ns, "done_ns": c.done_ns, "bytes": c.bytes})
        return out

    def wait(self, count, timeout_ms=60000):
        """Polls until `count` completions arrived (raises after timeout_ms of silence)."""
        got = []
        while len(got) < count:
            batch = self.poll(timeout_ms=timeout_ms)
            if not batch:
                raise TimeoutError("server returned %d of %d completions" % (len(got), count))
            got.extend(batch)
        return got

    def set_fft_route(self, k, log2_bytes, route):
        _check(self._L.rs_server_set_fft_route(self._h, k, log2_bytes, route))

    def stats(self):
        s = Stats()
        _check(self._L.rs_server_stats_get(self._h, ctypes.byref(s)))
        return {n: getattr(s, n) for n, _ in Stats._fields_}

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.rs_server_free(h)
            self._h = None
        self._keep = {}

    def __del__(self):
        self.close()
