"""Serving masked grouped moments over staged Blocked-ELL partitions
(cs_b200_serve_*): a device-resident persistent request loop with HBM-budget
admission and continuous batching."""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi
from .device import BlockedELL

TWOSUM_F64_COMBINE = 2


class Request:
    """Host-side request: numpy inputs (copied into pinned buffers) and pinned outputs."""

    def __init__(self, group_count: int, row_keep: np.ndarray | None, row_labels: np.ndarray | None,
                 feature_keep: np.ndarray | None, cols: int, scheme: int = TWOSUM_F64_COMBINE, ddof: int = 1,
                 want_moments: bool = True):
        self.G = int(group_count)
        self.cols = cols

        def pin(a, dtype):
            if a is None:
                return None
            t = torch.from_numpy(np.ascontiguousarray(a).view(dtype)).pin_memory()
            return t

        self.row_keep = pin(row_keep.astype(np.uint8) if row_keep is not None else None, np.uint8)
        self.row_labels = pin(row_labels.astype(np.uint32).view(np.int32) if row_labels is not None else None,
                              np.int32)
        self.feature_keep = pin(feature_keep.astype(np.uint8) if feature_keep is not None else None, np.uint8)
        shape = (self.G, cols)
        self.sum = torch.empty(shape, dtype=torch.float32).pin_memory()
        self.sumsq = torch.empty(shape, dtype=torch.float32).pin_memory()
        self.mean = torch.empty(shape, dtype=torch.float32).pin_memory() if want_moments else None
        self.var = torch.empty(shape, dtype=torch.float32).pin_memory() if want_moments else None
        self.group_rows = torch.empty(self.G, dtype=torch.int32).pin_memory()
        self.c = _abi.ServeRequest(self.G, scheme, ddof, 0, _p(self.row_keep), _p(self.row_labels),
                                   _p(self.feature_keep), _p(self.sum), _p(self.sumsq), _p(self.mean), _p(self.var),
                                   _p(self.group_rows))

    def results(self) -> dict:
        out = {"sum": self.sum.numpy().copy(), "sumsq": self.sumsq.numpy().copy(),
               "group_rows": self.group_rows.numpy().view(np.uint32).copy()}
        if self.mean is not None:
            out["mean"] = self.mean.numpy().copy()
            out["var"] = self.var.numpy().copy()
        return out


def _p(t):
    return None if t is None else t.data_ptr()


class Server:
    def __init__(self, parts: list[BlockedELL], scratch_budget_bytes: int = 16 << 30, max_inflight: int = 32,
                 chunk_rows: int = 0, idle_exit_us: int = 0, ctas_per_sm: int = 0):
        self.lib = _abi.load()
        self.parts = parts
        views = (_abi.BlockedEllView * len(parts))(*[p.view() for p in parts])
        self._views = views
        cfg = _abi.ServeConfig(scratch_budget_bytes, max_inflight, chunk_rows, idle_exit_us, ctas_per_sm)
        h = C.c_void_p()
        _abi.check(self.lib.cs_b200_serve_open(views, len(parts), C.byref(cfg), C.byref(h)), "serve_open")
        self.handle = h
        self.total_rows = sum(p.rows for p in parts)
        self.cols = parts[0].cols

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.cs_b200_serve_close(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def submit(self, req: Request) -> int:
        t = _abi.u64()
        _abi.check(self.lib.cs_b200_serve_submit(self.handle, C.byref(req.c), C.byref(t)), "serve_submit")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 30000) -> float:
        ms = C.c_double()
        _abi.check(self.lib.cs_b200_serve_wait(self.handle, ticket, timeout_ms, C.byref(ms)), "serve_wait")
        self.lib.cs_b200_serve_release(self.handle, ticket)
        return ms.value

    def stats(self) -> dict:
        st = _abi.ServeStats()
        _abi.check(self.lib.cs_b200_serve_stats(self.handle, C.byref(st)), "serve_stats")
        out = {k: getattr(st, k) for k, _ in _abi.ServeStats._fields_ if k not in ("pad", "items", "item_ns")}
        kinds = ["none", "start", "hist", "scan", "scatter", "acc", "combine", "other"]
        out["items"] = {kinds[k]: int(st.items[k]) for k in range(1, 7)}
        out["item_ms"] = {kinds[k]: st.item_ns[k] / 1e6 for k in range(1, 7)}
        return out

    def run_trace(self, requests: list[Request], req_index, arrival_s):
        """Open-loop arrivals; returns (latency ms [n], makespan s, phase ms [n, 4]: admitted,
        started, device done, results on the host -- each measured from submit)."""
        n = len(req_index)
        arr = (_abi.ServeRequest * len(requests))(*[r.c for r in requests])
        idx = (_abi.u32 * n)(*[int(i) for i in req_index])
        at = (C.c_double * n)(*[float(a) for a in arrival_s])
        lat = (C.c_double * n)()
        ph = (C.c_double * (4 * n))()
        mk = C.c_double()
        _abi.check(self.lib.cs_b200_serve_run_trace(self.handle, arr, idx, at, n, lat, C.byref(mk), ph), "run_trace")
        return (np.frombuffer(lat, dtype=np.float64).copy(), mk.value,
                np.frombuffer(ph, dtype=np.float64).reshape(n, 4).copy())
