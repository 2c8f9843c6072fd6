"""Batched CSR -> Sliced-ELL conversion with nnz bucket plans over many uneven
partitions (cs_b200_batch_sliced_*): one persistent launch per wave from a
device work queue, replayed from a CUDA graph, tiles from the autotuner."""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _abi
from .device import CSR, SlicedELL, ptr, stream_handle

ARENA_ALIGN = 256


def _align(x: int, a: int = ARENA_ALIGN) -> int:
    return (x + a - 1) // a * a


def block_bytes(slice_count: int, total_slots: int) -> int:
    """Arena bytes of one converted partition: header arrays, columns, values."""
    return _align((3 * slice_count + 1) * 4) + _align(total_slots * 4) + _align(total_slots * 2)


def part_bounds(parts: list[CSR], candidates, stream=None) -> list[int]:
    """Per partition, the arena bytes of its block at its most padded candidate height."""
    lib = _abi.load()
    bounds = []
    cand = (_abi.u32 * len(candidates))(*candidates)
    out = torch.zeros(len(candidates), dtype=torch.int64, device="cuda")
    for p in parts:
        if p.rows == 0:
            bounds.append(0)
            continue
        out.zero_()
        v = p.view()
        _abi.check(lib.cs_b200_sliced_ell_candidates(C.byref(v), cand, len(candidates), ptr(out),
                                                     stream_handle(stream)), "sliced candidates")
        padded = out.cpu().tolist()
        worst = 0
        for h, slots in zip(candidates, padded):
            hh = max(1, min(h, p.rows))
            worst = max(worst, block_bytes((p.rows + hh - 1) // hh, int(slots)))
        bounds.append(worst)
    return bounds


def arena_bound(parts: list[CSR], candidates, stream=None) -> int:
    """Arena bytes that hold every partition at its most padded candidate height."""
    return max(sum(part_bounds(parts, candidates, stream)), ARENA_ALIGN)


@dataclass
class PartResult:
    status: int
    slice_rows: int
    slice_count: int
    total_slots: int
    score: float
    plan_status: int
    sliced: SlicedELL | None
    plan: dict | None


class BatchSlicedConverter:
    """Holds the plan (queue, descriptors, graph), the plan outputs and the arena."""

    def __init__(self, parts: list[CSR], candidates=(16, 32, 64), bucket_count: int = 16, with_plan: bool = True,
                 arena_bytes: int | None = None, tiles: dict | None = None, stream=None):
        self.lib = _abi.load()
        self.parts = parts
        self.candidates = tuple(int(c) for c in candidates)
        self.stream = stream
        if arena_bytes is None:
            arena_bytes = arena_bound(parts, self.candidates, stream)
        self.arena = torch.empty(_align(arena_bytes), dtype=torch.uint8, device="cuda")
        self.plan_out = []
        arr = (_abi.BatchPart * max(len(parts), 1))()
        for i, p in enumerate(parts):
            arr[i].src = p.view()
            arr[i].bucket_count = bucket_count
            if with_plan:
                b = 1 if p.rows == 0 else max(1, min(bucket_count, p.rows)) + 1
                o = {"nnz": torch.empty(max(p.rows, 1), dtype=torch.int32, device="cuda"),
                     "sorted": torch.empty(max(p.rows, 1), dtype=torch.int32, device="cuda"),
                     "order": torch.empty(max(p.rows, 1), dtype=torch.int32, device="cuda"),
                     "bucket_offsets": torch.empty(b, dtype=torch.int32, device="cuda"),
                     "pow2_bins": torch.empty(34, dtype=torch.int32, device="cuda")}
                self.plan_out.append(o)
                arr[i].d_major_nnz = o["nnz"].data_ptr()
                arr[i].d_sorted_nnz = o["sorted"].data_ptr()
                arr[i].d_order = o["order"].data_ptr()
                arr[i].d_bucket_offsets = o["bucket_offsets"].data_ptr()
                arr[i].d_pow2_offsets = o["pow2_bins"].data_ptr()
            else:
                self.plan_out.append(None)
        self._parts_c = arr
        cand = (_abi.u32 * len(self.candidates))(*self.candidates)
        t = None
        if tiles is not None:
            t = _abi.BatchTiles(tiles["layout_rows"], tiles["emit_rows"], tiles["emit_lanes"],
                                tiles.get("ctas_per_sm", 0))
        h = C.c_void_p()
        _abi.check(self.lib.cs_b200_batch_sliced_create(arr, len(parts), cand, len(self.candidates),
                                                        self.arena.data_ptr(), self.arena.numel(),
                                                        C.byref(t) if t is not None else None, C.byref(h)),
                   "batch_sliced_create")
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.cs_b200_batch_sliced_destroy(h)
            self.handle = None

    def tiles(self) -> dict:
        t = _abi.BatchTiles()
        g, n = _abi.u32(), _abi.u32()
        _abi.check(self.lib.cs_b200_batch_sliced_tiles(self.handle, C.byref(t), C.byref(g), C.byref(n)), "tiles")
        return {"layout_rows": t.layout_rows, "emit_rows": t.emit_rows, "emit_lanes": t.emit_lanes,
                "ctas_per_sm": t.ctas_per_sm, "grid": g.value, "items": n.value}

    def autotune(self) -> dict:
        t = _abi.BatchTiles()
        _abi.check(self.lib.cs_b200_batch_sliced_autotune(self.handle, stream_handle(self.stream), C.byref(t)),
                   "batch_sliced_autotune")
        return self.tiles()

    def run(self) -> None:
        _abi.check(self.lib.cs_b200_batch_sliced_run(self.handle, stream_handle(self.stream)), "batch_sliced_run")

    def next_wave(self, arena: torch.Tensor | None = None) -> int:
        if arena is not None:
            self.arena = arena
        n = _abi.u32()
        _abi.check(self.lib.cs_b200_batch_sliced_next_wave(self.handle, self.arena.data_ptr(), self.arena.numel(),
                                                           C.byref(n)), "batch_sliced_next_wave")
        return n.value

    def reset(self, arena: torch.Tensor | None = None) -> None:
        """All partitions form the next wave again."""
        if arena is not None:
            self.arena = arena
        _abi.check(self.lib.cs_b200_batch_sliced_reset(self.handle, self.arena.data_ptr(), self.arena.numel()),
                   "batch_sliced_reset")

    def raw_results(self):
        res = (_abi.BatchSlicedResult * max(len(self.parts), 1))()
        d, e = _abi.u32(), _abi.u32()
        _abi.check(self.lib.cs_b200_batch_sliced_results(self.handle, res, C.byref(d), C.byref(e),
                                                         stream_handle(self.stream)), "batch_sliced_results")
        return res, d.value, e.value

    def results(self, arena: torch.Tensor | None = None) -> tuple[list[PartResult], int, int]:
        """Per-partition results; Sliced-ELL tensors are views into `arena` (the
        arena of the wave that converted them; default the current one)."""
        res, deferred, err = self.raw_results()
        a = self.arena if arena is None else arena
        out = []
        for i, p in enumerate(self.parts):
            r = res[i]
            sl = None
            if r.status == 0 and r.arena_offset != 0xFFFFFFFFFFFFFFFF and p.rows > 0:
                S, n = r.slice_count, r.total_slots
                base = r.arena_offset
                hdr = _align((3 * S + 1) * 4)
                cb = _align(n * 4)
                words = a[base:base + (3 * S + 1) * 4].view(torch.int32)
                sl = SlicedELL(p.rows, p.cols, p.nnz, r.slice_rows, words[:S + 1], words[S + 1:2 * S + 1],
                               words[2 * S + 1:3 * S + 1], a[base + hdr:base + hdr + n * 4].view(torch.int32),
                               a[base + hdr + cb:base + hdr + cb + n * 2].view(torch.float16))
            out.append(PartResult(r.status, r.slice_rows, r.slice_count, r.total_slots, r.score, r.plan_status, sl,
                                  self.plan_out[i]))
        return out, deferred, err
