"""Device-resident formats over torch tensors and the conversion launchers.

Mirrors the reference's device views (include/CellShard/runtime/device/
sharded_device.cuh:67-98): u32 arrays are held as torch.int32 tensors (same
bits) and fp16 values as torch.float16.  Every function here calls the C ABI
of libcellshard_b200.so; nothing computes on the host.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _abi

COMPRESSED_BY_ROW = 0
COMPRESSED_BY_COL = 1
INVALID_COL = 0xFFFFFFFF


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    return t.data_ptr() if t.numel() > 0 else None


def u32(t) -> torch.Tensor:
    """int32 view of a uint32 array (numpy / tensor), moved to the current device."""
    if isinstance(t, torch.Tensor):
        return t if t.dtype == torch.int32 else t.to(torch.int32)
    import numpy as np

    a = np.ascontiguousarray(t, dtype=np.uint32).view(np.int32)
    return torch.from_numpy(a.copy()).cuda()


@dataclass
class CSR:
    rows: int
    cols: int
    ptr: torch.Tensor  # int32 [major + 1]
    idx: torch.Tensor  # int32 [nnz]
    val: torch.Tensor  # float16 [nnz]
    axis: int = COMPRESSED_BY_ROW

    @property
    def nnz(self) -> int:
        return int(self.idx.numel())

    def view(self) -> _abi.CompressedView:
        v = _abi.CompressedView()
        v.rows, v.cols, v.nnz, v.axis = self.rows, self.cols, self.nnz, self.axis
        v.majorPtr, v.minorIdx, v.val = ptr(self.ptr), ptr(self.idx), ptr(self.val)
        return v


@dataclass
class BlockedELL:
    rows: int
    cols: int
    block_size: int
    ell_cols: int
    bci: torch.Tensor  # int32 [row_blocks * ell_width]
    val: torch.Tensor  # float16 [rows * ell_cols]
    nnz: int = 0

    @property
    def row_blocks(self) -> int:
        return (self.rows + self.block_size - 1) // self.block_size

    @property
    def ell_width(self) -> int:
        return self.ell_cols // self.block_size if self.block_size else 0

    def view(self) -> _abi.BlockedEllView:
        v = _abi.BlockedEllView()
        v.rows, v.cols, v.nnz, v.block_size, v.ell_cols = self.rows, self.cols, self.nnz, self.block_size, self.ell_cols
        v.blockColIdx, v.val = ptr(self.bci), ptr(self.val)
        return v


@dataclass
class SlicedELL:
    rows: int
    cols: int
    nnz: int
    slice_rows: int
    slice_row_offsets: torch.Tensor  # int32 [S + 1]
    slice_widths: torch.Tensor       # int32 [S]
    slice_slot_offsets: torch.Tensor # int32 [S]
    col_idx: torch.Tensor            # int32 [total_slots]
    val: torch.Tensor                # float16 [total_slots]

    @property
    def slice_count(self) -> int:
        return int(self.slice_widths.numel())

    def view(self) -> _abi.SlicedEllView:
        v = _abi.SlicedEllView()
        v.rows, v.cols, v.nnz, v.slice_count, v.slice_rows = (self.rows, self.cols, self.nnz, self.slice_count,
                                                              self.slice_rows)
        v.slice_row_offsets, v.slice_widths = ptr(self.slice_row_offsets), ptr(self.slice_widths)
        v.slice_slot_offsets, v.col_idx, v.val = ptr(self.slice_slot_offsets), ptr(self.col_idx), ptr(self.val)
        return v


def _scratch(nbytes: int) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device="cuda")


def blocked_ell_shape(csr: CSR, block_size: int, keep_bitmaps: bool = True, stream=None):
    """Shape pass; returns (ell_width, total_blocks, scratch, status) (synchronises)."""
    lib = _abi.load()
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_blocked_ell_scratch_bytes(csr.rows, csr.cols, block_size, C.byref(nbytes)), "scratch")
    scratch = _scratch(nbytes.value) if keep_bitmaps else None
    shape = torch.zeros(2, dtype=torch.int64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    v = csr.view()
    _abi.check(lib.cs_b200_blocked_ell_shape(C.byref(v), block_size, ptr(shape), ptr(scratch),
                                             nbytes.value if keep_bitmaps else 0, ptr(status), stream_handle(stream)),
               "blocked_ell_shape")
    sh = shape.cpu()
    return int(sh[0]), int(sh[1]), scratch, status


def blocked_ell_from_csr(csr: CSR, block_size: int, stream=None, check_status: bool = True) -> BlockedELL:
    """Device CSR -> device Blocked-ELL (convert::blocked_ell_from_compressed on the GPU)."""
    lib = _abi.load()
    width, _total, scratch, status = blocked_ell_shape(csr, block_size, True, stream)
    rb = (csr.rows + block_size - 1) // block_size
    ell_cols = width * block_size
    out = BlockedELL(csr.rows, csr.cols, block_size, ell_cols,
                     torch.empty(rb * width, dtype=torch.int32, device="cuda"),
                     torch.empty(csr.rows * ell_cols, dtype=torch.float16, device="cuda"), 0)
    nnz = torch.zeros(1, dtype=torch.int32, device="cuda")
    v, dv = csr.view(), out.view()
    _abi.check(lib.cs_b200_blocked_ell_emit(C.byref(v), C.byref(dv), ptr(nnz), ptr(scratch), scratch.numel(),
                                            ptr(status), stream_handle(stream)), "blocked_ell_emit")
    out.nnz = int(nnz.cpu().view(torch.int32)[0]) & 0xFFFFFFFF
    if check_status:
        st = int(status.cpu()[0])
        if st:
            raise _abi.CellShardError(f"blocked_ell conversion flagged invalid input (status 0x{st:x})")
    return out


def sliced_ell_from_csr(csr: CSR, slice_rows: int, stream=None) -> SlicedELL:
    """Device CSR -> device Sliced-ELL (convert::sliced_ell_from_compressed on the GPU).
    Synchronises once to size the slot arrays."""
    lib = _abi.load()
    rows = csr.rows
    h = max(1, min(slice_rows, rows)) if rows else 0
    S = (rows + h - 1) // h if rows else 0
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_sliced_ell_scratch_bytes(rows, slice_rows, C.byref(nbytes)), "sliced scratch")
    scratch = _scratch(nbytes.value)
    offs = torch.empty(S + 1, dtype=torch.int32, device="cuda")
    widths = torch.empty(max(S, 1), dtype=torch.int32, device="cuda")
    slots = torch.empty(max(S, 1), dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int64, device="cuda")
    v = csr.view()
    s = stream_handle(stream)
    _abi.check(lib.cs_b200_sliced_ell_layout(C.byref(v), slice_rows, ptr(offs), ptr(widths), ptr(slots), ptr(total),
                                             ptr(scratch), nbytes.value, s), "sliced_ell_layout")
    n_slots = int(total.item())
    out = SlicedELL(rows, csr.cols, csr.nnz, h, offs, widths[:S], slots[:S],
                    torch.empty(n_slots, dtype=torch.int32, device="cuda"),
                    torch.empty(n_slots, dtype=torch.float16, device="cuda"))
    dv = out.view()
    _abi.check(lib.cs_b200_sliced_ell_emit(C.byref(v), C.byref(dv), s), "sliced_ell_emit")
    return out


def blocked_ell_row_ptr(bell: BlockedELL, stream=None) -> torch.Tensor:
    """Row pointers of a device Blocked-ELL's live entries (count_blocked_ell_row_nnz_,
    src/convert/sliced_ell_from_blocked_ell.cuh:36-62, prefix-summed on the GPU)."""
    lib = _abi.load()
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_blocked_ell_row_ptr_scratch_bytes(bell.rows, C.byref(nbytes)), "row_ptr scratch")
    scratch = _scratch(nbytes.value)
    rp = torch.empty(bell.rows + 1, dtype=torch.int32, device="cuda")
    v = bell.view()
    _abi.check(lib.cs_b200_blocked_ell_row_ptr(C.byref(v), ptr(rp), ptr(scratch), nbytes.value, stream_handle(stream)),
               "blocked_ell_row_ptr")
    return rp


def sliced_ell_from_blocked_ell(bell: BlockedELL, slice_rows: int, stream=None) -> SlicedELL:
    """Device Blocked-ELL -> device Sliced-ELL (convert::sliced_ell_from_blocked_ell on the
    GPU): live-entry row pointers, the CSR layout pass over them, then the emit.
    Synchronises once to size the slot arrays."""
    lib = _abi.load()
    rows = bell.rows
    h = max(1, min(slice_rows, rows)) if rows else 0
    S = (rows + h - 1) // h if rows else 0
    rp = blocked_ell_row_ptr(bell, stream)
    rv = _abi.CompressedView()
    rv.rows, rv.cols, rv.nnz, rv.axis = rows, bell.cols, bell.nnz, COMPRESSED_BY_ROW
    rv.majorPtr = ptr(rp)
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_sliced_ell_scratch_bytes(rows, slice_rows, C.byref(nbytes)), "sliced scratch")
    scratch = _scratch(nbytes.value)
    offs = torch.empty(S + 1, dtype=torch.int32, device="cuda")
    widths = torch.empty(max(S, 1), dtype=torch.int32, device="cuda")
    slots = torch.empty(max(S, 1), dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = stream_handle(stream)
    _abi.check(lib.cs_b200_sliced_ell_layout(C.byref(rv), slice_rows, ptr(offs), ptr(widths), ptr(slots), ptr(total),
                                             ptr(scratch), nbytes.value, s), "sliced_ell_layout")
    n_slots = int(total.item())
    out = SlicedELL(rows, bell.cols, bell.nnz, h, offs, widths[:S], slots[:S],
                    torch.empty(n_slots, dtype=torch.int32, device="cuda"),
                    torch.empty(n_slots, dtype=torch.float16, device="cuda"))
    bv, dv = bell.view(), out.view()
    _abi.check(lib.cs_b200_sliced_ell_emit_from_blocked_ell(C.byref(bv), C.byref(dv), s),
               "sliced_ell_emit_from_blocked_ell")
    return out


def transpose(csr: CSR, stream=None, check_status: bool = True) -> CSR:
    """build_compressed_transpose_raw on the GPU: a (cDim x uDim) compressed matrix ->
    its (uDim x cDim) transpose, minor indices ascending in each major segment."""
    lib = _abi.load()
    cdim = csr.rows if csr.axis == COMPRESSED_BY_ROW else csr.cols
    udim = csr.cols if csr.axis == COMPRESSED_BY_ROW else csr.rows
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_compressed_transpose_scratch_bytes(cdim, udim, csr.nnz, C.byref(nbytes)), "scratch")
    scratch = _scratch(nbytes.value)
    optr = torch.empty(udim + 1, dtype=torch.int32, device="cuda")
    oidx = torch.empty(csr.nnz, dtype=torch.int32, device="cuda")
    oval = torch.empty(csr.nnz, dtype=torch.float16, device="cuda")
    _abi.check(lib.cs_b200_build_compressed_transpose(cdim, udim, csr.nnz, ptr(csr.ptr), ptr(csr.idx), ptr(csr.val),
                                                      ptr(optr), None, ptr(oidx), ptr(oval), ptr(scratch),
                                                      nbytes.value, stream_handle(stream)), "compressed_transpose")
    if check_status:
        st = int(scratch[:4].view(torch.int32).item())
        if st:
            raise _abi.CellShardError(f"transpose flagged invalid input (status 0x{st:x})")
    axis = COMPRESSED_BY_COL if csr.axis == COMPRESSED_BY_ROW else COMPRESSED_BY_ROW
    return CSR(csr.rows, csr.cols, optr, oidx, oval, axis)


def major_nnz_plan(major_ptr: torch.Tensor, major_dim: int, buckets: int, stream=None) -> dict:
    """bucket::build_major_nnz_bucket_plan_raw on the GPU plus power-of-two bins."""
    lib = _abi.load()
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_major_nnz_bucket_sort_scratch_bytes(major_dim, C.byref(nbytes)), "sort scratch")
    scratch = _scratch(nbytes.value)
    n = max(major_dim, 1)
    out = {k: torch.empty(n, dtype=torch.int32, device="cuda") for k in ("nnz", "sorted", "order_in", "order")}
    nb = 1 if major_dim == 0 else min(max(buckets, 1), major_dim)
    out["bucket_offsets"] = torch.empty(nb + 1, dtype=torch.int32, device="cuda")
    out["pow2_bins"] = torch.empty(34, dtype=torch.int32, device="cuda")
    s = stream_handle(stream)
    _abi.check(lib.cs_b200_build_major_nnz_bucket_plan(ptr(major_ptr), major_dim, ptr(out["nnz"]), ptr(out["sorted"]),
                                                       ptr(out["order_in"]), ptr(out["order"]),
                                                       ptr(out["bucket_offsets"]), buckets, ptr(scratch),
                                                       nbytes.value, s), "major_nnz_bucket_plan")
    _abi.check(lib.cs_b200_pow2_nnz_bin_offsets(ptr(out["sorted"]), major_dim, ptr(out["pow2_bins"]), s), "pow2 bins")
    return out


def rebuild_major_order(csr: CSR, order: torch.Tensor, stream=None):
    """bucket::rebuild_compressed_major_order_raw on the GPU; returns (CSR, inverse)."""
    lib = _abi.load()
    n = csr.rows if csr.axis == COMPRESSED_BY_ROW else csr.cols
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_major_nnz_bucket_scan_scratch_bytes(n, C.byref(nbytes)), "scan scratch")
    scratch = _scratch(nbytes.value)
    dptr = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    didx = torch.empty(csr.nnz, dtype=torch.int32, device="cuda")
    dval = torch.empty(csr.nnz, dtype=torch.float16, device="cuda")
    inv = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    _abi.check(lib.cs_b200_rebuild_compressed_major_order(ptr(csr.ptr), ptr(csr.idx), ptr(csr.val), n, ptr(order),
                                                          ptr(dptr), ptr(didx), ptr(dval), ptr(inv), ptr(scratch),
                                                          nbytes.value, stream_handle(stream)), "rebuild")
    return CSR(csr.rows, csr.cols, dptr, didx, dval, csr.axis), inv


@dataclass
class BucketedPartition:
    """Execution-bucketed partition on the device (cellshard::bucketed_blocked_ell_partition /
    bucketed_sliced_ell_partition, io/csh5/api.cuh:316-327,394-406): the segments as device
    views over shared back-to-back buffers, the exec <-> canonical row maps and, for
    Blocked-ELL, the identity column maps."""
    plan: dict
    segments: list
    segment_row_offsets: list
    exec_to_canonical_rows: torch.Tensor
    canonical_to_exec_rows: torch.Tensor
    exec_to_canonical_cols: torch.Tensor | None = None
    canonical_to_exec_cols: torch.Tensor | None = None
    idx: torch.Tensor | None = None
    val: torch.Tensor | None = None


def _plan_dict(p: _abi.ExecBucketPlan) -> dict:
    return {k: getattr(p, k) for k, _ in _abi.ExecBucketPlan._fields_}


def _segments_arrays(room: int):
    import numpy as np

    arrs = [np.zeros(room + 1, np.uint32), np.zeros(room + 1, np.uint32), np.zeros(room, np.uint32)]
    segs = _abi.ExecBucketSegments()
    segs.max_segments = room
    segs.unit_offsets, segs.row_offsets, segs.widths = (a.ctypes.data for a in arrs)
    return segs, arrs


def bucketed_blocked_ell(bell: BlockedELL, requested: int, stream=None) -> BucketedPartition:
    """build_bucketed_blocked_ell_partition on the GPU (requested 0: choose_bucket_count_for_part's
    count).  Synchronises once, after the plan, to size the segments."""
    lib = _abi.load()
    RB = bell.row_blocks if bell.rows else 0
    room = max(1, min(max(requested, 8), max(RB, 1)))
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_bucketed_blocked_ell_scratch_bytes(bell.rows, bell.block_size, room, C.byref(nbytes)),
               "bucketed scratch")
    scratch = _scratch(nbytes.value)
    plan = _abi.ExecBucketPlan()
    segs, (unit_off, row_off, widths) = _segments_arrays(room)
    v = bell.view()
    s = stream_handle(stream)
    _abi.check(lib.cs_b200_bucketed_blocked_ell_plan(C.byref(v), requested, ptr(scratch), nbytes.value,
                                                     C.byref(plan), C.byref(segs), s), "bucketed_blocked_ell_plan")
    S, B = plan.segment_count, bell.block_size
    bci = torch.empty(max(plan.index_entries, 1), dtype=torch.int32, device="cuda")
    val = torch.empty(max(plan.value_entries, 1), dtype=torch.float16, device="cuda")
    maps = torch.empty(2 * bell.rows + 2 * bell.cols + 1, dtype=torch.int32, device="cuda")
    r, c = bell.rows, bell.cols
    e2c, c2e, e2cc, c2ec = maps[:r], maps[r:2 * r], maps[2 * r:2 * r + c], maps[2 * r + c:2 * r + 2 * c]
    _abi.check(lib.cs_b200_bucketed_blocked_ell_fill(C.byref(v), ptr(scratch), C.byref(plan), bci.data_ptr(),
                                                     val.data_ptr(), ptr(e2c), ptr(c2e), ptr(e2cc), ptr(c2ec), s),
               "bucketed_blocked_ell_fill")
    segments, io, vo = [], 0, 0
    for k in range(S):
        nrb, w, rows = int(unit_off[k + 1] - unit_off[k]), int(widths[k]), int(row_off[k + 1] - row_off[k])
        segments.append(BlockedELL(rows, bell.cols, B, w * B, bci[io:io + nrb * w], val[vo:vo + rows * w * B], 0))
        io += nrb * w
        vo += rows * w * B
    return BucketedPartition(_plan_dict(plan), segments, [int(x) for x in row_off[:S + 1]], e2c, c2e, e2cc, c2ec,
                             bci, val)


def bucketed_sliced_ell(sell: SlicedELL, requested: int, stream=None) -> BucketedPartition:
    """build_bucketed_sliced_ell_partition on the GPU (requested 0: choose_bucket_count_for_sliced_part's
    count); each segment is a one-slice Sliced-ELL."""
    lib = _abi.load()
    rows = sell.rows
    room = max(1, min(max(requested, 8), max(rows, 1)))
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_bucketed_sliced_ell_scratch_bytes(rows, room, C.byref(nbytes)), "bucketed scratch")
    scratch = _scratch(nbytes.value)
    plan = _abi.ExecBucketPlan()
    segs, (unit_off, row_off, widths) = _segments_arrays(room)
    v = sell.view()
    s = stream_handle(stream)
    _abi.check(lib.cs_b200_bucketed_sliced_ell_plan(C.byref(v), requested, ptr(scratch), nbytes.value,
                                                    C.byref(plan), C.byref(segs), s), "bucketed_sliced_ell_plan")
    S = plan.segment_count
    col = torch.empty(max(plan.index_entries, 1), dtype=torch.int32, device="cuda")
    val = torch.empty(max(plan.value_entries, 1), dtype=torch.float16, device="cuda")
    maps = torch.empty(2 * rows + 1, dtype=torch.int32, device="cuda")
    e2c, c2e = maps[:rows], maps[rows:2 * rows]
    _abi.check(lib.cs_b200_bucketed_sliced_ell_fill(C.byref(v), ptr(scratch), C.byref(plan), col.data_ptr(),
                                                    val.data_ptr(), ptr(e2c), ptr(c2e), s), "bucketed_sliced_ell_fill")
    segments, o = [], 0
    for k in range(S):
        n, w = int(unit_off[k + 1] - unit_off[k]), int(widths[k])
        z = torch.zeros(1, dtype=torch.int32, device="cuda")
        segments.append(SlicedELL(n, sell.cols, 0, n, torch.tensor([0, n], dtype=torch.int32, device="cuda"),
                                  torch.tensor([w], dtype=torch.int32, device="cuda"), z,
                                  col[o:o + n * w], val[o:o + n * w]))
        o += n * w
    return BucketedPartition(_plan_dict(plan), segments, [int(x) for x in row_off[:S + 1]], e2c, c2e, None, None,
                             col, val)


def blocked_ell_from_coo(rows: int, cols_src: int, row_idx: torch.Tensor, col_idx: torch.Tensor, val: torch.Tensor,
                         block_size: int, cols: int, feature_to_global: torch.Tensor | None = None, stream=None):
    """COO -> Blocked-ELL on the GPU (convert::blocked_ell_from_coo_cuda): plan (one host read of
    the largest column, one of the width), then the emit.  Returns the Blocked-ELL and the two
    nnz counts (the host routine's: stored nonzero values; the GPU routine's: those with
    column < cols)."""
    lib = _abi.load()
    n = int(row_idx.numel())
    v = _abi.CooView()
    v.rows, v.cols, v.nnz = rows, cols_src, n
    v.rowIdx, v.colIdx, v.val = ptr(row_idx), ptr(col_idx), ptr(val)
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_coo_blocked_ell_scratch_bytes(n, rows, cols, block_size, C.byref(nbytes)), "coo scratch")
    scratch = _scratch(nbytes.value)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    width, total = C.c_uint32(), C.c_uint64()
    s = stream_handle(stream)
    fm = ptr(feature_to_global) if feature_to_global is not None else None
    _abi.check(lib.cs_b200_coo_blocked_ell_plan(C.byref(v), fm, cols, block_size, ptr(scratch), nbytes.value,
                                                C.byref(width), C.byref(total), ptr(status), s), "coo plan")
    W = width.value
    RB = (rows + block_size - 1) // block_size
    out = BlockedELL(rows, cols, block_size, W * block_size,
                     torch.empty(max(RB * W, 1), dtype=torch.int32, device="cuda"),
                     torch.empty(max(rows * W * block_size, 1), dtype=torch.float16, device="cuda"), 0)
    nnz = torch.zeros(2, dtype=torch.int64, device="cuda")
    dv = out.view()
    dv.blockColIdx, dv.val = out.bci.data_ptr(), out.val.data_ptr()
    _abi.check(lib.cs_b200_coo_blocked_ell_emit(C.byref(v), fm, cols, ptr(scratch), nbytes.value, C.byref(dv),
                                                nnz.data_ptr(), s), "coo emit")
    counts = [int(x) for x in nnz.cpu()]
    out.nnz = counts[1]
    out.bci = out.bci[:RB * W]
    out.val = out.val[:rows * W * block_size]
    return out, counts, int(status.item()), total.value


def cspack_store(path, m) -> None:
    """Writes a device CSR / Blocked-ELL / Sliced-ELL as one .cspack raw record
    (the reference's store_*_raw layout, src/io/pack/packfile.cu)."""
    lib = _abi.load()
    torch.cuda.synchronize()
    p = str(path).encode()
    v = m.view()
    fn = {CSR: lib.cs_b200_cspack_store_compressed, BlockedELL: lib.cs_b200_cspack_store_blocked_ell,
          SlicedELL: lib.cs_b200_cspack_store_sliced_ell}[type(m)]
    _abi.check(fn(p, C.byref(v)), "cspack store")


def cspack_peek(path) -> _abi.CspackInfo:
    info = _abi.CspackInfo()
    _abi.check(_abi.load().cs_b200_cspack_peek(str(path).encode(), C.byref(info)), "cspack peek")
    return info


def cspack_load(path):
    """Reads one .cspack raw record into device memory (CSR, Blocked-ELL or Sliced-ELL;
    COO records come back as (rows, cols, row_idx, col_idx, val))."""
    lib = _abi.load()
    info = cspack_peek(path)
    p = str(path).encode()
    dev = dict(device="cuda")
    if info.format == 6:
        B = info.block_size
        rb = (info.rows + B - 1) // B if B else 0
        W = info.ell_cols // B if B else 0
        m = BlockedELL(info.rows, info.cols, B, info.ell_cols, torch.empty(max(rb * W, 1), dtype=torch.int32, **dev),
                       torch.empty(max(info.rows * info.ell_cols, 1), dtype=torch.float16, **dev), info.nnz)
        v = m.view()
        v.blockColIdx, v.val = m.bci.data_ptr(), m.val.data_ptr()
        _abi.check(lib.cs_b200_cspack_load_blocked_ell(p, C.byref(v)), "cspack load")
        m.bci, m.val = m.bci[:rb * W], m.val[:info.rows * info.ell_cols]
        return m
    if info.format == 7:
        S, T = info.slice_count, info.total_slots
        m = SlicedELL(info.rows, info.cols, info.nnz, 0, torch.empty(S + 1, dtype=torch.int32, **dev),
                      torch.empty(max(S, 1), dtype=torch.int32, **dev), torch.empty(max(S, 1), dtype=torch.int32, **dev),
                      torch.empty(max(T, 1), dtype=torch.int32, **dev), torch.empty(max(T, 1), dtype=torch.float16, **dev))
        v = m.view()
        v.slice_row_offsets, v.slice_widths, v.slice_slot_offsets = (m.slice_row_offsets.data_ptr(),
                                                                     m.slice_widths.data_ptr(),
                                                                     m.slice_slot_offsets.data_ptr())
        v.col_idx, v.val = m.col_idx.data_ptr(), m.val.data_ptr()
        _abi.check(lib.cs_b200_cspack_load_sliced_ell(p, C.byref(v)), "cspack load")
        m.slice_widths, m.slice_slot_offsets = m.slice_widths[:S], m.slice_slot_offsets[:S]
        m.col_idx, m.val = m.col_idx[:T], m.val[:T]
        return m
    if info.format == 2:
        major = info.cols if info.axis == COMPRESSED_BY_COL else info.rows
        m = CSR(info.rows, info.cols, torch.empty(major + 1, dtype=torch.int32, **dev),
                torch.empty(max(info.nnz, 1), dtype=torch.int32, **dev),
                torch.empty(max(info.nnz, 1), dtype=torch.float16, **dev), info.axis)
        v = _abi.CompressedView()
        v.rows, v.cols, v.nnz, v.axis = info.rows, info.cols, info.nnz, info.axis
        v.majorPtr, v.minorIdx, v.val = m.ptr.data_ptr(), m.idx.data_ptr(), m.val.data_ptr()
        _abi.check(lib.cs_b200_cspack_load_compressed(p, C.byref(v)), "cspack load")
        m.idx, m.val = m.idx[:info.nnz], m.val[:info.nnz]
        return m
    if info.format == 3:
        n = info.nnz
        r, c = torch.empty(max(n, 1), dtype=torch.int32, **dev), torch.empty(max(n, 1), dtype=torch.int32, **dev)
        val = torch.empty(max(n, 1), dtype=torch.float16, **dev)
        v = _abi.CooView()
        v.rows, v.cols, v.nnz = info.rows, info.cols, n
        v.rowIdx, v.colIdx, v.val = r.data_ptr(), c.data_ptr(), val.data_ptr()
        _abi.check(lib.cs_b200_cspack_load_coo(p, C.byref(v)), "cspack load")
        return info.rows, info.cols, r[:n], c[:n], val[:n]
    raise _abi.CellShardError(f"cspack: format {info.format} not handled")


def cspack_store_coo(path, rows: int, cols: int, row_idx: torch.Tensor, col_idx: torch.Tensor,
                     val: torch.Tensor) -> None:
    torch.cuda.synchronize()
    v = _abi.CooView()
    v.rows, v.cols, v.nnz = rows, cols, int(row_idx.numel())
    v.rowIdx, v.colIdx, v.val = ptr(row_idx), ptr(col_idx), ptr(val)
    _abi.check(_abi.load().cs_b200_cspack_store_coo(str(path).encode(), C.byref(v)), "cspack store")
