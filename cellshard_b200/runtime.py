"""Python mirror of the reference's mask_groups runtime
(include/CellShard/runtime/mask_groups.cuh) over the C ABI.

`compute_sparse_group_reduce*` keep the reference's argument meaning: group
bitmasks per feature (<= 32 groups), a row/feature mask view, filter params,
per-row outputs.  `compute_sparse_group_moments` is the row-label grouped
per-feature moments entry point (no reference counterpart).  Results are
device tensors; nothing here synchronises except where a value must be read.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _abi
from .device import BlockedELL, CSR, SlicedELL, ptr, stream_handle

MAX_MASK_GROUPS = 32
MAX_MOMENT_GROUPS = 4096

PHASE_PREPARE = 1
PHASE_ACCUMULATE = 2
PHASE_COMBINE = 4
PHASE_ALL = 7

PLAIN_F32 = 0
TWOSUM_F32 = 1
TWOSUM_F64_COMBINE = 2


@dataclass
class FilterParams:
    """runtime::sparse_group_filter_params (mask_groups.cuh:36-41)."""

    min_total: float = 0.0
    min_detected_features: int = 0
    max_group_fraction: float = 1.0
    fraction_group_index: int = 0

    def c(self) -> _abi.GroupFilterParams:
        return _abi.GroupFilterParams(self.min_total, self.min_detected_features, self.max_group_fraction,
                                      self.fraction_group_index)


def _mask_view(row_keep=None, feature_keep=None, row_remap=None, feature_remap=None) -> _abi.RowFeatureMaskView:
    m = _abi.RowFeatureMaskView()
    m.row_keep, m.feature_keep = ptr(row_keep), ptr(feature_keep)
    m.row_remap, m.feature_remap = ptr(row_remap), ptr(feature_remap)
    return m


def compute_sparse_group_reduce(src, feature_group_masks: torch.Tensor | None, group_count: int,
                                row_keep=None, feature_keep=None, filt: FilterParams | None = None, stream=None):
    """Masked per-row feature-group reduction (runtime::compute_sparse_group_reduce and
    compute_sparse_group_reduce_compressed_fallback, mask_groups.cu:811-918)."""
    lib = _abi.load()
    rows = src.rows
    dev = "cuda"
    res = {
        "row_totals": torch.empty(rows, dtype=torch.float32, device=dev),
        "detected_features": torch.empty(rows, dtype=torch.int32, device=dev),
        "max_values": torch.empty(rows, dtype=torch.float32, device=dev),
        "row_keep": torch.empty(rows, dtype=torch.uint8, device=dev),
        "group_counts": torch.empty(rows * group_count, dtype=torch.float32, device=dev) if group_count else None,
        "group_percentages": torch.empty(rows * group_count, dtype=torch.float32, device=dev) if group_count else None,
    }
    out = _abi.GroupReduceOut(ptr(res["row_totals"]), ptr(res["detected_features"]), ptr(res["max_values"]),
                              ptr(res["row_keep"]), ptr(res["group_counts"]), ptr(res["group_percentages"]))
    m = _mask_view(row_keep, feature_keep)
    f = (filt or FilterParams()).c()
    v = src.view()
    if isinstance(src, BlockedELL):
        fn, name = lib.cs_b200_group_reduce_blocked_ell, "group_reduce_blocked_ell"
    elif isinstance(src, SlicedELL):
        fn, name = lib.cs_b200_group_reduce_sliced_ell, "group_reduce_sliced_ell"
    elif isinstance(src, CSR):
        fn, name = lib.cs_b200_group_reduce_compressed, "group_reduce_compressed"
    else:
        raise TypeError(type(src))
    _abi.check(fn(C.byref(v), ptr(feature_group_masks), group_count, C.byref(m), C.byref(f), C.byref(out),
                  stream_handle(stream)), name)
    return res


def manual_reoptimize_masked_sparse(src: BlockedELL, row_keep=None, feature_keep=None, row_remap=None,
                                    feature_remap=None, output_rows: int = 0, output_cols: int = 0, stream=None):
    """Masked + remapped Blocked-ELL -> CSR (runtime::manual_reoptimize_masked_sparse,
    mask_groups.cu:960-1034).  Synchronises once to size the output, as the reference does."""
    lib = _abi.load()
    out_rows = output_rows if output_rows else src.rows
    out_cols = output_cols if output_cols else src.cols
    m = _mask_view(row_keep, feature_keep, row_remap, feature_remap)
    v = src.view()
    nbytes = C.c_size_t()
    _abi.check(lib.cs_b200_reoptimize_scratch_bytes(src.rows, out_rows, C.byref(nbytes)), "reoptimize scratch")
    scratch = torch.empty(max(nbytes.value, 16), dtype=torch.uint8, device="cuda")
    major = torch.empty(out_rows + 1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = stream_handle(stream)
    _abi.check(lib.cs_b200_reoptimize_count(C.byref(v), C.byref(m), out_rows, out_cols, ptr(major), ptr(scratch),
                                            nbytes.value, ptr(status), s), "reoptimize_count")
    nnz = int(major[out_rows].item()) & 0xFFFFFFFF
    idx = torch.empty(nnz, dtype=torch.int32, device="cuda")
    val = torch.empty(nnz, dtype=torch.float16, device="cuda")
    _abi.check(lib.cs_b200_reoptimize_emit(C.byref(v), C.byref(m), out_rows, out_cols, ptr(major), ptr(idx),
                                           ptr(val), s), "reoptimize_emit")
    st = int(status.item())
    if st:
        raise _abi.CellShardError(f"reoptimize flagged invalid input (status 0x{st:x})")
    meta = {
        "kept_rows": out_rows,
        "kept_features": out_cols,
        "live_nnz": nnz,
        "bytes_before": src.rows * src.ell_cols * 2 + src.row_blocks * src.ell_width * 4,
        "bytes_after": (out_rows + 1) * 4 + nnz * 6,
    }
    return CSR(out_rows, out_cols, major, idx, val), meta


STATUS_CAPACITY = 1 << 5


# the vector filter "auto" takes when a shard qualifies (the faster of the two
# on the 500,000 x 32,768 Blocked-ELL-16 shard at 70 % rows / 60 % features)
_AUTO_VECTOR_FILTER = "marked"


def filter_blocked_ell_to_compressed(parts, output_rows: int, output_cols: int, keep_rows=None, keep_cols=None,
                                     row_remap=None, col_remap=None, stream=None, method: str = "auto"):
    """Filtered Blocked-ELL -> CSR over the partitions of one shard, rows concatenated in
    order (convert::filter_blocked_ell_to_compressed, src/convert/
    filtered_blocked_ell_to_compressed.cuh:264-382, and the filter stage of
    repack::build_repacked_shard_blocked_ell).  Synchronises once to size the output.
    Returns (CSR, stats) with the reference's stats fields; kept_rows / kept_row_slots
    count every kept source row (the repack operator's figures).

    Routes: "marked" (cs_b200_filter_blocked_ell_marked: one pass counts each kept row and
    marks its 8-value groups holding kept entries, a scan places the rows, a second pass
    reads only the marked groups), "onepass" (cs_b200_filter_blocked_ell_onepass: each row
    counted, placed by a decoupled look-back and written from L2), both for shards with no
    remaps, block sizes multiples of 8 and output_rows >= their rows, into arrays sized by
    the parts' stored nnz; "two_pass" (count + emit, any shard).  "auto" takes the faster
    vector route when the shard qualifies and count + emit otherwise, or when the stored nnz
    proves too small.  A forced vector route raises where it does not apply."""
    lib = _abi.load()
    parts = list(parts) if isinstance(parts, (list, tuple)) else [parts]
    views = (_abi.BlockedEllView * len(parts))(*[p.view() for p in parts])
    shard_rows = sum(p.rows for p in parts)
    m = _mask_view(keep_rows, keep_cols, row_remap, col_remap)
    major = torch.empty(output_rows + 1, dtype=torch.int32, device="cuda")
    kept = torch.zeros(2, dtype=torch.int64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = stream_handle(stream)
    idx = val = None
    nnz = None
    qualifies = (row_remap is None and col_remap is None and output_rows >= shard_rows
                 and all(p.rows == 0 or (p.block_size % 8 == 0 and p.val.data_ptr() % 16 == 0) for p in parts))
    if method not in ("auto", "marked", "onepass", "two_pass"):
        raise ValueError(f"unknown filter method {method!r}")
    if method in ("marked", "onepass") and not qualifies:
        raise _abi.CellShardError(f"the {method} filter needs no remaps, block sizes multiple of 8 and "
                                  "output_rows >= the shard's rows")
    if method != "two_pass" and qualifies:
        route = _AUTO_VECTOR_FILTER if method == "auto" else method
        bytes_fn = getattr(lib, f"cs_b200_filter_blocked_ell_{route}_scratch_bytes")
        run_fn = getattr(lib, f"cs_b200_filter_blocked_ell_{route}")
        cap = sum(int(p.nnz) for p in parts)
        nb = C.c_size_t()
        _abi.check(bytes_fn(views, len(parts), C.byref(nb)), f"{route} scratch")
        scratch = torch.empty(max(nb.value, 16), dtype=torch.uint8, device="cuda")
        idx = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        val = torch.empty(max(cap, 1), dtype=torch.float16, device="cuda")
        _abi.check(run_fn(views, len(parts), C.byref(m), output_rows, output_cols, ptr(major), ptr(idx), ptr(val),
                          cap, ptr(kept), ptr(scratch), nb.value, ptr(status), s), f"filter_blocked_ell_{route}")
        st = int(status.item())
        if st & STATUS_CAPACITY and method == "auto":
            status.zero_()
            idx = val = None  # the stored nnz under-counts: count + emit below
        else:
            nnz = int(major[output_rows].item()) & 0xFFFFFFFF
            idx, val = idx[:nnz], val[:nnz]
    if idx is None:
        nbytes = C.c_size_t()
        _abi.check(lib.cs_b200_filter_blocked_ell_scratch_bytes(shard_rows, output_rows, C.byref(nbytes)), "scratch")
        scratch = torch.empty(max(nbytes.value, 16), dtype=torch.uint8, device="cuda")
        _abi.check(lib.cs_b200_filter_blocked_ell_count(views, len(parts), C.byref(m), output_rows, output_cols,
                                                        ptr(major), ptr(kept), ptr(scratch), nbytes.value,
                                                        ptr(status), s), "filter_blocked_ell_count")
        nnz = int(major[output_rows].item()) & 0xFFFFFFFF
        idx = torch.empty(nnz, dtype=torch.int32, device="cuda")
        val = torch.empty(nnz, dtype=torch.float16, device="cuda")
        _abi.check(lib.cs_b200_filter_blocked_ell_emit(views, len(parts), C.byref(m), output_rows, output_cols,
                                                       ptr(major), ptr(idx), ptr(val), s), "filter_blocked_ell_emit")
    st = int(status.item())
    if st:
        raise _abi.CellShardError(f"filter flagged invalid input (status 0x{st:x})")
    kept_rows, kept_slots = (int(x) for x in kept.tolist())
    dead = max(kept_slots - nnz, 0)
    stats = {"kept_rows": kept_rows, "output_rows": output_rows, "output_cols": output_cols, "live_nnz": nnz,
             "kept_row_slots": kept_slots, "dead_slots": dead,
             "live_fill_ratio": 1.0 if kept_slots == 0 else nnz / kept_slots, "dead_value_bytes": dead * 2}
    return CSR(output_rows, output_cols, major, idx, val), stats


def build_repacked_blocked_ell(parts, output_rows: int, output_cols: int, block_size: int, bucket_count: int,
                               keep_rows=None, keep_cols=None, row_remap=None, col_remap=None, stream=None):
    """repack::build_repacked_shard_blocked_ell (src/repack/operators/sharded_blocked_ell.cuh:
    393-726) over a list of partitions: filter -> CSR, nnz bucket plan and row rebuild,
    then the rebuilt CSR as Blocked-ELL of block_size.  Returns
    (filtered CSR, plan, rebuilt CSR, Blocked-ELL, stats)."""
    from .device import blocked_ell_from_csr, major_nnz_plan, rebuild_major_order

    filtered, stats = filter_blocked_ell_to_compressed(parts, output_rows, output_cols, keep_rows, keep_cols,
                                                       row_remap, col_remap, stream)
    plan = major_nnz_plan(filtered.ptr, output_rows, bucket_count, stream)
    rebuilt, _inverse = rebuild_major_order(filtered, plan["order"], stream)
    bell = blocked_ell_from_csr(rebuilt, block_size, stream)
    stats["ell_width"] = bell.ell_width
    return filtered, plan, rebuilt, bell, stats


class MomentsWorkspace:
    """Caller-held scratch for compute_sparse_group_moments (grows monotonically, like the
    reference's sparse_group_reduce_workspace)."""

    def __init__(self):
        self.scratch: torch.Tensor | None = None

    def reserve(self, nbytes: int) -> torch.Tensor:
        if self.scratch is None or self.scratch.numel() < nbytes:
            self.scratch = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")
        return self.scratch


def group_moments_scratch_bytes(src: BlockedELL, group_count: int, scheme: int = TWOSUM_F64_COMBINE,
                                ddof: int = 1, chunk_rows: int = 0) -> int:
    lib = _abi.load()
    p = _abi.GroupMomentsParams(group_count, scheme, ddof, chunk_rows)
    v = src.view()
    n = C.c_size_t()
    _abi.check(lib.cs_b200_group_moments_scratch_bytes(C.byref(v), C.byref(p), C.byref(n)), "moments scratch")
    return n.value


def build_moments_index(src: BlockedELL, status: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """The partition's column-block index (cs_b200_group_moments_build_index), built once
    and passed as ``index=`` to later reductions over the same partition, which then skip
    rebuilding it.  Order errors in blockColIdx go to ``status`` (int32[1]) when given."""
    lib = _abi.load()
    v = src.view()
    n = C.c_size_t()
    _abi.check(lib.cs_b200_group_moments_index_bytes(C.byref(v), C.byref(n)), "moments index bytes")
    index = torch.empty(max(n.value, 16), dtype=torch.uint8, device="cuda")
    _abi.check(lib.cs_b200_group_moments_build_index(C.byref(v), ptr(index), ptr(status), stream_handle(stream)),
               "moments index")
    return index


def compute_sparse_group_moments(src: BlockedELL, group_count: int, row_keep=None, feature_keep=None,
                                 row_labels=None, scheme: int = TWOSUM_F64_COMBINE, ddof: int = 1,
                                 chunk_rows: int = 0, workspace: MomentsWorkspace | None = None, out=None,
                                 want_f64: bool = False, phases: int = 7, stream=None, index=None):
    """Per-(group, feature) sum / sum of squares / mean / variance over kept rows of a
    Blocked-ELL partition; returns a dict of device tensors ([G, cols]).  ``index``: the
    partition's column-block index from build_moments_index (None = rebuilt by this call)."""
    lib = _abi.load()
    G, cols = group_count, src.cols
    p = _abi.GroupMomentsParams(G, scheme, ddof, chunk_rows, ptr(index))
    v = src.view()
    n = C.c_size_t()
    _abi.check(lib.cs_b200_group_moments_scratch_bytes(C.byref(v), C.byref(p), C.byref(n)), "moments scratch")
    ws = workspace or MomentsWorkspace()
    scratch = ws.reserve(n.value)
    if out is None:
        out = {
            "sum": torch.empty((G, cols), dtype=torch.float32, device="cuda"),
            "sumsq": torch.empty((G, cols), dtype=torch.float32, device="cuda"),
            "mean": torch.empty((G, cols), dtype=torch.float32, device="cuda"),
            "var": torch.empty((G, cols), dtype=torch.float32, device="cuda"),
            "group_rows": torch.empty(G, dtype=torch.int32, device="cuda"),
            "status": torch.zeros(1, dtype=torch.int32, device="cuda"),
        }
        if want_f64:
            out["mean64"] = torch.empty((G, cols), dtype=torch.float64, device="cuda")
            out["var64"] = torch.empty((G, cols), dtype=torch.float64, device="cuda")
    o = _abi.GroupMomentsOut(ptr(out["sum"]), ptr(out["sumsq"]), ptr(out.get("mean")), ptr(out.get("var")),
                             ptr(out.get("mean64")), ptr(out.get("var64")), ptr(out.get("group_rows")),
                             ptr(out.get("status")))
    if phases == PHASE_ALL:
        _abi.check(lib.cs_b200_group_moments_blocked_ell(C.byref(v), ptr(row_keep), ptr(feature_keep),
                                                         ptr(row_labels), C.byref(p), C.byref(o), ptr(scratch),
                                                         scratch.numel(), stream_handle(stream)),
                   "group_moments_blocked_ell")
    else:
        _abi.check(lib.cs_b200_group_moments_phases(C.byref(v), ptr(row_keep), ptr(feature_keep), ptr(row_labels),
                                                    C.byref(p), C.byref(o), ptr(scratch), scratch.numel(), phases,
                                                    stream_handle(stream)), "group_moments_phases")
    return out


def group_moments_parts_scratch_bytes(parts, group_count: int, scheme: int = TWOSUM_F64_COMBINE, ddof: int = 1,
                                      chunk_rows: int = 0) -> int:
    lib = _abi.load()
    p = _abi.GroupMomentsParams(group_count, scheme, ddof, chunk_rows)
    views = (_abi.BlockedEllView * len(parts))(*[q.view() for q in parts])
    n = C.c_size_t()
    _abi.check(lib.cs_b200_group_moments_parts_scratch_bytes(views, len(parts), C.byref(p), C.byref(n)),
               "moments parts scratch")
    return n.value


def compute_sparse_group_moments_parts(parts, group_count: int, row_keep=None, feature_keep=None, row_labels=None,
                                       scheme: int = TWOSUM_F64_COMBINE, ddof: int = 1, chunk_rows: int = 0,
                                       indexes=None, workspace: MomentsWorkspace | None = None, out=None,
                                       want_f64: bool = False, stream=None):
    """The moments reduction over a shard given as its Blocked-ELL partitions, in one call
    (cs_b200_group_moments_blocked_ell_parts).  ``row_keep`` / ``row_labels`` cover the rows of
    all partitions in order; ``indexes``: each partition's column-block index from
    build_moments_index (None, or a None entry, = built by the call)."""
    lib = _abi.load()
    G, cols = group_count, parts[0].cols
    p = _abi.GroupMomentsParams(G, scheme, ddof, chunk_rows)
    views = (_abi.BlockedEllView * len(parts))(*[q.view() for q in parts])
    n = C.c_size_t()
    _abi.check(lib.cs_b200_group_moments_parts_scratch_bytes(views, len(parts), C.byref(p), C.byref(n)),
               "moments parts scratch")
    ws = workspace or MomentsWorkspace()
    scratch = ws.reserve(n.value)
    if out is None:
        out = {k: torch.empty((G, cols), dtype=torch.float32, device="cuda") for k in ("sum", "sumsq", "mean", "var")}
        out["group_rows"] = torch.empty(G, dtype=torch.int32, device="cuda")
        out["status"] = torch.zeros(1, dtype=torch.int32, device="cuda")
        if want_f64:
            out["mean64"] = torch.empty((G, cols), dtype=torch.float64, device="cuda")
            out["var64"] = torch.empty((G, cols), dtype=torch.float64, device="cuda")
    keys = ("sum", "sumsq", "mean", "var", "mean64", "var64", "group_rows", "status")
    o = _abi.GroupMomentsOut(*[ptr(out.get(k)) for k in keys])
    idx = None
    if indexes is not None:
        idx = (C.c_void_p * len(parts))(*[ptr(x) for x in indexes])
    _abi.check(lib.cs_b200_group_moments_blocked_ell_parts(views, len(parts), idx, ptr(row_keep), ptr(feature_keep),
                                                           ptr(row_labels), C.byref(p), C.byref(o), ptr(scratch),
                                                           scratch.numel(), stream_handle(stream)),
               "group_moments_blocked_ell_parts")
    return out


def compute_sparse_group_moments_to_host(src: BlockedELL, group_count: int, host_out: dict, row_keep=None,
                                         feature_keep=None, row_labels=None, scheme: int = TWOSUM_F64_COMBINE,
                                         ddof: int = 1, chunk_rows: int = 0, parts: int = 0,
                                         workspace: MomentsWorkspace | None = None, out=None, stream=None,
                                         index=None):
    """compute_sparse_group_moments with the results copied into ``host_out`` (pinned CPU
    tensors keyed like the device outputs: sum, sumsq, mean, var, mean64, var64,
    group_rows, status), the groups split into ``parts`` ranges whose copies overlap the
    next range's work (cs_b200_group_moments_to_host).  Synchronise the stream before
    reading ``host_out``.  Returns the device outputs.  ``index`` as in
    compute_sparse_group_moments."""
    lib = _abi.load()
    G, cols = group_count, src.cols
    p = _abi.GroupMomentsParams(G, scheme, ddof, chunk_rows, ptr(index))
    v = src.view()
    n = C.c_size_t()
    _abi.check(lib.cs_b200_group_moments_scratch_bytes(C.byref(v), C.byref(p), C.byref(n)), "moments scratch")
    ws = workspace or MomentsWorkspace()
    scratch = ws.reserve(n.value)
    if out is None:
        out = {k: torch.empty((G, cols), dtype=torch.float32, device="cuda") for k in ("sum", "sumsq", "mean", "var")}
        out["group_rows"] = torch.empty(G, dtype=torch.int32, device="cuda")
        out["status"] = torch.zeros(1, dtype=torch.int32, device="cuda")
        if "mean64" in host_out or "var64" in host_out:
            out["mean64"] = torch.empty((G, cols), dtype=torch.float64, device="cuda")
            out["var64"] = torch.empty((G, cols), dtype=torch.float64, device="cuda")

    def hptr(k):
        t = host_out.get(k)
        if t is None:
            return None
        if t.is_cuda or t.numel() != out[k].numel() or t.dtype != out[k].dtype:
            raise ValueError(f"host_out[{k!r}] must be a CPU tensor shaped and typed like the device output")
        return t.data_ptr()

    keys = ("sum", "sumsq", "mean", "var", "mean64", "var64", "group_rows", "status")
    o = _abi.GroupMomentsOut(*[ptr(out.get(k)) for k in keys])
    h = _abi.GroupMomentsOut(*[hptr(k) for k in keys])
    _abi.check(lib.cs_b200_group_moments_to_host(C.byref(v), ptr(row_keep), ptr(feature_keep), ptr(row_labels),
                                                 C.byref(p), C.byref(o), C.byref(h), ptr(scratch), scratch.numel(),
                                                 parts, stream_handle(stream)), "group_moments_to_host")
    return out
