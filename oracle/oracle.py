"""TEST ORACLE ONLY: numpy wrappers over the C restatement (_build/libcs_oracle.so)
and the reference bridges (_ref/libcs_ref.so, _ref/libcs_ref_gpu.so,
_ref/libcs_ref_bucket.so).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "libcs_oracle.so"
REF_LIB = HERE / "_ref" / "libcs_ref.so"
REF_GPU_LIB = HERE / "_ref" / "libcs_ref_gpu.so"

vp = C.c_void_p
u32 = C.c_uint32


def build_restatement() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "restate"], check=True)


_o = None


def lib() -> C.CDLL:
    global _o
    if _o is None:
        if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < (HERE / "cs_oracle.c").stat().st_mtime:
            build_restatement()
        _o = C.CDLL(str(ORACLE_LIB))
    return _o


def _p(a):
    return None if a is None else a.ctypes.data_as(vp)


def h2f(bits: np.ndarray) -> np.ndarray:
    return np.asarray(bits, dtype=np.uint16).view(np.float16).astype(np.float32)


# ---------------------------------------------------------------------------
# mask_groups per-row reduce
# ---------------------------------------------------------------------------
class ReduceOut(C.Structure):
    _fields_ = [("row_totals", vp), ("detected", vp), ("max_values", vp), ("row_keep", vp),
                ("group_counts", vp), ("group_percentages", vp)]


def _reduce_outputs(rows, G):
    res = {
        "row_totals": np.zeros(rows, np.float32),
        "detected_features": np.zeros(rows, np.uint32),
        "max_values": np.zeros(rows, np.float32),
        "row_keep": np.zeros(rows, np.uint8),
        "group_counts": np.zeros(rows * G, np.float32) if G else None,
        "group_percentages": np.zeros(rows * G, np.float32) if G else None,
    }
    out = ReduceOut(_p(res["row_totals"]), _p(res["detected_features"]), _p(res["max_values"]),
                    _p(res["row_keep"]), _p(res["group_counts"]), _p(res["group_percentages"]))
    return res, out


def _f(filt):
    return (C.c_float(filt[0]), u32(filt[1]), C.c_float(filt[2]), u32(filt[3]))


def group_reduce_csr(rows, cols, ptr, idx, val, masks, G, row_keep, feature_keep, filt):
    res, out = _reduce_outputs(rows, G)
    ok = lib().cso_group_reduce_csr(u32(rows), u32(cols), _p(ptr), _p(idx), _p(val), _p(masks), u32(G),
                                    _p(row_keep), _p(feature_keep), *_f(filt), C.byref(out))
    assert ok == 1
    return res


def group_reduce_bell(rows, cols, B, ell_cols, bci, val, masks, G, row_keep, feature_keep, filt):
    res, out = _reduce_outputs(rows, G)
    ok = lib().cso_group_reduce_bell(u32(rows), u32(cols), u32(B), u32(ell_cols), _p(bci), _p(val), _p(masks),
                                     u32(G), _p(row_keep), _p(feature_keep), *_f(filt), C.byref(out))
    assert ok == 1
    return res


def group_reduce_sell(rows, cols, slice_rows, offsets, widths, slot_offsets, col_idx, val, masks, G, row_keep,
                      feature_keep, filt):
    res, out = _reduce_outputs(rows, G)
    ok = lib().cso_group_reduce_sell(u32(rows), u32(cols), u32(len(widths)), u32(slice_rows), _p(offsets),
                                     _p(widths), _p(slot_offsets), _p(col_idx), _p(val), _p(masks), u32(G),
                                     _p(row_keep), _p(feature_keep), *_f(filt), C.byref(out))
    assert ok == 1
    return res


def reoptimize_bell(rows, cols, B, ell_cols, bci, val, row_keep, feature_keep, row_remap, feature_remap, out_rows,
                    out_cols):
    cap = max(rows * ell_cols, 1)
    major = np.zeros(out_rows + 1, np.uint32)
    idx = np.zeros(cap, np.uint32)
    v = np.zeros(cap, np.uint16)
    f = lib().cso_reoptimize_bell
    f.restype = C.c_longlong
    n = f(u32(rows), u32(cols), u32(B), u32(ell_cols), _p(bci), _p(val), _p(row_keep), _p(feature_keep),
          _p(row_remap), _p(feature_remap), u32(out_rows), u32(out_cols), _p(major), _p(idx), _p(v))
    if n < 0:
        raise ValueError("remap collision")
    return major, idx[:n].copy(), v[:n].copy()


# ---------------------------------------------------------------------------
# grouped moments (FP64)
# ---------------------------------------------------------------------------
def group_moments_bell(rows, cols, B, ell_cols, bci, val, row_keep, feature_keep, labels, G, ddof=1,
                       nthreads=1):
    gc = G * cols
    s, q, m, v = (np.zeros(gc, np.float64) for _ in range(4))
    n = np.zeros(G, np.uint32)
    ok = lib().cso_group_moments_bell(u32(rows), u32(cols), u32(B), u32(ell_cols), _p(bci), _p(val), _p(row_keep),
                                      _p(feature_keep), _p(labels), u32(G), u32(ddof), _p(s), _p(q), _p(m), _p(v),
                                      _p(n), C.c_int(nthreads))
    assert ok == 1
    shp = (G, cols)
    return {"sum": s.reshape(shp), "sumsq": q.reshape(shp), "mean": m.reshape(shp), "var": v.reshape(shp),
            "group_rows": n}


def group_moments_bell_slabs(fetch, rows, cols, B, ell_cols, row_keep, feature_keep, labels, G, ddof=1,
                            slab_rows=32768, nthreads=1):
    """FP64 moments of a Blocked-ELL matrix too large to hold on the host at once.

    ``fetch(r0, r1)`` returns the host (bci, val) of rows [r0, r1) (r0 a multiple of B).
    Per-slab FP64 sums and sums of squares are added; integer counts keep them exact,
    so the totals equal one call over all rows.  The finishing rule is the one in
    cs_oracle.c's moments worker: mean = S / n; var = max(Q - S * mean, 0) / (n - ddof)
    when n > ddof; features the mask drops are all zero."""
    slab_rows = max(B, slab_rows // B * B)
    s = np.zeros((G, cols), np.float64)
    q = np.zeros((G, cols), np.float64)
    n = np.zeros(G, np.int64)
    for r0 in range(0, rows, slab_rows):
        r1 = min(rows, r0 + slab_rows)
        bci, val = fetch(r0, r1)
        part = group_moments_bell(r1 - r0, cols, B, ell_cols, bci, val, row_keep[r0:r1], None, labels[r0:r1], G,
                                  ddof=ddof, nthreads=nthreads)
        s += part["sum"]
        q += part["sumsq"]
        n += part["group_rows"].astype(np.int64)
    keep = np.ones(cols, bool) if feature_keep is None else feature_keep.astype(bool)
    s[:, ~keep] = 0.0
    q[:, ~keep] = 0.0
    nn = n.astype(np.float64)[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        mean = np.where(nn > 0, s / np.maximum(nn, 1.0), 0.0)
        m2 = np.maximum(q - s * mean, 0.0)
        var = np.where(nn > ddof, m2 / np.maximum(nn - ddof, 1.0), 0.0)
    mean[:, ~keep] = 0.0
    var[:, ~keep] = 0.0
    return {"sum": s, "sumsq": q, "mean": mean, "var": var, "group_rows": n.astype(np.uint32)}


def moments_max_rel(got: dict, ref: dict) -> dict:
    """Largest relative error per output against the FP64 result: |got - ref| / |ref| for
    sum, sumsq and mean (entries equal to the reference count as 0); variance relative to
    max(|var|, 1e-12 * sumsq / n) so that exact zeros compare absolutely."""
    out = {}
    n = ref["group_rows"].astype(np.float64)
    for k in ("sum", "sumsq", "mean", "var"):
        g = np.asarray(got[k], np.float64)
        e = ref[k]
        d = np.abs(g - e)
        scale = np.abs(e)
        if k == "var":
            scale = np.maximum(scale, 1e-12 * ref["sumsq"] / np.maximum(n, 1.0)[:, None])
        err = np.where(d == 0.0, 0.0, d / np.maximum(scale, 1e-30))
        out[k] = float(err.max(initial=0.0))
    return out


def group_moments_csr(rows, cols, ptr, idx, val, row_keep, feature_keep, labels, G, ddof=1, nthreads=1):
    gc = G * cols
    s, q, m, v = (np.zeros(gc, np.float64) for _ in range(4))
    n = np.zeros(G, np.uint32)
    ok = lib().cso_group_moments_csr(u32(rows), u32(cols), _p(ptr), _p(idx), _p(val), _p(row_keep),
                                     _p(feature_keep), _p(labels), u32(G), u32(ddof), _p(s), _p(q), _p(m), _p(v),
                                     _p(n), C.c_int(nthreads))
    assert ok == 1
    shp = (G, cols)
    return {"sum": s.reshape(shp), "sumsq": q.reshape(shp), "mean": m.reshape(shp), "var": v.reshape(shp),
            "group_rows": n}


# ---------------------------------------------------------------------------
# conversions, transpose, bucketing (restatement)
# ---------------------------------------------------------------------------
def blocked_ell_shape(rows, cols, ptr, idx, B):
    w = u32()
    t = C.c_uint64()
    assert lib().cso_blocked_ell_shape(u32(rows), u32(cols), _p(ptr), _p(idx), u32(B), C.byref(w), C.byref(t)) == 1
    return w.value, t.value


def blocked_ell_from_csr(rows, cols, ptr, idx, val, B):
    W, _ = blocked_ell_shape(rows, cols, ptr, idx, B)
    rb = (rows + B - 1) // B
    bci = np.zeros(max(rb * W, 1), np.uint32)
    out = np.zeros(max(rows * W * B, 1), np.uint16)
    f = lib().cso_blocked_ell_from_csr
    f.restype = u32
    nnz = f(u32(rows), u32(cols), _p(ptr), _p(idx), _p(val), u32(B), u32(W), _p(bci), _p(out))
    return {"ell_width": W, "ell_cols": W * B, "bci": bci[:rb * W], "val": out[:rows * W * B], "nnz": int(nnz)}


def sliced_ell_from_csr(rows, ptr, idx, val, slice_rows):
    f = lib().cso_sliced_slice_count
    f.restype = u32
    S = f(u32(rows), u32(slice_rows))
    offsets = np.zeros(S + 1, np.uint32)
    widths = np.zeros(max(S, 1), np.uint32)
    slot_off = np.zeros(max(S, 1), np.uint32)
    g = lib().cso_sliced_ell_layout
    g.restype = C.c_uint64
    total = g(u32(rows), _p(ptr), u32(slice_rows), _p(offsets), _p(widths), _p(slot_off))
    col_idx = np.zeros(max(total, 1), np.uint32)
    v = np.zeros(max(total, 1), np.uint16)
    lib().cso_sliced_ell_fill(u32(rows), _p(ptr), _p(idx), _p(val), u32(slice_rows), _p(offsets), _p(widths),
                              _p(slot_off), _p(col_idx), _p(v))
    return {"slice_count": S, "offsets": offsets, "widths": widths[:S], "slot_offsets": slot_off[:S],
            "col_idx": col_idx[:total], "val": v[:total], "total_slots": int(total)}


def bell_live_csr(rows, cols, B, ell_cols, bci, val):
    """Restated count_blocked_ell_row_nnz_ + the emit order of
    convert::sliced_ell_from_blocked_ell (src/convert/sliced_ell_from_blocked_ell.cuh:36-62,
    251-270): the Blocked-ELL's live entries (valid slot, column < cols, value != 0
    as a float) per row, slots then lanes in order, as CSR."""
    f = lib().cso_bell_live_csr
    f.restype = C.c_uint64
    n = f(u32(rows), u32(cols), u32(B), u32(ell_cols), _p(bci), _p(val), None, None, None)
    ptr = np.zeros(rows + 1, np.uint32)
    idx = np.zeros(max(n, 1), np.uint32)
    v = np.zeros(max(n, 1), np.uint16)
    f(u32(rows), u32(cols), u32(B), u32(ell_cols), _p(bci), _p(val), _p(ptr), _p(idx), _p(v))
    return ptr, idx[:n], v[:n]


def sliced_ell_from_bell(rows, cols, B, ell_cols, bci, val, slice_rows):
    """Restated convert::sliced_ell_from_blocked_ell (sliced_ell_from_blocked_ell.cuh:233-276):
    the uniform layout and fill of the live entries."""
    ptr, idx, v = bell_live_csr(rows, cols, B, ell_cols, bci, val)
    r = sliced_ell_from_csr(rows, ptr, idx, v, slice_rows)
    r["row_ptr"] = ptr
    return r


def sliced_padded_slots(rows, ptr, candidate):
    f = lib().cso_sliced_padded_slots
    f.restype = C.c_uint64
    return int(f(u32(rows), _p(ptr), u32(candidate)))


def choose_sliced_slice_rows(rows, nnz, ptr, candidates):
    """Restated convert::choose_sliced_ell_slice_rows_from_compressed
    (src/convert/sliced_ell_from_blocked_ell.cuh:64-109,196-221): per candidate
    h clamped to [1, rows], score = padded_slots / nnz + 0.25 * slices / rows;
    lower score (1e-12 slack), then fewer padded bytes, then larger h.
    Returns (h, score, padded_bytes)."""
    best = None
    for h in candidates:
        if h == 0:
            continue
        hh = max(1, min(h, rows))
        S = (rows + hh - 1) // hh
        padded = sliced_padded_slots(rows, ptr, hh)
        nbytes = padded * 6 + (2 * S + 1) * 4
        score = (1.0 if nnz == 0 else padded / nnz) + 0.25 * (S / rows)
        if (best is None or score + 1e-12 < best[1] or (score <= best[1] + 1e-12 and nbytes < best[2])
                or (score <= best[1] + 1e-12 and nbytes == best[2] and hh > best[0])):
            best = (hh, score, nbytes)
    return best


def csr_transpose(cDim, uDim, ptr, idx, val):
    nnz = int(ptr[cDim]) if cDim else 0
    out_ptr = np.zeros(uDim + 1, np.uint32)
    out_idx = np.zeros(max(nnz, 1), np.uint32)
    out_val = np.zeros(max(nnz, 1), np.uint16)
    lib().cso_csr_transpose(u32(cDim), u32(uDim), _p(ptr), _p(idx), _p(val), _p(out_ptr), _p(out_idx), _p(out_val))
    return out_ptr, out_idx[:nnz], out_val[:nnz]


def major_nnz_plan(major_ptr, n, requested):
    nnz = np.zeros(max(n, 1), np.uint32)
    srt = np.zeros(max(n, 1), np.uint32)
    order = np.zeros(max(n, 1), np.uint32)
    B = 1 if n == 0 else min(max(requested, 1), n)
    offs = np.zeros(B + 1, np.uint32)
    lib().cso_major_nnz_plan(_p(major_ptr), u32(n), u32(requested), _p(nnz), _p(srt), _p(order), _p(offs))
    return nnz[:n], srt[:n], order[:n], offs


def pow2_bins(sorted_nnz):
    bins = np.zeros(34, np.uint32)
    lib().cso_pow2_bins(_p(np.ascontiguousarray(sorted_nnz, np.uint32)), u32(len(sorted_nnz)), _p(bins))
    return bins


def rebuild(ptr, idx, val, n, order):
    nnz = int(ptr[n]) if n else 0
    dptr = np.zeros(n + 1, np.uint32)
    didx = np.zeros(max(nnz, 1), np.uint32)
    dval = np.zeros(max(nnz, 1), np.uint16)
    inv = np.zeros(max(n, 1), np.uint32)
    lib().cso_rebuild(_p(ptr), _p(idx), _p(val), u32(n), _p(order), _p(dptr), _p(didx), _p(dval), _p(inv))
    return dptr, didx[:nnz], dval[:nnz], inv[:n]



# ---------------------------------------------------------------------------
# execution bucketing (src/io/csh5/execution_builders_part.hh:1011-1596)
# ---------------------------------------------------------------------------
def _seg_room(units, requested):
    return max(1, min(max(requested, 8), max(units, 1)))


def bell_bucketed(rows, B, ell_cols, bci, val, requested):
    """build_bucketed_execution_partition restated: the kept layout, its bytes
    and the segments' contents packed back to back."""
    o = lib()
    W = ell_cols // B if B else 0
    RB = (rows + B - 1) // B if B else 0
    room = _seg_room(RB, requested)
    order, widths = np.zeros(max(RB, 1), np.uint32), np.zeros(max(RB, 1), np.uint32)
    seg_rb, seg_w = np.zeros(room + 1, np.uint32), np.zeros(room, np.uint32)
    nbytes = C.c_uint64()
    o.cso_bell_exec_build_layout.restype = u32
    S = o.cso_bell_exec_build_layout(u32(rows), u32(B), u32(W), _p(np.ascontiguousarray(bci, np.uint32)),
                                     u32(requested), _p(order), _p(widths), _p(seg_rb), _p(seg_w), C.byref(nbytes))
    seg_rows = []
    for s in range(S):
        n = sum(min(B, rows - int(rb) * B) for rb in order[seg_rb[s]:seg_rb[s + 1]])
        seg_rows.append(n)
    n_idx = sum(int(seg_rb[s + 1] - seg_rb[s]) * int(seg_w[s]) for s in range(S))
    n_val = sum(seg_rows[s] * int(seg_w[s]) * B for s in range(S))
    seg_bci, seg_val = np.zeros(max(n_idx, 1), np.uint32), np.zeros(max(n_val, 1), np.uint16)
    e2c, c2e = np.zeros(max(rows, 1), np.uint32), np.zeros(max(rows, 1), np.uint32)
    o.cso_bell_exec_fill.restype = None
    o.cso_bell_exec_fill(u32(rows), u32(B), u32(W), _p(np.ascontiguousarray(bci, np.uint32)),
                         _p(np.ascontiguousarray(val, np.uint16)), _p(order), u32(S), _p(seg_rb), _p(seg_w),
                         _p(seg_bci), _p(seg_val), _p(e2c), _p(c2e))
    return {"segment_count": S, "bytes": nbytes.value, "order": order[:RB], "widths": widths[:RB],
            "seg_rb": seg_rb[:S + 1], "seg_w": seg_w[:S], "seg_rows": np.array(seg_rows, np.uint32),
            "seg_bci": seg_bci[:n_idx], "seg_val": seg_val[:n_val], "e2c": e2c[:rows], "c2e": c2e[:rows]}


def bell_choose_bucket_count(rows, B, ell_cols, bci):
    count, nbytes = C.c_uint32(), C.c_uint64()
    assert lib().cso_bell_choose_bucket_count(u32(rows), u32(B), u32(ell_cols // B if B else 0),
                                              _p(np.ascontiguousarray(bci, np.uint32)), C.byref(count),
                                              C.byref(nbytes)) == 1
    return count.value, nbytes.value


def _sell_args(offsets, widths, col_idx):
    return (_p(np.ascontiguousarray(offsets, np.uint32)), _p(np.ascontiguousarray(widths, np.uint32)),
            _p(np.ascontiguousarray(col_idx, np.uint32)))


def sell_bucketed(rows, offsets, widths, col_idx, val, requested):
    """build_bucketed_sliced_execution_partition restated."""
    o = lib()
    S_src = len(widths)
    room = _seg_room(rows, requested)
    order, rw, sw = (np.zeros(max(rows, 1), np.uint32) for _ in range(3))
    seg_row, seg_w = np.zeros(room + 1, np.uint32), np.zeros(room, np.uint32)
    nbytes = C.c_uint64()
    S = o.cso_sell_exec_build_layout(u32(rows), u32(S_src), *_sell_args(offsets, widths, col_idx), u32(requested),
                                     _p(order), _p(rw), _p(sw), _p(seg_row), _p(seg_w), C.byref(nbytes))
    assert S >= 0
    n = sum(int(seg_row[s + 1] - seg_row[s]) * int(seg_w[s]) for s in range(S))
    seg_col, seg_val = np.zeros(max(n, 1), np.uint32), np.zeros(max(n, 1), np.uint16)
    e2c, c2e = np.zeros(max(rows, 1), np.uint32), np.zeros(max(rows, 1), np.uint32)
    o.cso_sell_exec_fill.restype = None
    o.cso_sell_exec_fill(u32(rows), u32(S_src), *_sell_args(offsets, widths, col_idx),
                         _p(np.ascontiguousarray(val, np.uint16)), _p(order), u32(S), _p(seg_row), _p(seg_w),
                         _p(seg_col), _p(seg_val), _p(e2c), _p(c2e))
    return {"segment_count": S, "bytes": nbytes.value, "order": order[:rows], "row_widths": rw[:rows],
            "seg_row": seg_row[:S + 1], "seg_w": seg_w[:S], "seg_col": seg_col[:n], "seg_val": seg_val[:n],
            "e2c": e2c[:rows], "c2e": c2e[:rows]}


def sell_choose_bucket_count(rows, offsets, widths, col_idx):
    count, nbytes = C.c_uint32(), C.c_uint64()
    assert lib().cso_sell_choose_bucket_count(u32(rows), u32(len(widths)), *_sell_args(offsets, widths, col_idx),
                                              C.byref(count), C.byref(nbytes)) == 1
    return count.value, nbytes.value


def bell_bucket_plan(rows, B, ell_cols, bci):
    """bucket::build_plan restated: (order, width_sorted) of the row blocks."""
    RB = (rows + B - 1) // B if B else 0
    order, ws = np.zeros(max(RB, 1), np.uint32), np.zeros(max(RB, 1), np.uint32)
    lib().cso_bell_bucket_plan.restype = None
    lib().cso_bell_bucket_plan(u32(rows), u32(B), u32(ell_cols // B if B else 0),
                               _p(np.ascontiguousarray(bci, np.uint32)), _p(order), _p(ws))
    return order[:RB], ws[:RB]


def bell_estimate_bucketed_bytes(rows, B, order, width_sorted, buckets):
    f = lib().cso_bell_estimate_bucketed_bytes
    f.restype = C.c_uint64
    return f(u32(rows), u32(B), _p(np.ascontiguousarray(order, np.uint32)),
             _p(np.ascontiguousarray(width_sorted, np.uint32)), u32(len(order)), u32(buckets))


def bell_choose_ingest_bucket_count(rows, B, ell_cols, bci):
    f = lib().cso_bell_choose_ingest_bucket_count
    f.restype = u32
    return f(u32(rows), u32(B), u32(ell_cols // B if B else 0), _p(np.ascontiguousarray(bci, np.uint32)))


class HostCoo(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("storage", vp), ("rowIdx", vp), ("colIdx", vp),
                ("val", vp)]


def blocked_ell_from_coo(rows, cols, row, col, val, B, fmap=None):
    """Restated convert::blocked_ell_from_coo (blocked_ell_from_compressed.cuh:349-437): ell width,
    block columns, values, nnz (host count, GPU-path count) and total blocks; None when a
    row index is out of range."""
    f = lib().cso_blocked_ell_from_coo
    f.restype = C.c_longlong
    row, col = np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.uint16)
    m = None if fmap is None else np.ascontiguousarray(fmap, np.uint32)
    nz, tot = np.zeros(2, np.uint64), C.c_uint64()
    W = f(u32(rows), u32(cols), u32(len(row)), _p(row), _p(col), _p(val), _p(m), u32(B), None, None, _p(nz),
          C.byref(tot))
    if W < 0:
        return None
    RB = (rows + B - 1) // B
    bci, v = np.zeros(max(RB * W, 1), np.uint32), np.zeros(max(rows * W * B, 1), np.uint16)
    f(u32(rows), u32(cols), u32(len(row)), _p(row), _p(col), _p(val), _p(m), u32(B), _p(bci), _p(v), _p(nz),
      C.byref(tot))
    return {"ell_width": int(W), "ell_cols": int(W) * B, "bci": bci[:RB * W], "val": v[:rows * W * B],
            "nnz_host": int(nz[0]), "nnz_gpu": int(nz[1]), "total_blocks": tot.value}


def choose_block_size_from_coo(rows, cols, row, col, B_candidates, fmap=None):
    """choose_blocked_ell_block_size_from_coo restated: (block_size, fill_ratio, padded_bytes)."""
    f = lib().cso_coo_block_shape
    row, col = np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32)
    m = None if fmap is None else np.ascontiguousarray(fmap, np.uint32)
    best = None
    for B in B_candidates:
        if B == 0:
            continue
        w, tot = C.c_uint32(), C.c_uint64()
        assert f(u32(rows), u32(len(row)), _p(row), _p(col), _p(m), u32(B), C.byref(w), C.byref(tot)) == 1
        RB = (rows + B - 1) // B
        padded = rows * w.value * B * 2
        fill = 1.0 if (RB == 0 or w.value == 0) else tot.value / float(RB * w.value)
        if (best is None or padded + 1 < best[2] or (padded == best[2] and fill > best[1] + 1e-9)
                or (padded == best[2] and fill + 1e-9 >= best[1] and B > best[0])):
            best = (B, fill, padded)
    return best


# ---------------------------------------------------------------------------
# .cspack raw records (src/io/pack/packfile.cu:13-47,265-272,351-369,597-621,715-721)
# ---------------------------------------------------------------------------
CSPACK_COMPRESSED, CSPACK_COO, CSPACK_BLOCKED_ELL, CSPACK_SLICED_ELL = 2, 3, 6, 7


def cspack_record(fmt, rows, cols, nnz, parts):
    """Bytes of one record: the 13-byte header (u8 format, u32 rows, cols, nnz)
    then the format's words and arrays, little-endian, no padding."""
    head = np.array([fmt], np.uint8).tobytes() + np.array([rows, cols, nnz], np.uint32).tobytes()
    return head + b"".join(np.ascontiguousarray(p).tobytes() for p in parts)


def cspack_blocked_ell(rows, cols, nnz, B, ell_cols, bci, val):
    return cspack_record(CSPACK_BLOCKED_ELL, rows, cols, nnz,
                         [np.array([B, ell_cols], np.uint32), np.asarray(bci, np.uint32), np.asarray(val, np.uint16)])


def cspack_sliced_ell(rows, cols, nnz, offsets, widths, col_idx, val):
    return cspack_record(CSPACK_SLICED_ELL, rows, cols, nnz,
                         [np.array([len(widths)], np.uint32), np.asarray(offsets, np.uint32),
                          np.asarray(widths, np.uint32), np.asarray(col_idx, np.uint32), np.asarray(val, np.uint16)])


def cspack_compressed(rows, cols, nnz, axis, ptr, idx, val):
    major = cols if axis == 1 else rows
    parts = [np.array([axis], np.uint32), np.asarray(val, np.uint16)]
    if major:
        parts.append(np.asarray(ptr, np.uint32))
    parts.append(np.asarray(idx, np.uint32))
    return cspack_record(CSPACK_COMPRESSED, rows, cols, nnz, parts)


def cspack_coo(rows, cols, row, col, val):
    return cspack_record(CSPACK_COO, rows, cols, len(row),
                         [np.asarray(val, np.uint16), np.asarray(row, np.uint32), np.asarray(col, np.uint32)])

# ---------------------------------------------------------------------------
# the reference's own code (compiled from its sources into _ref/)
# ---------------------------------------------------------------------------
class HostCompressed(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("axis", u32), ("flags", u32),
                ("storage", vp), ("majorPtr", vp), ("minorIdx", vp), ("val", vp), ("_pad", C.c_uint64)]


class HostBlockedEll(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("block_size", u32), ("ell_cols", u32),
                ("flags", u32), ("storage", vp), ("blockColIdx", vp), ("val", vp)]


class HostSlicedEll(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("slice_count", u32), ("flags", u32),
                ("storage", vp), ("slice_row_offsets", vp), ("slice_widths", vp), ("col_idx", vp),
                ("val", vp)]


class BlockedTune(C.Structure):
    _fields_ = [("block_size", C.c_uint), ("fill_ratio", C.c_double), ("padded_bytes", C.c_size_t)]


class SlicedTune(C.Structure):
    _fields_ = [("slice_rows", C.c_uint), ("slice_count", C.c_uint), ("padded_slots", C.c_size_t),
                ("padded_bytes", C.c_size_t), ("storage_ratio", C.c_double), ("slice_penalty", C.c_double),
                ("score", C.c_double)]


_r = None


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _r
    if _r is None:
        r = C.CDLL(str(REF_LIB))
        r.csref_free.argtypes = [vp]
        r.csref_free.restype = None
        for name in ("csref_blocked_ell_from_compressed", "csref_sliced_ell_from_compressed"):
            getattr(r, name).argtypes = [vp, C.c_uint, vp]
        for name in ("csref_choose_blocked_ell_block_size", "csref_choose_sliced_ell_slice_rows_from_compressed"):
            getattr(r, name).argtypes = [vp, vp, C.c_uint, vp]
        r.csref_sliced_total_slots.argtypes = [vp]
        r.csref_sliced_total_slots.restype = u32
        r.csref_sliced_ell_from_blocked_ell.argtypes = [vp, C.c_uint, vp]
        r.csref_choose_sliced_ell_slice_rows_from_blocked_ell.argtypes = [vp, vp, C.c_uint, vp]
        _r = r
    return _r


def host_csr(rows, cols, ptr, idx, val):
    h = HostCompressed()
    h.rows, h.cols, h.nnz, h.axis = rows, cols, len(idx), 0
    h.majorPtr, h.minorIdx, h.val = _p(ptr), _p(idx), _p(val)
    return h


def ref_blocked_ell_from_compressed(rows, cols, ptr, idx, val, B):
    src = host_csr(rows, cols, ptr, idx, val)
    dst = HostBlockedEll()
    ok = ref().csref_blocked_ell_from_compressed(C.byref(src), C.c_uint(B), C.byref(dst))
    if ok != 1:
        return None
    rb = (dst.rows + B - 1) // B
    W = dst.ell_cols // B if B else 0
    bci = np.ctypeslib.as_array(C.cast(dst.blockColIdx, C.POINTER(u32)), (rb * W,)).copy() if rb * W else \
        np.zeros(0, np.uint32)
    n = dst.rows * dst.ell_cols
    v = np.ctypeslib.as_array(C.cast(dst.val, C.POINTER(C.c_uint16)), (n,)).copy() if n else np.zeros(0, np.uint16)
    res = {"ell_cols": dst.ell_cols, "ell_width": W, "bci": bci, "val": v, "nnz": dst.nnz}
    ref().csref_free(dst.storage)
    return res


def ref_choose_blocked_ell_block_size(rows, cols, ptr, idx, val, candidates):
    src = host_csr(rows, cols, ptr, idx, val)
    c = (C.c_uint * len(candidates))(*candidates)
    out = BlockedTune()
    ok = ref().csref_choose_blocked_ell_block_size(C.byref(src), c, C.c_uint(len(candidates)), C.byref(out))
    return (out.block_size, out.fill_ratio, out.padded_bytes) if ok == 1 else None


def ref_sliced_ell_from_compressed(rows, cols, ptr, idx, val, slice_rows):
    src = host_csr(rows, cols, ptr, idx, val)
    dst = HostSlicedEll()
    ok = ref().csref_sliced_ell_from_compressed(C.byref(src), C.c_uint(slice_rows), C.byref(dst))
    if ok != 1:
        return None
    S = dst.slice_count
    f = ref().csref_sliced_total_slots
    f.restype = u32
    total = f(C.byref(dst))

    def arr(p, n, t):
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(t)), (n,)).copy() if n else np.zeros(0, np.dtype(t))

    res = {"slice_count": S, "offsets": arr(dst.slice_row_offsets, S + 1 if dst.storage else 0, u32),
           "widths": arr(dst.slice_row_offsets and dst.slice_widths, S, u32),
           "col_idx": arr(dst.col_idx, total, u32), "val": arr(dst.val, total, C.c_uint16), "nnz": dst.nnz,
           "total_slots": int(total)}
    if dst.storage:
        ref().csref_free(dst.storage)
    return res


def host_bell(rows, cols, nnz, B, ell_cols, bci, val):
    h = HostBlockedEll()
    h.rows, h.cols, h.nnz, h.block_size, h.ell_cols = rows, cols, nnz, B, ell_cols
    h.blockColIdx, h.val = _p(bci), _p(val)
    return h


def _sliced_result(dst):
    S = dst.slice_count
    total = ref().csref_sliced_total_slots(C.byref(dst))

    def arr(p, n, t):
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(t)), (n,)).copy() if n else np.zeros(0, np.dtype(t))

    res = {"slice_count": S, "offsets": arr(dst.slice_row_offsets, S + 1 if dst.storage else 0, u32),
           "widths": arr(dst.slice_widths, S, u32), "col_idx": arr(dst.col_idx, total, u32),
           "val": arr(dst.val, total, C.c_uint16), "nnz": dst.nnz, "total_slots": int(total)}
    if dst.storage:
        ref().csref_free(dst.storage)
    return res


def ref_sliced_ell_from_blocked_ell(rows, cols, nnz, B, ell_cols, bci, val, slice_rows):
    """convert::sliced_ell_from_blocked_ell of the reference, run on the host."""
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    dst = HostSlicedEll()
    ok = ref().csref_sliced_ell_from_blocked_ell(C.byref(src), C.c_uint(slice_rows), C.byref(dst))
    return _sliced_result(dst) if ok == 1 else None


def ref_choose_sliced_ell_slice_rows_from_blocked_ell(rows, cols, nnz, B, ell_cols, bci, val, candidates):
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    c = (C.c_uint * len(candidates))(*candidates)
    out = SlicedTune()
    ok = ref().csref_choose_sliced_ell_slice_rows_from_blocked_ell(C.byref(src), c, C.c_uint(len(candidates)),
                                                                   C.byref(out))
    if ok != 1:
        return None
    return {k: getattr(out, k) for k, _ in SlicedTune._fields_}


def ref_choose_sliced_ell_slice_rows(rows, cols, ptr, idx, val, candidates):
    src = host_csr(rows, cols, ptr, idx, val)
    c = (C.c_uint * len(candidates))(*candidates)
    out = SlicedTune()
    ok = ref().csref_choose_sliced_ell_slice_rows_from_compressed(C.byref(src), c, C.c_uint(len(candidates)),
                                                                  C.byref(out))
    if ok != 1:
        return None
    return {k: getattr(out, k) for k, _ in SlicedTune._fields_}


def host_coo(rows, cols, row, col, val):
    h = HostCoo()
    h.rows, h.cols, h.nnz = rows, cols, len(row)
    h.rowIdx, h.colIdx, h.val = _p(row), _p(col), _p(val)
    return h


def _bell_result(dst, B, free):
    rb = (dst.rows + B - 1) // B
    W = dst.ell_cols // B if B else 0
    bci = np.ctypeslib.as_array(C.cast(dst.blockColIdx, C.POINTER(u32)), (rb * W,)).copy() if rb * W else \
        np.zeros(0, np.uint32)
    n = dst.rows * dst.ell_cols
    v = np.ctypeslib.as_array(C.cast(dst.val, C.POINTER(C.c_uint16)), (n,)).copy() if n else np.zeros(0, np.uint16)
    res = {"ell_cols": dst.ell_cols, "ell_width": W, "bci": bci, "val": v, "nnz": dst.nnz, "rows": dst.rows,
           "cols": dst.cols}
    if dst.storage:
        free(dst.storage)
    return res


def ref_blocked_ell_from_coo(rows, cols_src, cols, row, col, val, B, fmap=None):
    """convert::blocked_ell_from_coo of the reference (host loops)."""
    row, col = np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.uint16)
    m = None if fmap is None else np.ascontiguousarray(fmap, np.uint32)
    src = host_coo(rows, cols_src, row, col, val)
    dst = HostBlockedEll()
    r = ref()
    r.csref_blocked_ell_from_coo.argtypes = [vp, u32, vp, C.c_uint, vp]
    ok = r.csref_blocked_ell_from_coo(C.byref(src), cols, _p(m), B, C.byref(dst))
    return _bell_result(dst, B, r.csref_free) if ok == 1 else None


def ref_choose_block_size_from_coo(rows, cols_src, cols, row, col, val, candidates, fmap=None):
    row, col = np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.uint16)
    m = None if fmap is None else np.ascontiguousarray(fmap, np.uint32)
    src = host_coo(rows, cols_src, row, col, val)
    c = (C.c_uint * len(candidates))(*candidates)
    out = BlockedTune()
    r = ref()
    r.csref_choose_blocked_ell_block_size_from_coo.argtypes = [vp, u32, vp, vp, C.c_uint, vp]
    ok = r.csref_choose_blocked_ell_block_size_from_coo(C.byref(src), cols, _p(m), c, len(candidates), C.byref(out))
    return (out.block_size, out.fill_ratio, out.padded_bytes) if ok == 1 else None


def ref_gpu_blocked_ell_from_coo_cuda(rows, cols_src, cols, row, col, val, B, fmap=None):
    """convert::blocked_ell_from_coo_cuda of the reference, run on the GPU."""
    row, col = np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.uint16)
    m = None if fmap is None else np.ascontiguousarray(fmap, np.uint32)
    src = host_coo(rows, cols_src, row, col, val)
    dst = HostBlockedEll()
    g = ref_gpu()
    g.csrefgpu_blocked_ell_from_coo_cuda.argtypes = [vp, u32, vp, C.c_uint, vp]
    g.csrefgpu_free.argtypes = [vp]
    g.csrefgpu_free.restype = None
    ok = g.csrefgpu_blocked_ell_from_coo_cuda(C.byref(src), cols, _p(m), B, C.byref(dst))
    return _bell_result(dst, B, g.csrefgpu_free) if ok == 1 else None


def ref_gpu_choose_block_size_from_coo_cuda(rows, cols_src, cols, row, col, val, candidates, fmap=None):
    row, col = np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.uint16)
    m = None if fmap is None else np.ascontiguousarray(fmap, np.uint32)
    src = host_coo(rows, cols_src, row, col, val)
    c = (C.c_uint * len(candidates))(*candidates)
    out = BlockedTune()
    g = ref_gpu()
    g.csrefgpu_choose_blocked_ell_block_size_from_coo_cuda.argtypes = [vp, u32, vp, vp, C.c_uint, vp]
    ok = g.csrefgpu_choose_blocked_ell_block_size_from_coo_cuda(C.byref(src), cols, _p(m), c, len(candidates),
                                                                C.byref(out))
    return (out.block_size, out.fill_ratio, out.padded_bytes) if ok == 1 else None


_rg = None


def ref_gpu_available() -> bool:
    return REF_GPU_LIB.exists()


def ref_gpu() -> C.CDLL:
    global _rg
    if _rg is None:
        g = C.CDLL(str(REF_GPU_LIB))
        g.csrefgpu_filter_blocked_ell.argtypes = [vp, u32, u32, vp, vp, vp]
        for name in ("csrefgpu_group_reduce_blocked_ell", "csrefgpu_group_reduce_sliced_ell",
                     "csrefgpu_group_reduce_compressed"):
            getattr(g, name).argtypes = [vp, vp, u32, vp, vp, vp]
        g.csrefgpu_reoptimize.argtypes = [vp, vp, u32, u32, vp, vp, vp, u32, vp]
        g.csrefgpu_transpose.argtypes = [u32, u32, u32, vp, vp, vp, vp, vp, vp]
        g.csrefgpu_major_nnz_plan.argtypes = [vp, u32, vp, vp, vp, vp, vp, u32]
        g.csrefgpu_rebuild.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp, vp]
        g.csrefgpu_sliced_ell_from_compressed_cuda.argtypes = [vp, C.c_uint, vp]
        fp = C.POINTER(C.c_float)
        g.csrefgpu_transpose_timed.argtypes = [u32, u32, u32, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, fp]
        g.csrefgpu_major_nnz_plan_timed.argtypes = [vp, u32, vp, vp, vp, vp, vp, u32, C.c_int, C.c_int, fp]
        g.csrefgpu_group_reduce_blocked_ell_timed.argtypes = [vp, vp, u32, vp, vp, C.c_int, C.c_int, fp]
        g.csrefgpu_group_reduce_sliced_ell_timed.argtypes = [vp, vp, u32, vp, vp, C.c_int, C.c_int, fp]
        g.csrefgpu_group_reduce_compressed_timed.argtypes = [vp, vp, u32, vp, vp, C.c_int, C.c_int, fp]
        _rg = g
    return _rg


# ---------------------------------------------------------------------------
# the reference's execution-bucketing builders (_ref/libcs_ref_bucket.so)
# ---------------------------------------------------------------------------
REF_BUCKET_LIB = HERE / "_ref" / "libcs_ref_bucket.so"


class HostBucketedBell(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("segment_count", u32), ("segments", vp),
                ("segment_row_offsets", vp), ("exec_to_canonical_rows", vp), ("canonical_to_exec_rows", vp),
                ("exec_to_canonical_cols", vp), ("canonical_to_exec_cols", vp)]


class HostBucketedSell(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("segment_count", u32), ("segments", vp),
                ("segment_row_offsets", vp), ("exec_to_canonical_rows", vp), ("canonical_to_exec_rows", vp),
                ("canonical_slice_count", u32), ("canonical_slice_row_offsets", vp),
                ("canonical_slice_widths", vp)]


_rb = None


def ref_bucket_available() -> bool:
    return REF_BUCKET_LIB.exists()


def ref_bucket() -> C.CDLL:
    global _rb
    if _rb is None:
        b = C.CDLL(str(REF_BUCKET_LIB))
        b.csrefb_build_bucketed_blocked_ell.argtypes = [vp, u32, vp, vp]
        b.csrefb_build_bucketed_sliced_ell.argtypes = [vp, u32, vp, vp]
        b.csrefb_choose_bucket_count_for_part.argtypes = [vp, vp, vp]
        b.csrefb_choose_bucket_count_for_sliced_part.argtypes = [vp, vp, vp]
        for name in ("csrefb_clear_bucketed_blocked_ell", "csrefb_clear_bucketed_sliced_ell"):
            getattr(b, name).argtypes = [vp]
            getattr(b, name).restype = None
        _rb = b
    return _rb


def _arr(p, n, t):
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(t)), (n,)).copy() if n and p else np.zeros(0, np.dtype(t))


def read_bucketed_bell(out):
    """Host bucketed Blocked-ELL struct -> dict (reference layout)."""
    S, rows, cols = out.segment_count, out.rows, out.cols
    segs = []
    base = C.cast(out.segments, C.POINTER(HostBlockedEll)) if S else None
    for s in range(S):
        m = base[s]
        B = m.block_size
        rb = (m.rows + B - 1) // B if B else 0
        w = m.ell_cols // B if B else 0
        segs.append({"rows": m.rows, "cols": m.cols, "nnz": m.nnz, "block_size": B, "ell_cols": m.ell_cols,
                     "bci": _arr(m.blockColIdx, rb * w, u32), "val": _arr(m.val, m.rows * m.ell_cols, C.c_uint16)})
    return {"rows": rows, "cols": cols, "nnz": out.nnz, "segment_count": S, "segments": segs,
            "segment_row_offsets": _arr(out.segment_row_offsets, S + 1, u32),
            "e2c": _arr(out.exec_to_canonical_rows, rows, u32), "c2e": _arr(out.canonical_to_exec_rows, rows, u32),
            "e2c_cols": _arr(out.exec_to_canonical_cols, cols, u32),
            "c2e_cols": _arr(out.canonical_to_exec_cols, cols, u32)}


def read_bucketed_sell(out):
    S, rows = out.segment_count, out.rows
    segs = []
    base = C.cast(out.segments, C.POINTER(HostSlicedEll)) if S else None
    for s in range(S):
        m = base[s]
        offs = _arr(m.slice_row_offsets, m.slice_count + 1, u32) if m.slice_count else np.zeros(1, np.uint32)
        widths = _arr(m.slice_widths, m.slice_count, u32)
        total = int(sum(int(offs[i + 1] - offs[i]) * int(widths[i]) for i in range(m.slice_count)))
        segs.append({"rows": m.rows, "cols": m.cols, "nnz": m.nnz, "slice_count": m.slice_count,
                     "offsets": offs, "widths": widths, "col_idx": _arr(m.col_idx, total, u32),
                     "val": _arr(m.val, total, C.c_uint16)})
    cs = out.canonical_slice_count
    return {"rows": rows, "cols": out.cols, "nnz": out.nnz, "segment_count": S, "segments": segs,
            "segment_row_offsets": _arr(out.segment_row_offsets, S + 1, u32),
            "e2c": _arr(out.exec_to_canonical_rows, rows, u32), "c2e": _arr(out.canonical_to_exec_rows, rows, u32),
            "canonical_slice_count": cs, "canonical_slice_row_offsets": _arr(out.canonical_slice_row_offsets,
                                                                             cs + 1, u32),
            "canonical_slice_widths": _arr(out.canonical_slice_widths, cs, u32)}


def host_sell(rows, cols, nnz, offsets, widths, col_idx, val):
    h = HostSlicedEll()
    h.rows, h.cols, h.nnz, h.slice_count = rows, cols, nnz, len(widths)
    h.slice_row_offsets, h.slice_widths, h.col_idx, h.val = _p(offsets), _p(widths), _p(col_idx), _p(val)
    return h


def ref_build_bucketed_bell(rows, cols, nnz, B, ell_cols, bci, val, requested):
    """build_bucketed_blocked_ell_partition of the reference, on the host."""
    bci, val = np.ascontiguousarray(bci, np.uint32), np.ascontiguousarray(val, np.uint16)
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    out, nbytes = HostBucketedBell(), C.c_uint64()
    ok = ref_bucket().csrefb_build_bucketed_blocked_ell(C.byref(src), requested, C.byref(out), C.byref(nbytes))
    res = read_bucketed_bell(out) if ok == 1 else None
    ref_bucket().csrefb_clear_bucketed_blocked_ell(C.byref(out))
    if res is not None:
        res["bytes"] = nbytes.value
    return res


def ref_choose_bucket_count_for_part(rows, cols, nnz, B, ell_cols, bci, val):
    bci, val = np.ascontiguousarray(bci, np.uint32), np.ascontiguousarray(val, np.uint16)
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    count, nbytes = C.c_uint32(), C.c_uint64()
    assert ref_bucket().csrefb_choose_bucket_count_for_part(C.byref(src), C.byref(count), C.byref(nbytes)) == 1
    return count.value, nbytes.value


def ref_build_bucketed_sell(rows, cols, nnz, offsets, widths, col_idx, val, requested):
    arrs = [np.ascontiguousarray(a, np.uint32) for a in (offsets, widths, col_idx)]
    val = np.ascontiguousarray(val, np.uint16)
    src = host_sell(rows, cols, nnz, *arrs, val)
    out, nbytes = HostBucketedSell(), C.c_uint64()
    ok = ref_bucket().csrefb_build_bucketed_sliced_ell(C.byref(src), requested, C.byref(out), C.byref(nbytes))
    res = read_bucketed_sell(out) if ok == 1 else None
    ref_bucket().csrefb_clear_bucketed_sliced_ell(C.byref(out))
    if res is not None:
        res["bytes"] = nbytes.value
    return res


def ref_choose_bucket_count_for_sliced_part(rows, cols, nnz, offsets, widths, col_idx, val):
    arrs = [np.ascontiguousarray(a, np.uint32) for a in (offsets, widths, col_idx)]
    val = np.ascontiguousarray(val, np.uint16)
    src = host_sell(rows, cols, nnz, *arrs, val)
    count, nbytes = C.c_uint32(), C.c_uint64()
    assert ref_bucket().csrefb_choose_bucket_count_for_sliced_part(C.byref(src), C.byref(count),
                                                                   C.byref(nbytes)) == 1
    return count.value, nbytes.value



def ref_cspack_store(fmt, path, rows, cols, nnz, *arrays):
    """The reference's store_*_raw writing one record to `path`."""
    b = ref_bucket()
    a = [np.ascontiguousarray(x) for x in arrays]
    s = str(path).encode()
    if fmt == CSPACK_BLOCKED_ELL:
        B, ell_cols, bci, val = arrays
        bci, val = np.ascontiguousarray(bci, np.uint32), np.ascontiguousarray(val, np.uint16)
        b.csrefb_store_blocked_ell_raw.argtypes = [C.c_char_p, u32, u32, u32, u32, u32, vp, vp]
        return b.csrefb_store_blocked_ell_raw(s, rows, cols, nnz, B, ell_cols, _p(bci), _p(val))
    if fmt == CSPACK_SLICED_ELL:
        offs, widths, col, val = (np.ascontiguousarray(x, t) for x, t in zip(arrays, (np.uint32, np.uint32,
                                                                                      np.uint32, np.uint16)))
        b.csrefb_store_sliced_ell_raw.argtypes = [C.c_char_p, u32, u32, u32, u32, vp, vp, vp, vp]
        return b.csrefb_store_sliced_ell_raw(s, rows, cols, nnz, len(widths), _p(offs), _p(widths), _p(col), _p(val))
    if fmt == CSPACK_COMPRESSED:
        axis, ptr, idx, val = arrays
        ptr, idx, val = (np.ascontiguousarray(x, t) for x, t in zip((ptr, idx, val), (np.uint32, np.uint32,
                                                                                        np.uint16)))
        b.csrefb_store_compressed_raw.argtypes = [C.c_char_p, u32, u32, u32, u32, vp, vp, vp]
        return b.csrefb_store_compressed_raw(s, rows, cols, nnz, axis, _p(ptr), _p(idx), _p(val))
    row, col, val = (np.ascontiguousarray(x, t) for x, t in zip(arrays, (np.uint32, np.uint32, np.uint16)))
    b.csrefb_store_coo_raw.argtypes = [C.c_char_p, u32, u32, u32, vp, vp, vp]
    return b.csrefb_store_coo_raw(s, rows, cols, nnz, _p(row), _p(col), _p(val))


# ---------------------------------------------------------------------------
# the reference's ingest-time chooser (_ref/libcs_ref_ingest.so; its plan runs on the GPU)
# ---------------------------------------------------------------------------
REF_INGEST_LIB = HERE / "_ref" / "libcs_ref_ingest.so"
_ri = None


def ref_ingest_available() -> bool:
    return REF_INGEST_LIB.exists()


def ref_ingest() -> C.CDLL:
    global _ri
    if _ri is None:
        r = C.CDLL(str(REF_INGEST_LIB))
        r.csrefi_bucket_plan.argtypes = [vp, vp, vp]
        r.csrefi_estimate_bucketed_bytes.argtypes = [vp, vp, vp, u32, u32]
        r.csrefi_estimate_bucketed_bytes.restype = C.c_ulonglong
        r.csrefi_choose_bucket_count_for_part.argtypes = [vp, vp]
        _ri = r
    return _ri


def ref_bucket_plan(rows, cols, nnz, B, ell_cols, bci, val):
    bci, val = np.ascontiguousarray(bci, np.uint32), np.ascontiguousarray(val, np.uint16)
    RB = (rows + B - 1) // B
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    order, ws = np.zeros(max(RB, 1), np.uint32), np.zeros(max(RB, 1), np.uint32)
    assert ref_ingest().csrefi_bucket_plan(C.byref(src), _p(order), _p(ws)) == 1
    return order[:RB], ws[:RB]


def ref_estimate_bucketed_bytes(rows, cols, nnz, B, ell_cols, bci, val, order, ws, buckets):
    bci, val = np.ascontiguousarray(bci, np.uint32), np.ascontiguousarray(val, np.uint16)
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    return ref_ingest().csrefi_estimate_bucketed_bytes(C.byref(src), _p(np.ascontiguousarray(order, np.uint32)),
                                                       _p(np.ascontiguousarray(ws, np.uint32)), len(order), buckets)


def ref_choose_ingest_bucket_count(rows, cols, nnz, B, ell_cols, bci, val):
    bci, val = np.ascontiguousarray(bci, np.uint32), np.ascontiguousarray(val, np.uint16)
    src = host_bell(rows, cols, nnz, B, ell_cols, bci, val)
    count = C.c_uint32()
    assert ref_ingest().csrefi_choose_bucket_count_for_part(C.byref(src), C.byref(count)) == 1
    return count.value


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# CPU baselines: the reference's host conversions (and the restated CPU paths
# where the reference has none) timed over independent partitions on a pool
# of host threads.  ctypes releases the GIL inside the foreign call, so the
# threads run in parallel.  Outputs are freed, not copied back.
# ---------------------------------------------------------------------------
def _pool_time(parts, one, threads, seconds):
    """Runs one(part) over `parts` on `threads` threads, repeating the list until
    `seconds` of wall time have passed (at least once); returns (seconds, passes)."""
    import time
    from concurrent.futures import ThreadPoolExecutor

    t0 = time.perf_counter()
    passes = 0
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        while True:
            list(ex.map(one, parts))
            passes += 1
            if time.perf_counter() - t0 >= seconds or passes >= 50:
                break
    return (time.perf_counter() - t0) / passes, passes


def ref_time_blocked_ell_from_compressed(parts, B, threads, seconds=3.0):
    """convert::blocked_ell_from_compressed (the reference's host routine) on every
    (rows, cols, ptr, idx, val) partition; seconds per pass over all partitions."""
    def one(p):
        rows, cols, ptr, idx, val = p
        src = host_csr(rows, cols, ptr, idx, val)
        dst = HostBlockedEll()
        assert ref().csref_blocked_ell_from_compressed(C.byref(src), C.c_uint(B), C.byref(dst)) == 1
        ref().csref_free(dst.storage)

    return _pool_time(parts, one, threads, seconds)


def ref_time_sliced_ell_from_compressed(parts, slice_rows, threads, seconds=3.0, candidates=None):
    """convert::sliced_ell_from_compressed (host) at `slice_rows`, or, with
    `candidates`, choose_sliced_ell_slice_rows_from_compressed first and convert at
    its choice; seconds per pass over all partitions."""
    def one(p):
        rows, cols, ptr, idx, val = p
        src = host_csr(rows, cols, ptr, idx, val)
        h = slice_rows
        if candidates:
            c = (C.c_uint * len(candidates))(*candidates)
            out = SlicedTune()
            assert ref().csref_choose_sliced_ell_slice_rows_from_compressed(C.byref(src), c, C.c_uint(len(candidates)),
                                                                            C.byref(out)) == 1
            h = out.slice_rows
        dst = HostSlicedEll()
        assert ref().csref_sliced_ell_from_compressed(C.byref(src), C.c_uint(h), C.byref(dst)) == 1
        ref().csref_free(dst.storage)

    return _pool_time(parts, one, threads, seconds)


def time_restated(fn, parts, threads, seconds=3.0):
    """Seconds per pass of a restated CPU routine fn(part) over `parts`."""
    return _pool_time(parts, fn, threads, seconds)


def ref_time_sliced_ell_from_blocked_ell(parts, slice_rows, threads, seconds=3.0):
    """convert::sliced_ell_from_blocked_ell (the reference's host routine) on every
    (rows, cols, B, ell_cols, bci, val) Blocked-ELL partition; seconds per pass."""
    def one(p):
        rows, cols, B, ell_cols, bci, val = p
        src = host_bell(rows, cols, 0, B, ell_cols, bci, val)
        dst = HostSlicedEll()
        assert ref().csref_sliced_ell_from_blocked_ell(C.byref(src), C.c_uint(slice_rows), C.byref(dst)) == 1
        if dst.storage:
            ref().csref_free(dst.storage)

    return _pool_time(parts, one, threads, seconds)


class _FilterOut:
    """Output arrays of the restated filter for one partition, allocated once so
    the timed passes run the filter alone."""

    def __init__(self, rows, ell_cols):
        cap = max(rows * ell_cols, 1)
        self.major = np.zeros(rows + 1, np.uint32)
        self.idx = np.zeros(cap, np.uint32)
        self.val = np.zeros(cap, np.uint16)


def _filter_one(p, out):
    rows, cols, B, ell_cols, bci, val, row_keep, feature_keep = p
    f = lib().cso_reoptimize_bell
    f.restype = C.c_longlong
    n = f(u32(rows), u32(cols), u32(B), u32(ell_cols), _p(bci), _p(val), _p(row_keep), _p(feature_keep), None, None,
          u32(rows), u32(cols), _p(out.major), _p(out.idx), _p(out.val))
    assert n >= 0
    return n


def time_filter_bell(parts, threads, seconds=3.0):
    """The restated filtered Blocked-ELL -> CSR (cso_reoptimize_bell: kept rows,
    kept features, no remaps) on every (rows, cols, B, ell_cols, bci, val,
    row_keep, feature_keep) partition; seconds per pass."""
    outs = {id(p): _FilterOut(p[0], p[3]) for p in parts}
    return _pool_time(parts, lambda p: _filter_one(p, outs[id(p)]), threads, seconds)


def time_repack_bell(parts, B_out, buckets, threads, seconds=3.0):
    """The restated repack of every Blocked-ELL partition: filter to CSR, nnz plan
    over `buckets` buckets, row rebuild in plan order (all restated), then the
    reference's convert::blocked_ell_from_compressed at block B_out; seconds per pass."""
    outs = {id(p): _FilterOut(p[0], p[3]) for p in parts}

    def one(p):
        o = outs[id(p)]
        rows, cols = p[0], p[1]
        n = _filter_one(p, o)
        ptr, idx, val = o.major, o.idx[:n], o.val[:n]
        _, _, order, _ = major_nnz_plan(ptr, rows, buckets)
        dptr, didx, dval, _ = rebuild(ptr, idx, val, rows, order)
        src = host_csr(rows, cols, dptr, didx, dval)
        dst = HostBlockedEll()
        assert ref().csref_blocked_ell_from_compressed(C.byref(src), C.c_uint(B_out), C.byref(dst)) == 1
        ref().csref_free(dst.storage)

    return _pool_time(parts, one, threads, seconds)


def time_rebuild(parts, threads, seconds=3.0):
    """The restated row rebuild (cso_rebuild) of every (rows, cols, ptr, idx, val)
    partition in its nnz-plan order (the plan made once, outside the timing);
    seconds per pass."""
    prepared = []
    for rows, cols, ptr, idx, val in parts:
        _, _, order, _ = major_nnz_plan(ptr, rows, 64)
        nnz = int(ptr[rows]) if rows else 0
        prepared.append((rows, ptr, idx, val, order, np.zeros(rows + 1, np.uint32), np.zeros(max(nnz, 1), np.uint32),
                         np.zeros(max(nnz, 1), np.uint16), np.zeros(max(rows, 1), np.uint32)))

    def one(q):
        rows, ptr, idx, val, order, dptr, didx, dval, inv = q
        lib().cso_rebuild(_p(ptr), _p(idx), _p(val), u32(rows), _p(order), _p(dptr), _p(didx), _p(dval), _p(inv))

    return _pool_time(prepared, one, threads, seconds)
