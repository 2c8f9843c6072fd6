"""Execution bucketing on the GPU (build_bucketed_blocked_ell_partition,
build_bucketed_sliced_ell_partition and the two bucket-count choosers) against
the reference's own builders (golden/ref_bucketing.npz and, where
oracle/_ref is present, the compiled builders live) and the restatement."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
INVALID = 0xFFFFFFFF


def _dev_bell(rows, cols, nnz, B, ell_cols, bci, val):
    import torch

    from cellshard_b200.device import BlockedELL

    return BlockedELL(rows, cols, B, ell_cols,
                      torch.from_numpy(np.ascontiguousarray(bci, np.uint32).view(np.int32).copy()).cuda(),
                      torch.from_numpy(np.ascontiguousarray(val, np.uint16).view(np.float16).copy()).cuda(), nnz)


def _dev_sell(rows, cols, nnz, offsets, widths, col, val):
    import torch

    from cellshard_b200.device import SlicedELL

    offsets, widths = np.asarray(offsets, np.int64), np.asarray(widths, np.int64)
    slots = np.concatenate([[0], np.cumsum(np.diff(offsets) * widths)[:-1]]) if len(widths) else np.zeros(0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32).copy()).cuda()
    return SlicedELL(rows, cols, nnz, 0, t(offsets), t(widths), t(slots), t(col),
                     torch.from_numpy(np.ascontiguousarray(val, np.uint16).view(np.float16).copy()).cuda())


def _flat(bp):
    p = bp.plan
    return np_u32(bp.idx)[:p["index_entries"]], np_u16(bp.val)[:p["value_entries"]]


def test_blocked_matches_reference_vectors(cuda):
    """Golden outputs of the reference's builders on its own Blocked-ELL
    conversions (B = 4 takes the per-half copy, B = 16 the 16-byte one)."""
    from cellshard_b200.device import bucketed_blocked_ell

    conv, gold = np.load(GOLD / "ref_conversions.npz"), np.load(GOLD / "ref_bucketing.npz")
    checked = 0
    for n in sorted({k.split("/")[0] for k in gold.files}):
        rows, cols = (int(x) for x in conv[f"{n}/shape"])
        for B in (4, 16):
            key = f"{n}/bell{B}"
            ell_cols, nnz = (int(x) for x in conv[f"{key}/meta"])
            bell = _dev_bell(rows, cols, nnz, B, ell_cols, conv[f"{key}/bci"], conv[f"{key}/val"])
            for req in (1, 2, 3, 8):
                g = f"{key}/bucket{req}"
                bp = bucketed_blocked_ell(bell, req)
                S, nbytes = (int(x) for x in gold[f"{g}/meta"])
                assert bp.plan["segment_count"] == S and bp.plan["bytes"] == nbytes, g
                seg = gold[f"{g}/seg"].reshape(-1, 3)
                assert [s.rows for s in bp.segments] == list(seg[:, 0]), g
                assert [s.ell_cols for s in bp.segments] == list(seg[:, 1]), g
                bci, val = _flat(bp)
                assert np.array_equal(bci, gold[f"{g}/bci"]) and np.array_equal(val, gold[f"{g}/val"]), g
                assert np.array_equal(np_u32(bp.exec_to_canonical_rows), gold[f"{g}/e2c"]), g
                checked += 1
            chosen = bucketed_blocked_ell(bell, 0)
            assert (chosen.plan["bucket_count"], chosen.plan["bytes"]) == tuple(int(x) for x in gold[f"{key}/choose"])
    assert checked >= 40


def test_sliced_matches_reference_vectors(cuda):
    from cellshard_b200.device import bucketed_sliced_ell

    conv, gold = np.load(GOLD / "ref_conversions.npz"), np.load(GOLD / "ref_bucketing.npz")
    checked = 0
    for n in sorted({k.split("/")[0] for k in gold.files}):
        rows, cols = (int(x) for x in conv[f"{n}/shape"])
        for h in (3, 32):
            key = f"{n}/sell{h}"
            if f"{key}/choose" not in gold.files:
                continue
            nnz = int(conv[f"{key}/meta"][1])
            sell = _dev_sell(rows, cols, nnz, *(conv[f"{key}/{f}"] for f in ("offsets", "widths", "col_idx", "val")))
            for req in (1, 2, 3, 8):
                g = f"{key}/bucket{req}"
                bp = bucketed_sliced_ell(sell, req)
                S, nbytes = (int(x) for x in gold[f"{g}/meta"])
                assert bp.plan["segment_count"] == S and bp.plan["bytes"] == nbytes, g
                seg = gold[f"{g}/seg"].reshape(-1, 3)
                assert [s.rows for s in bp.segments] == list(seg[:, 0]), g
                col, val = _flat(bp)
                assert np.array_equal(col, gold[f"{g}/col_idx"]) and np.array_equal(val, gold[f"{g}/val"]), g
                assert np.array_equal(np_u32(bp.exec_to_canonical_rows), gold[f"{g}/e2c"]), g
                checked += 1
            chosen = bucketed_sliced_ell(sell, 0)
            assert (chosen.plan["bucket_count"], chosen.plan["bytes"]) == tuple(int(x) for x in gold[f"{key}/choose"])
    assert checked >= 20


@pytest.mark.parametrize("rows,cols,B,density,empty", [
    (1000, 2000, 16, 0.01, 0.3),   # heavy tail: several segments kept
    (333, 500, 8, 0.05, 0.2),      # partial last row block, 16-byte copy
    (200, 300, 5, 0.1, 0.1),       # per-half copy (B not a multiple of 8)
    (64, 4096, 16, 0.3, 0.0),      # long rows: several 2048-slot chunks per row block
    (96, 96, 8, 1.0, 0.0),         # dense: every row block the same width, buckets merge
    (40, 50, 16, 0.0, 1.0),        # no entries: zero-width segments
    (300, 900, 32, 0.02, 0.5),     # B = 32, more than one row block per chunk of slots
])
def test_blocked_vs_restatement(cuda, orc, rows, cols, B, density, empty):
    from cellshard_b200.device import blocked_ell_from_csr, bucketed_blocked_ell

    ptr, idx, val = random_csr(rows, cols, density, rows + B, empty)
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), B)
    bci, bval = np_u32(bell.bci), np_u16(bell.val)
    for req in (1, 2, 3, 8, 0):
        bp = bucketed_blocked_ell(bell, req)
        want = req if req else orc.bell_choose_bucket_count(rows, B, bell.ell_cols, bci)[0]
        ref = orc.bell_bucketed(rows, B, bell.ell_cols, bci, bval, want)
        assert bp.plan["segment_count"] == ref["segment_count"] and bp.plan["bytes"] == ref["bytes"], req
        assert bp.plan["bucket_count"] == want
        assert bp.segment_row_offsets == [0] + list(np.cumsum(ref["seg_rows"]).astype(int))
        got_bci, got_val = _flat(bp)
        assert np.array_equal(got_bci, ref["seg_bci"]) and np.array_equal(got_val, ref["seg_val"]), req
        assert np.array_equal(np_u32(bp.exec_to_canonical_rows), ref["e2c"])
        assert np.array_equal(np_u32(bp.canonical_to_exec_rows), ref["c2e"])
        ident = np.arange(cols, dtype=np.uint32)
        assert np.array_equal(np_u32(bp.exec_to_canonical_cols), ident)
        assert np.array_equal(np_u32(bp.canonical_to_exec_cols), ident)


def test_blocked_unaligned_values_take_the_per_half_copy(cuda, orc):
    import torch

    from cellshard_b200.device import BlockedELL, blocked_ell_from_csr, bucketed_blocked_ell

    rows, cols = 500, 800
    ptr, idx, val = random_csr(rows, cols, 0.03, 31, 0.3)
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), 16)
    buf = torch.empty(bell.val.numel() + 1, dtype=torch.float16, device="cuda")
    buf[1:] = bell.val
    shifted = BlockedELL(rows, cols, 16, bell.ell_cols, bell.bci, buf[1:], bell.nnz)
    assert shifted.val.data_ptr() % 16 != 0
    a, b = bucketed_blocked_ell(bell, 4), bucketed_blocked_ell(shifted, 4)
    assert a.plan == b.plan
    for x, y in zip(_flat(a), _flat(b)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("rows,cols,density,empty,h", [
    (1000, 2000, 0.01, 0.3, 32),   # several segments kept
    (333, 500, 0.05, 0.2, 7),      # ragged last slice
    (64, 4096, 0.3, 0.0, 16),      # long rows
    (40, 50, 0.0, 1.0, 8),         # no entries
])
def test_sliced_vs_restatement(cuda, orc, rows, cols, density, empty, h):
    from cellshard_b200.device import bucketed_sliced_ell

    ptr, idx, val = random_csr(rows, cols, density, rows + h, empty)
    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, h)
    col = s["col_idx"].copy()
    sv = s["val"].copy()
    sell = _dev_sell(rows, cols, len(idx), s["offsets"], s["widths"], col, sv)
    for req in (1, 2, 3, 8, 0):
        bp = bucketed_sliced_ell(sell, req)
        want = req if req else orc.sell_choose_bucket_count(rows, s["offsets"], s["widths"], col)[0]
        ref = orc.sell_bucketed(rows, s["offsets"], s["widths"], col, sv, want)
        assert bp.plan["segment_count"] == ref["segment_count"] and bp.plan["bytes"] == ref["bytes"], req
        assert bp.segment_row_offsets == list(ref["seg_row"].astype(int))
        got_col, got_val = _flat(bp)
        assert np.array_equal(got_col, ref["seg_col"]) and np.array_equal(got_val, ref["seg_val"]), req
        assert np.array_equal(np_u32(bp.exec_to_canonical_rows), ref["e2c"])
        assert np.array_equal(np_u32(bp.canonical_to_exec_rows), ref["c2e"])


def _host_bell(lib_abi, rows, cols, nnz, B, ell_cols, bci, val):
    src = lib_abi.HostBlockedEll()
    src.rows, src.cols, src.nnz, src.block_size, src.ell_cols = rows, cols, nnz, B, ell_cols
    src.blockColIdx, src.val = bci.ctypes.data, val.ctypes.data
    return src


def test_host_api_vs_live_reference(cuda, orc):
    """cs_b200_build_bucketed_blocked_ell_partition / _sliced_ and the choosers with
    the reference's host signatures, field by field against the reference's own
    builders (segment nnz fields, row offsets, maps, canonical slices)."""
    from cellshard_b200 import _abi

    if not orc.ref_bucket_available():
        pytest.skip("reference bucketing bridge not built")
    lib = _abi.load()
    rows, cols, B = 700, 1500, 16
    ptr, idx, val = random_csr(rows, cols, 0.02, 41, 0.3)
    b = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
    bci, bval = np.ascontiguousarray(b["bci"]), np.ascontiguousarray(b["val"])
    src = _host_bell(_abi, rows, cols, b["nnz"], B, b["ell_cols"], bci, bval)
    for req in (1, 3, 8):
        out, nbytes = _abi.HostBucketedBlockedEll(), C.c_uint64()
        assert lib.cs_b200_build_bucketed_blocked_ell_partition(C.byref(out), C.byref(src), req, C.byref(nbytes)) == 1
        mine = orc.read_bucketed_bell(out)
        lib.cs_b200_host_bucketed_blocked_ell_clear(C.byref(out))
        ref = orc.ref_build_bucketed_bell(rows, cols, b["nnz"], B, b["ell_cols"], bci, bval, req)
        assert nbytes.value == ref["bytes"]
        for k in ("rows", "cols", "nnz", "segment_count"):
            assert mine[k] == ref[k], k
        for k in ("segment_row_offsets", "e2c", "c2e", "e2c_cols", "c2e_cols"):
            assert np.array_equal(mine[k], ref[k]), k
        for x, y in zip(mine["segments"], ref["segments"]):
            for k in ("rows", "cols", "nnz", "block_size", "ell_cols"):
                assert x[k] == y[k], k
            assert np.array_equal(x["bci"], y["bci"]) and np.array_equal(x["val"], y["val"])
    count, nbytes = C.c_uint32(), C.c_uint64()
    assert lib.cs_b200_choose_bucket_count_for_part(C.byref(src), C.byref(count), C.byref(nbytes)) == 1
    assert (count.value, nbytes.value) == orc.ref_choose_bucket_count_for_part(rows, cols, b["nnz"], B, b["ell_cols"],
                                                                               bci, bval)

    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, 32)
    arrs = [np.ascontiguousarray(s[k], np.uint32) for k in ("offsets", "widths", "col_idx")]
    sv = np.ascontiguousarray(s["val"], np.uint16)
    ssrc = orc.host_sell(rows, cols, len(idx), *arrs, sv)
    ssrc_mine = _abi.HostSlicedEll.from_buffer_copy(ssrc)
    for req in (1, 2, 8):
        out, nbytes = _abi.HostBucketedSlicedEll(), C.c_uint64()
        assert lib.cs_b200_build_bucketed_sliced_ell_partition(C.byref(out), C.byref(ssrc_mine), req,
                                                               C.byref(nbytes)) == 1
        mine = orc.read_bucketed_sell(orc.HostBucketedSell.from_buffer_copy(out))
        lib.cs_b200_host_bucketed_sliced_ell_clear(C.byref(out))
        ref = orc.ref_build_bucketed_sell(rows, cols, len(idx), *arrs, sv, req)
        assert nbytes.value == ref["bytes"]
        for k in ("rows", "cols", "nnz", "segment_count", "canonical_slice_count"):
            assert mine[k] == ref[k], k
        for k in ("segment_row_offsets", "e2c", "c2e", "canonical_slice_row_offsets", "canonical_slice_widths"):
            assert np.array_equal(mine[k], ref[k]), k
        for x, y in zip(mine["segments"], ref["segments"]):
            for k in ("rows", "cols", "nnz", "slice_count"):
                assert x[k] == y[k], k
            for k in ("offsets", "widths", "col_idx", "val"):
                assert np.array_equal(x[k], y[k]), k
    assert lib.cs_b200_choose_bucket_count_for_sliced_part(C.byref(ssrc_mine), C.byref(count), C.byref(nbytes)) == 1
    assert (count.value, nbytes.value) == orc.ref_choose_bucket_count_for_sliced_part(rows, cols, len(idx), *arrs, sv)


def test_synthetic_round_trip(cuda):
    """50,000 x 32,768 Blocked-ELL-16 of the grouped-reduction generator (the
    heavy-tailed rows bucketing is for): every execution row block holds its
    source row block's valid block columns compacted in slot order, with their
    values, padding after them, and the row maps invert each other."""
    import torch

    from cellshard_b200 import synth
    from cellshard_b200.device import blocked_ell_from_csr, bucketed_blocked_ell

    bell = blocked_ell_from_csr(synth.make_csr(synth.grouped_reduction_spec(50_000)), 16)
    bp = bucketed_blocked_ell(bell, 0)
    B, W, RB = bell.block_size, bell.ell_width, bell.row_blocks
    assert 1 <= bp.plan["segment_count"] <= 8 and bp.plan["bytes"] <= bp.plan["original_bytes"]
    e2c, c2e = bp.exec_to_canonical_rows.long(), bp.canonical_to_exec_rows.long()
    assert torch.equal(e2c[c2e], torch.arange(bell.rows, device="cuda"))
    for k, seg in enumerate(bp.segments):
        r0, w = bp.segment_row_offsets[k], seg.ell_width
        nrb = (seg.rows + B - 1) // B
        src_rb = e2c[r0:r0 + seg.rows:B] // B
        sbci = bell.bci.view(RB, W)[src_rb]
        valid = sbci != -1
        cnt = valid.sum(1)
        order = torch.argsort((~valid).to(torch.int8), dim=1, stable=True)[:, :w]
        slot = torch.arange(w, device="cuda")[None, :]
        want_bci = torch.where(slot < cnt[:, None], torch.gather(sbci, 1, order), torch.full_like(order, -1).int())
        assert torch.equal(seg.bci.view(nrb, w), want_bci.int())
        for a in range(0, seg.rows, 8192):  # values, a slab of rows at a time
            b = min(seg.rows, a + 8192)
            sval = bell.val.view(bell.rows, W, B)[e2c[r0 + a:r0 + b]]
            o = order.repeat_interleave(B, 0)[a:b]
            g = torch.gather(sval, 1, o[:, :, None].expand(-1, -1, B))
            keep = slot < cnt.repeat_interleave(B)[a:b, None]
            want = torch.where(keep[:, :, None], g, torch.zeros_like(g))
            assert torch.equal(seg.val.view(seg.rows, w, B)[a:b].view(torch.int16), want.view(torch.int16))


@pytest.mark.parametrize("rows,cols,B,density,empty", [
    (1000, 2000, 16, 0.01, 0.3),
    (333, 500, 8, 0.05, 0.2),     # partial last row block, sorted with the others here
    (200, 300, 5, 0.1, 0.1),
    (96, 96, 8, 1.0, 0.0),        # equal widths: the hash orders the row blocks
    (17, 40, 16, 0.2, 0.0),       # two row blocks
])
def test_ingest_plan_and_choice(cuda, orc, rows, cols, B, density, empty):
    """bucket::build_plan and the ingest chooser: the device plan against the
    restatement and the reference's own GPU plan, the device choice against
    the restatement, the reference's chooser and its estimate."""
    import torch

    from cellshard_b200 import _abi
    from cellshard_b200.device import blocked_ell_from_csr, ptr, stream_handle

    ptr_, idx, val = random_csr(rows, cols, density, rows + 3 * B, empty)
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr_, idx, val), B)
    bci, bval = np_u32(bell.bci), np_u16(bell.val)
    lib = _abi.load()
    RB = bell.row_blocks
    nb = C.c_size_t()
    assert lib.cs_b200_blocked_ell_bucket_plan_scratch_bytes(rows, B, C.byref(nb)) == 1
    scr = torch.empty(max(nb.value, 16), dtype=torch.uint8, device="cuda")
    order = torch.empty(RB, dtype=torch.int32, device="cuda")
    ws = torch.empty(RB, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.int64, device="cuda")
    v = bell.view()
    assert lib.cs_b200_blocked_ell_bucket_plan(C.byref(v), ptr(order), ptr(ws), ptr(scr), nb.value,
                                               stream_handle()) == 1
    assert lib.cs_b200_choose_bucket_count_from_plan(C.byref(v), ptr(order), ptr(ws), out.data_ptr(),
                                                     out.data_ptr() + 8, stream_handle()) == 1
    o, w = np_u32(order), np_u32(ws)
    ro, rw = orc.bell_bucket_plan(rows, B, bell.ell_cols, bci)
    assert np.array_equal(o, ro) and np.array_equal(w, rw)
    count = int(out[0].item()) & 0xFFFFFFFF
    assert count == orc.bell_choose_ingest_bucket_count(rows, B, bell.ell_cols, bci)
    est = [orc.bell_estimate_bucketed_bytes(rows, B, o, w, b) for b in range(1, min(8, RB) + 1)]
    f = orc.lib().cso_packed_blocked_ell_bytes
    f.restype = C.c_uint64
    orig = f(C.c_uint32(rows), C.c_uint32(bell.ell_cols), C.c_uint32(B))
    assert int(out[1].item()) == (min(orig, est[count - 1]) if est else orig)
    h = _abi.HostBlockedEll()
    h.rows, h.cols, h.nnz, h.block_size, h.ell_cols = rows, cols, bell.nnz, B, bell.ell_cols
    hb = np.ascontiguousarray(bci)
    h.blockColIdx = hb.ctypes.data
    c = C.c_uint32()
    assert lib.cs_b200_choose_ingest_bucket_count_for_part(C.byref(h), 0, C.byref(c)) == 1 and c.value == count
    if orc.ref_ingest_available():
        po, pw = orc.ref_bucket_plan(rows, cols, bell.nnz, B, bell.ell_cols, bci, bval)
        assert np.array_equal(o, po) and np.array_equal(w, pw)
        assert count == orc.ref_choose_ingest_bucket_count(rows, cols, bell.nnz, B, bell.ell_cols, bci, bval)
        for b in range(1, min(8, RB) + 1):
            assert est[b - 1] == orc.ref_estimate_bucketed_bytes(rows, cols, bell.nnz, B, bell.ell_cols, bci, bval,
                                                                 po, pw, b)
