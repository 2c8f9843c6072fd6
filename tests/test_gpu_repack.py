"""Filtered Blocked-ELL -> CSR over a shard's partitions and the repack
(filter -> nnz bucket plan -> row rebuild -> Blocked-ELL), against the
restatement composed from the pinned pieces (masked reoptimize per partition,
nnz plan, rebuild, CSR -> Blocked-ELL), plus the reference's own filter run on
the B200 to record its row pointers."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
INVALID = 0xFFFFFFFF


def _shard(seed, part_specs, cols):
    """Partitions (rows, block_size) of one shard, each a Blocked-ELL from a random CSR."""
    from cellshard_b200.device import blocked_ell_from_csr

    parts, host = [], []
    for k, (rows, B) in enumerate(part_specs):
        ptr, idx, val = random_csr(rows, cols, 0.08, seed + k, 0.15)
        bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), B)
        parts.append(bell)
        host.append((rows, B, bell.ell_cols, np_u32(bell.bci), np_u16(bell.val)))
    return parts, host


def _masks(rng, shard_rows, cols, out_rows, out_cols):
    keep_rows = (rng.random(shard_rows) < 0.8).astype(np.uint8)
    keep_cols = (rng.random(cols) < 0.85).astype(np.uint8)
    row_remap = np.full(shard_rows, INVALID, np.uint32)
    kept = np.flatnonzero(keep_rows)
    targets = rng.permutation(out_rows)[: min(len(kept), out_rows)]
    row_remap[kept[: len(targets)]] = targets  # kept rows past out_rows map nowhere
    col_remap = rng.permutation(cols).astype(np.uint32)  # some land >= out_cols and drop
    return keep_rows, keep_cols, row_remap, col_remap


def _oracle_filter(orc, host, cols, keep_rows, keep_cols, row_remap, col_remap, out_rows, out_cols):
    """Per partition the restated masked reoptimize; output rows are filled by
    exactly one source row, so the partition results merge row by row."""
    per_row = [[] for _ in range(out_rows)]
    off = 0
    for rows, B, ell_cols, bci, val in host:
        major, idx, v = orc.reoptimize_bell(rows, cols, B, ell_cols, bci, val, keep_rows[off:off + rows], keep_cols,
                                            row_remap[off:off + rows], col_remap, out_rows, out_cols)
        for r in range(out_rows):
            a, b = int(major[r]), int(major[r + 1])
            if b > a:
                per_row[r].append((idx[a:b], v[a:b]))
        off += rows
    ptr = np.zeros(out_rows + 1, np.uint32)
    idxs, vals = [], []
    for r in range(out_rows):
        assert len(per_row[r]) <= 1
        n = 0
        for i, v in per_row[r]:
            idxs.append(i)
            vals.append(v)
            n += len(i)
        ptr[r + 1] = ptr[r] + n
    cat = lambda xs, t: np.concatenate(xs).astype(t) if xs else np.zeros(0, t)
    return ptr, cat(idxs, np.uint32), cat(vals, np.uint16)


@pytest.mark.parametrize("part_specs,cols,out_rows,out_cols", [
    ([(300, 16)], 257, 280, 200),                        # one partition, output narrower
    ([(130, 16), (77, 8), (200, 4)], 300, 320, 300),     # three partitions, mixed block sizes
    ([(64, 16), (1, 16), (90, 2)], 50, 100, 60),         # a one-row partition
])
def test_filter_parts_vs_restatement(cuda, orc, part_specs, cols, out_rows, out_cols):
    import torch

    from cellshard_b200 import runtime

    parts, host = _shard(7, part_specs, cols)
    shard_rows = sum(r for r, _ in part_specs)
    rng = np.random.default_rng(3)
    kr, kc, rr, cr = _masks(rng, shard_rows, cols, out_rows, out_cols)
    dev = lambda a, t: torch.from_numpy(a.view(t).copy()).cuda()
    csr, stats = runtime.filter_blocked_ell_to_compressed(parts, out_rows, out_cols, dev(kr, np.uint8),
                                                          dev(kc, np.uint8), dev(rr, np.int32), dev(cr, np.int32))
    ptr, idx, val = _oracle_filter(orc, host, cols, kr, kc, rr, cr, out_rows, out_cols)
    assert np.array_equal(np_u32(csr.ptr), ptr)
    assert np.array_equal(np_u32(csr.idx), idx) and np.array_equal(np_u16(csr.val), val)
    kept = np.flatnonzero(kr)
    ell = np.concatenate([np.full(r, h[2], np.int64) for r, h in zip((r for r, _ in part_specs), host)])
    assert stats["kept_rows"] == len(kept) and stats["kept_row_slots"] == int(ell[kept].sum())
    assert stats["live_nnz"] == len(idx)


def test_repack_vs_restatement(cuda, orc):
    import torch

    from cellshard_b200 import runtime

    part_specs, cols, out_rows, out_cols = [(200, 16), (150, 8)], 400, 330, 380
    parts, host = _shard(11, part_specs, cols)
    rng = np.random.default_rng(5)
    kr, kc, rr, cr = _masks(rng, 350, cols, out_rows, out_cols)
    dev = lambda a, t: torch.from_numpy(a.view(t).copy()).cuda()
    filtered, plan, rebuilt, bell, stats = runtime.build_repacked_blocked_ell(
        parts, out_rows, out_cols, 8, 6, dev(kr, np.uint8), dev(kc, np.uint8), dev(rr, np.int32), dev(cr, np.int32))
    ptr, idx, val = _oracle_filter(orc, host, cols, kr, kc, rr, cr, out_rows, out_cols)
    _nnz, _sorted, order, offs = orc.major_nnz_plan(ptr, out_rows, 6)
    assert np.array_equal(np_u32(plan["order"])[:out_rows], order)
    assert np.array_equal(np_u32(plan["bucket_offsets"]), offs)
    rptr, ridx, rval, _inv = orc.rebuild(ptr, idx, val, out_rows, order)
    assert np.array_equal(np_u32(rebuilt.ptr), rptr) and np.array_equal(np_u32(rebuilt.idx), ridx)
    ref = orc.blocked_ell_from_csr(out_rows, out_cols, rptr, ridx, rval, 8)
    assert bell.ell_cols == ref["ell_cols"] and stats["ell_width"] == ref["ell_width"]
    assert np.array_equal(np_u32(bell.bci), ref["bci"]) and np.array_equal(np_u16(bell.val), ref["val"])


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libcs_ref_gpu.so").exists(), reason="reference GPU bridge")
def test_reference_filter_row_pointers_are_shifted(cuda, orc):
    """The reference's filter exclusive-scans counts it stored one slot up: its row
    pointers read [0, 0, c0, c0 + c1, ...] and its nnz misses the last row.  This
    library returns the CSR row pointers [0, c0, c0 + c1, ...]."""
    import torch

    from cellshard_b200 import _abi, runtime

    parts, host = _shard(21, [(257, 16)], 120)
    rng = np.random.default_rng(8)
    kr, kc, rr, cr = _masks(rng, 257, 120, 240, 110)
    dev = lambda a, t: torch.from_numpy(a.view(t).copy()).cuda()
    m_t = [dev(kr, np.uint8), dev(kc, np.uint8), dev(rr, np.int32), dev(cr, np.int32)]
    csr, _ = runtime.filter_blocked_ell_to_compressed(parts, 240, 110, *m_t)
    counts = np.diff(np_u32(csr.ptr).astype(np.int64))
    m = _abi.RowFeatureMaskView(*(t.data_ptr() for t in m_t))
    rptr = torch.empty(241, dtype=torch.int32, device="cuda")
    live = C.c_uint32()
    v = parts[0].view()
    assert orc.ref_gpu().csrefgpu_filter_blocked_ell(C.byref(v), 240, 110, C.byref(m), rptr.data_ptr(),
                                                     C.byref(live)) == 1
    shifted = np.concatenate([[0, 0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    assert np.array_equal(np_u32(rptr), shifted)
    assert live.value == int(shifted[-1])


@pytest.mark.parametrize("method", ["onepass", "marked"])
@pytest.mark.parametrize("part_specs,cols,out_rows", [
    ([(300, 16)], 257, 300),
    ([(130, 16), (77, 8), (2000, 16)], 3000, 2500),   # output rows past the shard's stay empty
    ([(64, 32), (1, 16), (9000, 8)], 500, 9065),
])
def test_filter_onepass_matches_count_emit(cuda, orc, part_specs, cols, out_rows, method):
    """The vector filters -- one pass (rows counted, placed by a look-back, emitted from
    L2) and marked (count + mark, scan, re-read of the marked groups) -- give the count +
    emit CSR bit for bit, with the same kept-row statistics, and both equal the
    restatement's masked reoptimize without remaps."""
    from cellshard_b200 import runtime

    parts, host = _shard(61, part_specs, cols)
    shard_rows = sum(r for r, _ in part_specs)
    rng = np.random.default_rng(5)
    keep_rows = (rng.random(shard_rows) < 0.7).astype(np.uint8)
    keep_cols = (rng.random(cols) < 0.6).astype(np.uint8)
    import torch

    rk, fk = torch.from_numpy(keep_rows).cuda(), torch.from_numpy(keep_cols).cuda()
    a, sa = runtime.filter_blocked_ell_to_compressed(parts, out_rows, cols, rk, fk, method=method)
    b, sb = runtime.filter_blocked_ell_to_compressed(parts, out_rows, cols, rk, fk, method="two_pass")
    assert sa == sb
    assert np.array_equal(np_u32(a.ptr), np_u32(b.ptr))
    assert np.array_equal(np_u32(a.idx), np_u32(b.idx))
    assert np.array_equal(np_u16(a.val), np_u16(b.val))
    ident = np.arange(shard_rows, dtype=np.uint32)
    ptr, idx, val = _oracle_filter(orc, host, cols, keep_rows, keep_cols, ident, np.arange(cols, dtype=np.uint32),
                                   out_rows, cols)
    assert np.array_equal(np_u32(a.ptr), ptr) and np.array_equal(np_u32(a.idx), idx)
    assert np.array_equal(np_u16(a.val), val)


@pytest.mark.parametrize("method", ["onepass", "marked"])
@pytest.mark.parametrize("cols", [9000, 40000, 70000])
@pytest.mark.parametrize("drop", ["last_row", "last_partition", "first_rows", "all"])
def test_filter_onepass_long_rows_and_dropped_tail(cuda, orc, drop, cols, method):
    """Rows of 9,000 columns (two 8,192-slot steps of the one-pass kernel, the
    last ragged: the per-step counts of the whole row go through one scan) and of
    40,000 columns (more steps than that: one scan per step), of 70,000 columns (the
    marked route's emit compacts its mark words in five chunks), and a dropped final
    row or partition, the first rows, or every row dropped (dropped rows carry no
    entries but must still get their row pointers and the total): bit-exact vs
    count + emit and the restatement, for both vector routes."""
    import torch

    from cellshard_b200 import runtime

    specs = [(40, 16), (33, 8)]
    parts, host = _shard(81, specs, cols)
    assert cols < 32768 or max(p.ell_cols for p in parts) > 32768
    shard_rows = sum(r for r, _ in specs)
    rng = np.random.default_rng(9)
    keep_rows = (rng.random(shard_rows) < 0.7).astype(np.uint8)
    if drop == "last_row":
        keep_rows[-1] = 0
    elif drop == "last_partition":
        keep_rows[specs[0][0]:] = 0
    elif drop == "first_rows":
        keep_rows[:7] = 0
    else:
        keep_rows[:] = 0
    keep_cols = (rng.random(cols) < 0.6).astype(np.uint8)
    out_rows = shard_rows + 5
    rk, fk = torch.from_numpy(keep_rows).cuda(), torch.from_numpy(keep_cols).cuda()
    a, sa = runtime.filter_blocked_ell_to_compressed(parts, out_rows, cols, rk, fk, method=method)
    b, sb = runtime.filter_blocked_ell_to_compressed(parts, out_rows, cols, rk, fk, method="two_pass")
    assert sa == sb
    assert np.array_equal(np_u32(a.ptr), np_u32(b.ptr))
    assert np.array_equal(np_u32(a.idx), np_u32(b.idx)) and np.array_equal(np_u16(a.val), np_u16(b.val))
    ident = np.arange(shard_rows, dtype=np.uint32)
    ptr, idx, val = _oracle_filter(orc, host, cols, keep_rows, keep_cols, ident, np.arange(cols, dtype=np.uint32),
                                   out_rows, cols)
    assert np.array_equal(np_u32(a.ptr), ptr) and np.array_equal(np_u32(a.idx), idx)
    assert np.array_equal(np_u16(a.val), val)


@pytest.mark.parametrize("method", ["onepass", "marked"])
def test_filter_onepass_capacity_falls_back(cuda, method):
    """A view whose stored nnz under-counts its nonzeros gives the vector filters too
    little room: they flag CS_STATUS_CAPACITY (a forced vector route raises) and the
    default route reruns count + emit with the same result as always."""
    import torch

    from cellshard_b200 import _abi, runtime
    from cellshard_b200.device import BlockedELL

    parts, _host = _shard(71, [(500, 16)], 400)
    p = parts[0]
    short = BlockedELL(p.rows, p.cols, p.block_size, p.ell_cols, p.bci, p.val, nnz=p.nnz // 3)
    rk = torch.ones(p.rows, dtype=torch.uint8, device="cuda")
    with pytest.raises(_abi.CellShardError):
        runtime.filter_blocked_ell_to_compressed([short], p.rows, p.cols, rk, None, method=method)
    a, _ = runtime.filter_blocked_ell_to_compressed([short], p.rows, p.cols, rk, None)
    b, _ = runtime.filter_blocked_ell_to_compressed([p], p.rows, p.cols, rk, None, method="two_pass")
    assert np.array_equal(np_u32(a.ptr), np_u32(b.ptr)) and np.array_equal(np_u32(a.idx), np_u32(b.idx))
    assert np.array_equal(np_u16(a.val), np_u16(b.val))
