"""COO -> Blocked-ELL on the GPU against the restatement, the reference's host
routines (golden vectors and live) and the reference's own GPU routine run on
the B200: block columns, values, both nnz counts, the block-size chooser, the
two key layouts, repeated entries and dropped rows."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _t(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(dtype).copy()).cuda()


def _run(rows, cols, row, col, val, B, fmap=None, cols_src=None):
    import numpy as _np
    import torch

    from cellshard_b200.device import blocked_ell_from_coo

    fm = _t(fmap.astype(_np.uint32), _np.int32) if fmap is not None else None
    return blocked_ell_from_coo(rows, cols if cols_src is None else cols_src, _t(row.astype(_np.uint32), _np.int32),
                                _t(col.astype(_np.uint32), _np.int32), _t(val.astype(_np.uint16), _np.float16), B,
                                cols, fm)


def _coo(rows, cols, density, seed, dups=0, shuffle=True):
    ptr, idx, val = random_csr(rows, cols, density, seed, 0.2)
    rng = np.random.default_rng(seed)
    row = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))
    col, v = idx.copy(), val.copy()
    if dups and len(row) > 4:
        k = rng.integers(0, len(row), dups)
        row, col, v = np.concatenate([row, row[k]]), np.concatenate([col, col[k]]), np.concatenate([v, v[k] ^ 0x400])
    if shuffle:
        p = rng.permutation(len(row))
        row, col, v = row[p], col[p], v[p]
    return row.astype(np.uint32), col.astype(np.uint32), v.astype(np.uint16)


def test_matches_reference_vectors(cuda):
    conv, gold = np.load(GOLD / "ref_conversions.npz"), np.load(GOLD / "ref_coo.npz")
    checked = 0
    for n in sorted({k.split("/")[0] for k in gold.files}):
        rows, cols = (int(x) for x in conv[f"{n}/shape"])
        row, col, val = (gold[f"{n}/coo/{k}"] for k in ("row", "col", "val"))
        fmap = gold[f"{n}/coo/map"] if f"{n}/coo/map" in gold.files else None
        for B in (2, 3, 8, 16):
            out, counts, status, _tot = _run(rows, cols, row, col, val, B, fmap)
            ell_cols, nnz = (int(x) for x in gold[f"{n}/coo{B}/meta"])
            assert out.ell_cols == ell_cols and counts[0] == nnz and status == 0, (n, B)
            assert np.array_equal(np_u32(out.bci), gold[f"{n}/coo{B}/bci"]), (n, B)
            assert np.array_equal(np_u16(out.val), gold[f"{n}/coo{B}/val"]), (n, B)
            checked += 1
    assert checked >= 20


@pytest.mark.parametrize("rows,cols,density,B,dups,remap", [
    (1000, 2000, 0.01, 16, 0, False),     # 16-byte values, no repeats: also vs the reference GPU routine
    (333, 500, 0.05, 8, 7, False),        # repeated (row, column): the last value stays
    (200, 300, 0.1, 5, 0, True),          # block size 5, a column map
    (64, 4096, 0.3, 16, 3, True),         # long rows
    (40, 50, 0.0, 4, 0, False),           # no entries
])
def test_vs_restatement_and_references(cuda, orc, rows, cols, density, B, dups, remap):
    row, col, val = _coo(rows, cols, density, rows + B, dups)
    fmap = np.random.default_rng(3).permutation(cols).astype(np.uint32) if remap else None
    out, counts, status, total = _run(rows, cols, row, col, val, B, fmap)
    ref = orc.blocked_ell_from_coo(rows, cols, row, col, val, B, fmap)
    assert status == 0 and out.ell_cols == ref["ell_cols"] and total == ref["total_blocks"]
    assert np.array_equal(np_u32(out.bci), ref["bci"]) and np.array_equal(np_u16(out.val), ref["val"])
    assert counts == [ref["nnz_host"], ref["nnz_gpu"]]
    if orc.ref_available():
        h = orc.ref_blocked_ell_from_coo(rows, cols, cols, row, col, val, B, fmap)
        assert h["ell_cols"] == out.ell_cols and h["nnz"] == counts[0]
        assert np.array_equal(h["bci"], np_u32(out.bci)) and np.array_equal(h["val"], np_u16(out.val))
    if orc.ref_gpu_available() and dups == 0 and len(row):
        # The reference's GPU routine places the same block columns, but its value
        # scatter takes each entry's group from an exclusive scan of the head flags,
        # which counts the entry's own group head for every entry after the first:
        # those entries land one slot to the right.  Every cell where its values
        # differ from this build's is a cell such an entry left or reached.
        g = orc.ref_gpu_blocked_ell_from_coo_cuda(rows, cols, cols, row, col, val, B, fmap)
        assert g["ell_cols"] == out.ell_cols and np.array_equal(g["bci"], np_u32(out.bci))
        diff = set(np.flatnonzero(g["val"] != np_u16(out.val)).tolist())
        assert diff <= _shifted_cells(rows, B, out.ell_cols, row, col, fmap, ref["bci"])


def _shifted_cells(rows, B, ell_cols, row, col, fmap, bci):
    """Cells left and reached by the entries after the first of each (row block,
    block column) group when they are written one slot to the right."""
    W = ell_cols // B
    c = fmap[col] if fmap is not None else col
    key = (row.astype(np.int64) // B) * (1 << 32) + c.astype(np.int64) // B
    order = np.argsort(key, kind="stable")
    cells, prev = set(), None
    for i in order:
        rb, bc = int(row[i]) // B, int(c[i]) // B
        slots = bci[rb * W:(rb + 1) * W]
        slot = int(np.searchsorted(slots[slots != 0xFFFFFFFF], bc))
        if prev == (rb, bc):
            base = int(row[i]) * ell_cols + int(c[i]) % B
            cells.add(base + slot * B)
            cells.add(base + (slot + 1) * B)
        prev = (rb, bc)
    return cells


def test_wide_keys_take_two_sorts(cuda, orc):
    """A column map into 2^31 columns: row block and block column no longer fit
    one 32-bit key, so the entries are sorted by block column, then row block."""
    rows, cols = 300, 400
    row, col, val = _coo(rows, cols, 0.05, 11)
    fmap = (np.random.default_rng(2).permutation(cols).astype(np.uint64) * 5_000_000 + 7).astype(np.uint32)
    big = int(fmap.max()) + 1
    out, counts, status, _ = _run(rows, big, row, col, val, 4, fmap, cols_src=cols)
    ref = orc.blocked_ell_from_coo(rows, big, row, col, val, 4, fmap)
    assert status == 0 and out.ell_cols == ref["ell_cols"]
    assert np.array_equal(np_u32(out.bci), ref["bci"]) and np.array_equal(np_u16(out.val), ref["val"])
    assert counts == [ref["nnz_host"], ref["nnz_gpu"]]


def test_rows_out_of_range_are_dropped_and_flagged(cuda, orc):
    """Dropped rows send the entries through the (row block, block column) sort
    route, here with repeated entries too."""
    rows, cols = 100, 120
    row, col, val = _coo(rows, cols, 0.1, 5, dups=6)
    bad = row.copy()
    bad[::17] = rows + 3
    out, counts, status, _ = _run(rows, cols, bad, col, val, 8)
    keep = bad < rows
    ref = orc.blocked_ell_from_coo(rows, cols, bad[keep], col[keep], val[keep], 8)
    assert status & 4  # CS_STATUS_INDEX_RANGE
    assert np.array_equal(np_u32(out.bci), ref["bci"]) and np.array_equal(np_u16(out.val), ref["val"])
    from cellshard_b200 import _abi

    lib = _abi.load()
    h = _abi.HostCoo()
    h.rows, h.cols, h.nnz = rows, cols, len(bad)
    b, c, v = np.ascontiguousarray(bad), np.ascontiguousarray(col), np.ascontiguousarray(val)
    h.rowIdx, h.colIdx, h.val = b.ctypes.data, c.ctypes.data, v.ctypes.data
    dst = _abi.HostBlockedEll()
    assert lib.cs_b200_blocked_ell_from_coo(C.byref(h), cols, None, 8, C.byref(dst)) == 0
    assert b"row index" in lib.cs_b200_last_error()


def test_host_signatures_and_chooser(cuda, orc):
    from cellshard_b200 import _abi

    lib = _abi.load()
    rows, cols = 700, 900
    row, col, val = _coo(rows, cols, 0.02, 21, dups=4)
    fmap = np.random.default_rng(9).permutation(cols).astype(np.uint32)
    h = _abi.HostCoo()
    h.rows, h.cols, h.nnz = rows, cols, len(row)
    h.rowIdx, h.colIdx, h.val = row.ctypes.data, col.ctypes.data, val.ctypes.data
    cands = [2, 4, 8, 16, 32]
    ca = (C.c_uint * len(cands))(*cands)
    t = _abi.BlockedEllTuneResult()
    assert lib.cs_b200_choose_blocked_ell_block_size_from_coo(C.byref(h), cols, fmap.ctypes.data, ca, len(cands),
                                                              C.byref(t)) == 1
    want = orc.choose_block_size_from_coo(rows, cols, row, col, cands, fmap)
    assert (t.block_size, t.fill_ratio, t.padded_bytes) == want
    if orc.ref_available():
        assert want == orc.ref_choose_block_size_from_coo(rows, cols, cols, row, col, val, cands, fmap)
    if orc.ref_gpu_available():
        assert want == orc.ref_gpu_choose_block_size_from_coo_cuda(rows, cols, cols, row, col, val, cands, fmap)
    for fn, idx in (("cs_b200_blocked_ell_from_coo", "nnz_host"), ("cs_b200_blocked_ell_from_coo_cuda", "nnz_gpu")):
        dst = _abi.HostBlockedEll()
        args = (C.byref(h), cols, fmap.ctypes.data, t.block_size, C.byref(dst)) + ((0,) if fn.endswith("cuda") else ())
        assert getattr(lib, fn)(*args) == 1
        ref = orc.blocked_ell_from_coo(rows, cols, row, col, val, t.block_size, fmap)
        RB = (rows + t.block_size - 1) // t.block_size
        W = dst.ell_cols // t.block_size
        bci = np.ctypeslib.as_array(C.cast(dst.blockColIdx, C.POINTER(C.c_uint32)), (RB * W,)).copy()
        v = np.ctypeslib.as_array(C.cast(dst.val, C.POINTER(C.c_uint16)), (rows * dst.ell_cols,)).copy()
        assert dst.ell_cols == ref["ell_cols"] and dst.nnz == ref[idx] and dst.cols == cols
        assert np.array_equal(bci, ref["bci"]) and np.array_equal(v, ref["val"])
        lib.cs_b200_host_blocked_ell_clear(C.byref(dst))


@pytest.mark.parametrize("remap,B", [(False, 16), (True, 8), (False, 3)])
def test_row_ordered_input_takes_the_csr_route(cuda, orc, remap, B):
    """COO written row by row (columns in any order inside a row, some repeated
    next to each other) goes through row pointers and the CSR -> Blocked-ELL
    kernels; the result is the host routine's, repeats keeping the last value."""
    rows, cols = 500, 700
    ptr, idx, val = random_csr(rows, cols, 0.04, 77 + B, 0.2)
    rng = np.random.default_rng(B)
    rr, cc, vv = [], [], []
    for r in range(rows):
        a, b = int(ptr[r]), int(ptr[r + 1])
        c, v = idx[a:b].copy(), val[a:b].copy()
        if len(c) > 2:
            p = rng.permutation(len(c))
            c, v = c[p], v[p]
            if r % 5 == 0:  # repeat one column with another value
                c, v = np.append(c, c[0]), np.append(v, v[0] ^ 0x400)
        rr.append(np.full(len(c), r, np.uint32))
        cc.append(c)
        vv.append(v)
    row, col, v = np.concatenate(rr), np.concatenate(cc).astype(np.uint32), np.concatenate(vv).astype(np.uint16)
    fmap = rng.permutation(cols).astype(np.uint32) if remap else None
    out, counts, status, total = _run(rows, cols, row, col, v, B, fmap)
    ref = orc.blocked_ell_from_coo(rows, cols, row, col, v, B, fmap)
    assert status == 0 and out.ell_cols == ref["ell_cols"] and total == ref["total_blocks"]
    assert np.array_equal(np_u32(out.bci), ref["bci"]) and np.array_equal(np_u16(out.val), ref["val"])
    assert counts == [ref["nnz_host"], ref["nnz_gpu"]]
    if orc.ref_available():
        h = orc.ref_blocked_ell_from_coo(rows, cols, cols, row, col, v, B, fmap)
        assert h["nnz"] == counts[0] and np.array_equal(h["val"], np_u16(out.val))
