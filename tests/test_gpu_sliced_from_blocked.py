"""Blocked-ELL -> Sliced-ELL on the GPU: bit-exact against the reference's own
convert::sliced_ell_from_blocked_ell (golden vectors and the live bridge), the
restatement, and the chooser choose_sliced_ell_slice_rows_from_blocked_ell."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"


def _dev_bell(rows, cols, nnz, B, ell_cols, bci, val):
    import torch

    from cellshard_b200.device import BlockedELL

    return BlockedELL(rows, cols, B, ell_cols,
                      torch.from_numpy(np.ascontiguousarray(bci, np.uint32).view(np.int32).copy()).cuda(),
                      torch.from_numpy(np.ascontiguousarray(val, np.uint16).view(np.float16).copy()).cuda(), nnz)


def _host(s):
    return np_u32(s.slice_widths), np_u32(s.col_idx), np_u16(s.val)


def test_matches_reference_vectors(cuda):
    """Golden outputs of the reference on its own Blocked-ELL conversions (B = 3,
    4, 16; -0.0 and NaN planted in the B = 4 matrices), two slice heights."""
    from cellshard_b200.device import sliced_ell_from_blocked_ell

    gold = np.load(GOLD / "ref_conversions.npz")
    checked = 0
    for n in sorted({k.split("/")[0] for k in gold.files}):
        rows, cols = (int(x) for x in gold[f"{n}/shape"])
        for B in (3, 4, 16):
            key = f"{n}/bell{B}"
            if f"{key}/sell3/meta" not in gold.files:
                continue
            ell_cols, nnz = (int(x) for x in gold[f"{key}/meta"])
            bval = gold[f"{key}/val_special"] if f"{key}/val_special" in gold.files else gold[f"{key}/val"]
            bell = _dev_bell(rows, cols, nnz, B, ell_cols, gold[f"{key}/bci"], bval)
            for h in (3, 32):
                out = sliced_ell_from_blocked_ell(bell, h)
                S, _nnz, total = (int(x) for x in gold[f"{key}/sell{h}/meta"])
                w, col, val = _host(out)
                assert out.slice_count == S and len(col) == total, (key, h)
                assert np.array_equal(w, gold[f"{key}/sell{h}/widths"]), (key, h)
                assert np.array_equal(col, gold[f"{key}/sell{h}/col_idx"]), (key, h)
                assert np.array_equal(val, gold[f"{key}/sell{h}/val"]), (key, h)
                checked += 1
    assert checked >= 30


@pytest.mark.parametrize("rows,cols,B,density,h", [
    (1000, 777, 16, 0.05, 32),   # vector path, last column block partial
    (333, 500, 8, 0.2, 7),       # vector path, rows not a multiple of B or h
    (200, 300, 5, 0.1, 16),      # per-value path (B not a multiple of 8)
    (64, 4096, 16, 0.3, 64),     # long rows: many 256-value steps
    (40, 50, 16, 0.0, 8),        # no live entries at all
])
def test_vs_restatement_and_live_reference(cuda, orc, rows, cols, B, density, h):
    import torch

    from cellshard_b200.device import blocked_ell_from_csr, blocked_ell_row_ptr, sliced_ell_from_blocked_ell

    ptr, idx, val = random_csr(rows, cols, density, rows + cols, 0.15, integer=(B % 2 == 0))
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), B)
    # plant zeros, -0.0 and NaN among the stored values
    v = bell.val.view(torch.int16)
    if v.numel() >= 4:
        g = torch.Generator().manual_seed(rows)
        pos = torch.randint(0, v.numel(), (max(4, v.numel() // 50),), generator=g).cuda()
        v[pos[0::3]] = 0
        v[pos[1::3]] = torch.tensor(0x8000 - 65536, dtype=torch.int16)
        v[pos[2::3]] = 0x7E00
    bci, bval = np_u32(bell.bci), np_u16(bell.val)
    out = sliced_ell_from_blocked_ell(bell, h)
    ref = orc.sliced_ell_from_bell(rows, cols, B, bell.ell_cols, bci, bval, h)
    assert np.array_equal(np_u32(blocked_ell_row_ptr(bell)), ref["row_ptr"])
    w, col, val_o = _host(out)
    assert np.array_equal(np_u32(out.slice_row_offsets), ref["offsets"])
    assert np.array_equal(w, ref["widths"]) and np.array_equal(np_u32(out.slice_slot_offsets), ref["slot_offsets"])
    assert np.array_equal(col, ref["col_idx"]) and np.array_equal(val_o, ref["val"])
    if orc.ref_available():
        live = orc.ref_sliced_ell_from_blocked_ell(rows, cols, bell.nnz, B, bell.ell_cols, bci, bval, h)
        assert np.array_equal(col, live["col_idx"]) and np.array_equal(val_o, live["val"])


def test_unaligned_values_take_the_per_value_path(cuda, orc):
    import torch

    from cellshard_b200.device import BlockedELL, blocked_ell_from_csr, sliced_ell_from_blocked_ell

    rows, cols = 300, 640
    ptr, idx, val = random_csr(rows, cols, 0.06, 17, 0.1)
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), 16)
    buf = torch.empty(bell.val.numel() + 1, dtype=torch.float16, device="cuda")
    buf[1:] = bell.val
    shifted = BlockedELL(rows, cols, 16, bell.ell_cols, bell.bci, buf[1:], bell.nnz)
    assert shifted.val.data_ptr() % 16 != 0
    a, b = sliced_ell_from_blocked_ell(bell, 32), sliced_ell_from_blocked_ell(shifted, 32)
    assert np.array_equal(np_u32(a.col_idx), np_u32(b.col_idx)) and np.array_equal(np_u16(a.val), np_u16(b.val))


def test_host_api_and_chooser_vs_reference(cuda, orc):
    """cs_b200_sliced_ell_from_blocked_ell / choose_..._from_blocked_ell with the
    reference's host signature, against the reference's own functions."""
    from cellshard_b200 import _abi

    if not orc.ref_available():
        pytest.skip("reference bridge not built")
    lib = _abi.load()
    rows, cols, B = 500, 900, 16
    ptr, idx, val = random_csr(rows, cols, 0.04, 5, 0.2)
    b = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
    src = _abi.HostBlockedEll()
    src.rows, src.cols, src.nnz, src.block_size, src.ell_cols = rows, cols, b["nnz"], B, b["ell_cols"]
    bci, bval = np.ascontiguousarray(b["bci"]), np.ascontiguousarray(b["val"])
    src.blockColIdx, src.val = bci.ctypes.data, bval.ctypes.data
    cands = (C.c_uint * 4)(8, 16, 32, 64)
    mine = _abi.SlicedEllTuneResult()
    assert lib.cs_b200_choose_sliced_ell_slice_rows_from_blocked_ell(C.byref(src), cands, 4, C.byref(mine)) == 1
    ref = orc.ref_choose_sliced_ell_slice_rows_from_blocked_ell(rows, cols, b["nnz"], B, b["ell_cols"], bci, bval,
                                                                [8, 16, 32, 64])
    for k in ("slice_rows", "slice_count", "padded_slots", "padded_bytes", "storage_ratio", "slice_penalty", "score"):
        assert getattr(mine, k) == ref[k], k
    dst = _abi.HostSlicedEll()
    assert lib.cs_b200_sliced_ell_from_blocked_ell(C.byref(src), mine.slice_rows, C.byref(dst)) == 1
    live = orc.ref_sliced_ell_from_blocked_ell(rows, cols, b["nnz"], B, b["ell_cols"], bci, bval, mine.slice_rows)
    S = dst.slice_count
    assert S == live["slice_count"] and dst.nnz == live["nnz"] == b["nnz"]
    total = live["total_slots"]
    col = np.ctypeslib.as_array(C.cast(dst.col_idx, C.POINTER(C.c_uint32)), (total,)).copy()
    v = np.ctypeslib.as_array(C.cast(dst.val, C.POINTER(C.c_uint16)), (total,)).copy()
    widths = np.ctypeslib.as_array(C.cast(dst.slice_widths, C.POINTER(C.c_uint32)), (S,)).copy()
    lib.cs_b200_host_sliced_ell_clear(C.byref(dst))
    assert np.array_equal(widths, live["widths"])
    assert np.array_equal(col, live["col_idx"]) and np.array_equal(v, live["val"])
