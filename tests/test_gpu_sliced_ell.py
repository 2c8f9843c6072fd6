"""CSR -> Sliced-ELL on the GPU: bit-exact against the reference's own
convert::sliced_ell_from_compressed (golden vectors and the live bridge), its
chooser, and its GPU route sliced_ell_from_compressed_cuda."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
ROOT = Path(__file__).resolve().parents[1]


def _host(s):
    return (np_u32(s.slice_row_offsets), np_u32(s.slice_widths), np_u32(s.col_idx), np_u16(s.val))


def test_sliced_ell_matches_reference_vectors(cuda):
    from cellshard_b200.device import sliced_ell_from_csr

    gold = np.load(GOLD / "ref_conversions.npz")
    checked = 0
    for n in sorted({k.split("/")[0] for k in gold.files}):
        rows, cols = (int(x) for x in gold[f"{n}/shape"])
        for h in (1, 3, 16, 32, 64):
            key = f"{n}/sell{h}/meta"
            if key not in gold.files:
                continue
            out = sliced_ell_from_csr(to_device_csr(rows, cols, gold[f"{n}/ptr"], gold[f"{n}/idx"], gold[f"{n}/val"]), h)
            offs, widths, col, val = _host(out)
            S, _nnz, total = (int(x) for x in gold[key])
            assert out.slice_count == S and len(col) == total
            assert np.array_equal(offs, gold[f"{n}/sell{h}/offsets"])
            assert np.array_equal(widths, gold[f"{n}/sell{h}/widths"])
            assert np.array_equal(col, gold[f"{n}/sell{h}/col_idx"])
            assert np.array_equal(val, gold[f"{n}/sell{h}/val"])
            checked += 1
    assert checked >= 20


@pytest.mark.parametrize("h", [7, 16, 32, 64])
def test_sliced_ell_generated_matrix_vs_restatement(cuda, orc, h):
    """8,192 x 2,000 NB/Zipf matrix, per slice height."""
    from cellshard_b200 import synth
    from cellshard_b200.device import sliced_ell_from_csr

    csr = synth.make_csr(synth.plain_conversion_spec())
    ptr, idx, val = np_u32(csr.ptr), np_u32(csr.idx), np_u16(csr.val)
    out = sliced_ell_from_csr(csr, h)
    ref = orc.sliced_ell_from_csr(csr.rows, ptr, idx, val, h)
    offs, widths, col, v = _host(out)
    assert np.array_equal(offs, ref["offsets"]) and np.array_equal(widths, ref["widths"])
    assert np.array_equal(np_u32(out.slice_slot_offsets), ref["slot_offsets"])
    assert np.array_equal(col, ref["col_idx"]) and np.array_equal(v, ref["val"])
    if orc.ref_available():
        live = orc.ref_sliced_ell_from_compressed(csr.rows, csr.cols, ptr, idx, val, h)
        assert np.array_equal(col, live["col_idx"]) and np.array_equal(v, live["val"])


def test_sliced_host_api_chooser_and_csc(cuda, orc):
    from cellshard_b200 import _abi

    lib = _abi.load()
    gold = np.load(GOLD / "ref_conversions.npz")
    for n in ("small", "wide", "dense", "empty_rows", "all_empty"):
        rows, cols = (int(x) for x in gold[f"{n}/shape"])
        ptr, idx, val = gold[f"{n}/ptr"], gold[f"{n}/idx"], gold[f"{n}/val"]
        src = _abi.HostCompressed()
        src.rows, src.cols, src.nnz, src.axis = rows, cols, len(idx), 0
        src.majorPtr, src.minorIdx, src.val = ptr.ctypes.data, idx.ctypes.data, val.ctypes.data
        cand = (C.c_uint * 4)(8, 16, 32, 64)
        tune = _abi.SlicedEllTuneResult()
        _abi.check(lib.cs_b200_choose_sliced_ell_slice_rows_from_compressed(C.byref(src), cand, 4, C.byref(tune)),
                   "choose")
        g = [int(x) for x in gold[f"{n}/choose_sell"]]
        assert [tune.slice_rows, tune.slice_count, tune.padded_slots, tune.padded_bytes] == g
        assert tune.score == float(gold[f"{n}/choose_sell_f"][2])
        dst = _abi.HostSlicedEll()
        _abi.check(lib.cs_b200_sliced_ell_from_compressed(C.byref(src), 16, C.byref(dst)), "host sliced")
        S, _nnz, total = (int(x) for x in gold[f"{n}/sell16/meta"])
        assert dst.slice_count == S
        if total:
            col = np.ctypeslib.as_array(C.cast(dst.col_idx, C.POINTER(C.c_uint32)), (total,))
            assert np.array_equal(col, gold[f"{n}/sell16/col_idx"])
        lib.cs_b200_host_sliced_ell_clear(C.byref(dst))
        # the same matrix given column-compressed (the reference's CPU CSC route)
        tptr, tidx, tval = orc.csr_transpose(rows, cols, ptr, idx, val)
        csc = _abi.HostCompressed()
        csc.rows, csc.cols, csc.nnz, csc.axis = rows, cols, len(tidx), 1
        csc.majorPtr, csc.minorIdx, csc.val = tptr.ctypes.data, tidx.ctypes.data, tval.ctypes.data
        dst2 = _abi.HostSlicedEll()
        _abi.check(lib.cs_b200_sliced_ell_from_compressed(C.byref(csc), 16, C.byref(dst2)), "host sliced csc")
        if total:
            col2 = np.ctypeslib.as_array(C.cast(dst2.col_idx, C.POINTER(C.c_uint32)), (total,))
            assert np.array_equal(col2, gold[f"{n}/sell16/col_idx"])
        lib.cs_b200_host_sliced_ell_clear(C.byref(dst2))


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libcs_ref_gpu.so").exists(), reason="reference GPU bridge")
def test_sliced_matches_reference_gpu_route(cuda, orc):
    """sliced_ell_from_compressed_cuda (the reference's own GPU emit) on the same input."""
    from cellshard_b200.device import sliced_ell_from_csr

    rows, cols = 700, 333
    ptr, idx, val = random_csr(rows, cols, 0.07, 17, 0.1)
    src = orc.host_csr(rows, cols, ptr, idx, val)
    dst = orc.HostSlicedEll()
    assert orc.ref_gpu().csrefgpu_sliced_ell_from_compressed_cuda(C.byref(src), 32, C.byref(dst)) == 1
    f = orc.ref().csref_sliced_total_slots
    total = f(C.byref(dst))
    ref_col = np.ctypeslib.as_array(C.cast(dst.col_idx, C.POINTER(C.c_uint32)), (total,)).copy()
    ref_val = np.ctypeslib.as_array(C.cast(dst.val, C.POINTER(C.c_uint16)), (total,)).copy()
    orc.ref().csref_free(dst.storage)
    out = sliced_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), 32)
    assert np.array_equal(np_u32(out.col_idx), ref_col)
    assert np.array_equal(np_u16(out.val), ref_val)
