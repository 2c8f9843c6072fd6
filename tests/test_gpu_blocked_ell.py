"""CSR -> Blocked-ELL on the GPU: bit-exact against the reference's own
conversion (golden vectors from convert::blocked_ell_from_compressed, and the
live reference bridge when built) and the C restatement."""

from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"


def _convert(rows, cols, ptr, idx, val, B):
    from cellshard_b200.device import blocked_ell_from_csr

    return blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), B)


def test_blocked_ell_matches_reference_vectors(cuda):
    gold = np.load(GOLD / "ref_conversions.npz")
    names = sorted({k.split("/")[0] for k in gold.files})
    n_checked = 0
    for n in names:
        rows, cols = (int(x) for x in gold[f"{n}/shape"])
        ptr, idx, val = gold[f"{n}/ptr"], gold[f"{n}/idx"], gold[f"{n}/val"]
        for B in (1, 2, 3, 4, 8, 16):
            out = _convert(rows, cols, ptr, idx, val, B)
            ell_cols, nnz = (int(x) for x in gold[f"{n}/bell{B}/meta"])
            assert out.ell_cols == ell_cols, (n, B)
            assert out.nnz == nnz, (n, B)
            assert np.array_equal(np_u32(out.bci), gold[f"{n}/bell{B}/bci"]), (n, B)
            assert np.array_equal(np_u16(out.val), gold[f"{n}/bell{B}/val"]), (n, B)
            n_checked += 1
    assert n_checked == len(names) * 6


@pytest.mark.parametrize("seed,rows,cols,B", [(1, 1000, 777, 16), (2, 513, 2000, 16), (3, 64, 31, 32),
                                              (4, 300, 4097, 8), (5, 17, 5, 2)])
def test_blocked_ell_random_vs_restatement(cuda, orc, seed, rows, cols, B):
    ptr, idx, val = random_csr(rows, cols, 0.06, seed, 0.1, integer=(seed % 2 == 0), dup_rows=seed % 3,
                               unsorted_rows=seed % 2)
    out = _convert(rows, cols, ptr, idx, val, B)
    ref = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
    assert out.ell_cols == ref["ell_cols"] and out.nnz == ref["nnz"]
    assert np.array_equal(np_u32(out.bci), ref["bci"])
    assert np.array_equal(np_u16(out.val), ref["val"])
    if orc.ref_available():
        live = orc.ref_blocked_ell_from_compressed(rows, cols, ptr, idx, val, B)
        assert np.array_equal(np_u16(out.val), live["val"]) and out.nnz == live["nnz"]


def test_blocked_ell_generated_plain_conversion(cuda, orc):
    """8,192 x 2,000 NB/Zipf matrix (lognormal mean 120, clipped [10, 1000]) at block 16."""
    from cellshard_b200 import synth
    from cellshard_b200.device import blocked_ell_from_csr

    csr = synth.make_csr(synth.plain_conversion_spec())
    ptr, idx, val = np_u32(csr.ptr), np_u32(csr.idx), np_u16(csr.val)
    # generator properties: ascending unique in-range columns, positive integer counts
    assert ptr[-1] == len(idx)
    d = np.diff(idx.astype(np.int64))
    starts = ptr[1:-1]
    inner = np.ones(len(d), bool)
    inner[starts[starts < len(idx)] - 1] = False
    assert np.all(d[inner] > 0) and idx.max() < 2000
    vf = val.view(np.float16).astype(np.float32)
    assert vf.min() >= 1 and np.all(vf == np.round(vf))
    out = blocked_ell_from_csr(csr, 16)
    ref = orc.blocked_ell_from_csr(8192, 2000, ptr, idx, val, 16)
    assert out.ell_cols == ref["ell_cols"] and out.nnz == ref["nnz"] == len(idx)
    assert np.array_equal(np_u32(out.bci), ref["bci"])
    assert np.array_equal(np_u16(out.val), ref["val"])
    if orc.ref_available():
        # the reference's own convert::blocked_ell_from_compressed on the whole matrix
        live = orc.ref_blocked_ell_from_compressed(8192, 2000, ptr, idx, val, 16)
        assert live["ell_cols"] == out.ell_cols and live["nnz"] == out.nnz
        assert np.array_equal(np_u32(out.bci), live["bci"])
        assert np.array_equal(np_u16(out.val), live["val"])


def test_blocked_ell_host_api_and_chooser(cuda, orc):
    import ctypes as C

    from cellshard_b200 import _abi

    gold = np.load(GOLD / "ref_conversions.npz")
    lib = _abi.load()
    for n in ("small", "wide", "empty_rows", "all_empty"):
        rows, cols = (int(x) for x in gold[f"{n}/shape"])
        ptr, idx, val = gold[f"{n}/ptr"], gold[f"{n}/idx"], gold[f"{n}/val"]
        src = _abi.HostCompressed()
        src.rows, src.cols, src.nnz, src.axis = rows, cols, len(idx), 0
        src.majorPtr, src.minorIdx, src.val = ptr.ctypes.data, idx.ctypes.data, val.ctypes.data
        dst = _abi.HostBlockedEll()
        _abi.check(lib.cs_b200_blocked_ell_from_compressed(C.byref(src), 4, C.byref(dst)), "host convert")
        ell_cols, nnz = (int(x) for x in gold[f"{n}/bell4/meta"])
        assert dst.ell_cols == ell_cols and dst.nnz == nnz
        if rows * ell_cols:
            v = np.ctypeslib.as_array(C.cast(dst.val, C.POINTER(C.c_uint16)), (rows * ell_cols,))
            assert np.array_equal(v, gold[f"{n}/bell4/val"])
        lib.cs_b200_host_blocked_ell_clear(C.byref(dst))
        cand = (C.c_uint * 4)(4, 8, 16, 32)
        tune = _abi.BlockedEllTuneResult()
        _abi.check(lib.cs_b200_choose_blocked_ell_block_size(C.byref(src), cand, 4, C.byref(tune)), "choose")
        bsz, pbytes = (int(x) for x in gold[f"{n}/choose_bell"])
        assert (tune.block_size, tune.padded_bytes) == (bsz, pbytes)
        assert tune.fill_ratio == float(gold[f"{n}/choose_bell_fill"][0])


def test_blocked_ell_flags_out_of_range_columns(cuda):
    from cellshard_b200 import _abi

    ptr = np.array([0, 2, 3], np.uint32)
    idx = np.array([1, 9, 0], np.uint32)  # 9 >= cols
    val = np.array([1, 2, 3], np.float16).view(np.uint16)
    with pytest.raises(_abi.CellShardError, match="status"):
        _convert(2, 4, ptr, idx, val, 2)
