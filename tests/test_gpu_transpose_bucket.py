"""Transpose and nnz bucketing on the GPU.

Transpose: bit-exact vs the stable counting-sort restatement and vs the
reference's own build_compressed_transpose_raw (cuSPARSE csr2cscEx2 path)
run on the same device buffers.  Bucketing: plan bit-exact vs the
restatement and the reference's CUB plan; power-of-two bins by property;
rebuild vs the restatement, and the reference's rebuild recorded as the
shifted-scan result it produces.
"""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
ref_gpu = pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libcs_ref_gpu.so").exists(),
                             reason="reference GPU bridge not built")


@pytest.mark.parametrize("rows,cols,seed", [(300, 200, 1), (1000, 777, 2), (64, 40000, 3), (5, 3, 4)])
def test_transpose_vs_restatement(cuda, orc, rows, cols, seed):
    from cellshard_b200.device import transpose

    ptr, idx, val = random_csr(rows, cols, 0.05 if cols < 10000 else 0.002, seed, 0.2, integer=(seed % 2 == 0))
    t = transpose(to_device_csr(rows, cols, ptr, idx, val))
    rptr, ridx, rval = orc.csr_transpose(rows, cols, ptr, idx, val)
    assert np.array_equal(np_u32(t.ptr), rptr)
    assert np.array_equal(np_u32(t.idx), ridx)
    assert np.array_equal(np_u16(t.val), rval)


def test_transpose_generated_and_roundtrip(cuda, orc):
    from cellshard_b200 import synth
    from cellshard_b200.device import CSR, transpose

    csr = synth.make_csr(synth.plain_conversion_spec())
    t = transpose(csr)
    ptr, idx, val = np_u32(csr.ptr), np_u32(csr.idx), np_u16(csr.val)
    rptr, ridx, rval = orc.csr_transpose(csr.rows, csr.cols, ptr, idx, val)
    assert np.array_equal(np_u32(t.ptr), rptr) and np.array_equal(np_u32(t.idx), ridx)
    assert np.array_equal(np_u16(t.val), rval)
    back = transpose(CSR(csr.cols, csr.rows, t.ptr, t.idx, t.val))
    assert np.array_equal(np_u32(back.ptr), ptr) and np.array_equal(np_u32(back.idx), idx)
    assert np.array_equal(np_u16(back.val), val)
    if (ROOT / "oracle" / "_ref" / "libcs_ref_gpu.so").exists():
        # the reference's own cuSPARSE route on the whole 8,192 x 2,000 matrix
        import torch

        optr = torch.empty(csr.cols + 1, dtype=torch.int32, device="cuda")
        oidx = torch.empty(csr.nnz, dtype=torch.int32, device="cuda")
        oval = torch.empty(csr.nnz, dtype=torch.float16, device="cuda")
        assert orc.ref_gpu().csrefgpu_transpose(csr.rows, csr.cols, csr.nnz, csr.ptr.data_ptr(), csr.idx.data_ptr(),
                                                csr.val.data_ptr(), optr.data_ptr(), oidx.data_ptr(),
                                                oval.data_ptr()) == 1
        assert np.array_equal(np_u32(t.ptr), np_u32(optr)) and np.array_equal(np_u32(t.idx), np_u32(oidx))
        assert np.array_equal(np_u16(t.val), np_u16(oval))


def test_transpose_keeps_repeated_columns_in_row_order(cuda, orc):
    """A row repeating a column keeps both entries, in CSR order (stable)."""
    from cellshard_b200.device import transpose

    ptr = np.array([0, 3, 4, 6], np.uint32)
    idx = np.array([1, 1, 2, 0, 2, 1], np.uint32)
    val = np.array([1, 2, 3, 4, 5, 6], np.float16).view(np.uint16)
    t = transpose(to_device_csr(3, 3, ptr, idx, val))
    rptr, ridx, rval = orc.csr_transpose(3, 3, ptr, idx, val)
    assert np.array_equal(np_u32(t.ptr), rptr) and np.array_equal(np_u32(t.idx), ridx)
    assert np.array_equal(np_u16(t.val), rval)


@pytest.mark.parametrize("rows,cols,density,unsorted,dups", [
    (3000, 20000, 0.01, 0, 0),    # many pass-1 buckets, uneven rows
    (130, 4096, 0.3, 0, 0),       # dense rows
    (2000, 9000, 0.02, 7, 0),     # some rows unsorted
    (500, 300, 0.05, 0, 4),       # repeated columns
])
def test_transpose_shapes_unsorted_and_repeated(cuda, orc, rows, cols, density, unsorted, dups):
    """Stable transpose of sorted, unsorted and column-repeating rows."""
    from cellshard_b200.device import transpose

    ptr, idx, val = random_csr(rows, cols, density, 21, 0.15, unsorted_rows=unsorted, dup_rows=dups)
    t = transpose(to_device_csr(rows, cols, ptr, idx, val))
    rptr, ridx, rval = orc.csr_transpose(rows, cols, ptr, idx, val)
    assert np.array_equal(np_u32(t.ptr), rptr)
    assert np.array_equal(np_u32(t.idx), ridx)
    assert np.array_equal(np_u16(t.val), rval)


@ref_gpu
def test_transpose_vs_reference_cusparse(cuda, orc):
    import torch

    rows, cols = 900, 500
    ptr, idx, val = random_csr(rows, cols, 0.04, 8, 0.1)
    from cellshard_b200.device import transpose

    d = to_device_csr(rows, cols, ptr, idx, val)
    mine = transpose(d)
    optr = torch.empty(cols + 1, dtype=torch.int32, device="cuda")
    oidx = torch.empty(len(idx), dtype=torch.int32, device="cuda")
    oval = torch.empty(len(idx), dtype=torch.float16, device="cuda")
    assert orc.ref_gpu().csrefgpu_transpose(rows, cols, len(idx), d.ptr.data_ptr(), d.idx.data_ptr(),
                                            d.val.data_ptr(), optr.data_ptr(), oidx.data_ptr(),
                                            oval.data_ptr()) == 1
    assert np.array_equal(np_u32(mine.ptr), np_u32(optr))
    assert np.array_equal(np_u32(mine.idx), np_u32(oidx))
    assert np.array_equal(np_u16(mine.val), np_u16(oval))


@pytest.mark.parametrize("rows,buckets,seed", [(1000, 7, 1), (8192, 16, 2), (3, 10, 3), (70000, 64, 4)])
def test_bucket_plan_vs_restatement(cuda, orc, rows, buckets, seed):
    from cellshard_b200.device import major_nnz_plan, u32

    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 3000 if seed == 4 else 50, rows).astype(np.uint32)
    counts[rng.random(rows) < 0.05] = 70000  # keys above 16 bits exercise the high digit passes
    ptr = np.zeros(rows + 1, np.uint64)
    np.cumsum(counts, out=ptr[1:])
    ptr = ptr.astype(np.uint32)
    out = major_nnz_plan(u32(ptr), rows, buckets)
    nnz, srt, order, offs = orc.major_nnz_plan(ptr, rows, buckets)
    assert np.array_equal(np_u32(out["nnz"])[:rows], nnz)
    assert np.array_equal(np_u32(out["sorted"])[:rows], srt)
    assert np.array_equal(np_u32(out["order"])[:rows], order)
    assert np.array_equal(np_u32(out["order_in"])[:rows], np.arange(rows, dtype=np.uint32))
    assert np.array_equal(np_u32(out["bucket_offsets"]), offs)
    assert np.array_equal(np_u32(out["pow2_bins"]), orc.pow2_bins(srt))


def test_rebuild_and_shard_variants(cuda, orc):
    import torch

    from cellshard_b200 import _abi
    from cellshard_b200.device import major_nnz_plan, rebuild_major_order

    rows, cols = 2000, 300
    ptr, idx, val = random_csr(rows, cols, 0.05, 21, 0.15)
    d = to_device_csr(rows, cols, ptr, idx, val)
    plan = major_nnz_plan(d.ptr, rows, 8)
    rb, inv = rebuild_major_order(d, plan["order"])
    order = np_u32(plan["order"])[:rows]
    rptr, ridx, rval, rinv = orc.rebuild(ptr, idx, val, rows, order)
    assert np.array_equal(np_u32(rb.ptr), rptr) and np.array_equal(np_u32(rb.idx), ridx)
    assert np.array_equal(np_u16(rb.val), rval) and np.array_equal(np_u32(inv)[:rows], rinv)
    # shard variant: the same rows split into 5 uneven parts
    lib = _abi.load()
    cuts = [0, 100, 650, 651, 1500, rows]
    parts_ptr, parts_idx, parts_val = [], [], []
    for a, b in zip(cuts[:-1], cuts[1:]):
        pp = (ptr[a:b + 1] - ptr[a]).astype(np.uint32)
        parts_ptr.append(torch.from_numpy(pp.view(np.int32).copy()).cuda())
        parts_idx.append(torch.from_numpy(idx[ptr[a]:ptr[b]].view(np.int32).copy()).cuda())
        parts_val.append(torch.from_numpy(val[ptr[a]:ptr[b]].view(np.float16).copy()).cuda())

    def table(ts):
        return torch.tensor([t.data_ptr() if t.numel() else 0 for t in ts], dtype=torch.int64, device="cuda")

    tp, ti, tv = table(parts_ptr), table(parts_idx), table(parts_val)
    offs = torch.tensor(cuts, dtype=torch.int32, device="cuda")
    n = C.c_size_t()
    _abi.check(lib.cs_b200_major_nnz_bucket_sort_scratch_bytes(rows, C.byref(n)), "scratch")
    scratch = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    o = {k: torch.empty(rows, dtype=torch.int32, device="cuda") for k in ("nnz", "sorted", "oin", "order")}
    boffs = torch.empty(9, dtype=torch.int32, device="cuda")
    _abi.check(lib.cs_b200_build_shard_major_nnz_bucket_plan(tp.data_ptr(), offs.data_ptr(), 5, rows,
                                                             o["nnz"].data_ptr(), o["sorted"].data_ptr(),
                                                             o["oin"].data_ptr(), o["order"].data_ptr(),
                                                             boffs.data_ptr(), 8, scratch.data_ptr(), n.value, None),
               "shard plan")
    assert np.array_equal(np_u32(o["order"]), order)
    assert np.array_equal(np_u32(boffs), np_u32(plan["bucket_offsets"]))
    dptr = torch.empty(rows + 1, dtype=torch.int32, device="cuda")
    didx = torch.empty(len(idx), dtype=torch.int32, device="cuda")
    dval = torch.empty(len(idx), dtype=torch.float16, device="cuda")
    dinv = torch.empty(rows, dtype=torch.int32, device="cuda")
    _abi.check(lib.cs_b200_major_nnz_bucket_scan_scratch_bytes(rows, C.byref(n)), "scan scratch")
    sc = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    _abi.check(lib.cs_b200_rebuild_bucketed_shard_compressed(tp.data_ptr(), ti.data_ptr(), tv.data_ptr(),
                                                             offs.data_ptr(), 5, rows, o["order"].data_ptr(),
                                                             dptr.data_ptr(), didx.data_ptr(), dval.data_ptr(),
                                                             dinv.data_ptr(), sc.data_ptr(), n.value, None),
               "shard rebuild")
    assert np.array_equal(np_u32(dptr), rptr) and np.array_equal(np_u32(didx), ridx)
    assert np.array_equal(np_u16(dval), rval) and np.array_equal(np_u32(dinv), rinv)


@ref_gpu
def test_plan_vs_reference_cub_and_reference_rebuild_shift(cuda, orc):
    import torch

    from cellshard_b200.device import major_nnz_plan

    rows, cols = 3000, 100
    ptr, idx, val = random_csr(rows, cols, 0.1, 31, 0.1)
    d = to_device_csr(rows, cols, ptr, idx, val)
    mine = major_nnz_plan(d.ptr, rows, 12)
    ref = {k: torch.empty(rows, dtype=torch.int32, device="cuda") for k in ("nnz", "sorted", "oin", "order")}
    offs = torch.empty(13, dtype=torch.int32, device="cuda")
    assert orc.ref_gpu().csrefgpu_major_nnz_plan(d.ptr.data_ptr(), rows, ref["nnz"].data_ptr(),
                                                 ref["sorted"].data_ptr(), ref["oin"].data_ptr(),
                                                 ref["order"].data_ptr(), offs.data_ptr(), 12) == 1
    for k_m, k_r in (("nnz", "nnz"), ("sorted", "sorted"), ("order", "order"), ("order_in", "oin")):
        assert np.array_equal(np_u32(mine[k_m])[:rows], np_u32(ref[k_r])), k_m
    assert np.array_equal(np_u32(mine["bucket_offsets"]), np_u32(offs))
    # the reference rebuild's row pointer is the exclusive scan of counts that
    # were already shifted one slot: [0, 0, c0, c0 + c1, ...]
    rptr = torch.empty(rows + 1, dtype=torch.int32, device="cuda")
    ridx = torch.zeros(len(idx), dtype=torch.int32, device="cuda")
    rval = torch.zeros(len(idx), dtype=torch.float16, device="cuda")
    rinv = torch.empty(rows, dtype=torch.int32, device="cuda")
    assert orc.ref_gpu().csrefgpu_rebuild(d.ptr.data_ptr(), d.idx.data_ptr(), d.val.data_ptr(), rows,
                                          ref["order"].data_ptr(), rptr.data_ptr(), ridx.data_ptr(), rval.data_ptr(),
                                          rinv.data_ptr()) == 1
    counts = np.diff(ptr.astype(np.int64))[np_u32(ref["order"])]
    shifted = np.concatenate([[0, 0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    assert np.array_equal(np_u32(rptr), shifted)
    assert np.array_equal(np_u32(rinv), np.argsort(np_u32(ref["order"])).astype(np.uint32))


@pytest.mark.parametrize("rows,cols,density,seed", [
    (600, 64, 0.9, 31),     # dense, narrow panels
    (1000, 5000, 0.5, 32),  # dense rows, hundreds of panels
    (4097, 257, 0.08, 33),  # ragged last tile and panel
    (70000, 300, 0.02, 34), # many tiles
])
def test_transpose_sorted_row_edges(cuda, orc, rows, cols, density, seed):
    """The stable transpose of sorted rows at dense, ragged and many-tile shapes, bit-exact vs the restatement."""
    from cellshard_b200.device import transpose

    ptr, idx, val = random_csr(rows, cols, density, seed, 0.1, integer=False)
    t = transpose(to_device_csr(rows, cols, ptr, idx, val))
    rptr, ridx, rval = orc.csr_transpose(rows, cols, ptr, idx, val)
    assert np.array_equal(np_u32(t.ptr), rptr)
    assert np.array_equal(np_u32(t.idx), ridx)
    assert np.array_equal(np_u16(t.val), rval)


def _stack_csr(parts):
    """Row-wise concatenation of (rows, ptr, idx, val) CSR pieces with the same column count."""
    ptrs, idxs, vals, base = [np.zeros(1, np.uint32)], [], [], 0
    for _, ptr, idx, val in parts:
        ptrs.append(ptr[1:].astype(np.uint64) + base)
        idxs.append(idx)
        vals.append(val)
        base += int(ptr[-1])
    return (sum(p[0] for p in parts), np.concatenate(ptrs).astype(np.uint32), np.concatenate(idxs).astype(np.uint32),
            np.concatenate(vals).astype(np.uint16))


@pytest.mark.parametrize("case", ["dense_first_tile", "long_rows_among_short"])
def test_transpose_uneven_rows(cuda, orc, case):
    """A block of rows far denser than the rest, and single near-dense rows among
    sparse ones, bit-exact vs the restatement."""
    from cellshard_b200.device import transpose

    cols = 3000
    if case == "dense_first_tile":
        pieces = [(512, *random_csr(512, cols, 0.9, 41, 0.0, integer=False)),
                  (6000, *random_csr(6000, cols, 0.002, 42, 0.3, integer=False))]
    else:
        pieces = []
        for k in range(12):
            pieces.append((300, *random_csr(300, cols, 0.01, 50 + k, 0.1, integer=False)))
            pieces.append((3, *random_csr(3, cols, 0.95, 70 + k, 0.0, integer=False)))
    rows, ptr, idx, val = _stack_csr(pieces)
    t = transpose(to_device_csr(rows, cols, ptr, idx, val))
    rptr, ridx, rval = orc.csr_transpose(rows, cols, ptr, idx, val)
    assert np.array_equal(np_u32(t.ptr), rptr)
    assert np.array_equal(np_u32(t.idx), ridx)
    assert np.array_equal(np_u16(t.val), rval)
