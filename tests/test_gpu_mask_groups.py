"""mask_groups drop-in on the GPU, called through the C ABI.

Reads like the reference's tests/mask_groups_runtime_test.cu: the same 4 x 5
matrix in Blocked-ELL, CSR and Sliced-ELL with 3 feature groups, row and
feature masks and the same filter; then seeded random cases against the C
restatement, and against the reference's own kernels (compiled from its
sources into oracle/_ref/libcs_ref_gpu.so) on the same device buffers.

Tolerance: 1e-3 absolute for the known answers (the reference test's
close_enough, :21-23); integer-valued random data must match bit for bit
except group_percentages and the fraction filter, which the reference computes
with --use_fast_math division (CMakeLists.txt:183): 2 ulp there.
"""

import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cases import np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
KA = json.loads((GOLD / "mask_groups_known_answers.json").read_text())
ROOT = Path(__file__).resolve().parents[1]


def t(a, dtype=None):
    import torch

    a = np.asarray(a)
    if dtype == "u32":
        return torch.from_numpy(a.astype(np.uint64).astype(np.uint32).view(np.int32).copy()).cuda()
    if dtype == "u8":
        return torch.from_numpy(a.astype(np.uint8).copy()).cuda()
    if dtype == "f16":
        return torch.from_numpy(a.astype(np.float32).astype(np.float16).copy()).cuda()
    raise ValueError(dtype)


def close(a, b, tol=1e-3):
    return abs(float(a) - float(b)) <= tol


def _known():
    from cellshard_b200.device import BlockedELL, CSR, SlicedELL
    from cellshard_b200.runtime import FilterParams

    b = KA["blocked"]
    bell = BlockedELL(4, 5, b["block_size"], b["ell_cols"], t(b["block_cols"], "u32"), t(b["values"], "f16"), 10)
    c = KA["compressed"]
    csr = CSR(4, 5, t(c["ptr"], "u32"), t(c["idx"], "u32"), t(c["values"], "f16"))
    s = KA["sliced"]
    sell = SlicedELL(4, 5, s["nnz"], s["slice_rows"], t(s["offsets"], "u32"), t(s["widths"], "u32"),
                     t(s["slot_offsets"], "u32"), t(s["col_idx"], "u32"), t(s["values"], "f16"))
    f = KA["filter"]
    return bell, csr, sell, FilterParams(f[0], f[1], f[2], f[3])


def host(res):
    return {k: (None if v is None else v.cpu().numpy()) for k, v in res.items()}


def test_known_answers_through_c_abi(cuda):
    from cellshard_b200 import runtime

    bell, csr, sell, filt = _known()
    gm, rk, fk = t(KA["group_masks"], "u32"), t(KA["row_keep"], "u8"), t(KA["feature_keep"], "u8")
    r = host(runtime.compute_sparse_group_reduce(bell, gm, 3, rk, fk, filt))
    e = KA["expect_blocked"]
    assert all(close(a, b) for a, b in zip(r["row_totals"], e["row_totals"]))
    assert list(r["detected_features"]) == e["detected"]
    assert list(r["row_keep"]) == e["keep"]
    for k, v in e["group_counts"].items():
        assert close(r["group_counts"][int(k)], v)
    for k, v in e["group_percentages"].items():
        assert close(r["group_percentages"][int(k)], v)
    r = host(runtime.compute_sparse_group_reduce(bell, None, 0, None, None, filt))
    assert r["group_counts"] is None and close(r["row_totals"][0], 15) and r["detected_features"][0] == 3
    r = host(runtime.compute_sparse_group_reduce(csr, gm, 3, rk, fk, filt))
    assert close(r["row_totals"][2], 7) and close(r["group_counts"][8], 2)
    r = host(runtime.compute_sparse_group_reduce(sell, gm, 3, rk, fk, filt))
    assert close(r["row_totals"][0], 8) and close(r["row_totals"][3], 18)
    rr = KA["reoptimize"]
    out, meta = runtime.manual_reoptimize_masked_sparse(bell, rk, fk, t(rr["row_remap"], "u32"),
                                                        t(rr["feature_remap"], "u32"), rr["output_rows"],
                                                        rr["output_cols"])
    e = KA["expect_reoptimize"]
    assert (meta["kept_rows"], meta["kept_features"], meta["live_nnz"]) == (e["kept_rows"], e["kept_features"],
                                                                            e["live_nnz"])


def _random_inputs(rows, cols, seed, integer=True):
    ptr, idx, val = random_csr(rows, cols, 0.08, seed, 0.1, integer)
    rng = np.random.default_rng(seed)
    masks = rng.integers(0, 2 ** 32, cols, dtype=np.uint64).astype(np.uint32) & np.uint32(0x1F_FFFF)
    masks[rng.random(cols) < 0.3] = 0
    rk = (rng.random(rows) < 0.75).astype(np.uint8)
    fk = (rng.random(cols) < 0.8).astype(np.uint8)
    return ptr, idx, val, masks, rk, fk


def _cmp(r, o, exact=True):
    assert np.array_equal(r["row_keep"], o["row_keep"]) or not exact
    assert np.array_equal(r["detected_features"].view(np.uint32), o["detected_features"])
    if exact:
        assert np.array_equal(r["row_totals"], o["row_totals"])
        assert np.array_equal(r["max_values"], o["max_values"])
        assert np.array_equal(r["group_counts"], o["group_counts"])
        assert np.array_equal(r["group_percentages"], o["group_percentages"])
    else:
        assert np.allclose(r["row_totals"], o["row_totals"], rtol=1e-5, atol=1e-3)
        assert np.array_equal(r["max_values"], o["max_values"])
        assert np.allclose(r["group_counts"], o["group_counts"], rtol=1e-5, atol=1e-3)


@pytest.mark.parametrize("seed,integer", [(1, True), (2, True), (3, False)])
def test_random_all_formats_vs_restatement(cuda, orc, seed, integer):
    import torch

    from cellshard_b200 import runtime
    from cellshard_b200.device import SlicedELL, blocked_ell_from_csr

    rows, cols, G = 700, 300, 21
    ptr, idx, val, masks, rk, fk = _random_inputs(rows, cols, seed, integer)
    filt = runtime.FilterParams(3.0, 2, 0.5, 4)
    fa = (3.0, 2, 0.5, 4)
    csr = to_device_csr(rows, cols, ptr, idx, val)
    gm, drk, dfk = t(masks, "u32"), t(rk, "u8"), t(fk, "u8")
    r = host(runtime.compute_sparse_group_reduce(csr, gm, G, drk, dfk, filt))
    o = orc.group_reduce_csr(rows, cols, ptr, idx, val, masks, G, rk, fk, fa)
    _cmp(r, o, integer)
    bell = blocked_ell_from_csr(csr, 16)
    r = host(runtime.compute_sparse_group_reduce(bell, gm, G, drk, dfk, filt))
    o = orc.group_reduce_bell(rows, cols, 16, bell.ell_cols, np_u32(bell.bci), bell.val.cpu().numpy().view(np.uint16),
                              masks, G, rk, fk, fa)
    _cmp(r, o, integer)
    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, 32)
    sell = SlicedELL(rows, cols, len(idx), 32, t(s["offsets"], "u32"), t(s["widths"], "u32"),
                     t(s["slot_offsets"], "u32"), t(s["col_idx"], "u32"),
                     torch.from_numpy(s["val"].view(np.float16).copy()).cuda())
    r = host(runtime.compute_sparse_group_reduce(sell, gm, G, drk, dfk, filt))
    o = orc.group_reduce_sell(rows, cols, 32, s["offsets"], s["widths"], s["slot_offsets"], s["col_idx"], s["val"],
                              masks, G, rk, fk, fa)
    _cmp(r, o, integer)


def test_reoptimize_random_vs_restatement(cuda, orc):
    from cellshard_b200 import runtime
    from cellshard_b200.device import blocked_ell_from_csr

    rows, cols = 500, 260
    ptr, idx, val, _m, rk, fk = _random_inputs(rows, cols, 11)
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), 8)
    rng = np.random.default_rng(4)
    kept = np.flatnonzero(rk)
    row_remap = np.full(rows, 0xFFFFFFFF, np.uint32)
    row_remap[kept] = rng.permutation(len(kept)).astype(np.uint32)
    feat_remap = np.full(cols, 0xFFFFFFFF, np.uint32)
    kf = np.flatnonzero(fk)
    feat_remap[kf] = np.arange(len(kf), dtype=np.uint32)
    out_rows, out_cols = len(kept) - 5, len(kf) - 3
    out, meta = runtime.manual_reoptimize_masked_sparse(bell, t(rk, "u8"), t(fk, "u8"), t(row_remap, "u32"),
                                                        t(feat_remap, "u32"), out_rows, out_cols)
    major, oidx, oval = orc.reoptimize_bell(rows, cols, 8, bell.ell_cols, np_u32(bell.bci),
                                            bell.val.cpu().numpy().view(np.uint16), rk, fk, row_remap, feat_remap,
                                            out_rows, out_cols)
    assert np.array_equal(np_u32(out.ptr), major)
    assert np.array_equal(np_u32(out.idx), oidx)
    assert np.array_equal(out.val.cpu().numpy().view(np.uint16), oval)
    assert meta["live_nnz"] == int(major[-1])


ref_gpu = pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libcs_ref_gpu.so").exists(),
                             reason="reference GPU bridge not built")


@ref_gpu
def test_reference_kernels_agree_on_known_answers(cuda, orc):
    """The reference's own kernels on the known-answer inputs: confirms the two
    expectations of its test that its kernel does not produce (fixture notes)."""
    import ctypes as C

    import torch

    from cellshard_b200 import _abi

    bell, _csr, _sell, _f = _known()
    rows, G = 4, 3
    outs = {k: torch.zeros(rows * (G if k.startswith("group") else 1),
                           dtype=torch.uint8 if k == "row_keep" else torch.float32, device="cuda")
            for k in ("row_totals", "detected_features", "max_values", "row_keep", "group_counts",
                      "group_percentages")}
    o = _abi.GroupReduceOut(*(outs[k].data_ptr() for k in ("row_totals", "detected_features", "max_values",
                                                             "row_keep", "group_counts", "group_percentages")))
    m = _abi.RowFeatureMaskView()
    rk, fk, gm = t(KA["row_keep"], "u8"), t(KA["feature_keep"], "u8"), t(KA["group_masks"], "u32")
    m.row_keep, m.feature_keep = rk.data_ptr(), fk.data_ptr()
    f = _abi.GroupFilterParams(*KA["filter"])
    v = bell.view()
    assert orc.ref_gpu().csrefgpu_group_reduce_blocked_ell(C.byref(v), C.c_void_p(gm.data_ptr()), G, C.byref(m),
                                                           C.byref(f), C.byref(o)) == 1
    keep = outs["row_keep"].cpu().numpy()
    gc = outs["group_counts"].cpu().numpy()
    assert list(keep) == KA["expect_blocked"]["keep"]
    assert gc[8] == KA["expect_blocked"]["group_counts"]["8"]


@ref_gpu
def test_reference_test_binary_exit_code(cuda):
    exe = ROOT / "oracle" / "_ref" / "mask_groups_runtime_test"
    if not exe.exists():
        pytest.skip("reference test binary not built")
    rc = subprocess.run([str(exe)], capture_output=True, timeout=120).returncode
    assert rc == KA["reference_test_asserts"]["expected_exit_code"]


@ref_gpu
@pytest.mark.parametrize("seed", [5, 6])
def test_random_vs_reference_kernels(cuda, orc, seed):
    import ctypes as C

    import torch

    from cellshard_b200 import _abi, runtime
    from cellshard_b200.device import blocked_ell_from_csr

    rows, cols, G = 900, 333, 17
    ptr, idx, val, masks, rk, fk = _random_inputs(rows, cols, seed)
    csr = to_device_csr(rows, cols, ptr, idx, val)
    bell = blocked_ell_from_csr(csr, 16)
    gm, drk, dfk = t(masks, "u32"), t(rk, "u8"), t(fk, "u8")
    filt = runtime.FilterParams(2.0, 3, 0.6, 1)
    for src, fn in ((bell, "csrefgpu_group_reduce_blocked_ell"), (csr, "csrefgpu_group_reduce_compressed")):
        mine = host(runtime.compute_sparse_group_reduce(src, gm, G, drk, dfk, filt))
        outs = {k: torch.zeros_like(torch.from_numpy(v)).cuda() for k, v in mine.items()}
        o = _abi.GroupReduceOut(*(outs[k].data_ptr() for k in ("row_totals", "detected_features", "max_values",
                                                                 "row_keep", "group_counts", "group_percentages")))
        m = _abi.RowFeatureMaskView()
        m.row_keep, m.feature_keep = drk.data_ptr(), dfk.data_ptr()
        f = filt.c()
        v = src.view()
        assert getattr(orc.ref_gpu(), fn)(C.byref(v), C.c_void_p(gm.data_ptr()), G, C.byref(m), C.byref(f),
                                          C.byref(o)) == 1
        ref = host(outs)
        for k in ("row_totals", "detected_features", "max_values", "group_counts"):
            assert np.array_equal(mine[k], ref[k]), (fn, k)
        p, q = mine["group_percentages"].view(np.int32), ref["group_percentages"].view(np.int32)
        assert np.max(np.abs(p.astype(np.int64) - q.astype(np.int64))) <= 2, fn
        diff = np.flatnonzero(mine["row_keep"] != ref["row_keep"])
        assert len(diff) <= 2, (fn, diff)  # fast-math fraction right at the threshold


def _shifted(t):
    """The same values starting one element past an aligned allocation, so
    the kernels take their unaligned (per-entry) path."""
    import torch

    buf = torch.empty(t.numel() + 1, dtype=t.dtype, device=t.device)
    buf[1:] = t
    return buf[1:]


@pytest.mark.parametrize("seed", [7, 8])
def test_unaligned_views_match_vector_path(cuda, orc, seed):
    """Compressed and Sliced-ELL reduces over 16-byte-aligned arrays (quad
    loads, ragged heads and tails) and over arrays shifted by one element
    (per-entry loads) agree with each other and with the restatement."""
    from dataclasses import replace

    import torch

    from cellshard_b200 import runtime
    from cellshard_b200.device import SlicedELL

    rows, cols, G = 640, 515, 9
    ptr, idx, val, masks, rk, fk = _random_inputs(rows, cols, seed)
    filt = runtime.FilterParams(3.0, 2, 0.5, 2)
    fa = (3.0, 2, 0.5, 2)
    csr = to_device_csr(rows, cols, ptr, idx, val)
    gm, drk, dfk = t(masks, "u32"), t(rk, "u8"), t(fk, "u8")
    o = orc.group_reduce_csr(rows, cols, ptr, idx, val, masks, G, rk, fk, fa)
    a = host(runtime.compute_sparse_group_reduce(csr, gm, G, drk, dfk, filt))
    csr_u = replace(csr, idx=_shifted(csr.idx), val=_shifted(csr.val))
    assert csr_u.idx.data_ptr() % 16 != 0
    u = host(runtime.compute_sparse_group_reduce(csr_u, gm, G, drk, dfk, filt))
    _cmp(a, o)
    _cmp(u, o)
    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, 32)
    sell = SlicedELL(rows, cols, len(idx), 32, t(s["offsets"], "u32"), t(s["widths"], "u32"),
                     t(s["slot_offsets"], "u32"), t(s["col_idx"], "u32"),
                     torch.from_numpy(s["val"].view(np.float16).copy()).cuda())
    o = orc.group_reduce_sell(rows, cols, 32, s["offsets"], s["widths"], s["slot_offsets"], s["col_idx"], s["val"],
                              masks, G, rk, fk, fa)
    _cmp(host(runtime.compute_sparse_group_reduce(sell, gm, G, drk, dfk, filt)), o)
    sell_u = replace(sell, col_idx=_shifted(sell.col_idx), val=_shifted(sell.val))
    _cmp(host(runtime.compute_sparse_group_reduce(sell_u, gm, G, drk, dfk, filt)), o)


def _bell_case(rows, cols, G, seed, integer, density=0.08):
    ptr, idx, val = random_csr(rows, cols, density, seed, 0.1, integer)
    rng = np.random.default_rng(seed + 100)
    masks = rng.integers(0, 2 ** 32, cols, dtype=np.uint64).astype(np.uint32)
    masks[rng.random(cols) < 0.3] = 0
    rk = (rng.random(rows) < 0.75).astype(np.uint8)
    fk = (rng.random(cols) < 0.8).astype(np.uint8)
    return ptr, idx, val, masks, rk, fk


def _cmp_nan(r, o, exact=True):
    """_cmp for outputs that may hold NaN / inf (equal NaNs count as equal)."""
    assert np.array_equal(r["detected_features"].view(np.uint32), o["detected_features"])
    assert np.array_equal(r["row_keep"], o["row_keep"])
    for k in ("row_totals", "max_values", "group_counts", "group_percentages"):
        if r[k] is None:
            assert o[k] is None or o[k].size == 0
            continue
        if exact or k == "max_values":
            assert np.array_equal(r[k], o[k], equal_nan=True), k
        else:
            assert np.allclose(r[k], o[k], rtol=1e-5, atol=1e-3, equal_nan=True), k


@pytest.mark.parametrize("G,rows,cols,integer,masked", [
    (0, 700, 300, True, True),      # totals only (pipelined tensor-core kernel)
    (5, 700, 300, True, False),     # no row / feature masks
    (12, 700, 515, True, True),     # two group tiles, last column block partial
    (12, 700, 515, False, True),
    (16, 700, 300, True, True),     # register tensor-core kernel
    (24, 333, 333, True, True),
    (32, 700, 300, True, True),
    (32, 700, 300, False, True),
    (8, 48, 50000, True, True),     # a wide column table beside the many-warp pipeline
    (8, 48, 70000, True, True),     # the table leaves room for 16 warps only
    (8, 48, 90000, True, True),     # column table too large for shared memory
])
def test_bell16_tensor_core_paths(cuda, orc, G, rows, cols, integer, masked):
    """Blocked-ELL-16 reduces on the tensor-core kernels (every group-count
    class, partial last column block, padding slots, rows not a multiple of 16)
    against the restatement."""
    from cellshard_b200 import runtime
    from cellshard_b200.device import blocked_ell_from_csr

    ptr, idx, val, masks, rk, fk = _bell_case(rows, cols, G, 11 + G, integer,
                                              density=0.08 if cols < 10000 else 0.002)
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), 16)
    filt = runtime.FilterParams(3.0, 2, 0.5, min(G - 1, 9) if G else 0)
    fa = (3.0, 2, 0.5, min(G - 1, 9) if G else 0)
    gm = t(masks, "u32") if G else None
    r = host(runtime.compute_sparse_group_reduce(bell, gm, G, t(rk, "u8") if masked else None,
                                                 t(fk, "u8") if masked else None, filt))
    o = orc.group_reduce_bell(rows, cols, 16, bell.ell_cols, np_u32(bell.bci), bell.val.cpu().numpy().view(np.uint16),
                              masks if G else None, G, rk if masked else None, fk if masked else None, fa)
    _cmp_nan(r, o, integer)


@pytest.mark.parametrize("G", [3, 12, 20])
def test_bell16_nonfinite_rows_take_per_row_path(cuda, orc, G):
    """inf / NaN values (in kept and dropped columns) give the reference's
    per-value results: their row blocks are redone on the per-row path."""
    import torch

    from cellshard_b200 import runtime
    from cellshard_b200.device import blocked_ell_from_csr

    rows, cols = 200, 300
    ptr, idx, val, masks, rk, fk = _bell_case(rows, cols, G, 3, True)
    val = val.copy()
    special = np.array([np.inf, -np.inf, np.nan], np.float16).view(np.uint16)
    rng = np.random.default_rng(9)
    for p in rng.choice(len(val), size=6, replace=False):
        val[p] = special[p % 3]
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), 16)
    filt = runtime.FilterParams(3.0, 2, 0.5, 1)
    r = host(runtime.compute_sparse_group_reduce(bell, t(masks, "u32"), G, t(rk, "u8"), t(fk, "u8"), filt))
    o = orc.group_reduce_bell(rows, cols, 16, bell.ell_cols, np_u32(bell.bci), bell.val.cpu().numpy().view(np.uint16),
                              masks, G, rk, fk, (3.0, 2, 0.5, 1))
    assert not np.all(np.isfinite(o["row_totals"]))
    _cmp_nan(r, o)
    # the per-row kernel (values not 16-byte aligned) agrees
    from dataclasses import replace

    r2 = host(runtime.compute_sparse_group_reduce(replace(bell, val=_shifted(bell.val)), t(masks, "u32"), G,
                                                  t(rk, "u8"), t(fk, "u8"), filt))
    _cmp_nan(r2, o)
