"""Reference GPU points: the reference's own GPU code (built from its sources
for sm_100a: the cuSPARSE transpose route, the CUB nnz plan, the mask_groups
Blocked-ELL kernel) timed beside this library's kernels on the same device
buffers, with both outputs compared.

The matrix is the grouped-reduction workload's generator at 100,000 rows by
default (32,768 columns, ~4 % density); CS_REFPOINT_ROWS=500000 gives the
full size.  Times are CUDA events around repeated calls after warm-up
(the reference's calls through oracle/_ref timed inside the bridge, so its
allocations are outside the timed region).  One JSON line is printed.
"""

import ctypes as C
import json
import os

import numpy as np
import pytest

from cases import np_u16, np_u32

pytestmark = pytest.mark.gpu

REPS = 5


def _percent_ulps(ours, ref):
    """group_percentages within 2 ulp of the reference kernels' (they divide with
    --use_fast_math); every value is a non-negative float, so the ulp distance is
    the difference of the bit patterns."""
    import torch

    a = ours["group_percentages"].view(torch.int32).long()
    b = ref["group_percentages"].view(torch.int32).long()
    assert int((a - b).abs().max()) <= 2


def _time_ours(fn, reps=REPS, warmup=2):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def test_reference_gpu_points(cuda, orc):
    if not orc.ref_gpu_available():
        pytest.skip("reference GPU library not built")
    import torch

    from cellshard_b200 import _abi, runtime, synth
    from cellshard_b200.device import blocked_ell_from_csr, ptr, stream_handle

    rows = int(os.environ.get("CS_REFPOINT_ROWS", "100000"))
    spec = synth.grouped_reduction_spec(rows)
    csr = synth.make_csr(spec)
    R, Cc, nnz = csr.rows, csr.cols, csr.nnz
    lib, rg = _abi.load(), orc.ref_gpu()
    out = {"rows": R, "cols": Cc, "nnz": nnz}
    ms_ref = C.c_float()

    # transpose: this library's two-pass sort vs cuSPARSE csr2cscEx2 through the reference
    nb = C.c_size_t()
    lib.cs_b200_compressed_transpose_scratch_bytes(R, Cc, nnz, C.byref(nb))
    scr = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    o = [torch.empty(Cc + 1, dtype=torch.int32, device="cuda"), torch.empty(nnz, dtype=torch.int32, device="cuda"),
         torch.empty(nnz, dtype=torch.float16, device="cuda")]
    r = [torch.empty_like(t) for t in o]
    ms = _time_ours(lambda: lib.cs_b200_build_compressed_transpose(R, Cc, nnz, ptr(csr.ptr), ptr(csr.idx),
                                                                   ptr(csr.val), ptr(o[0]), None, ptr(o[1]),
                                                                   ptr(o[2]), ptr(scr), nb.value, stream_handle()))
    assert rg.csrefgpu_transpose_timed(R, Cc, nnz, ptr(csr.ptr), ptr(csr.idx), ptr(csr.val), ptr(r[0]), ptr(r[1]),
                                       ptr(r[2]), 2, REPS, C.byref(ms_ref)) == 1
    for a, b in zip(o, r):
        assert torch.equal(a, b)
    out["transpose_ms"] = {"ours": ms, "reference_cusparse": ms_ref.value}
    del o, r, scr
    torch.cuda.empty_cache()

    # nnz plan: this library's radix passes vs the reference's CUB SortPairs route
    B = 64
    plan = [torch.empty(R, dtype=torch.int32, device="cuda") for _ in range(4)]
    offs = torch.empty(B + 1, dtype=torch.int32, device="cuda")
    rplan = [torch.empty_like(t) for t in plan]
    roffs = torch.empty_like(offs)
    lib.cs_b200_major_nnz_bucket_sort_scratch_bytes(R, C.byref(nb))
    sscr = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    ms = _time_ours(lambda: lib.cs_b200_build_major_nnz_bucket_plan(ptr(csr.ptr), R, *[ptr(t) for t in plan],
                                                                    ptr(offs), B, ptr(sscr), nb.value,
                                                                    stream_handle()))
    assert rg.csrefgpu_major_nnz_plan_timed(ptr(csr.ptr), R, *[ptr(t) for t in rplan], ptr(roffs), B, 2, REPS,
                                            C.byref(ms_ref)) == 1
    for a, b in zip(plan + [offs], rplan + [roffs]):
        assert torch.equal(a, b)
    out["nnz_plan_ms"] = {"ours": ms, "reference_cub": ms_ref.value}

    # mask_groups reduce over the compressed, Sliced-ELL and Blocked-ELL forms:
    # this library's kernels vs the reference's
    rng = np.random.default_rng(5)
    G = 8
    masks = (rng.integers(0, 1 << G, Cc) & rng.integers(0, 2, Cc) * 0xFF).astype(np.uint32)
    d_masks = torch.from_numpy(masks.view(np.int32)).cuda()
    rk = torch.from_numpy((rng.random(R) < 0.7).astype(np.uint8)).cuda()
    fk = torch.from_numpy((rng.random(Cc) < 0.6).astype(np.uint8)).cuda()
    filt = runtime.FilterParams(10.0, 5, 0.9, 0)
    mv = _abi.RowFeatureMaskView(ptr(rk), ptr(fk), None, None)
    fp = filt.c()

    def compare(ours, bridge, v):
        ref = {k: torch.empty_like(t) for k, t in ours.items() if t is not None}
        ro = _abi.GroupReduceOut(ptr(ref["row_totals"]), ptr(ref["detected_features"]), ptr(ref["max_values"]),
                                 ptr(ref["row_keep"]), ptr(ref["group_counts"]), ptr(ref["group_percentages"]))
        assert bridge(C.byref(v), ptr(d_masks), G, C.byref(mv), C.byref(fp), C.byref(ro)) == 1
        torch.cuda.synchronize()
        for k in ("row_totals", "detected_features", "max_values", "row_keep", "group_counts"):
            assert torch.equal(ours[k], ref[k]), k
        _percent_ulps(ours, ref)

    ours = runtime.compute_sparse_group_reduce(csr, d_masks, G, rk, fk, filt)
    ms = _time_ours(lambda: runtime.compute_sparse_group_reduce(csr, d_masks, G, rk, fk, filt))
    v = csr.view()
    assert rg.csrefgpu_group_reduce_compressed_timed(C.byref(v), ptr(d_masks), G, C.byref(mv), C.byref(fp), 2, REPS,
                                                     C.byref(ms_ref)) == 1
    compare(ours, rg.csrefgpu_group_reduce_compressed, v)
    out["mask_groups_reduce_compressed_ms"] = {"ours": ms, "reference": ms_ref.value}

    from cellshard_b200.device import sliced_ell_from_csr

    sell = sliced_ell_from_csr(csr, 32)
    ours = runtime.compute_sparse_group_reduce(sell, d_masks, G, rk, fk, filt)
    ms = _time_ours(lambda: runtime.compute_sparse_group_reduce(sell, d_masks, G, rk, fk, filt))
    v = sell.view()
    assert rg.csrefgpu_group_reduce_sliced_ell_timed(C.byref(v), ptr(d_masks), G, C.byref(mv), C.byref(fp), 2, REPS,
                                                     C.byref(ms_ref)) == 1
    compare(ours, rg.csrefgpu_group_reduce_sliced_ell, v)
    out["mask_groups_reduce_sliced_ms"] = {"ours": ms, "reference": ms_ref.value,
                                           "bytes": int(sell.col_idx.numel()) * 6}
    del sell
    torch.cuda.empty_cache()

    bell = blocked_ell_from_csr(csr, 16)
    del csr
    torch.cuda.empty_cache()
    ours = runtime.compute_sparse_group_reduce(bell, d_masks, G, rk, fk, filt)
    ms = _time_ours(lambda: runtime.compute_sparse_group_reduce(bell, d_masks, G, rk, fk, filt))
    v = bell.view()
    assert rg.csrefgpu_group_reduce_blocked_ell_timed(C.byref(v), ptr(d_masks), G, C.byref(mv), C.byref(fp), 2, REPS,
                                                      C.byref(ms_ref)) == 1
    ref = {k: torch.empty_like(t) for k, t in ours.items() if t is not None}
    ro = _abi.GroupReduceOut(ptr(ref["row_totals"]), ptr(ref["detected_features"]), ptr(ref["max_values"]),
                             ptr(ref["row_keep"]), ptr(ref["group_counts"]), ptr(ref["group_percentages"]))
    assert rg.csrefgpu_group_reduce_blocked_ell(C.byref(v), ptr(d_masks), G, C.byref(mv), C.byref(fp),
                                                C.byref(ro)) == 1
    torch.cuda.synchronize()
    for k in ("row_totals", "detected_features", "max_values", "row_keep", "group_counts"):
        assert torch.equal(ours[k], ref[k]), k
    _percent_ulps(ours, ref)
    bytes_read = R * bell.ell_cols * 2 + bell.row_blocks * bell.ell_width * 4
    out["mask_groups_reduce_ms"] = {"ours": ms, "reference": ms_ref.value, "bytes_read": bytes_read}
    print(json.dumps({"reference_gpu_points": out}))
