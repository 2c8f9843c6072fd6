"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point the header declares, the ctypes mirrors match the C layouts, and
host-side argument validation rejects bad calls with a message."""

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from cellshard_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "cellshard_b200.h"


def declared_entry_points():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"CS_API\s+[\w\s\*]*?\b(cs_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(cs_lib):
    names = declared_entry_points()
    assert len(names) >= 15
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_abi.LIB_PATH)], capture_output=True, text=True,
                        check=True).stdout
    exported = set(re.findall(r"\bT (cs_b200_\w+)", nm))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(cs_lib, n)
    assert set(names) <= set(_abi.PROTOTYPES), sorted(set(names) - set(_abi.PROTOTYPES))


LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include "cellshard_b200.h"
#define S(T) printf(#T " %zu\n", sizeof(T));
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  S(cs_compressed_view) O(cs_compressed_view, val)
  S(cs_blocked_ell_view) O(cs_blocked_ell_view, blockColIdx) O(cs_blocked_ell_view, val)
  S(cs_sliced_ell_view) O(cs_sliced_ell_view, slice_row_offsets) O(cs_sliced_ell_view, val)
  S(cs_host_compressed) O(cs_host_compressed, storage) O(cs_host_compressed, val)
  S(cs_host_blocked_ell) O(cs_host_blocked_ell, storage) O(cs_host_blocked_ell, val)
  S(cs_host_sliced_ell) O(cs_host_sliced_ell, storage) O(cs_host_sliced_ell, val)
  S(cs_blocked_ell_tune_result) S(cs_sliced_ell_tune_result)
  S(cs_row_feature_mask_view) S(cs_group_filter_params) S(cs_group_reduce_out)
  S(cs_group_moments_params) S(cs_group_moments_out)
  S(cs_batch_part) O(cs_batch_part, d_major_nnz) O(cs_batch_part, d_pow2_offsets)
  S(cs_batch_tiles) S(cs_batch_sliced_result) O(cs_batch_sliced_result, view)
  S(cs_serve_config) S(cs_serve_request) O(cs_serve_request, group_rows) S(cs_serve_stats)
  S(cs_partition_record) O(cs_partition_record, host_view)
  S(cs_staged_part) O(cs_staged_part, group_begin) O(cs_staged_part, device_id)
  S(cs_cached_allocation) S(cs_sharded_device) O(cs_sharded_device, cache)
  S(cs_host_bucketed_blocked_ell) O(cs_host_bucketed_blocked_ell, canonical_to_exec_cols)
  S(cs_host_bucketed_sliced_ell) O(cs_host_bucketed_sliced_ell, canonical_slice_widths)
  S(cs_exec_bucket_plan) O(cs_exec_bucket_plan, value_entries) S(cs_exec_bucket_segments)
  S(cs_host_coo) O(cs_host_coo, val) S(cs_coo_view) O(cs_coo_view, val) S(cs_cspack_info)
  return 0;
}
"""

PAIRS = {
    "cs_compressed_view": _abi.CompressedView,
    "cs_blocked_ell_view": _abi.BlockedEllView,
    "cs_sliced_ell_view": _abi.SlicedEllView,
    "cs_host_compressed": _abi.HostCompressed,
    "cs_host_blocked_ell": _abi.HostBlockedEll,
    "cs_host_sliced_ell": _abi.HostSlicedEll,
    "cs_blocked_ell_tune_result": _abi.BlockedEllTuneResult,
    "cs_sliced_ell_tune_result": _abi.SlicedEllTuneResult,
    "cs_row_feature_mask_view": _abi.RowFeatureMaskView,
    "cs_group_filter_params": _abi.GroupFilterParams,
    "cs_group_reduce_out": _abi.GroupReduceOut,
    "cs_group_moments_params": _abi.GroupMomentsParams,
    "cs_group_moments_out": _abi.GroupMomentsOut,
    "cs_batch_part": _abi.BatchPart,
    "cs_batch_tiles": _abi.BatchTiles,
    "cs_batch_sliced_result": _abi.BatchSlicedResult,
    "cs_serve_config": _abi.ServeConfig,
    "cs_serve_request": _abi.ServeRequest,
    "cs_serve_stats": _abi.ServeStats,
    "cs_partition_record": _abi.PartitionRecord,
    "cs_staged_part": _abi.StagedPart,
    "cs_cached_allocation": _abi.CachedAllocation,
    "cs_sharded_device": _abi.ShardedDevice,
    "cs_host_bucketed_blocked_ell": _abi.HostBucketedBlockedEll,
    "cs_host_bucketed_sliced_ell": _abi.HostBucketedSlicedEll,
    "cs_exec_bucket_plan": _abi.ExecBucketPlan,
    "cs_exec_bucket_segments": _abi.ExecBucketSegments,
    "cs_host_coo": _abi.HostCoo,
    "cs_coo_view": _abi.CooView,
    "cs_cspack_info": _abi.CspackInfo,
}


def test_ctypes_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        k, v = line.split()
        got[k] = int(v)
    for cname, ct in PAIRS.items():
        assert got[cname] == C.sizeof(ct), cname
    assert got["cs_blocked_ell_view.val"] == _abi.BlockedEllView.val.offset
    assert got["cs_sliced_ell_view.val"] == _abi.SlicedEllView.val.offset
    assert got["cs_host_compressed.val"] == _abi.HostCompressed.val.offset
    assert got["cs_host_sliced_ell.val"] == _abi.HostSlicedEll.val.offset
    assert got["cs_batch_part.d_major_nnz"] == _abi.BatchPart.d_major_nnz.offset
    assert got["cs_batch_part.d_pow2_offsets"] == _abi.BatchPart.d_pow2_offsets.offset
    assert got["cs_host_bucketed_blocked_ell.canonical_to_exec_cols"] == \
        _abi.HostBucketedBlockedEll.canonical_to_exec_cols.offset
    assert got["cs_host_bucketed_sliced_ell.canonical_slice_widths"] == \
        _abi.HostBucketedSlicedEll.canonical_slice_widths.offset
    assert got["cs_exec_bucket_plan.value_entries"] == _abi.ExecBucketPlan.value_entries.offset
    assert got["cs_host_coo.val"] == _abi.HostCoo.val.offset and got["cs_coo_view.val"] == _abi.CooView.val.offset
    assert got["cs_batch_sliced_result.view"] == _abi.BatchSlicedResult.view.offset
    assert got["cs_serve_request.group_rows"] == _abi.ServeRequest.group_rows.offset
    assert got["cs_partition_record.host_view"] == _abi.PartitionRecord.host_view.offset
    assert got["cs_staged_part.group_begin"] == _abi.StagedPart.group_begin.offset
    assert got["cs_staged_part.device_id"] == _abi.StagedPart.device_id.offset
    assert got["cs_sharded_device.cache"] == _abi.ShardedDevice.cache.offset


def test_abi_version_and_host_validation(cs_lib):
    assert cs_lib.cs_b200_abi_version() == 2
    v = _abi.BlockedEllView()
    v.rows, v.cols, v.block_size, v.ell_cols = 100, 64, 16, 64
    n = C.c_size_t()
    bad = _abi.GroupMomentsParams(0, 2, 1, 0)
    assert cs_lib.cs_b200_group_moments_scratch_bytes(C.byref(v), C.byref(bad), C.byref(n)) == 0
    assert b"group_count" in cs_lib.cs_b200_last_error()
    ok = _abi.GroupMomentsParams(8, 2, 1, 0)
    assert cs_lib.cs_b200_group_moments_scratch_bytes(C.byref(v), C.byref(ok), C.byref(n)) == 1
    assert n.value > 100 * 4
    v.ell_cols = 60  # not a multiple of the block size
    assert cs_lib.cs_b200_group_moments_scratch_bytes(C.byref(v), C.byref(ok), C.byref(n)) == 0
    # more than 32 feature groups is rejected before any device work (mask_groups.cu:729,819)
    v.ell_cols = 64
    f = _abi.GroupFilterParams(0.0, 0, 1.0, 0)
    out = _abi.GroupReduceOut(1, 1, 1, 1, 1, 1)
    m = _abi.RowFeatureMaskView()
    assert cs_lib.cs_b200_group_reduce_blocked_ell(C.byref(v), None, 33, C.byref(m), C.byref(f), C.byref(out),
                                                   None) == 0
    assert b"33" in cs_lib.cs_b200_last_error()
    assert cs_lib.cs_b200_blocked_ell_scratch_bytes(10, 10, 0, C.byref(n)) == 0
    assert cs_lib.cs_b200_blocked_ell_scratch_bytes(1000, 32768, 16, C.byref(n)) == 1
    assert n.value >= 63 * 64 * 4


def test_missing_library_fails_loudly(tmp_path):
    saved = _abi._lib
    try:
        _abi._lib = None
        with pytest.raises(_abi.CellShardError, match="no CPU fallback"):
            _abi.load(tmp_path / "absent.so")
    finally:
        _abi._lib = saved


def test_sharded_device_table_on_the_host(cs_lib):
    """The residency table of device::sharded_device grows on the host with no device
    work: records start empty (device -1), keep their contents when the table grows,
    and staging outside the table is refused with a message before any CUDA call."""
    st = _abi.ShardedDevice()
    assert cs_lib.cs_b200_sharded_device_reserve(C.byref(st), 3) == 1
    assert st.capacity == 3 and all(st.parts[i].device_id == -1 and not st.parts[i].view for i in range(3))
    st.parts[1].group_begin, st.parts[1].group_end = 7, 9
    assert cs_lib.cs_b200_sharded_device_reserve(C.byref(st), 2) == 1 and st.capacity == 3
    assert cs_lib.cs_b200_sharded_device_reserve(C.byref(st), 8) == 1 and st.capacity == 8
    assert (st.parts[1].group_begin, st.parts[1].group_end) == (7, 9) and st.parts[7].device_id == -1
    st.parts[1].group_begin = st.parts[1].group_end = 0
    h = _abi.HostBlockedEll()
    h.rows, h.cols, h.block_size, h.ell_cols = 16, 16, 16, 16
    assert cs_lib.cs_b200_stage_partition_blocked_ell(C.byref(st), 8, C.byref(h), 0, None) == 0
    assert b"outside" in cs_lib.cs_b200_last_error()
    arr = (C.POINTER(_abi.HostBlockedEll) * 2)(C.pointer(h), C.pointer(h))
    assert cs_lib.cs_b200_stage_shard_blocked_ell(C.byref(st), 7, 2, arr, 0, None) == 0
    # not resident: releasing is a no-op success
    assert cs_lib.cs_b200_release_staged_partition(C.byref(st), 2) == 1
    assert cs_lib.cs_b200_sharded_device_clear(C.byref(st)) == 1
    assert st.capacity == 0 and not st.parts and st.cache_count == 0


def test_staged_group_bytes(cs_lib):
    """A packed group: the views back to back in one 256-byte-rounded block, then each
    partition's arrays rounded to 256 bytes; one partition alone is the single-upload
    footprint."""
    import numpy as np

    def bell(rows, W, B=4):
        h = _abi.HostBlockedEll()
        h.rows, h.cols, h.block_size, h.ell_cols = rows, 64, B, W * B
        return h

    parts = [bell(37, 3), bell(64, 5), bell(21, 2)]
    arr = (C.POINTER(_abi.HostBlockedEll) * 3)(*[C.pointer(p) for p in parts])
    n = C.c_size_t()
    assert cs_lib.cs_b200_staged_bytes_blocked_ell(arr, 3, C.byref(n)) == 1
    r = lambda x: (x + 255) // 256 * 256
    want = r(3 * C.sizeof(_abi.BlockedEllView)) + sum(
        r(((p.rows + 3) // 4) * (p.ell_cols // 4) * 4) + r(p.rows * p.ell_cols * 2) for p in parts)
    assert n.value == want
    one = C.c_size_t()
    assert cs_lib.cs_b200_staged_bytes_blocked_ell(arr, 1, C.byref(n)) == 1
    assert cs_lib.cs_b200_device_partition_bytes_blocked_ell(C.byref(parts[0]), C.byref(one)) == 1
    assert n.value == one.value
    assert np.int64(n.value) > 0
