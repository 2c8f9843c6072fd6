"""ctypes mirror of include/cellshard_b200.h.

Structures follow the C layouts field for field (16-byte aligned structs get
explicit tail padding so ctypes.sizeof matches the C sizeof; the layout test
compiles the header with gcc and compares).
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

u32 = C.c_uint32
u64 = C.c_uint64
vp = C.c_void_p
sz = C.c_size_t

LIB_PATH = Path(__file__).resolve().parent / "libcellshard_b200.so"


class CompressedView(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("axis", u32),
                ("majorPtr", vp), ("minorIdx", vp), ("val", vp), ("_pad", C.c_uint64)]


class BlockedEllView(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("block_size", u32), ("ell_cols", u32),
                ("blockColIdx", vp), ("val", vp), ("_pad", C.c_uint64)]


class SlicedEllView(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("slice_count", u32), ("slice_rows", u32),
                ("slice_row_offsets", vp), ("slice_widths", vp), ("slice_slot_offsets", vp),
                ("col_idx", vp), ("val", vp)]


class HostCompressed(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("axis", u32), ("flags", u32),
                ("storage", vp), ("majorPtr", vp), ("minorIdx", vp), ("val", vp), ("_pad", C.c_uint64)]


class HostBlockedEll(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("block_size", u32), ("ell_cols", u32),
                ("flags", u32), ("storage", vp), ("blockColIdx", vp), ("val", vp)]


class HostSlicedEll(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("slice_count", u32), ("flags", u32),
                ("storage", vp), ("slice_row_offsets", vp), ("slice_widths", vp), ("col_idx", vp),
                ("val", vp)]


class HostCoo(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("storage", vp), ("rowIdx", vp), ("colIdx", vp),
                ("val", vp)]


class CooView(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("rowIdx", vp), ("colIdx", vp), ("val", vp),
                ("_pad", C.c_uint64)]


class CspackInfo(C.Structure):
    _fields_ = [("format", u32), ("rows", u32), ("cols", u32), ("nnz", u32), ("axis", u32), ("block_size", u32),
                ("ell_cols", u32), ("slice_count", u32), ("total_slots", u32)]


class HostBucketedBlockedEll(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("segment_count", u32), ("segments", vp),
                ("segment_row_offsets", vp), ("exec_to_canonical_rows", vp), ("canonical_to_exec_rows", vp),
                ("exec_to_canonical_cols", vp), ("canonical_to_exec_cols", vp)]


class HostBucketedSlicedEll(C.Structure):
    _fields_ = [("rows", u32), ("cols", u32), ("nnz", u32), ("segment_count", u32), ("segments", vp),
                ("segment_row_offsets", vp), ("exec_to_canonical_rows", vp), ("canonical_to_exec_rows", vp),
                ("canonical_slice_count", u32), ("canonical_slice_row_offsets", vp),
                ("canonical_slice_widths", vp)]


class ExecBucketPlan(C.Structure):
    _fields_ = [("segment_count", u32), ("bucket_count", u32), ("units", u32), ("block_size", u32),
                ("bytes", u64), ("original_bytes", u64), ("index_entries", u64), ("value_entries", u64)]


class ExecBucketSegments(C.Structure):
    _fields_ = [("max_segments", u32), ("unit_offsets", vp), ("row_offsets", vp), ("widths", vp)]


class BlockedEllTuneResult(C.Structure):
    _fields_ = [("block_size", C.c_uint), ("fill_ratio", C.c_double), ("padded_bytes", sz)]


class SlicedEllTuneResult(C.Structure):
    _fields_ = [("slice_rows", C.c_uint), ("slice_count", C.c_uint), ("padded_slots", sz),
                ("padded_bytes", sz), ("storage_ratio", C.c_double), ("slice_penalty", C.c_double),
                ("score", C.c_double)]


class RowFeatureMaskView(C.Structure):
    _fields_ = [("row_keep", vp), ("feature_keep", vp), ("row_remap", vp), ("feature_remap", vp)]


class GroupFilterParams(C.Structure):
    _fields_ = [("min_total", C.c_float), ("min_detected_features", u32),
                ("max_group_fraction", C.c_float), ("fraction_group_index", u32)]


class GroupReduceOut(C.Structure):
    _fields_ = [("row_totals", vp), ("detected_features", vp), ("max_values", vp), ("row_keep", vp),
                ("group_counts", vp), ("group_percentages", vp)]


class GroupMomentsParams(C.Structure):
    _fields_ = [("group_count", u32), ("scheme", u32), ("ddof", u32), ("chunk_rows", u32), ("index", vp),
                ("_align16", C.c_ubyte * 8)]


class GroupMomentsOut(C.Structure):
    _fields_ = [("sum", vp), ("sumsq", vp), ("mean", vp), ("var", vp), ("mean64", vp), ("var64", vp),
                ("group_rows", vp), ("status", vp)]


class BatchPart(C.Structure):
    _fields_ = [("src", CompressedView), ("bucket_count", u32), ("pad0", u32 * 3), ("d_major_nnz", vp),
                ("d_sorted_nnz", vp), ("d_order", vp), ("d_bucket_offsets", vp), ("d_pow2_offsets", vp),
                ("_pad", C.c_uint64)]


class BatchTiles(C.Structure):
    _fields_ = [("layout_rows", u32), ("emit_rows", u32), ("emit_lanes", u32), ("ctas_per_sm", u32)]


class BatchSlicedResult(C.Structure):
    _fields_ = [("status", u32), ("slice_rows", u32), ("slice_count", u32), ("plan_status", u32),
                ("total_slots", u64), ("arena_offset", u64), ("arena_bytes", u64), ("score", C.c_double),
                ("view", SlicedEllView)]


class PartitionRecord(C.Structure):
    _fields_ = [("allocation", vp), ("allocation_bytes", sz), ("view", vp), ("a0", vp), ("a1", vp), ("a2", vp),
                ("a3", vp), ("device_id", C.c_int), ("format", u32), ("host_view", C.c_ubyte * 64)]


class StagedPart(C.Structure):
    """device::partition_record (one record of a sharded_device residency table)."""
    _fields_ = [("allocation", vp), ("allocation_bytes", sz), ("storage", vp), ("view", vp), ("a0", vp), ("a1", vp),
                ("a2", vp), ("a3", vp), ("group_begin", C.c_ulong), ("group_end", C.c_ulong), ("device_id", C.c_int),
                ("_align16", C.c_ubyte * 12)]


class CachedAllocation(C.Structure):
    _fields_ = [("ptr", vp), ("bytes", sz), ("device_id", C.c_int)]


class ShardedDevice(C.Structure):
    _fields_ = [("capacity", C.c_ulong), ("parts", C.POINTER(StagedPart)), ("cache_count", C.c_ulong),
                ("cache_capacity", C.c_ulong), ("cache", C.POINTER(CachedAllocation))]


class ServeConfig(C.Structure):
    _fields_ = [("scratch_budget_bytes", u64), ("max_inflight", u32), ("chunk_rows", u32), ("idle_exit_us", u32),
                ("ctas_per_sm", u32)]


class ServeRequest(C.Structure):
    _fields_ = [("group_count", u32), ("scheme", u32), ("ddof", u32), ("flags", u32), ("row_keep", vp),
                ("row_labels", vp), ("feature_keep", vp), ("sum", vp), ("sumsq", vp), ("mean", vp), ("var", vp),
                ("group_rows", vp)]


class ServeStats(C.Structure):
    _fields_ = [("admitted", u64), ("completed", u64), ("pending", u64), ("kernel_launches", u64),
                ("scratch_in_use", u64), ("scratch_budget", u64), ("device_error", u32), ("pad", u32),
                ("items", u64 * 8), ("item_ns", u64 * 8)]


SERVE_DEVICE_INPUTS = 1
SERVE_DEVICE_OUTPUTS = 2
SERVE_QUEUED, SERVE_RUNNING, SERVE_DONE = 0, 1, 2

BATCH_DEFERRED = 1 << 8
BATCH_WAIT_TIMEOUT = 1 << 9
BATCH_TOO_LARGE = 1 << 10
BATCH_NO_CANDIDATE = 1 << 11
BATCH_EXCEEDS_ARENA = 1 << 12

P = C.POINTER

# name -> (restype, argtypes)
PROTOTYPES: dict[str, tuple] = {
    "cs_b200_abi_version": (C.c_int, []),
    "cs_b200_last_error": (C.c_char_p, []),
    "cs_b200_host_compressed_clear": (None, [P(HostCompressed)]),
    "cs_b200_host_blocked_ell_clear": (None, [P(HostBlockedEll)]),
    "cs_b200_host_sliced_ell_clear": (None, [P(HostSlicedEll)]),
    "cs_b200_blocked_ell_scratch_bytes": (C.c_int, [u32, u32, u32, P(sz)]),
    "cs_b200_blocked_ell_shape": (C.c_int, [P(CompressedView), u32, vp, vp, sz, vp, vp]),
    "cs_b200_blocked_ell_emit": (C.c_int, [P(CompressedView), P(BlockedEllView), vp, vp, sz, vp, vp]),
    "cs_b200_blocked_ell_from_compressed": (C.c_int, [P(HostCompressed), C.c_uint, P(HostBlockedEll)]),
    "cs_b200_choose_blocked_ell_block_size": (C.c_int, [P(HostCompressed), P(C.c_uint), C.c_uint,
                                                         P(BlockedEllTuneResult)]),
    "cs_b200_sliced_ell_scratch_bytes": (C.c_int, [u32, u32, P(sz)]),
    "cs_b200_sliced_ell_layout": (C.c_int, [P(CompressedView), u32, vp, vp, vp, vp, vp, sz, vp]),
    "cs_b200_sliced_ell_emit": (C.c_int, [P(CompressedView), P(SlicedEllView), vp]),
    "cs_b200_sliced_ell_candidates": (C.c_int, [P(CompressedView), vp, u32, vp, vp]),
    "cs_b200_sliced_ell_from_compressed": (C.c_int, [P(HostCompressed), C.c_uint, P(HostSlicedEll)]),
    "cs_b200_choose_sliced_ell_slice_rows_from_compressed": (C.c_int, [P(HostCompressed), P(C.c_uint), C.c_uint,
                                                                        P(SlicedEllTuneResult)]),
    "cs_b200_blocked_ell_row_ptr_scratch_bytes": (C.c_int, [u32, P(sz)]),
    "cs_b200_blocked_ell_row_ptr": (C.c_int, [P(BlockedEllView), vp, vp, sz, vp]),
    "cs_b200_sliced_ell_emit_from_blocked_ell": (C.c_int, [P(BlockedEllView), P(SlicedEllView), vp]),
    "cs_b200_sliced_ell_from_blocked_ell": (C.c_int, [P(HostBlockedEll), C.c_uint, P(HostSlicedEll)]),
    "cs_b200_choose_sliced_ell_slice_rows_from_blocked_ell": (C.c_int, [P(HostBlockedEll), P(C.c_uint), C.c_uint,
                                                                         P(SlicedEllTuneResult)]),
    "cs_b200_filter_blocked_ell_scratch_bytes": (C.c_int, [u32, u32, P(sz)]),
    "cs_b200_filter_blocked_ell_count": (C.c_int, [P(BlockedEllView), u32, P(RowFeatureMaskView), u32, u32, vp, vp,
                                                    vp, sz, vp, vp]),
    "cs_b200_filter_blocked_ell_onepass_scratch_bytes": (C.c_int, [P(BlockedEllView), u32, P(sz)]),
    "cs_b200_filter_blocked_ell_onepass": (C.c_int, [P(BlockedEllView), u32, P(RowFeatureMaskView), u32, u32, vp, vp,
                                                     vp, u64, vp, vp, sz, vp, vp]),
    "cs_b200_filter_blocked_ell_marked_scratch_bytes": (C.c_int, [P(BlockedEllView), u32, P(sz)]),
    "cs_b200_filter_blocked_ell_marked": (C.c_int, [P(BlockedEllView), u32, P(RowFeatureMaskView), u32, u32, vp, vp,
                                                    vp, u64, vp, vp, sz, vp, vp]),
    "cs_b200_filter_blocked_ell_emit": (C.c_int, [P(BlockedEllView), u32, P(RowFeatureMaskView), u32, u32, vp, vp,
                                                   vp, vp]),
    "cs_b200_cspack_peek": (C.c_int, [C.c_char_p, P(CspackInfo)]),
    "cs_b200_cspack_store_blocked_ell": (C.c_int, [C.c_char_p, P(BlockedEllView)]),
    "cs_b200_cspack_load_blocked_ell": (C.c_int, [C.c_char_p, P(BlockedEllView)]),
    "cs_b200_cspack_store_sliced_ell": (C.c_int, [C.c_char_p, P(SlicedEllView)]),
    "cs_b200_cspack_load_sliced_ell": (C.c_int, [C.c_char_p, P(SlicedEllView)]),
    "cs_b200_cspack_store_compressed": (C.c_int, [C.c_char_p, P(CompressedView)]),
    "cs_b200_cspack_load_compressed": (C.c_int, [C.c_char_p, P(CompressedView)]),
    "cs_b200_cspack_store_coo": (C.c_int, [C.c_char_p, P(CooView)]),
    "cs_b200_cspack_load_coo": (C.c_int, [C.c_char_p, P(CooView)]),
    "cs_b200_coo_blocked_ell_scratch_bytes": (C.c_int, [u32, u32, u32, u32, P(sz)]),
    "cs_b200_coo_blocked_ell_plan": (C.c_int, [P(CooView), vp, u32, u32, vp, sz, P(u32), P(u64), vp, vp]),
    "cs_b200_coo_blocked_ell_emit": (C.c_int, [P(CooView), vp, u32, vp, sz, P(BlockedEllView), vp, vp]),
    "cs_b200_blocked_ell_from_coo": (C.c_int, [P(HostCoo), u32, vp, C.c_uint, P(HostBlockedEll)]),
    "cs_b200_blocked_ell_from_coo_cuda": (C.c_int, [P(HostCoo), u32, vp, C.c_uint, P(HostBlockedEll), C.c_int]),
    "cs_b200_choose_blocked_ell_block_size_from_coo": (C.c_int, [P(HostCoo), u32, vp, P(C.c_uint), C.c_uint,
                                                                  P(BlockedEllTuneResult)]),
    "cs_b200_bucketed_blocked_ell_scratch_bytes": (C.c_int, [u32, u32, u32, P(sz)]),
    "cs_b200_bucketed_blocked_ell_plan": (C.c_int, [P(BlockedEllView), u32, vp, sz, P(ExecBucketPlan),
                                                     P(ExecBucketSegments), vp]),
    "cs_b200_bucketed_blocked_ell_fill": (C.c_int, [P(BlockedEllView), vp, P(ExecBucketPlan), vp, vp, vp, vp, vp,
                                                     vp, vp]),
    "cs_b200_bucketed_sliced_ell_scratch_bytes": (C.c_int, [u32, u32, P(sz)]),
    "cs_b200_bucketed_sliced_ell_plan": (C.c_int, [P(SlicedEllView), u32, vp, sz, P(ExecBucketPlan),
                                                    P(ExecBucketSegments), vp]),
    "cs_b200_bucketed_sliced_ell_fill": (C.c_int, [P(SlicedEllView), vp, P(ExecBucketPlan), vp, vp, vp, vp, vp]),
    "cs_b200_build_bucketed_blocked_ell_partition": (C.c_int, [P(HostBucketedBlockedEll), P(HostBlockedEll), u32,
                                                                P(u64)]),
    "cs_b200_choose_bucket_count_for_part": (C.c_int, [P(HostBlockedEll), P(u32), P(u64)]),
    "cs_b200_host_bucketed_blocked_ell_clear": (None, [P(HostBucketedBlockedEll)]),
    "cs_b200_build_bucketed_sliced_ell_partition": (C.c_int, [P(HostBucketedSlicedEll), P(HostSlicedEll), u32,
                                                               P(u64)]),
    "cs_b200_choose_bucket_count_for_sliced_part": (C.c_int, [P(HostSlicedEll), P(u32), P(u64)]),
    "cs_b200_host_bucketed_sliced_ell_clear": (None, [P(HostBucketedSlicedEll)]),
    "cs_b200_blocked_ell_bucket_plan_scratch_bytes": (C.c_int, [u32, u32, P(sz)]),
    "cs_b200_blocked_ell_bucket_plan": (C.c_int, [P(BlockedEllView), vp, vp, vp, sz, vp]),
    "cs_b200_choose_bucket_count_from_plan": (C.c_int, [P(BlockedEllView), vp, vp, vp, vp, vp]),
    "cs_b200_choose_ingest_bucket_count_for_part": (C.c_int, [P(HostBlockedEll), C.c_int, P(u32)]),
    "cs_b200_compressed_transpose_scratch_bytes": (C.c_int, [u32, u32, u32, P(sz)]),
    "cs_b200_build_compressed_transpose": (C.c_int, [u32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "cs_b200_major_nnz_bucket_sort_scratch_bytes": (C.c_int, [u32, P(sz)]),
    "cs_b200_major_nnz_bucket_scan_scratch_bytes": (C.c_int, [u32, P(sz)]),
    "cs_b200_build_major_nnz_bucket_plan": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, u32, vp, sz, vp]),
    "cs_b200_build_shard_major_nnz_bucket_plan": (C.c_int, [vp, vp, u32, u32, vp, vp, vp, vp, vp, u32, vp, sz, vp]),
    "cs_b200_pow2_nnz_bin_offsets": (C.c_int, [vp, u32, vp, vp]),
    "cs_b200_rebuild_compressed_major_order": (C.c_int, [vp, vp, vp, u32, vp, vp, vp, vp, vp, vp, sz, vp]),
    "cs_b200_rebuild_bucketed_shard_compressed": (C.c_int, [vp, vp, vp, vp, u32, u32, vp, vp, vp, vp, vp, vp, sz,
                                                             vp]),
    "cs_b200_group_reduce_blocked_ell": (C.c_int, [P(BlockedEllView), vp, u32, P(RowFeatureMaskView),
                                                   P(GroupFilterParams), P(GroupReduceOut), vp]),
    "cs_b200_group_reduce_sliced_ell": (C.c_int, [P(SlicedEllView), vp, u32, P(RowFeatureMaskView),
                                                  P(GroupFilterParams), P(GroupReduceOut), vp]),
    "cs_b200_group_reduce_compressed": (C.c_int, [P(CompressedView), vp, u32, P(RowFeatureMaskView),
                                                  P(GroupFilterParams), P(GroupReduceOut), vp]),
    "cs_b200_reoptimize_scratch_bytes": (C.c_int, [u32, u32, P(sz)]),
    "cs_b200_reoptimize_count": (C.c_int, [P(BlockedEllView), P(RowFeatureMaskView), u32, u32, vp, vp, sz, vp,
                                           vp]),
    "cs_b200_reoptimize_emit": (C.c_int, [P(BlockedEllView), P(RowFeatureMaskView), u32, u32, vp, vp, vp, vp]),
    "cs_b200_group_moments_scratch_bytes": (C.c_int, [P(BlockedEllView), P(GroupMomentsParams), P(sz)]),
    "cs_b200_group_moments_index_bytes": (C.c_int, [P(BlockedEllView), P(sz)]),
    "cs_b200_group_moments_parts_scratch_bytes": (C.c_int, [P(BlockedEllView), u32, P(GroupMomentsParams), P(sz)]),
    "cs_b200_group_moments_blocked_ell_parts": (C.c_int, [P(BlockedEllView), u32, P(vp), vp, vp, vp,
                                                          P(GroupMomentsParams), P(GroupMomentsOut), vp, sz, vp]),
    "cs_b200_group_moments_build_index": (C.c_int, [P(BlockedEllView), vp, vp, vp]),
    "cs_b200_group_moments_blocked_ell": (C.c_int, [P(BlockedEllView), vp, vp, vp, P(GroupMomentsParams),
                                                    P(GroupMomentsOut), vp, sz, vp]),
    "cs_b200_group_moments_blocked_ell_noalloc": (C.c_int, [P(BlockedEllView), vp, vp, vp, P(GroupMomentsParams),
                                                            P(GroupMomentsOut), vp]),
    "cs_b200_group_moments_phases": (C.c_int, [P(BlockedEllView), vp, vp, vp, P(GroupMomentsParams),
                                               P(GroupMomentsOut), vp, sz, u32, vp]),
    "cs_b200_group_moments_to_host": (C.c_int, [P(BlockedEllView), vp, vp, vp, P(GroupMomentsParams),
                                                P(GroupMomentsOut), P(GroupMomentsOut), vp, sz, u32, vp]),
    "cs_b200_synth_csr": (C.c_int, [u32, u32, vp, vp, vp, vp, u32, vp, u64, vp, vp, vp]),
    "cs_b200_batch_sliced_create": (C.c_int, [P(BatchPart), u32, P(u32), u32, vp, u64, P(BatchTiles), P(vp)]),
    "cs_b200_batch_sliced_autotune": (C.c_int, [vp, vp, P(BatchTiles)]),
    "cs_b200_batch_sliced_run": (C.c_int, [vp, vp]),
    "cs_b200_batch_sliced_results": (C.c_int, [vp, P(BatchSlicedResult), P(u32), P(u32), vp]),
    "cs_b200_batch_sliced_next_wave": (C.c_int, [vp, vp, u64, P(u32)]),
    "cs_b200_batch_sliced_reset": (C.c_int, [vp, vp, u64]),
    "cs_b200_batch_sliced_tiles": (C.c_int, [vp, P(BatchTiles), P(u32), P(u32)]),
    "cs_b200_batch_sliced_destroy": (None, [vp]),
    "cs_b200_device_partition_bytes_compressed": (C.c_int, [P(HostCompressed), P(sz)]),
    "cs_b200_device_partition_bytes_blocked_ell": (C.c_int, [P(HostBlockedEll), P(sz)]),
    "cs_b200_device_partition_bytes_sliced_ell": (C.c_int, [P(HostSlicedEll), P(sz)]),
    "cs_b200_upload_compressed": (C.c_int, [P(HostCompressed), P(PartitionRecord), vp]),
    "cs_b200_upload_blocked_ell": (C.c_int, [P(HostBlockedEll), P(PartitionRecord), vp]),
    "cs_b200_upload_sliced_ell": (C.c_int, [P(HostSlicedEll), P(PartitionRecord), vp]),
    "cs_b200_release_partition": (C.c_int, [P(PartitionRecord)]),
    "cs_b200_sharded_device_reserve": (C.c_int, [P(ShardedDevice), C.c_ulong]),
    "cs_b200_sharded_device_clear": (C.c_int, [P(ShardedDevice)]),
    "cs_b200_stage_partition_compressed": (C.c_int, [P(ShardedDevice), C.c_ulong, P(HostCompressed), C.c_int, vp]),
    "cs_b200_stage_partition_blocked_ell": (C.c_int, [P(ShardedDevice), C.c_ulong, P(HostBlockedEll), C.c_int, vp]),
    "cs_b200_stage_partition_sliced_ell": (C.c_int, [P(ShardedDevice), C.c_ulong, P(HostSlicedEll), C.c_int, vp]),
    "cs_b200_stage_shard_compressed": (C.c_int, [P(ShardedDevice), C.c_ulong, C.c_ulong, P(P(HostCompressed)),
                                                 C.c_int, vp]),
    "cs_b200_stage_shard_blocked_ell": (C.c_int, [P(ShardedDevice), C.c_ulong, C.c_ulong, P(P(HostBlockedEll)),
                                                  C.c_int, vp]),
    "cs_b200_stage_shard_sliced_ell": (C.c_int, [P(ShardedDevice), C.c_ulong, C.c_ulong, P(P(HostSlicedEll)),
                                                 C.c_int, vp]),
    "cs_b200_release_staged_partition": (C.c_int, [P(ShardedDevice), C.c_ulong]),
    "cs_b200_staged_bytes_compressed": (C.c_int, [P(P(HostCompressed)), C.c_ulong, P(sz)]),
    "cs_b200_staged_bytes_blocked_ell": (C.c_int, [P(P(HostBlockedEll)), C.c_ulong, P(sz)]),
    "cs_b200_staged_bytes_sliced_ell": (C.c_int, [P(P(HostSlicedEll)), C.c_ulong, P(sz)]),
    "cs_b200_serve_open": (C.c_int, [P(BlockedEllView), u32, P(ServeConfig), P(vp)]),
    "cs_b200_serve_submit": (C.c_int, [vp, P(ServeRequest), P(u64)]),
    "cs_b200_serve_poll": (C.c_int, [vp, u64, P(u32), P(C.c_double)]),
    "cs_b200_serve_wait": (C.c_int, [vp, u64, u32, P(C.c_double)]),
    "cs_b200_serve_release": (C.c_int, [vp, u64]),
    "cs_b200_serve_stats": (C.c_int, [vp, P(ServeStats)]),
    "cs_b200_serve_run_trace": (C.c_int, [vp, P(ServeRequest), P(u32), P(C.c_double), u32, P(C.c_double),
                                          P(C.c_double), P(C.c_double)]),
    "cs_b200_serve_close": (None, [vp]),
}


class CellShardError(RuntimeError):
    pass


_lib = None


def load(path: os.PathLike | None = None) -> C.CDLL:
    """Loads libcellshard_b200.so; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise CellShardError(
            f"{p} is missing: build it with `python -m cellshard_b200.build` (nvcc, sm_100a); "
            "there is no CPU fallback")
    lib = C.CDLL(str(p))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(ok: int, what: str) -> None:
    if ok != 1:
        msg = load().cs_b200_last_error()
        raise CellShardError(f"{what} failed: {msg.decode() if msg else 'unknown error'}")
