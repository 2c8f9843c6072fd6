/*
 * cellshard_b200.h -- C ABI of the B200-native CellShard sparse hot path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * launches hand-written sm_100a kernels from libcellshard_b200.so.  Device
 * pointers (prefix d_) must point to memory on the current CUDA device; host
 * pointers are plain malloc'd or pinned memory.
 *
 * Conventions kept from the reference (tumlinso/CellShard 0.1.0):
 *   - int return codes: 1 = success, 0 = failure (src/runtime/mask_groups.cu,
 *     src/convert/*, src/bucket/*).  On failure cs_b200_last_error() holds a
 *     one-line message for the calling host thread.
 *   - raw launchers are stream-ordered and never synchronise; host-struct
 *     convenience wrappers synchronise and return host-owned results.
 *   - u32 local indices, fp16 values (passed here as uint16_t IEEE bits).
 *
 * Device-side input validation (bad block-column order, duplicate columns,
 * out-of-range indices) cannot be reported by a return code without a sync,
 * so launchers that validate take a nullable `uint32_t *d_status` word into
 * which kernels OR CS_STATUS_* bits.  The caller clears it before the call
 * and reads it after its own synchronisation point.
 */
#ifndef CELLSHARD_B200_H_
#define CELLSHARD_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_B200_ABI_VERSION 2
#define CS_ALIGN16 __attribute__((aligned(16)))
#define CS_API __attribute__((visibility("default")))

typedef struct CUstream_st *cs_stream_t; /* == cudaStream_t */

enum {
    CS_COMPRESSED_BY_ROW = 0, /* sparse::compressed_by_row (formats/compressed.cuh:11-14) */
    CS_COMPRESSED_BY_COL = 1
};

#define CS_INVALID_COL 0xffffffffu   /* blocked_ell_invalid_col / sliced_ell_invalid_col */
#define CS_MAX_MASK_GROUPS 32u       /* runtime::CELLSHARD_MAX_MASK_GROUPS (mask_groups.cuh:14) */
#define CS_MAX_MOMENT_GROUPS 4096u   /* row-label groups of the moments reduction */

/* Device status bits (OR'd by kernels into *d_status). */
enum {
    CS_STATUS_OK = 0u,
    CS_STATUS_BLOCK_COL_ORDER = 1u << 0,    /* blockColIdx row not ascending / padding not trailing */
    CS_STATUS_DUPLICATE_COL = 1u << 1,      /* a row repeats a column index */
    CS_STATUS_INDEX_RANGE = 1u << 2,        /* an index is >= its dimension */
    CS_STATUS_REMAP_COLLISION = 1u << 3,    /* two kept rows remap to one output row */
    CS_STATUS_BAD_POINTERS = 1u << 4,       /* a CSR row pointer decreases or exceeds nnz */
    CS_STATUS_CAPACITY = 1u << 5,           /* the caller's output arrays are too small (nothing written past them) */
    CS_STATUS_WAIT_LIMIT = 1u << 6          /* a device-side wait gave up: the result is incomplete */
};

/* ------------------------------------------------------------------------ */
/* Device views: field for field the reference's POD views                   */
/* include/CellShard/runtime/device/sharded_device.cuh:67-98                 */
/* ------------------------------------------------------------------------ */

typedef struct CS_ALIGN16 cs_compressed_view {
    uint32_t rows, cols, nnz, axis;
    uint32_t *majorPtr;
    uint32_t *minorIdx;
    uint16_t *val;
} cs_compressed_view;

typedef struct CS_ALIGN16 cs_blocked_ell_view {
    uint32_t rows, cols, nnz, block_size, ell_cols;
    uint32_t *blockColIdx;
    uint16_t *val;
} cs_blocked_ell_view;

typedef struct CS_ALIGN16 cs_sliced_ell_view {
    uint32_t rows, cols, nnz, slice_count, slice_rows;
    uint32_t *slice_row_offsets;
    uint32_t *slice_widths;
    uint32_t *slice_slot_offsets;
    uint32_t *col_idx;
    uint16_t *val;
} cs_sliced_ell_view;

/* Host-owned formats: field for field sparse::compressed, sparse::blocked_ell
 * and sparse::sliced_ell (formats/compressed.cuh:24-37, blocked_ell.cuh:15-25,
 * sliced_ell.cuh:16-28).  Results written by this library own one malloc'd
 * packed block in `storage` laid out as the reference's sparse::allocate()
 * lays it out, so the reference's sparse::clear() frees them. */
typedef struct CS_ALIGN16 cs_host_compressed {
    uint32_t rows, cols, nnz, axis, flags;
    void *storage;
    uint32_t *majorPtr;
    uint32_t *minorIdx;
    uint16_t *val;
} cs_host_compressed;

typedef struct CS_ALIGN16 cs_host_blocked_ell {
    uint32_t rows, cols, nnz, block_size, ell_cols, flags;
    void *storage;
    uint32_t *blockColIdx;
    uint16_t *val;
} cs_host_blocked_ell;

typedef struct CS_ALIGN16 cs_host_sliced_ell {
    uint32_t rows, cols, nnz, slice_count, flags;
    void *storage;
    uint32_t *slice_row_offsets;
    uint32_t *slice_widths;
    uint32_t *col_idx;
    uint16_t *val;
} cs_host_sliced_ell;

/* convert::blocked_ell_tune_result (blocked_ell_from_compressed.cuh:16-20) */
typedef struct cs_blocked_ell_tune_result {
    unsigned int block_size;
    double fill_ratio;
    size_t padded_bytes;
} cs_blocked_ell_tune_result;

/* convert::sliced_ell_tune_result (sliced_ell_from_blocked_ell.cuh:18-26) */
typedef struct cs_sliced_ell_tune_result {
    unsigned int slice_rows;
    unsigned int slice_count;
    size_t padded_slots;
    size_t padded_bytes;
    double storage_ratio;
    double slice_penalty;
    double score;
} cs_sliced_ell_tune_result;

/* Releases a host result written by this library (sparse::clear semantics:
 * frees `storage` and zeroes the struct). */
CS_API void cs_b200_host_compressed_clear(cs_host_compressed *m);
CS_API void cs_b200_host_blocked_ell_clear(cs_host_blocked_ell *m);
CS_API void cs_b200_host_sliced_ell_clear(cs_host_sliced_ell *m);

/* runtime::row_feature_mask_view (mask_groups.cuh:29-34) */
typedef struct CS_ALIGN16 cs_row_feature_mask_view {
    const uint8_t *row_keep;
    const uint8_t *feature_keep;
    const uint32_t *row_remap;
    const uint32_t *feature_remap;
} cs_row_feature_mask_view;

/* ------------------------------------------------------------------------ */
/* Library                                                                   */
/* ------------------------------------------------------------------------ */

/* Returns CS_B200_ABI_VERSION.  No reference counterpart. */
CS_API int cs_b200_abi_version(void);

/* Last error message of the calling host thread ("" if none).  Replaces the
 * reference's fprintf(stderr) helpers (mask_groups.cu:44-48). */
CS_API const char *cs_b200_last_error(void);

/* ------------------------------------------------------------------------ */
/* CSR -> Blocked-ELL                                                         */
/* replaces convert::blocked_ell_from_compressed and                          */
/* convert::choose_blocked_ell_block_size (src/convert/                        */
/* blocked_ell_from_compressed.cuh:33-91,157-190,258-347), which the           */
/* reference runs as serial host loops.                                       */
/* ------------------------------------------------------------------------ */

/* Scratch of cs_b200_blocked_ell_shape when it keeps the per-row-block
 * column-block bitmaps for cs_b200_blocked_ell_emit. */
CS_API int cs_b200_blocked_ell_scratch_bytes(uint32_t rows, uint32_t cols, uint32_t block_size, size_t *out_bytes);

/* Shape pass (detail::count_blocked_ell_shape_): d_shape[0] <- ell_width
 * (max distinct column blocks over row blocks), d_shape[1] <- total distinct
 * (row block, column block) pairs.  d_shape must be zeroed by the caller.
 * d_scratch may be NULL (shape only, as the chooser needs). */
CS_API int cs_b200_blocked_ell_shape(const cs_compressed_view *src,
                              uint32_t block_size,
                              uint64_t *d_shape,
                              void *d_scratch,
                              size_t scratch_bytes,
                              uint32_t *d_status,
                              cs_stream_t stream);

/* Emit pass: dst->blockColIdx [row_blocks x ell_width] ascending with
 * CS_INVALID_COL padding, dst->val [rows x ell_cols] with the value of column
 * c of row r at r*ell_cols + slot*block_size + c%block_size and zeros
 * elsewhere; *d_nnz += number of written values that are nonzero as fp32
 * (the reference's dst->nnz).  d_scratch must hold the bitmaps of a
 * preceding cs_b200_blocked_ell_shape with the same src and block_size.
 * Repeated columns in a row resolve to the last one, as in the reference. */
CS_API int cs_b200_blocked_ell_emit(const cs_compressed_view *src,
                             const cs_blocked_ell_view *dst,
                             uint32_t *d_nnz,
                             const void *d_scratch,
                             size_t scratch_bytes,
                             uint32_t *d_status,
                             cs_stream_t stream);

/* Host convenience with the reference's signature and results:
 * convert::blocked_ell_from_compressed(src, block_size, dst).  Synchronous. */
CS_API int cs_b200_blocked_ell_from_compressed(const cs_host_compressed *src,
                                        unsigned int block_size,
                                        cs_host_blocked_ell *dst);

/* convert::choose_blocked_ell_block_size: same candidates loop, same
 * tie-breaking in double, shapes computed on the GPU.  Synchronous. */
CS_API int cs_b200_choose_blocked_ell_block_size(const cs_host_compressed *src,
                                          const unsigned int *candidates,
                                          unsigned int candidate_count,
                                          cs_blocked_ell_tune_result *out);

/* ------------------------------------------------------------------------ */
/* COO -> Blocked-ELL                                                         */
/* replaces convert::blocked_ell_from_coo[_auto] and                          */
/* choose_blocked_ell_block_size_from_coo (src/convert/                        */
/* blocked_ell_from_compressed.cuh:105-257,349-478, host loops) and their GPU  */
/* twins blocked_ell_from_coo_cuda[_auto] /                                   */
/* choose_blocked_ell_block_size_from_coo_cuda (src/convert/                   */
/* blocked_ell_from_coo_cuda.cuh:17-966).  Columns pass through the optional   */
/* feature_to_global map first.  Each row block's distinct block columns are  */
/* its slots, ascending; the width is the largest count.  Values land in COO  */
/* order, so a repeated (row, column) keeps its last value (the host          */
/* routine's rule; the reference's GPU scatter leaves the winner to the        */
/* hardware).  Entries whose row is out of range are dropped and flagged      */
/* CS_STATUS_INDEX_RANGE.                                                     */
/* ------------------------------------------------------------------------ */

/* sparse::coo (formats/triplet.cuh:14-25) and device::coo_view
 * (runtime/device/sharded_device.cuh:100-107) */
typedef struct CS_ALIGN16 cs_host_coo {
    uint32_t rows, cols, nnz;
    void *storage;
    uint32_t *rowIdx;
    uint32_t *colIdx;
    uint16_t *val;
} cs_host_coo;

typedef struct CS_ALIGN16 cs_coo_view {
    uint32_t rows, cols, nnz;
    uint32_t *rowIdx;
    uint32_t *colIdx;
    uint16_t *val;
} cs_coo_view;

/* Shape of one block size: width and the count of (row block, block column)
 * pairs; the plan stays in the scratch for the emit of the same block size.
 * Entries whose rows never decrease, with every mapped column below cols,
 * take the CSR route (row pointers from the row runs, then the CSR ->
 * Blocked-ELL shape and emit); others are sorted by (row block, block
 * column).  Synchronises (two small reads of sizes). */
CS_API int cs_b200_coo_blocked_ell_scratch_bytes(uint32_t nnz, uint32_t rows, uint32_t cols, uint32_t block_size,
                                                 size_t *out_bytes);
CS_API int cs_b200_coo_blocked_ell_plan(const cs_coo_view *src,
                                        const uint32_t *d_feature_to_global,
                                        uint32_t cols,
                                        uint32_t block_size,
                                        void *d_scratch,
                                        size_t scratch_bytes,
                                        uint32_t *ell_width_out,
                                        uint64_t *total_blocks_out,
                                        uint32_t *d_status,
                                        cs_stream_t stream);
/* dst: rows = src->rows, block_size, ell_cols = width * block_size, arrays
 * allocated by the caller.  d_nnz (u64[2], zeroed by the caller) <- the
 * stored values nonzero as floats, and those of them with column < cols
 * (the host routine's and the GPU routine's nnz respectively). */
CS_API int cs_b200_coo_blocked_ell_emit(const cs_coo_view *src,
                                        const uint32_t *d_feature_to_global,
                                        uint32_t cols,
                                        const void *d_scratch,
                                        size_t scratch_bytes,
                                        const cs_blocked_ell_view *dst,
                                        uint64_t *d_nnz,
                                        cs_stream_t stream);

/* Host signatures (host COO in, host Blocked-ELL out; synchronous).
 * feature_to_global is a host array of src->cols entries or NULL. */
CS_API int cs_b200_blocked_ell_from_coo(const cs_host_coo *src, uint32_t cols, const uint32_t *feature_to_global,
                                        unsigned int block_size, cs_host_blocked_ell *dst);
CS_API int cs_b200_blocked_ell_from_coo_cuda(const cs_host_coo *src, uint32_t cols,
                                             const uint32_t *feature_to_global, unsigned int block_size,
                                             cs_host_blocked_ell *dst, int device);
CS_API int cs_b200_choose_blocked_ell_block_size_from_coo(const cs_host_coo *src, uint32_t cols,
                                                          const uint32_t *feature_to_global,
                                                          const unsigned int *candidates,
                                                          unsigned int candidate_count,
                                                          cs_blocked_ell_tune_result *out);

/* ------------------------------------------------------------------------ */
/* CSR -> Sliced-ELL                                                          */
/* replaces convert::sliced_ell_from_compressed[_cuda] and                    */
/* choose_sliced_ell_slice_rows[_from_compressed] (src/convert/                */
/* sliced_ell_from_compressed.cuh:20-45,86-254; sliced_ell_from_blocked_ell.cuh:*/
/* 64-142,196-221), whose layout the reference computes on the host.          */
/* ------------------------------------------------------------------------ */

CS_API int cs_b200_sliced_ell_scratch_bytes(uint32_t rows, uint32_t slice_rows, size_t *out_bytes);

/* Layout pass for uniform slices of clamp(slice_rows, 1, rows) rows:
 * d_slice_row_offsets[S+1], d_slice_widths[S] (max row nnz of the slice),
 * d_slice_slot_offsets[S] (u32 running sum of rows_in_slice * width), and
 * d_total_slots[0] (u64, exact).  S = ceil(rows / clamp(slice_rows)). */
CS_API int cs_b200_sliced_ell_layout(const cs_compressed_view *src,
                                     uint32_t slice_rows,
                                     uint32_t *d_slice_row_offsets,
                                     uint32_t *d_slice_widths,
                                     uint32_t *d_slice_slot_offsets,
                                     uint64_t *d_total_slots,
                                     void *d_scratch,
                                     size_t scratch_bytes,
                                     cs_stream_t stream);

/* Emit pass: each row's entries in its first slots, CS_INVALID_COL / 0
 * padding after them.  dst carries the layout and uniform slice_rows. */
CS_API int cs_b200_sliced_ell_emit(const cs_compressed_view *src, const cs_sliced_ell_view *dst, cs_stream_t stream);

/* d_padded_slots[k] <- sum over slices of rows_in_slice * max row nnz for
 * candidate height candidates[k] (clamped to [1, rows]); at most 16. */
CS_API int cs_b200_sliced_ell_candidates(const cs_compressed_view *src,
                                         const uint32_t *candidates,
                                         uint32_t count,
                                         uint64_t *d_padded_slots,
                                         cs_stream_t stream);

/* Host convenience with the reference's signature and results:
 * convert::sliced_ell_from_compressed(src, slice_rows, dst), CSR or CSC
 * input.  Synchronous. */
CS_API int cs_b200_sliced_ell_from_compressed(const cs_host_compressed *src,
                                              unsigned int slice_rows,
                                              cs_host_sliced_ell *dst);

/* convert::choose_sliced_ell_slice_rows_from_compressed: same score,
 * penalty and tie-breaking in host doubles, padded slots from the GPU. */
CS_API int cs_b200_choose_sliced_ell_slice_rows_from_compressed(const cs_host_compressed *src,
                                                                const unsigned int *candidates,
                                                                unsigned int candidate_count,
                                                                cs_sliced_ell_tune_result *out);

/* ------------------------------------------------------------------------ */
/* Blocked-ELL -> Sliced-ELL                                                  */
/* replaces convert::sliced_ell_from_blocked_ell[_cuda],                      */
/* choose_sliced_ell_slice_rows_from_blocked_ell and the host row count       */
/* count_blocked_ell_row_nnz_ (src/convert/sliced_ell_from_blocked_ell.cuh:    */
/* 36-62,146-190,223-364).  A row's entries are its live values in slot then  */
/* lane order: valid block column, column < cols, value != 0 as a float.      */
/* ------------------------------------------------------------------------ */

CS_API int cs_b200_blocked_ell_row_ptr_scratch_bytes(uint32_t rows, size_t *out_bytes);

/* d_row_ptr[rows + 1] <- exclusive prefix of the rows' live-entry counts
 * (count_blocked_ell_row_nnz_, :36-62).  A cs_compressed_view with these
 * row pointers (minorIdx / val unused) is a valid input of
 * cs_b200_sliced_ell_layout and cs_b200_sliced_ell_candidates, which then
 * give the reference's uniform layout (build_uniform_sliced_layout_,
 * :111-142) and candidate padding for this Blocked-ELL. */
CS_API int cs_b200_blocked_ell_row_ptr(const cs_blocked_ell_view *src,
                                       uint32_t *d_row_ptr,
                                       void *d_scratch,
                                       size_t scratch_bytes,
                                       cs_stream_t stream);

/* Emit (emit_sliced_ell_from_blocked_ell_kernel, :146-190): each row's live
 * entries in its first slots, CS_INVALID_COL / 0 padding after them.  dst
 * carries the layout and the uniform slice_rows. */
CS_API int cs_b200_sliced_ell_emit_from_blocked_ell(const cs_blocked_ell_view *src,
                                                    const cs_sliced_ell_view *dst,
                                                    cs_stream_t stream);

/* Host convenience with the reference's signature and results:
 * convert::sliced_ell_from_blocked_ell(src, slice_rows, dst) (:233-276; the
 * result carries src->nnz, as the reference's does).  Synchronous. */
CS_API int cs_b200_sliced_ell_from_blocked_ell(const cs_host_blocked_ell *src,
                                               unsigned int slice_rows,
                                               cs_host_sliced_ell *dst);

/* convert::choose_sliced_ell_slice_rows_from_blocked_ell (:223-231): the
 * chooser's score over the live-entry counts, storage ratio over src->nnz. */
CS_API int cs_b200_choose_sliced_ell_slice_rows_from_blocked_ell(const cs_host_blocked_ell *src,
                                                                 const unsigned int *candidates,
                                                                 unsigned int candidate_count,
                                                                 cs_sliced_ell_tune_result *out);

/* ------------------------------------------------------------------------ */
/* Compressed transpose                                                       */
/* replaces convert::build_compressed_transpose_raw (src/convert/             */
/* compressed_transpose_raw.cuh:14-123), same arguments.  The output equals   */
/* the reference's cuSPARSE csr2cscEx2 path: row indices ascending inside     */
/* each column; deterministic.  d_heads is accepted and unused.  Scratch word */
/* 0 receives CS_STATUS bits (a row repeating a column sets                   */
/* CS_STATUS_DUPLICATE_COL; such input has no defined transpose here).        */
/* ------------------------------------------------------------------------ */

CS_API int cs_b200_compressed_transpose_scratch_bytes(uint32_t cDim, uint32_t uDim, uint32_t nnz, size_t *out_bytes);

CS_API int cs_b200_build_compressed_transpose(uint32_t cDim,
                                              uint32_t uDim,
                                              uint32_t nnz,
                                              const uint32_t *d_cAxPtr,
                                              const uint32_t *d_uAxIdx,
                                              const uint16_t *d_val,
                                              uint32_t *d_out_uAxPtr,
                                              uint32_t *d_heads,
                                              uint32_t *d_out_cAxIdx,
                                              uint16_t *d_out_val,
                                              void *d_scan_tmp,
                                              size_t scan_bytes,
                                              cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Major-axis nnz bucketing                                                   */
/* replaces bucket::build_major_nnz_bucket_plan_raw,                          */
/* build_shard_major_nnz_bucket_plan_raw, rebuild_compressed_major_order_raw, */
/* rebuild_bucketed_shard_compressed_raw and their scratch queries            */
/* (src/bucket/major_nnz_raw.cuh:34-320), same arguments.                     */
/* ------------------------------------------------------------------------ */

CS_API int cs_b200_major_nnz_bucket_sort_scratch_bytes(uint32_t major_dim, size_t *out_bytes);
CS_API int cs_b200_major_nnz_bucket_scan_scratch_bytes(uint32_t major_dim, size_t *out_bytes);

/* d_major_nnz[i] = ptr[i+1]-ptr[i]; d_major_order_in = identity;
 * d_major_nnz_sorted / d_major_order_out = stable ascending sort of the
 * counts; d_bucket_offsets (nullable) = clamp(requested, 1, major_dim) + 1
 * equal-count offsets, the first major_dim % B buckets one row larger. */
CS_API int cs_b200_build_major_nnz_bucket_plan(const uint32_t *d_major_ptr,
                                               uint32_t major_dim,
                                               uint32_t *d_major_nnz,
                                               uint32_t *d_major_nnz_sorted,
                                               uint32_t *d_major_order_in,
                                               uint32_t *d_major_order_out,
                                               uint32_t *d_bucket_offsets,
                                               uint32_t requested_bucket_count,
                                               void *d_sort_tmp,
                                               size_t sort_tmp_bytes,
                                               cs_stream_t stream);

/* The same over many parts: row r of the shard is local row
 * r - d_part_row_offsets[p] of part p (d_part_row_offsets[part_count+1]). */
CS_API int cs_b200_build_shard_major_nnz_bucket_plan(const uint32_t *const *d_part_major_ptr,
                                                     const uint32_t *d_part_row_offsets,
                                                     uint32_t part_count,
                                                     uint32_t shard_rows,
                                                     uint32_t *d_major_nnz,
                                                     uint32_t *d_major_nnz_sorted,
                                                     uint32_t *d_major_order_in,
                                                     uint32_t *d_major_order_out,
                                                     uint32_t *d_bucket_offsets,
                                                     uint32_t requested_bucket_count,
                                                     void *d_sort_tmp,
                                                     size_t sort_tmp_bytes,
                                                     cs_stream_t stream);

/* Power-of-two nnz bins over a sorted count array (no reference function):
 * d_bin_offsets[34]; bin k in [0, 32] is [d_bin_offsets[k], d_bin_offsets[k+1]),
 * holding counts in [2^k, 2^(k+1)) for k >= 1 and in [0, 2) for k = 0. */
CS_API int cs_b200_pow2_nnz_bin_offsets(const uint32_t *d_major_nnz_sorted,
                                        uint32_t major_dim,
                                        uint32_t *d_bin_offsets,
                                        cs_stream_t stream);

/* Rows permuted into plan order: d_dst_major_ptr[major_dim+1] is the
 * exclusive scan of the counts in plan order (the reference scans counts it
 * has already shifted by one slot, giving [0, 0, c0, ...]; this returns the
 * permuted CSR the function is documented to build); d_inverse (nullable). */
CS_API int cs_b200_rebuild_compressed_major_order(const uint32_t *d_src_major_ptr,
                                                  const uint32_t *d_src_minor_idx,
                                                  const uint16_t *d_src_val,
                                                  uint32_t major_dim,
                                                  const uint32_t *d_major_order,
                                                  uint32_t *d_dst_major_ptr,
                                                  uint32_t *d_dst_minor_idx,
                                                  uint16_t *d_dst_val,
                                                  uint32_t *d_inverse_major_order,
                                                  void *d_scan_tmp,
                                                  size_t scan_tmp_bytes,
                                                  cs_stream_t stream);

CS_API int cs_b200_rebuild_bucketed_shard_compressed(const uint32_t *const *d_part_major_ptr,
                                                     const uint32_t *const *d_part_minor_idx,
                                                     const uint16_t *const *d_part_val,
                                                     const uint32_t *d_part_row_offsets,
                                                     uint32_t part_count,
                                                     uint32_t shard_rows,
                                                     const uint32_t *d_major_order,
                                                     uint32_t *d_dst_major_ptr,
                                                     uint32_t *d_dst_minor_idx,
                                                     uint16_t *d_dst_val,
                                                     uint32_t *d_inverse_major_order,
                                                     void *d_scan_tmp,
                                                     size_t scan_tmp_bytes,
                                                     cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* mask_groups: masked per-row feature-group reduction                        */
/* replaces runtime::compute_sparse_group_reduce (mask_groups.cuh:185-204,     */
/* mask_groups.cu:811-918)                                                    */
/* ------------------------------------------------------------------------ */

/* runtime::sparse_group_filter_params (mask_groups.cuh:36-41) */
typedef struct CS_ALIGN16 cs_group_filter_params {
    float min_total;
    uint32_t min_detected_features;
    float max_group_fraction;
    uint32_t fraction_group_index;
} cs_group_filter_params;

/* Output arrays of one reduction (runtime::sparse_group_reduce_result,
 * mask_groups.cuh:43-52): rows entries each, group arrays rows x group_count,
 * row-major.  group_counts / group_percentages may be NULL when group_count
 * is 0. */
typedef struct CS_ALIGN16 cs_group_reduce_out {
    float *row_totals;
    uint32_t *detected_features;
    float *max_values;
    uint8_t *row_keep;
    float *group_counts;
    float *group_percentages;
} cs_group_reduce_out;

/* compute_group_reduce_blocked_ell_kernel (mask_groups.cu:107-199) via
 * compute_sparse_group_reduce(blocked_ell_view) (mask_groups.cu:811-845).
 * d_feature_group_masks: [cols] uint32 bitmasks, or NULL for no groups. */
CS_API int cs_b200_group_reduce_blocked_ell(const cs_blocked_ell_view *src,
                                     const uint32_t *d_feature_group_masks,
                                     uint32_t group_count,
                                     const cs_row_feature_mask_view *masks,
                                     const cs_group_filter_params *filter,
                                     const cs_group_reduce_out *out,
                                     cs_stream_t stream);

/* compute_sparse_group_reduce(sliced_ell_view) (mask_groups.cu:847-881). */
CS_API int cs_b200_group_reduce_sliced_ell(const cs_sliced_ell_view *src,
                                    const uint32_t *d_feature_group_masks,
                                    uint32_t group_count,
                                    const cs_row_feature_mask_view *masks,
                                    const cs_group_filter_params *filter,
                                    const cs_group_reduce_out *out,
                                    cs_stream_t stream);

/* compute_sparse_group_reduce_compressed_fallback (mask_groups.cu:883-918). */
CS_API int cs_b200_group_reduce_compressed(const cs_compressed_view *src,
                                    const uint32_t *d_feature_group_masks,
                                    uint32_t group_count,
                                    const cs_row_feature_mask_view *masks,
                                    const cs_group_filter_params *filter,
                                    const cs_group_reduce_out *out,
                                    cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* manual_reoptimize_masked_sparse: masked + remapped Blocked-ELL -> CSR      */
/* (mask_groups.cuh:220-224, mask_groups.cu:383-462,960-1034)                 */
/* ------------------------------------------------------------------------ */

/* Scratch for cs_b200_reoptimize_count (per-row claim words + scan). */
CS_API int cs_b200_reoptimize_scratch_bytes(uint32_t src_rows, uint32_t output_rows, size_t *out_bytes);

/* Pass 1: d_major_ptr[output_rows + 1] <- exclusive scan of kept nonzeros per
 * output row (count_masked_blocked_ell_rows_kernel + the serial scan at
 * mask_groups.cu:383-424, here one parallel scan).  Rows whose remap target
 * is >= output_rows are dropped, as in the reference.  Two kept source rows
 * with one target set CS_STATUS_REMAP_COLLISION. */
CS_API int cs_b200_reoptimize_count(const cs_blocked_ell_view *src,
                             const cs_row_feature_mask_view *masks,
                             uint32_t output_rows,
                             uint32_t output_cols,
                             uint32_t *d_major_ptr,
                             void *d_scratch,
                             size_t scratch_bytes,
                             uint32_t *d_status,
                             cs_stream_t stream);

/* Pass 2: deterministic scatter (scatter_masked_blocked_ell_to_compressed_kernel,
 * mask_groups.cu:426-462).  Within an output row the entries keep Blocked-ELL
 * slot order, which is ascending source column for a sorted blockColIdx. */
CS_API int cs_b200_reoptimize_emit(const cs_blocked_ell_view *src,
                            const cs_row_feature_mask_view *masks,
                            uint32_t output_rows,
                            uint32_t output_cols,
                            const uint32_t *d_major_ptr,
                            uint32_t *d_minor_idx,
                            uint16_t *d_val,
                            cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Filtered Blocked-ELL -> CSR over the partitions of one shard               */
/* replaces convert::filter_blocked_ell_to_compressed (src/convert/           */
/* filtered_blocked_ell_to_compressed.cuh:264-382) and the filter stage of    */
/* repack::build_repacked_shard_blocked_ell (src/repack/operators/            */
/* sharded_blocked_ell.cuh:393-566, kernels/sharded_blocked_ell.cuh:23-138).  */
/* parts: host array of device views, rows concatenated in order (the         */
/* reference's part_views / part_row_offsets); row masks and remaps index the */
/* shard's rows.  The entries kept are those of the masked reoptimize above.  */
/* ------------------------------------------------------------------------ */

#define CS_MAX_REPACK_PARTS 64u

CS_API int cs_b200_filter_blocked_ell_scratch_bytes(uint32_t shard_rows, uint32_t output_rows, size_t *out_bytes);

/* d_major_ptr[output_rows + 1] <- row pointers of the filtered CSR (the live
 * nnz is d_major_ptr[output_rows]); d_kept (nullable, u64[2]) <- kept rows
 * and their Blocked-ELL slots (the reference's d_kept_rows /
 * d_kept_row_slots).  The reference exclusive-scans counts already stored one
 * slot up, so its pointers read [0, 0, c0, c0 + c1, ...]; these are the CSR
 * row pointers the functions document. */
CS_API int cs_b200_filter_blocked_ell_count(const cs_blocked_ell_view *parts,
                                            uint32_t part_count,
                                            const cs_row_feature_mask_view *masks,
                                            uint32_t output_rows,
                                            uint32_t output_cols,
                                            uint32_t *d_major_ptr,
                                            uint64_t *d_kept,
                                            void *d_scratch,
                                            size_t scratch_bytes,
                                            uint32_t *d_status,
                                            cs_stream_t stream);

/* The same filter in ONE pass over the kept rows' values, for shards without
 * row or feature remaps whose block sizes are multiples of 8 (16-byte aligned
 * values) and output_rows >= the shard's rows: each kept row is counted, its
 * output offset found by a decoupled look-back over the rows before it, and
 * its entries written while its values are still in L2 (the count's loads
 * mark them evict_last; only the 8-value groups holding kept entries are read
 * again), so the values cross HBM once instead of twice (count + emit).  Rows
 * the row mask drops cost no pass over their values.  The output arrays hold
 * `capacity` entries (the stored nnz of the parts bounds the live entries); a
 * shard that needs more sets CS_STATUS_CAPACITY in *d_status and writes
 * nothing past them (run count + emit instead).  d_major_ptr, d_kept as for
 * count.  Returns 0 with a message (and launches nothing) when the shard does
 * not qualify.  Scratch: cs_b200_filter_blocked_ell_onepass_scratch_bytes
 * (8 bytes per row). */
CS_API int cs_b200_filter_blocked_ell_onepass_scratch_bytes(const cs_blocked_ell_view *parts,
                                                            uint32_t part_count,
                                                            size_t *out_bytes);
CS_API int cs_b200_filter_blocked_ell_onepass(const cs_blocked_ell_view *parts,
                                              uint32_t part_count,
                                              const cs_row_feature_mask_view *masks,
                                              uint32_t output_rows,
                                              uint32_t output_cols,
                                              uint32_t *d_major_ptr,
                                              uint32_t *d_minor_idx,
                                              uint16_t *d_val,
                                              uint64_t capacity,
                                              uint64_t *d_kept,
                                              void *d_scratch,
                                              size_t scratch_bytes,
                                              uint32_t *d_status,
                                              cs_stream_t stream);

/* The same filter for the same shards as the one-pass entry, in two passes
 * with no waits between CTAs: pass 1 reads every kept row's values once,
 * counts its kept entries and marks (one bit per 8-value group, in scratch)
 * the groups that hold any; a device scan turns the counts into d_major_ptr;
 * pass 2 reads only the marked groups again and writes their entries in slot
 * order.  Arguments, capacity, CS_STATUS_CAPACITY, d_major_ptr and d_kept as
 * for cs_b200_filter_blocked_ell_onepass.  Scratch:
 * cs_b200_filter_blocked_ell_marked_scratch_bytes (4 bytes per 256 slots of
 * the widest partition per row, plus the scan's). */
CS_API int cs_b200_filter_blocked_ell_marked_scratch_bytes(const cs_blocked_ell_view *parts,
                                                           uint32_t part_count,
                                                           size_t *out_bytes);
CS_API int cs_b200_filter_blocked_ell_marked(const cs_blocked_ell_view *parts,
                                             uint32_t part_count,
                                             const cs_row_feature_mask_view *masks,
                                             uint32_t output_rows,
                                             uint32_t output_cols,
                                             uint32_t *d_major_ptr,
                                             uint32_t *d_minor_idx,
                                             uint16_t *d_val,
                                             uint64_t capacity,
                                             uint64_t *d_kept,
                                             void *d_scratch,
                                             size_t scratch_bytes,
                                             uint32_t *d_status,
                                             cs_stream_t stream);

CS_API int cs_b200_filter_blocked_ell_emit(const cs_blocked_ell_view *parts,
                                           uint32_t part_count,
                                           const cs_row_feature_mask_view *masks,
                                           uint32_t output_rows,
                                           uint32_t output_cols,
                                           const uint32_t *d_major_ptr,
                                           uint32_t *d_minor_idx,
                                           uint16_t *d_val,
                                           cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Execution bucketing of one partition (the persisted execution layout)      */
/* replaces build_bucketed_blocked_ell_partition / build_bucketed_sliced_ell_ */
/* partition (include/CellShard/io/csh5/api.cuh:726-733, src/io/csh5/runtime/ */
/* fetch.cc:332-344 -> src/io/csh5/execution_builders_part.hh:1011-1596) and  */
/* choose_bucket_count_for_part / choose_bucket_count_for_sliced_part (:1249, */
/* :1572).  Blocked-ELL: row blocks stably sorted by their valid block        */
/* columns (a partial last row block stays last), equal row-block cuts, each  */
/* segment as wide as its widest row block, neighbouring equal widths merged  */
/* only when all are equal.  Sliced-ELL: rows stably sorted by live slots,    */
/* cut by the reference's byte-minimising dynamic programme into single-slice */
/* segments.  Both fall back to one segment when the cut layout packs no      */
/* smaller than the source.  Valid slots are compacted to the front of each   */
/* destination row (block); padding is the invalid column with zero values.   */
/* ------------------------------------------------------------------------ */

/* cellshard::bucketed_blocked_ell_partition (io/csh5/api.cuh:316-327) */
typedef struct cs_host_bucketed_blocked_ell {
    uint32_t rows, cols, nnz, segment_count;
    cs_host_blocked_ell *segments;
    uint32_t *segment_row_offsets;
    uint32_t *exec_to_canonical_rows;
    uint32_t *canonical_to_exec_rows;
    uint32_t *exec_to_canonical_cols;
    uint32_t *canonical_to_exec_cols;
} cs_host_bucketed_blocked_ell;

/* cellshard::bucketed_sliced_ell_partition (io/csh5/api.cuh:394-406) */
typedef struct cs_host_bucketed_sliced_ell {
    uint32_t rows, cols, nnz, segment_count;
    cs_host_sliced_ell *segments;
    uint32_t *segment_row_offsets;
    uint32_t *exec_to_canonical_rows;
    uint32_t *canonical_to_exec_rows;
    uint32_t canonical_slice_count;
    uint32_t *canonical_slice_row_offsets;
    uint32_t *canonical_slice_widths;
} cs_host_bucketed_sliced_ell;

/* A planned layout.  Segments are stored back to back: segment s's index
 * entries (block-column indices or column indices) start at the sum of the
 * earlier segments' index entries, its values likewise. */
typedef struct cs_exec_bucket_plan {
    uint32_t segment_count;
    uint32_t bucket_count;   /* the requested count it was built for (the chosen one when 0 was asked) */
    uint32_t units;          /* row blocks (Blocked-ELL) or rows (Sliced-ELL) */
    uint32_t block_size;     /* Blocked-ELL block size, 1 for Sliced-ELL */
    uint64_t bytes;          /* bucketed_bytes_out: packed bytes of the kept layout */
    uint64_t original_bytes; /* packed bytes of the source part */
    uint64_t index_entries;  /* all segments */
    uint64_t value_entries;  /* all segments */
} cs_exec_bucket_plan;

/* Host arrays of a plan: room for max_segments entries (+1 for offsets),
 * max_segments >= min(max(requested, 8), units). */
typedef struct cs_exec_bucket_segments {
    uint32_t max_segments;
    uint32_t *unit_offsets;  /* [S + 1] row blocks (Blocked-ELL) or rows (Sliced-ELL) of each segment */
    uint32_t *row_offsets;   /* [S + 1] execution rows of each segment */
    uint32_t *widths;        /* [S] width in blocks (Blocked-ELL) or slots (Sliced-ELL) */
} cs_exec_bucket_segments;

CS_API int cs_b200_bucketed_blocked_ell_scratch_bytes(uint32_t rows, uint32_t block_size, uint32_t max_segments,
                                                      size_t *out_bytes);
/* Plans on the device (valid-slot counts, the stable sort, the cuts and the
 * byte fallback) and synchronises the stream to return the plan.
 * requested 0 picks the count in 1..min(8, row blocks) with fewest packed
 * bytes (ties to the smaller), as choose_bucket_count_for_part. */
CS_API int cs_b200_bucketed_blocked_ell_plan(const cs_blocked_ell_view *part,
                                             uint32_t requested,
                                             void *d_scratch,
                                             size_t scratch_bytes,
                                             cs_exec_bucket_plan *plan,
                                             cs_exec_bucket_segments *segments,
                                             cs_stream_t stream);
/* Copies the part into the planned segments and writes the row maps and the
 * identity column maps (each of the four maps nullable). */
CS_API int cs_b200_bucketed_blocked_ell_fill(const cs_blocked_ell_view *part,
                                             const void *d_scratch,
                                             const cs_exec_bucket_plan *plan,
                                             uint32_t *d_seg_block_col_idx,
                                             uint16_t *d_seg_val,
                                             uint32_t *d_exec_to_canonical_rows,
                                             uint32_t *d_canonical_to_exec_rows,
                                             uint32_t *d_exec_to_canonical_cols,
                                             uint32_t *d_canonical_to_exec_cols,
                                             cs_stream_t stream);

CS_API int cs_b200_bucketed_sliced_ell_scratch_bytes(uint32_t rows, uint32_t max_segments, size_t *out_bytes);
/* Live-slot counts and the stable sort on the device; the split (a
 * sequential dynamic programme over the sorted widths, as the reference's)
 * runs on the host over the widths copied back.  requested 0 chooses as
 * choose_bucket_count_for_sliced_part. */
CS_API int cs_b200_bucketed_sliced_ell_plan(const cs_sliced_ell_view *part,
                                            uint32_t requested,
                                            void *d_scratch,
                                            size_t scratch_bytes,
                                            cs_exec_bucket_plan *plan,
                                            cs_exec_bucket_segments *segments,
                                            cs_stream_t stream);
CS_API int cs_b200_bucketed_sliced_ell_fill(const cs_sliced_ell_view *part,
                                            const void *d_scratch,
                                            const cs_exec_bucket_plan *plan,
                                            uint32_t *d_seg_col_idx,
                                            uint16_t *d_seg_val,
                                            uint32_t *d_exec_to_canonical_rows,
                                            uint32_t *d_canonical_to_exec_rows,
                                            cs_stream_t stream);

/* The ingest-time choice (bucket::build_plan, src/bucket/operators/
 * blocked_ell_bucket.cuh:149-210, and choose_bucket_count_for_part,
 * include/CellShard/ingest/internal/dataset/internal/convert_layout_support_part.hh:
 * 116-181): row blocks stably sorted by (valid width << 32 | hash of their
 * valid block columns); for 1..min(8, row blocks) equal cuts, an estimate of
 * index + value + row-map + offset bytes; the count must beat the source's
 * packed bytes (else 1).  Reads the block column indices only. */
CS_API int cs_b200_blocked_ell_bucket_plan_scratch_bytes(uint32_t rows, uint32_t block_size, size_t *out_bytes);
CS_API int cs_b200_blocked_ell_bucket_plan(const cs_blocked_ell_view *part,
                                           uint32_t *d_row_block_order,
                                           uint32_t *d_row_block_width_sorted,
                                           void *d_scratch,
                                           size_t scratch_bytes,
                                           cs_stream_t stream);
/* d_bucket_count <- the count; d_estimated_bytes <- its estimate, or the
 * source's packed bytes when no count beats them. */
CS_API int cs_b200_choose_bucket_count_from_plan(const cs_blocked_ell_view *part,
                                                 const uint32_t *d_row_block_order,
                                                 const uint32_t *d_row_block_width_sorted,
                                                 uint32_t *d_bucket_count,
                                                 uint64_t *d_estimated_bytes,
                                                 cs_stream_t stream);
/* The ingest chooser's host signature (part in host memory, device ordinal). */
CS_API int cs_b200_choose_ingest_bucket_count_for_part(const cs_host_blocked_ell *part,
                                                       int device,
                                                       uint32_t *bucket_count_out);

/* The reference's host signatures: H2D, plan + fill on the device, D2H into
 * host structs packed as the reference allocates them (its clear() frees
 * them).  bucketed_bytes_out nullable. */
CS_API int cs_b200_build_bucketed_blocked_ell_partition(cs_host_bucketed_blocked_ell *out,
                                                        const cs_host_blocked_ell *part,
                                                        uint32_t requested_bucket_count,
                                                        uint64_t *bucketed_bytes_out);
CS_API int cs_b200_choose_bucket_count_for_part(const cs_host_blocked_ell *part,
                                                uint32_t *bucket_count_out,
                                                uint64_t *bucketed_bytes_out);
CS_API void cs_b200_host_bucketed_blocked_ell_clear(cs_host_bucketed_blocked_ell *part);
CS_API int cs_b200_build_bucketed_sliced_ell_partition(cs_host_bucketed_sliced_ell *out,
                                                       const cs_host_sliced_ell *part,
                                                       uint32_t requested_bucket_count,
                                                       uint64_t *bucketed_bytes_out);
CS_API int cs_b200_choose_bucket_count_for_sliced_part(const cs_host_sliced_ell *part,
                                                       uint32_t *bucket_count_out,
                                                       uint64_t *bucketed_bytes_out);
CS_API void cs_b200_host_bucketed_sliced_ell_clear(cs_host_bucketed_sliced_ell *part);

/* ------------------------------------------------------------------------ */
/* .cspack raw partition records, file <-> device memory                       */
/* replaces store_*_raw / load_*_raw of src/io/pack/packfile.cu:191-770 (and   */
/* the host staging the reference does between them and device::upload):      */
/* the same bytes on disk, the arrays moved through two pinned staging        */
/* buffers so the file transfer and the PCIe copy overlap.  fp16 values.      */
/* Synchronous; call once the stream that produced the arrays has finished.   */
/* ------------------------------------------------------------------------ */

/* disk_header (io/common/raw_format.hh:26-31) and each format's leading words. */
typedef struct cs_cspack_info {
    uint32_t format; /* 2 compressed, 3 COO, 6 Blocked-ELL, 7 Sliced-ELL */
    uint32_t rows, cols, nnz;
    uint32_t axis;                 /* compressed */
    uint32_t block_size, ell_cols; /* Blocked-ELL */
    uint32_t slice_count, total_slots; /* Sliced-ELL */
} cs_cspack_info;

CS_API int cs_b200_cspack_peek(const char *path, cs_cspack_info *info);
CS_API int cs_b200_cspack_store_blocked_ell(const char *path, const cs_blocked_ell_view *part);
/* dst: shape from cs_b200_cspack_peek, arrays allocated by the caller. */
CS_API int cs_b200_cspack_load_blocked_ell(const char *path, const cs_blocked_ell_view *dst);
CS_API int cs_b200_cspack_store_sliced_ell(const char *path, const cs_sliced_ell_view *part);
/* also writes dst->slice_slot_offsets (when set) from the slice table. */
CS_API int cs_b200_cspack_load_sliced_ell(const char *path, const cs_sliced_ell_view *dst);
CS_API int cs_b200_cspack_store_compressed(const char *path, const cs_compressed_view *part);
CS_API int cs_b200_cspack_load_compressed(const char *path, const cs_compressed_view *dst);
CS_API int cs_b200_cspack_store_coo(const char *path, const cs_coo_view *part);
CS_API int cs_b200_cspack_load_coo(const char *path, const cs_coo_view *dst);

/* ------------------------------------------------------------------------ */
/* Row-label grouped per-feature moments (no reference counterpart: the new   */
/* entry point beside compute_sparse_group_reduce, same header style).        */
/* ------------------------------------------------------------------------ */

enum {
    CS_MOMENTS_PLAIN_F32 = 0,          /* one fp32 running sum per (group, feature) */
    CS_MOMENTS_TWOSUM_F32 = 1,         /* fp32 batch sums + two-sum compensation, fp32 combine */
    CS_MOMENTS_TWOSUM_F64_COMBINE = 2  /* as 1, cross-chunk combine and variance in fp64 */
};

typedef struct CS_ALIGN16 cs_group_moments_params {
    uint32_t group_count; /* G, 1..CS_MAX_MOMENT_GROUPS */
    uint32_t scheme;      /* CS_MOMENTS_* */
    uint32_t ddof;        /* variance divisor is n - ddof (0 or 1) */
    uint32_t chunk_rows;  /* rows per work chunk, 0 = default */
    /* Optional (NULL = built by every call): device address of the partition's
     * column-block index, built once by cs_b200_group_moments_build_index for
     * this partition (it depends only on blockColIdx, so it stays valid while
     * the staged partition does).  The prepare phase then skips the index pass
     * and the accumulation reads this one. */
    const void *index;
} cs_group_moments_params;

/* All arrays are device memory, [G x cols] row-major unless noted.  Only sum
 * and sumsq are required.  Features whose feature_keep is 0 report zeros. */
typedef struct CS_ALIGN16 cs_group_moments_out {
    float *sum;
    float *sumsq;
    float *mean;        /* nullable */
    float *var;         /* nullable */
    double *mean64;     /* nullable */
    double *var64;      /* nullable */
    uint32_t *group_rows; /* [G] kept rows per group, nullable */
    uint32_t *status;     /* nullable device status word */
} cs_group_moments_out;

CS_API int cs_b200_group_moments_scratch_bytes(const cs_blocked_ell_view *src,
                                        const cs_group_moments_params *params,
                                        size_t *out_bytes);

/* The column-block index of a Blocked-ELL partition, kept with the staged
 * partition so repeated reductions over it skip rebuilding it: one
 * (occupancy bitmap of 32 column blocks, slots before them) pair per row block
 * and 32 column blocks.  The build validates blockColIdx order into *d_status
 * (CS_STATUS_BLOCK_COL_ORDER; nullable) and is stream-ordered. */
CS_API int cs_b200_group_moments_index_bytes(const cs_blocked_ell_view *src, size_t *out_bytes);

/* No counterpart in the reference: the same reduction over a whole shard
 * given as its partitions' views, in one call (one label sort, one
 * accumulation launch over every partition's rows, one combine).  Rows are
 * numbered across the partitions in order (row r of partition k is global row
 * rows_0 + ... + rows_{k-1} + r), so d_row_keep and d_row_labels cover all
 * of them.  The partitions share cols and block_size; at most
 * CS_MOMENTS_MAX_PARTS.  d_indexes: nullable host array of each partition's
 * column-block index (cs_b200_group_moments_build_index); a NULL array or
 * entry is built in scratch by the call.  params->index is not used.
 * Stream-ordered, no synchronisation. */
#define CS_MOMENTS_MAX_PARTS 64u
CS_API int cs_b200_group_moments_parts_scratch_bytes(const cs_blocked_ell_view *parts, uint32_t count,
                                                     const cs_group_moments_params *params, size_t *out_bytes);
CS_API int cs_b200_group_moments_blocked_ell_parts(const cs_blocked_ell_view *parts, uint32_t count,
                                                   const void *const *d_indexes, const uint8_t *d_row_keep,
                                                   const uint8_t *d_feature_keep, const uint32_t *d_row_labels,
                                                   const cs_group_moments_params *params,
                                                   const cs_group_moments_out *out, void *d_scratch,
                                                   size_t scratch_bytes, cs_stream_t stream);
CS_API int cs_b200_group_moments_build_index(const cs_blocked_ell_view *src, void *d_index, uint32_t *d_status,
                                             cs_stream_t stream);

/* For every kept row r (d_row_keep[r] != 0, or all rows when NULL) with label
 * g = d_row_labels[r] < G (all rows in group 0 when NULL), and every stored
 * column f < cols: sum[g][f] += x, sumsq[g][f] += x*x, with x the fp16 value
 * widened to fp32.  blockColIdx rows must be ascending with CS_INVALID_COL
 * padding at the end (the layout cs_b200_blocked_ell_emit and
 * convert::blocked_ell_from_compressed produce); other layouts set
 * CS_STATUS_BLOCK_COL_ORDER.  Deterministic: the same inputs give the same
 * bits regardless of stream contention. */
CS_API int cs_b200_group_moments_blocked_ell(const cs_blocked_ell_view *src,
                                      const uint8_t *d_row_keep,
                                      const uint8_t *d_feature_keep,
                                      const uint32_t *d_row_labels,
                                      const cs_group_moments_params *params,
                                      const cs_group_moments_out *out,
                                      void *d_scratch,
                                      size_t scratch_bytes,
                                      cs_stream_t stream);

/* Size of the library-owned static scratch used by
 * cs_b200_group_moments_blocked_ell_noalloc (64 MiB per GPU that loads it). */
#define CS_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)

/* No counterpart in the reference.  The same reduction for callers that must
 * not allocate device memory (for example a plugin inside a process whose
 * device memory is owned by another allocator or capped by a fixed budget,
 * where cudaMalloc would synchronise the device mid-request and grow the
 * footprint behind the owner's back).  It allocates nothing: its scratch is
 * a fixed CS_NOALLOC_SCRATCH_BYTES device array inside the library, located
 * once per device with cudaGetSymbolAddress on the first call on that device
 * (make that first call before any stream capture).  Calls whose scratch need
 * (cs_b200_group_moments_scratch_bytes) exceeds CS_NOALLOC_SCRATCH_BYTES
 * return 0 with a message.  All calls share the array and it keeps the last
 * call's contents (nothing needs clearing: every byte read is written earlier
 * in the same call); calls that overlap on the GPU race on it, so the caller
 * serialises them.  The located address is kept for the life of the process:
 * do not call this again on a device after cudaDeviceReset. */
CS_API int cs_b200_group_moments_blocked_ell_noalloc(const cs_blocked_ell_view *src,
                                                     const uint8_t *d_row_keep,
                                                     const uint8_t *d_feature_keep,
                                                     const uint32_t *d_row_labels,
                                                     const cs_group_moments_params *params,
                                                     const cs_group_moments_out *out,
                                                     cs_stream_t stream);

/* The same work split into its three stream-ordered phases, for callers that
 * time or schedule them separately (the one-shot call above runs all three):
 * PREPARE builds the column-block index and sorts the kept rows by label,
 * ACCUMULATE streams the values (the dominant kernel), COMBINE adds the
 * per-chunk partials and writes the outputs.  Consecutive phase calls must
 * pass identical arguments and scratch. */
enum {
    CS_MOMENTS_PHASE_PREPARE = 1u,
    CS_MOMENTS_PHASE_ACCUMULATE = 2u,
    CS_MOMENTS_PHASE_COMBINE = 4u,
    CS_MOMENTS_PHASE_ALL = 7u
};

CS_API int cs_b200_group_moments_phases(const cs_blocked_ell_view *src,
                                        const uint8_t *d_row_keep,
                                        const uint8_t *d_feature_keep,
                                        const uint32_t *d_row_labels,
                                        const cs_group_moments_params *params,
                                        const cs_group_moments_out *out,
                                        void *d_scratch,
                                        size_t scratch_bytes,
                                        uint32_t phases,
                                        cs_stream_t stream);

/* No counterpart in the reference.  The one-shot reduction with its results
 * delivered to host memory: h_out holds host pointers (pinned memory, for the
 * copies to overlap) for the fields the caller wants back, each with its
 * device array in d_out.  The groups are split into `parts` ranges (0 = 2,
 * at most G): each range is accumulated and combined in turn, and its rows of
 * every requested array are copied to the host on a library-owned copy stream
 * while the next range computes.  Results equal the device-only call's bit
 * for bit.  Stream-ordered: `stream` waits for the copies, so synchronising
 * it makes h_out readable.  h_out->status, when given with d_out->status,
 * receives the device status word. */
CS_API int cs_b200_group_moments_to_host(const cs_blocked_ell_view *src,
                                         const uint8_t *d_row_keep,
                                         const uint8_t *d_feature_keep,
                                         const uint32_t *d_row_labels,
                                         const cs_group_moments_params *params,
                                         const cs_group_moments_out *d_out,
                                         const cs_group_moments_out *h_out,
                                         void *d_scratch,
                                         size_t scratch_bytes,
                                         uint32_t parts,
                                         cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Synthetic cell x gene data (no reference counterpart; feeds tests and the  */
/* benchmark with seeded NB counts on Zipf-popular columns).                  */
/* ------------------------------------------------------------------------ */

/* Fills d_minor_idx / d_val of a CSR whose d_row_ptr[rows + 1] is given.
 * Row r draws ptr[r+1]-ptr[r] distinct columns by successive sampling from
 * the popularity CDF d_col_cdf[cols] (uint64 thresholds, rank order) mapped
 * to columns through d_col_of_rank[cols], emitted ascending; value k of the
 * row is the zero-truncated count drawn from d_val_cdf[val_cdf_len] (value
 * i+1 for bucket i) times d_row_scale[r] (NULL = 1), rounded to fp16. */
CS_API int cs_b200_synth_csr(uint32_t rows,
                      uint32_t cols,
                      const uint32_t *d_row_ptr,
                      const uint64_t *d_col_cdf,
                      const uint32_t *d_col_of_rank,
                      const uint64_t *d_val_cdf,
                      uint32_t val_cdf_len,
                      const float *d_row_scale,
                      uint64_t seed,
                      uint32_t *d_minor_idx,
                      uint16_t *d_val,
                      cs_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Partition staging: replaces device::upload / release for the compressed,   */
/* Blocked-ELL and Sliced-ELL formats and device_partition_bytes              */
/* (runtime/device/sharded_device.cuh:343-756, 959-991, 1050-1083).  One      */
/* packed device allocation per partition: the device view descriptor, then   */
/* the payload arrays on 256-byte boundaries.  The upload synchronises the    */
/* given stream before returning, as device::upload does.  The Sliced-ELL     */
/* view gets its uniform slice height and u32 slot offsets on upload.         */
/* ------------------------------------------------------------------------ */
enum { CS_FORMAT_COMPRESSED = 1u, CS_FORMAT_BLOCKED_ELL = 2u, CS_FORMAT_SLICED_ELL = 3u };

/* device::partition_record (sharded_device.cuh:22-35) for one partition */
typedef struct CS_ALIGN16 cs_partition_record {
    void *allocation;          /* the packed device block (cudaMalloc) */
    size_t allocation_bytes;
    void *view;                /* device address of the cs_*_view at the block start */
    void *a0, *a1, *a2, *a3;   /* payload arrays (device) */
    int device_id;
    uint32_t format;           /* CS_FORMAT_* */
    unsigned char host_view[64]; /* host copy of the device view (a cs_*_view) */
} cs_partition_record;

CS_API int cs_b200_device_partition_bytes_compressed(const cs_host_compressed *src, size_t *out_bytes);
CS_API int cs_b200_device_partition_bytes_blocked_ell(const cs_host_blocked_ell *src, size_t *out_bytes);
CS_API int cs_b200_device_partition_bytes_sliced_ell(const cs_host_sliced_ell *src, size_t *out_bytes);
CS_API int cs_b200_upload_compressed(const cs_host_compressed *src, cs_partition_record *record, cs_stream_t stream);
CS_API int cs_b200_upload_blocked_ell(const cs_host_blocked_ell *src, cs_partition_record *record,
                                      cs_stream_t stream);
CS_API int cs_b200_upload_sliced_ell(const cs_host_sliced_ell *src, cs_partition_record *record, cs_stream_t stream);
/* device::release: frees the block on its device and zeroes the record. */
CS_API int cs_b200_release_partition(cs_partition_record *record);

/* ------------------------------------------------------------------------ */
/* Shard-level staging: the residency state of a sharded matrix on a device  */
/* (device::sharded_device<MatrixT>, runtime/device/sharded_device.cuh:22-52, */
/* 160-243, 992-1212, 1436-1721).  The three structs below are field for     */
/* field the reference's partition_record, cached_allocation and              */
/* sharded_device (one layout for every MatrixT), so a reference state table */
/* crosses this ABI unchanged.                                               */
/*                                                                          */
/* Device layout of one staged group (a single partition, or every partition */
/* of a shard in one packed allocation): the partitions' device views packed */
/* back to back at the start (record.view points at its own), then each     */
/* partition's arrays, every array on a 256-byte boundary.  Record arrays:   */
/*   compressed   a0 majorPtr, a1 minorIdx, a2 val                          */
/*   Blocked-ELL  a0 blockColIdx, a1 val                                    */
/*   Sliced-ELL   a0 slice_row_offsets, a1 slice_widths, a2 col_idx, a3 val;*/
/*                the u32 slot offsets of the device view sit at            */
/*                a1 + round_up(4 * slice_count, 256)                      */
/* The group's owner (its first partition) holds allocation /              */
/* allocation_bytes / storage; the others hold 0 there.  A released group's */
/* allocation goes to the state's cache (at most 16 entries; the smallest   */
/* cached block that fits is reused by the next upload on that device)     */
/* instead of cudaFree, as the reference's release_partition does.          */
/*                                                                          */
/* Stream order: payload arrays are copied with cudaMemcpyAsync on `stream`  */
/* (pinned host parts give truly asynchronous copies); the device views and */
/* the Sliced-ELL slot offsets are written by kernels on the same stream    */
/* whose arguments carry the data, so nothing on the host stack is read    */
/* after the call returns.  No call synchronises.  Like the reference, an   */
/* upload leaves `device_id` current and a release leaves the record's      */
/* device current.                                                           */
/* ------------------------------------------------------------------------ */

/* device::partition_record<MatrixT> (sharded_device.cuh:22-35) */
typedef struct CS_ALIGN16 cs_staged_part {
    void *allocation;          /* packed device block (group owner only) */
    size_t allocation_bytes;   /* bytes of that block (a cached block may be larger than needed) */
    void *storage;             /* == allocation on the owner */
    void *view;                /* device address of this partition's cs_*_view */
    void *a0, *a1, *a2, *a3;   /* device arrays, per format as listed above */
    unsigned long group_begin; /* partitions staged together: [group_begin, group_end) */
    unsigned long group_end;
    int device_id;             /* -1 when not resident */
} cs_staged_part;

/* device::cached_allocation (sharded_device.cuh:37-41) */
typedef struct cs_cached_allocation {
    void *ptr;
    size_t bytes;
    int device_id;
} cs_cached_allocation;

/* device::sharded_device<MatrixT> (sharded_device.cuh:44-51) */
typedef struct cs_sharded_device {
    unsigned long capacity;
    cs_staged_part *parts;       /* malloc'd by cs_b200_sharded_device_reserve */
    unsigned long cache_count;
    unsigned long cache_capacity;
    cs_cached_allocation *cache; /* malloc'd; at most 16 live entries */
} cs_sharded_device;

#define CS_STAGE_CACHE_ENTRIES 16u

/* device::reserve (sharded_device.cuh:160-178): grows the record table to
 * `capacity` records (new records zeroed, device_id -1); records move
 * bitwise. */
CS_API int cs_b200_sharded_device_reserve(cs_sharded_device *state, unsigned long capacity);
/* device::clear (sharded_device.cuh:136-158): releases every resident
 * partition, frees every cached block on its device and the tables. */
CS_API int cs_b200_sharded_device_clear(cs_sharded_device *state);

/* device::upload_partition_async (sharded_device.cuh:1019-1043, 1144-1166):
 * stages one host partition as record `part_id` on `device_id` (its group is
 * [part_id, part_id + 1)).  A partition already resident on that device is
 * left as it is; one resident elsewhere is released first. */
CS_API int cs_b200_stage_partition_compressed(cs_sharded_device *state, unsigned long part_id,
                                              const cs_host_compressed *src, int device_id, cs_stream_t stream);
CS_API int cs_b200_stage_partition_blocked_ell(cs_sharded_device *state, unsigned long part_id,
                                               const cs_host_blocked_ell *src, int device_id, cs_stream_t stream);
CS_API int cs_b200_stage_partition_sliced_ell(cs_sharded_device *state, unsigned long part_id,
                                              const cs_host_sliced_ell *src, int device_id, cs_stream_t stream);

/* device::upload_shard_async for the compressed and Blocked-ELL formats
 * (upload_{compressed,blocked_ell}_shard_current_device_async,
 * sharded_device.cuh:1223-1435): the `count` partitions `parts[0..count)`
 * become records [first_part, first_part + count), all in ONE packed
 * allocation with their views back to back (the reference does the same for
 * compressed and Blocked-ELL; Sliced-ELL shards are packed here too, where
 * the reference uploads them one partition at a time).  If every partition
 * of the range is already resident on `device_id` nothing happens;
 * otherwise the resident ones are released first. */
CS_API int cs_b200_stage_shard_compressed(cs_sharded_device *state, unsigned long first_part, unsigned long count,
                                          const cs_host_compressed *const *parts, int device_id, cs_stream_t stream);
CS_API int cs_b200_stage_shard_blocked_ell(cs_sharded_device *state, unsigned long first_part, unsigned long count,
                                           const cs_host_blocked_ell *const *parts, int device_id,
                                           cs_stream_t stream);
CS_API int cs_b200_stage_shard_sliced_ell(cs_sharded_device *state, unsigned long first_part, unsigned long count,
                                          const cs_host_sliced_ell *const *parts, int device_id, cs_stream_t stream);

/* device::release_partition (sharded_device.cuh:1168-1200): releases the
 * whole group record `part_id` belongs to; the owner's block goes to the
 * cache (cudaFree once 16 blocks are cached).  A record whose group range is
 * empty (a standalone upload) is freed on its own.  Not resident: success. */
CS_API int cs_b200_release_staged_partition(cs_sharded_device *state, unsigned long part_id);

/* Bytes one packed group of `count` partitions takes on the device (views +
 * arrays, 256-byte aligned): the shard-level counterpart of
 * cs_b200_device_partition_bytes_* (which is this with count 1). */
CS_API int cs_b200_staged_bytes_compressed(const cs_host_compressed *const *parts, unsigned long count,
                                           size_t *out_bytes);
CS_API int cs_b200_staged_bytes_blocked_ell(const cs_host_blocked_ell *const *parts, unsigned long count,
                                            size_t *out_bytes);
CS_API int cs_b200_staged_bytes_sliced_ell(const cs_host_sliced_ell *const *parts, unsigned long count,
                                           size_t *out_bytes);

/* ------------------------------------------------------------------------ */
/* Batched conversion of many uneven partitions (no reference counterpart:  */
/* the reference converts one partition per call, sliced_ell_from_          */
/* compressed.cuh:96-254, and plans one per call, major_nnz_raw.cuh:64-120). */
/* Per partition the results equal choose_sliced_ell_slice_rows_from_       */
/* compressed + sliced_ell_from_compressed at the chosen height, and        */
/* build_major_nnz_bucket_plan_raw, bit for bit.  All partitions of a wave   */
/* run in ONE persistent launch fed by a device work queue, replayed from a  */
/* CUDA graph; output blocks are taken from a caller arena first-fit in      */
/* partition order, and partitions that do not fit are deferred to the next  */
/* wave.                                                                     */
/* ------------------------------------------------------------------------ */
#define CS_BATCH_MAX_CANDIDATES 4

enum {
    CS_BATCH_DEFERRED = 1u << 8,      /* output did not fit the wave's arena */
    CS_BATCH_WAIT_TIMEOUT = 1u << 9,  /* a bounded device wait ran out; item skipped */
    CS_BATCH_TOO_LARGE = 1u << 10,    /* padded slots exceed the u32 slot offsets */
    CS_BATCH_NO_CANDIDATE = 1u << 11,
    CS_BATCH_EXCEEDS_ARENA = 1u << 12 /* the partition's block alone is larger than the arena */
};

typedef struct CS_ALIGN16 cs_batch_part {
    cs_compressed_view src;     /* device CSR (row-compressed) */
    uint32_t bucket_count;      /* requested nnz buckets; plan skipped if d_major_nnz is NULL */
    uint32_t pad0[3];
    uint32_t *d_major_nnz;      /* [rows] row nnz */
    uint32_t *d_sorted_nnz;     /* [rows] ascending */
    uint32_t *d_order;          /* [rows] stable: ties keep row order */
    uint32_t *d_bucket_offsets; /* [clamp(bucket_count, 1, rows) + 1]; [1] if rows == 0 */
    uint32_t *d_pow2_offsets;   /* [34] or NULL: bin k = nnz in [2^k, 2^(k+1)), bin 0 also 0 */
} cs_batch_part;

/* Launch-shape knobs picked by cs_b200_batch_sliced_autotune. */
typedef struct cs_batch_tiles {
    uint32_t layout_rows; /* rows per layout item (multiple of 32) */
    uint32_t emit_rows;   /* rows per emit item */
    uint32_t emit_lanes;  /* lanes per row in the emit: 32, 16, 8 or 4 (rows per warp 1..8) */
    uint32_t ctas_per_sm; /* 0 = as many as fit */
} cs_batch_tiles;

typedef struct CS_ALIGN16 cs_batch_sliced_result {
    uint32_t status;        /* 0, or CS_BATCH_* bits */
    uint32_t slice_rows;    /* chosen height (clamped to [1, rows]) */
    uint32_t slice_count;
    uint32_t plan_status;
    uint64_t total_slots;
    uint64_t arena_offset;  /* byte offset of the partition's block in its wave's arena */
    uint64_t arena_bytes;
    double score;           /* the chooser's score of the chosen height */
    cs_sliced_ell_view view; /* device view into the arena */
} cs_batch_sliced_result;

typedef struct cs_batch_plan cs_batch_plan;

/* Builds the queue, descriptors and the CUDA graph for wave 1 (all
 * partitions).  d_arena must be 256-byte aligned; tiles NULL = defaults.
 * 1..CS_BATCH_MAX_CANDIDATES non-zero candidate heights. */
CS_API int cs_b200_batch_sliced_create(const cs_batch_part *parts, uint32_t count, const uint32_t *candidates,
                                       uint32_t candidate_count, void *d_arena, uint64_t arena_bytes,
                                       const cs_batch_tiles *tiles, cs_batch_plan **out);
/* Times the tile candidates on this batch (each a full wave) and keeps the
 * fastest; cached per process by batch shape. */
CS_API int cs_b200_batch_sliced_autotune(cs_batch_plan *plan, cs_stream_t stream, cs_batch_tiles *chosen);
/* One wave: one graph launch (a state reset and the persistent kernel). */
CS_API int cs_b200_batch_sliced_run(cs_batch_plan *plan, cs_stream_t stream);
/* Copies every partition's result record to the host (synchronises). */
CS_API int cs_b200_batch_sliced_results(cs_batch_plan *plan, cs_batch_sliced_result *h_results, uint32_t *deferred,
                                        uint32_t *error_bits, cs_stream_t stream);
/* The partitions deferred by the last wave become the next wave, with a new
 * (or the same, once its blocks are consumed) arena. */
CS_API int cs_b200_batch_sliced_next_wave(cs_batch_plan *plan, void *d_arena, uint64_t arena_bytes,
                                          uint32_t *wave_size);
/* Every partition becomes the next wave again (e.g. to rerun the batch). */
CS_API int cs_b200_batch_sliced_reset(cs_batch_plan *plan, void *d_arena, uint64_t arena_bytes);
CS_API int cs_b200_batch_sliced_tiles(const cs_batch_plan *plan, cs_batch_tiles *out, uint32_t *grid,
                                      uint32_t *items);
CS_API void cs_b200_batch_sliced_destroy(cs_batch_plan *plan);

/* ------------------------------------------------------------------------ */
/* Serving: masked grouped moments requests over staged Blocked-ELL          */
/* partitions (no reference counterpart).  A device-resident persistent      */
/* kernel runs every admitted request as a dataflow of work items (label     */
/* histogram, scan, stable scatter, chunk accumulation, combine) that it     */
/* appends to its own device queue; the host scheduler admits requests from  */
/* a FIFO when a slot and their scratch fit the HBM budget, copies inputs    */
/* and results on a copy stream that overlaps the kernel, and relaunches the */
/* kernel after it exits on idle.  Results per request are the same bits     */
/* alone and in any mix.                                                      */
/* ------------------------------------------------------------------------ */
typedef struct cs_server cs_server;

typedef struct cs_serve_config {
    uint64_t scratch_budget_bytes; /* HBM for admitted requests (0 = 16 GiB) */
    uint32_t max_inflight;         /* request slots (0 = 32, at most 256) */
    uint32_t chunk_rows;           /* rows per accumulation chunk (0 = 2048, at most 2048) */
    uint32_t idle_exit_us;         /* the persistent kernel exits after this idle time (0 = 20000) */
    uint32_t ctas_per_sm;          /* 0 = occupancy */
} cs_serve_config;

enum {
    CS_SERVE_DEVICE_INPUTS = 1u,  /* row_keep / row_labels / feature_keep are device pointers */
    CS_SERVE_DEVICE_OUTPUTS = 2u  /* outputs are device pointers (no copy back) */
};

enum { CS_SERVE_QUEUED = 0u, CS_SERVE_RUNNING = 1u, CS_SERVE_DONE = 2u };

/* One request over the concatenation of the staged partitions (global rows
 * in partition order).  Host inputs and outputs must stay valid until the
 * request is done; pinned memory makes their copies asynchronous. */
typedef struct cs_serve_request {
    uint32_t group_count;           /* 1..1024 */
    uint32_t scheme;                /* CS_MOMENTS_* */
    uint32_t ddof;
    uint32_t flags;                 /* CS_SERVE_* */
    const uint8_t *row_keep;        /* [total rows] or NULL = all */
    const uint32_t *row_labels;     /* [total rows] or NULL = group 0; labels >= group_count are skipped */
    const uint8_t *feature_keep;    /* [cols] or NULL = all */
    float *sum, *sumsq;             /* [group_count x cols], required */
    float *mean, *var;              /* [group_count x cols] or NULL */
    uint32_t *group_rows;           /* [group_count] or NULL */
} cs_serve_request;

typedef struct cs_serve_stats {
    uint64_t admitted, completed, pending, kernel_launches;
    uint64_t scratch_in_use, scratch_budget;
    uint32_t device_error, pad;
    uint64_t items[8];   /* work items run, by kind (1 start, 2 hist, 3 scan, 4 scatter, 5 acc, 6 combine) */
    uint64_t item_ns[8]; /* device time spent in them (sum over CTAs) */
} cs_serve_stats;

CS_API int cs_b200_serve_open(const cs_blocked_ell_view *parts, uint32_t count, const cs_serve_config *config,
                              cs_server **out);
/* Queues a request (non-blocking); rejects one whose scratch exceeds the budget. */
CS_API int cs_b200_serve_submit(cs_server *server, const cs_serve_request *request, uint64_t *ticket);
CS_API int cs_b200_serve_poll(cs_server *server, uint64_t ticket, uint32_t *state, double *latency_ms);
/* Blocks until the ticket is done (results copied back); latency = submit -> done. */
CS_API int cs_b200_serve_wait(cs_server *server, uint64_t ticket, uint32_t timeout_ms, double *latency_ms);
/* Forgets a finished ticket. */
CS_API int cs_b200_serve_release(cs_server *server, uint64_t ticket);
CS_API int cs_b200_serve_stats(cs_server *server, cs_serve_stats *out);
/* Submits requests[req_index[i]] at arrival_s[i] seconds after the call
 * (open-loop arrivals), waits for all, returns per-request latency, the
 * makespan and (phase_ms, nullable, 4 per request) the times from submit to
 * admission, to the start item, to the device finishing, to results on the
 * host. */
CS_API int cs_b200_serve_run_trace(cs_server *server, const cs_serve_request *requests, const uint32_t *req_index,
                                   const double *arrival_s, uint32_t n, double *latency_ms, double *makespan_s,
                                   double *phase_ms);
/* Finishes admitted work (bounded), stops the kernel and frees everything. */
CS_API void cs_b200_serve_close(cs_server *server);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CELLSHARD_B200_H_ */
