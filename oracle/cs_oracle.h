/*
 * TEST ORACLE ONLY.  CPU restatement of the reference's hot-path algorithms,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
 * checker.  The product (libcellshard_b200) never links or calls it.
 * Each function cites the reference file:line it restates.
 */
#ifndef CS_ORACLE_H_
#define CS_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

float cso_h2f(uint16_t h);

/* ---- mask_groups per-row reduce (src/runtime/mask_groups.cu:107-381) ---- */
typedef struct cso_reduce_out {
    float *row_totals;
    uint32_t *detected;
    float *max_values;
    uint8_t *row_keep;
    float *group_counts;      /* rows x G, nullable */
    float *group_percentages; /* rows x G, nullable */
} cso_reduce_out;

int cso_group_reduce_csr(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                         const uint32_t *group_masks, uint32_t G, const uint8_t *row_keep, const uint8_t *feature_keep,
                         float min_total, uint32_t min_detected, float max_fraction, uint32_t fraction_index,
                         cso_reduce_out *out);
int cso_group_reduce_bell(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                          const uint16_t *val, const uint32_t *group_masks, uint32_t G, const uint8_t *row_keep,
                          const uint8_t *feature_keep, float min_total, uint32_t min_detected, float max_fraction,
                          uint32_t fraction_index, cso_reduce_out *out);
int cso_group_reduce_sell(uint32_t rows, uint32_t cols, uint32_t slice_count, uint32_t slice_rows,
                          const uint32_t *offsets, const uint32_t *widths, const uint32_t *slot_offsets,
                          const uint32_t *col_idx, const uint16_t *val, const uint32_t *group_masks, uint32_t G,
                          const uint8_t *row_keep, const uint8_t *feature_keep, float min_total,
                          uint32_t min_detected, float max_fraction, uint32_t fraction_index, cso_reduce_out *out);

/* ---- manual_reoptimize_masked_sparse (mask_groups.cu:383-462,960-1034) ---- */
/* Writes major_ptr[out_rows+1]; minor_idx/val must hold rows*ell_cols entries.
 * Within an output row entries follow Blocked-ELL slot order.  Returns nnz,
 * or -1 when two kept rows map to one output row. */
long long cso_reoptimize_bell(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                              const uint16_t *val, const uint8_t *row_keep, const uint8_t *feature_keep,
                              const uint32_t *row_remap, const uint32_t *feature_remap, uint32_t out_rows,
                              uint32_t out_cols, uint32_t *major_ptr, uint32_t *minor_idx, uint16_t *out_val);

/* ---- grouped moments, FP64 (no reference counterpart) ---- */
/* Outputs [G x cols] doubles; group_rows[G].  nthreads >= 1 (row-partitioned). */
int cso_group_moments_bell(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                           const uint16_t *val, const uint8_t *row_keep, const uint8_t *feature_keep,
                           const uint32_t *labels, uint32_t G, uint32_t ddof, double *sum, double *sumsq,
                           double *mean, double *var, uint32_t *group_rows, int nthreads);
int cso_group_moments_csr(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx,
                          const uint16_t *val, const uint8_t *row_keep, const uint8_t *feature_keep,
                          const uint32_t *labels, uint32_t G, uint32_t ddof, double *sum, double *sumsq, double *mean,
                          double *var, uint32_t *group_rows, int nthreads);
/* Plain fp32 running sums in row order (the "plain FP32" scheme's reference point). */
int cso_group_moments_bell_f32(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                               const uint16_t *val, const uint8_t *row_keep, const uint32_t *labels, uint32_t G,
                               float *sum, float *sumsq);

/* ---- CSR -> Blocked-ELL (src/convert/blocked_ell_from_compressed.cuh:33-91,258-347) ---- */
int cso_blocked_ell_shape(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx, uint32_t B,
                          uint32_t *ell_width, uint64_t *total_blocks);
/* bci[row_blocks*ell_width], val[rows*ell_width*B]; returns the nnz count. */
uint32_t cso_blocked_ell_from_csr(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx,
                                  const uint16_t *val, uint32_t B, uint32_t ell_width, uint32_t *bci,
                                  uint16_t *out_val);

/* ---- CSR -> Sliced-ELL (src/convert/sliced_ell_from_compressed.cuh:96-164,
 *      sliced_ell_from_blocked_ell.cuh:64-142) ---- */
uint32_t cso_sliced_slice_count(uint32_t rows, uint32_t slice_rows);
/* offsets[S+1], widths[S], slot_offsets[S]; returns total slots. */
uint64_t cso_sliced_ell_layout(uint32_t rows, const uint32_t *ptr, uint32_t slice_rows, uint32_t *offsets,
                               uint32_t *widths, uint32_t *slot_offsets);
void cso_sliced_ell_fill(uint32_t rows, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                         uint32_t slice_rows, const uint32_t *offsets, const uint32_t *widths,
                         const uint32_t *slot_offsets, uint32_t *col_idx, uint16_t *out_val);
/* evaluate_sliced_candidate_: padded slots for one candidate height. */
uint64_t cso_sliced_padded_slots(uint32_t rows, const uint32_t *ptr, uint32_t candidate);
uint64_t cso_bell_live_csr(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                           const uint16_t *val, uint32_t *ptr, uint32_t *idx, uint16_t *out_val);

/* ---- transpose: CSR (cDim x uDim) -> CSC, rows ascending in each column
 *      (cusparseCsr2cscEx2 result used by compressed_transpose_raw.cuh:43-81) ---- */
void cso_csr_transpose(uint32_t cDim, uint32_t uDim, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                       uint32_t *out_ptr, uint32_t *out_idx, uint16_t *out_val);

/* ---- major-axis nnz bucketing (src/bucket/major_nnz_raw.cuh:64-120,188-250) ---- */
void cso_major_nnz_plan(const uint32_t *major_ptr, uint32_t n, uint32_t requested, uint32_t *major_nnz,
                        uint32_t *sorted, uint32_t *order, uint32_t *bucket_offsets);
void cso_pow2_bins(const uint32_t *sorted, uint32_t n, uint32_t *bins /* 34 */);
void cso_rebuild(const uint32_t *ptr, const uint32_t *idx, const uint16_t *val, uint32_t n, const uint32_t *order,
                 uint32_t *dst_ptr, uint32_t *dst_idx, uint16_t *dst_val, uint32_t *inverse);

/* ---- execution bucketing (src/io/csh5/execution_builders_part.hh:1018-1596) ---- */
/* packed_blocked_ell_bytes (io/pack/packfile.cuh:110-116), fp16 values. */
uint64_t cso_packed_blocked_ell_bytes(uint32_t rows, uint32_t ell_cols, uint32_t B);
/* packed_sliced_ell_bytes (src/io/pack/packfile.cu:179-188), fp16 values. */
uint64_t cso_packed_sliced_ell_bytes(uint32_t slice_count, uint64_t total_slots);
/* Blocked-ELL: order[RB], widths[RB]; seg_rb[S+1], seg_w[S] with room for
 * min(requested, RB) segments.  Returns S (build_execution_bucket_layout). */
uint32_t cso_bell_exec_layout(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t requested,
                              uint32_t *order, uint32_t *widths, uint32_t *seg_rb, uint32_t *seg_w);
/* The layout build_bucketed_execution_partition keeps, and its byte count. */
uint32_t cso_bell_exec_build_layout(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t requested,
                                    uint32_t *order, uint32_t *widths, uint32_t *seg_rb, uint32_t *seg_w,
                                    uint64_t *bytes);
/* Segments packed back to back: seg_bci [sum RB_s * w_s], seg_val [sum rows_s * w_s * B]. */
void cso_bell_exec_fill(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, const uint16_t *val,
                        const uint32_t *order, uint32_t S, const uint32_t *seg_rb, const uint32_t *seg_w,
                        uint32_t *seg_bci, uint16_t *seg_val, uint32_t *exec_to_canonical,
                        uint32_t *canonical_to_exec);
int cso_bell_choose_bucket_count(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t *count,
                                 uint64_t *bytes);
/* Sliced-ELL: the split of ascending widths into <= requested segments. */
int cso_sell_exec_dp(uint32_t rows, const uint32_t *sorted_widths, uint32_t requested, uint32_t *seg_row,
                     uint32_t *seg_w);
int cso_sell_exec_build_layout(uint32_t rows, uint32_t S_src, const uint32_t *offsets, const uint32_t *widths,
                               const uint32_t *col_idx, uint32_t requested, uint32_t *order, uint32_t *row_widths,
                               uint32_t *sorted_widths, uint32_t *seg_row, uint32_t *seg_w, uint64_t *bytes);
/* Segments packed back to back: seg_col / seg_val [sum rows_s * w_s]. */
void cso_sell_exec_fill(uint32_t rows, uint32_t S_src, const uint32_t *offsets, const uint32_t *widths,
                        const uint32_t *col_idx, const uint16_t *val, const uint32_t *order, uint32_t S,
                        const uint32_t *seg_row, const uint32_t *seg_w, uint32_t *seg_col, uint16_t *seg_val,
                        uint32_t *exec_to_canonical, uint32_t *canonical_to_exec);
int cso_sell_choose_bucket_count(uint32_t rows, uint32_t S_src, const uint32_t *offsets, const uint32_t *widths,
                                 const uint32_t *col_idx, uint32_t *count, uint64_t *bytes);
/* Ingest-time choice (blocked_ell_bucket.cuh:70-210, convert_layout_support_part.hh:116-181). */
void cso_bell_bucket_plan(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t *order,
                          uint32_t *width_sorted);
uint64_t cso_bell_estimate_bucketed_bytes(uint32_t rows, uint32_t B, const uint32_t *order,
                                          const uint32_t *width_sorted, uint32_t RB, uint32_t buckets);
uint32_t cso_bell_choose_ingest_bucket_count(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci);
/* ---- COO -> Blocked-ELL (src/convert/blocked_ell_from_compressed.cuh:105-257,349-437,
 *      src/convert/blocked_ell_from_coo_cuda.cuh:179-198) ---- */
/* Returns the ell width (bci [RB x W], out_val [rows x W*B] when non-null), -1 on a
 * row out of range; nnz_out[0] host count, nnz_out[1] CUDA-path count. */
long long cso_blocked_ell_from_coo(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *row,
                                   const uint32_t *col, const uint16_t *val, const uint32_t *map, uint32_t B,
                                   uint32_t *bci, uint16_t *out_val, uint64_t *nnz_out, uint64_t *total_blocks);
int cso_coo_block_shape(uint32_t rows, uint32_t nnz, const uint32_t *row, const uint32_t *col, const uint32_t *map,
                        uint32_t B, uint32_t *width, uint64_t *total_blocks);

#ifdef __cplusplus
}
#endif

#endif
