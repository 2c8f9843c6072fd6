// TEST ORACLE ONLY -- never linked into libcellshard_b200.
//
// extern "C" bridge to the reference's own GPU code, compiled from the
// read-only reference tree with the reference's CUDA flags into
// oracle/_ref/libcs_ref_gpu.so (oracle/Makefile), together with
// src/runtime/mask_groups.cu.  The GPU parity tests run these beside
// libcellshard_b200 on the same device buffers:
//   runtime::compute_sparse_group_reduce / _compressed_fallback (mask_groups.cu:811-918)
//   runtime::manual_reoptimize_masked_sparse (mask_groups.cu:960-1034)
//   convert::build_compressed_transpose_raw (src/convert/compressed_transpose_raw.cuh:14)
//   bucket::build_major_nnz_bucket_plan_raw (src/bucket/major_nnz_raw.cuh:64)
//   bucket::rebuild_compressed_major_order_raw (src/bucket/major_nnz_raw.cuh:188)
//   convert::sliced_ell_from_compressed_cuda (src/convert/sliced_ell_from_compressed.cuh:166)
// The *_timed variants allocate once, run `warmup` untimed calls, then time
// `reps` calls of the reference function alone with CUDA events on its
// stream, for the reference GPU points beside this library's kernels.
#include <CellShard/runtime/mask_groups.cuh>

#include "src/bucket/major_nnz_raw.cuh"
#include "src/convert/compressed_transpose_raw.cuh"
#include "src/convert/sliced_ell_from_compressed.cuh"
#include "src/convert/filtered_blocked_ell_to_compressed.cuh"
#include "src/convert/blocked_ell_from_compressed.cuh"
#include "src/convert/blocked_ell_from_coo_cuda.cuh"

#include "cellshard_b200.h"

#include <cstdlib>
#include <cstring>

using namespace cellshard;

namespace {

runtime::row_feature_mask_view masks_of(const cs_row_feature_mask_view *m) {
    runtime::row_feature_mask_view r{};
    if (m != nullptr) {
        r.row_keep = m->row_keep;
        r.feature_keep = m->feature_keep;
        r.row_remap = m->row_remap;
        r.feature_remap = m->feature_remap;
    }
    return r;
}

int copy_out(runtime::sparse_group_reduce_workspace *ws, const runtime::sparse_group_reduce_result &res,
             const cs_group_reduce_out *out) {
    const std::size_t rows = res.rows;
    if (cudaStreamSynchronize(ws->stream) != cudaSuccess) return 0;
    cudaMemcpy(out->row_totals, res.row_totals, rows * 4u, cudaMemcpyDeviceToDevice);
    cudaMemcpy(out->detected_features, res.detected_features, rows * 4u, cudaMemcpyDeviceToDevice);
    cudaMemcpy(out->max_values, res.max_values, rows * 4u, cudaMemcpyDeviceToDevice);
    cudaMemcpy(out->row_keep, res.row_keep, rows, cudaMemcpyDeviceToDevice);
    if (res.group_count != 0u && out->group_counts != nullptr) {
        cudaMemcpy(out->group_counts, res.group_counts, rows * res.group_count * 4u, cudaMemcpyDeviceToDevice);
        cudaMemcpy(out->group_percentages, res.group_percentages, rows * res.group_count * 4u,
                   cudaMemcpyDeviceToDevice);
    }
    return cudaDeviceSynchronize() == cudaSuccess;
}

template <typename View, typename Fn>
int reduce_with(const View *v, const uint32_t *masks_dev, uint32_t group_count, const cs_row_feature_mask_view *m,
                const cs_group_filter_params *f, const cs_group_reduce_out *out, Fn fn) {
    runtime::sparse_group_reduce_workspace ws;
    runtime::init(&ws);
    if (!runtime::setup(&ws, 0)) return 0;
    runtime::group_mask_config_view groups{group_count, nullptr, masks_dev};
    runtime::row_feature_mask_view mv = masks_of(m);
    runtime::sparse_group_filter_params filter{f->min_total, f->min_detected_features, f->max_group_fraction,
                                               f->fraction_group_index};
    runtime::sparse_group_reduce_result res{};
    int ok = fn(v, &ws, &groups, &mv, &filter, &res);
    if (ok) ok = copy_out(&ws, res, out);
    runtime::clear(&ws);
    return ok;
}

} // namespace

extern "C" {

int csrefgpu_group_reduce_blocked_ell(const cs_blocked_ell_view *src, const uint32_t *d_masks, uint32_t group_count,
                                      const cs_row_feature_mask_view *m, const cs_group_filter_params *f,
                                      const cs_group_reduce_out *out) {
    const device::blocked_ell_view *v = reinterpret_cast<const device::blocked_ell_view *>(src);
    return reduce_with(v, d_masks, group_count, m, f, out,
                       [](const device::blocked_ell_view *vv, runtime::sparse_group_reduce_workspace *ws,
                          const runtime::group_mask_config_view *g, const runtime::row_feature_mask_view *mm,
                          const runtime::sparse_group_filter_params *ff, runtime::sparse_group_reduce_result *r) {
                           return runtime::compute_sparse_group_reduce(vv, ws, g, mm, ff, r);
                       });
}

int csrefgpu_group_reduce_sliced_ell(const cs_sliced_ell_view *src, const uint32_t *d_masks, uint32_t group_count,
                                     const cs_row_feature_mask_view *m, const cs_group_filter_params *f,
                                     const cs_group_reduce_out *out) {
    const device::sliced_ell_view *v = reinterpret_cast<const device::sliced_ell_view *>(src);
    return reduce_with(v, d_masks, group_count, m, f, out,
                       [](const device::sliced_ell_view *vv, runtime::sparse_group_reduce_workspace *ws,
                          const runtime::group_mask_config_view *g, const runtime::row_feature_mask_view *mm,
                          const runtime::sparse_group_filter_params *ff, runtime::sparse_group_reduce_result *r) {
                           return runtime::compute_sparse_group_reduce(vv, ws, g, mm, ff, r);
                       });
}

int csrefgpu_group_reduce_compressed(const cs_compressed_view *src, const uint32_t *d_masks, uint32_t group_count,
                                     const cs_row_feature_mask_view *m, const cs_group_filter_params *f,
                                     const cs_group_reduce_out *out) {
    const device::compressed_view *v = reinterpret_cast<const device::compressed_view *>(src);
    return reduce_with(v, d_masks, group_count, m, f, out,
                       [](const device::compressed_view *vv, runtime::sparse_group_reduce_workspace *ws,
                          const runtime::group_mask_config_view *g, const runtime::row_feature_mask_view *mm,
                          const runtime::sparse_group_filter_params *ff, runtime::sparse_group_reduce_result *r) {
                           return runtime::compute_sparse_group_reduce_compressed_fallback(vv, ws, g, mm, ff, r);
                       });
}

// Runs manual_reoptimize_masked_sparse and copies its CSR (major_ptr
// [out_rows + 1], then up to `cap` entries) into caller buffers; returns
// live_nnz through *nnz_out.
int csrefgpu_reoptimize(const cs_blocked_ell_view *src, const cs_row_feature_mask_view *m, uint32_t output_rows,
                        uint32_t output_cols, uint32_t *d_major_ptr, uint32_t *d_minor_idx, uint16_t *d_val,
                        uint32_t cap, uint32_t *nnz_out) {
    runtime::masked_sparse_reoptimize_workspace ws;
    runtime::init(&ws);
    if (!runtime::setup(&ws, 0)) return 0;
    runtime::row_feature_mask_view mv = masks_of(m);
    runtime::masked_sparse_reoptimize_config cfg{output_rows, output_cols, 0u, 0u,
                                                 runtime::sparse_mask_layout_compressed};
    runtime::masked_sparse_reoptimize_result res{};
    int ok = runtime::manual_reoptimize_masked_sparse(reinterpret_cast<const device::blocked_ell_view *>(src), &mv,
                                                      &cfg, &ws, &res);
    if (ok) {
        const uint32_t rows = res.compressed.rows;
        const uint32_t nnz = res.metadata.live_nnz;
        *nnz_out = nnz;
        cudaMemcpy(d_major_ptr, res.compressed.majorPtr, ((std::size_t) rows + 1u) * 4u, cudaMemcpyDeviceToDevice);
        const uint32_t n = nnz < cap ? nnz : cap;
        if (n != 0u) {
            cudaMemcpy(d_minor_idx, res.compressed.minorIdx, (std::size_t) n * 4u, cudaMemcpyDeviceToDevice);
            cudaMemcpy(d_val, res.compressed.val, (std::size_t) n * 2u, cudaMemcpyDeviceToDevice);
        }
        ok = cudaDeviceSynchronize() == cudaSuccess;
    }
    runtime::clear(&ws);
    return ok;
}

// cuSPARSE transpose path of build_compressed_transpose_raw; scratch sized by
// cusparseCsr2cscEx2_bufferSize so the vendor path (not the fallback) runs.
int csrefgpu_transpose(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *d_ptr, const uint32_t *d_idx,
                       const uint16_t *d_val, uint32_t *d_out_ptr, uint32_t *d_out_idx, uint16_t *d_out_val) {
    cusparseHandle_t handle = 0;
    std::size_t lib_bytes = 0;
    if (!convert::cusparse_utils::acquire((cudaStream_t) 0, &handle)) return 0;
    if (cusparseCsr2cscEx2_bufferSize(handle, (int) cDim, (int) uDim, (int) nnz, d_val,
                                      reinterpret_cast<const int *>(d_ptr), reinterpret_cast<const int *>(d_idx),
                                      d_out_val, reinterpret_cast<int *>(d_out_ptr),
                                      reinterpret_cast<int *>(d_out_idx), CUDA_R_16F, CUSPARSE_ACTION_NUMERIC,
                                      CUSPARSE_INDEX_BASE_ZERO, CUSPARSE_CSR2CSC_ALG1,
                                      &lib_bytes) != CUSPARSE_STATUS_SUCCESS)
        return 0;
    void *scratch = nullptr;
    uint32_t *heads = nullptr;
    const std::size_t bytes = lib_bytes < 256u ? 256u : lib_bytes;
    if (cudaMalloc(&scratch, bytes) != cudaSuccess) return 0;
    if (cudaMalloc((void **) &heads, ((std::size_t) uDim + 1u) * 4u) != cudaSuccess) {
        cudaFree(scratch);
        return 0;
    }
    int ok = convert::build_compressed_transpose_raw(cDim, uDim, nnz, d_ptr, d_idx,
                                                     reinterpret_cast<const __half *>(d_val), d_out_ptr, heads,
                                                     d_out_idx, reinterpret_cast<__half *>(d_out_val), scratch, bytes,
                                                     (cudaStream_t) 0);
    if (ok) ok = cudaDeviceSynchronize() == cudaSuccess;
    cudaFree(heads);
    cudaFree(scratch);
    return ok;
}

int csrefgpu_major_nnz_plan(const uint32_t *d_major_ptr, uint32_t major_dim, uint32_t *d_major_nnz,
                            uint32_t *d_sorted, uint32_t *d_order_in, uint32_t *d_order_out, uint32_t *d_offsets,
                            uint32_t requested) {
    std::size_t bytes = 0;
    if (!bucket::major_nnz_bucket_sort_scratch_bytes(major_dim, &bytes)) return 0;
    void *tmp = nullptr;
    if (cudaMalloc(&tmp, bytes < 256u ? 256u : bytes) != cudaSuccess) return 0;
    int ok = bucket::build_major_nnz_bucket_plan_raw(d_major_ptr, major_dim, d_major_nnz, d_sorted, d_order_in,
                                                     d_order_out, d_offsets, requested, tmp, bytes,
                                                     (cudaStream_t) 0);
    if (ok) ok = cudaDeviceSynchronize() == cudaSuccess;
    cudaFree(tmp);
    return ok;
}

int csrefgpu_rebuild(const uint32_t *d_ptr, const uint32_t *d_idx, const uint16_t *d_val, uint32_t major_dim,
                     const uint32_t *d_order, uint32_t *d_dst_ptr, uint32_t *d_dst_idx, uint16_t *d_dst_val,
                     uint32_t *d_inverse) {
    std::size_t bytes = 0;
    if (!bucket::major_nnz_bucket_scan_scratch_bytes(major_dim, &bytes)) return 0;
    void *tmp = nullptr;
    if (cudaMalloc(&tmp, bytes < 256u ? 256u : bytes) != cudaSuccess) return 0;
    int ok = bucket::rebuild_compressed_major_order_raw(d_ptr, d_idx, reinterpret_cast<const __half *>(d_val),
                                                        major_dim, d_order, d_dst_ptr, d_dst_idx,
                                                        reinterpret_cast<__half *>(d_dst_val), d_inverse, tmp, bytes,
                                                        (cudaStream_t) 0);
    if (ok) ok = cudaDeviceSynchronize() == cudaSuccess;
    cudaFree(tmp);
    return ok;
}

// convert::filter_blocked_ell_to_compressed (filtered_blocked_ell_to_compressed.cuh:264-382):
// its row pointers (output_rows + 1) into d_major_ptr_out and its nnz field.
int csrefgpu_filter_blocked_ell(const cs_blocked_ell_view *src, uint32_t output_rows, uint32_t output_cols,
                                const cs_row_feature_mask_view *m, uint32_t *d_major_ptr_out, uint32_t *live_nnz_out) {
    convert::filtered_blocked_ell_workspace ws;
    convert::init(&ws);
    if (!convert::setup(&ws, 0)) return 0;
    convert::filtered_blocked_ell_result r{};
    const device::blocked_ell_view *v = reinterpret_cast<const device::blocked_ell_view *>(src);
    int ok = convert::filter_blocked_ell_to_compressed(v, output_rows, output_cols, m->row_keep, m->feature_keep,
                                                       m->row_remap, m->feature_remap, &ws, &r);
    if (ok)
        ok = cudaStreamSynchronize(ws.stream) == cudaSuccess &&
             cudaMemcpy(d_major_ptr_out, r.filtered.majorPtr, ((std::size_t) output_rows + 1u) * 4u,
                        cudaMemcpyDeviceToDevice) == cudaSuccess;
    *live_nnz_out = r.filtered.nnz;
    convert::clear(&ws);
    return ok;
}

int csrefgpu_sliced_ell_from_compressed_cuda(const cs_host_compressed *src, unsigned int slice_rows,
                                             cs_host_sliced_ell *dst) {
    sparse::compressed s;
    sparse::init(&s, src->rows, src->cols, src->nnz, src->axis);
    s.majorPtr = src->majorPtr;
    s.minorIdx = src->minorIdx;
    s.val = reinterpret_cast<real::storage_t *>(src->val);
    sparse::sliced_ell d;
    sparse::init(&d);
    const int ok = convert::sliced_ell_from_compressed_cuda(&s, slice_rows, &d, 0, (cudaStream_t) 0);
    std::memcpy(dst, &d, sizeof(d));
    return ok;
}

} // extern "C"

namespace {
struct ev_timer {
    cudaEvent_t a = nullptr, b = nullptr;
    ev_timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~ev_timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

template <typename Call>
int time_calls(Call call, cudaStream_t stream, int warmup, int reps, float *ms_per_call) {
    int ok = 1;
    for (int i = 0; i < warmup && ok; ++i) ok = call();
    if (ok) ok = cudaStreamSynchronize(stream) == cudaSuccess;
    ev_timer t;
    cudaEventRecord(t.a, stream);
    for (int i = 0; i < reps && ok; ++i) ok = call();
    cudaEventRecord(t.b, stream);
    if (ok) ok = cudaEventSynchronize(t.b) == cudaSuccess;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, t.a, t.b);
    *ms_per_call = reps > 0 ? ms / (float) reps : 0.0f;
    return ok;
}
} // namespace

extern "C" {

int csrefgpu_transpose_timed(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *d_ptr, const uint32_t *d_idx,
                             const uint16_t *d_val, uint32_t *d_out_ptr, uint32_t *d_out_idx, uint16_t *d_out_val,
                             int warmup, int reps, float *ms_per_call) {
    cusparseHandle_t handle = 0;
    std::size_t lib_bytes = 0;
    if (!convert::cusparse_utils::acquire((cudaStream_t) 0, &handle)) return 0;
    if (cusparseCsr2cscEx2_bufferSize(handle, (int) cDim, (int) uDim, (int) nnz, d_val,
                                      reinterpret_cast<const int *>(d_ptr), reinterpret_cast<const int *>(d_idx),
                                      d_out_val, reinterpret_cast<int *>(d_out_ptr),
                                      reinterpret_cast<int *>(d_out_idx), CUDA_R_16F, CUSPARSE_ACTION_NUMERIC,
                                      CUSPARSE_INDEX_BASE_ZERO, CUSPARSE_CSR2CSC_ALG1,
                                      &lib_bytes) != CUSPARSE_STATUS_SUCCESS)
        return 0;
    void *scratch = nullptr;
    uint32_t *heads = nullptr;
    const std::size_t bytes = lib_bytes < 256u ? 256u : lib_bytes;
    if (cudaMalloc(&scratch, bytes) != cudaSuccess) return 0;
    if (cudaMalloc((void **) &heads, ((std::size_t) uDim + 1u) * 4u) != cudaSuccess) {
        cudaFree(scratch);
        return 0;
    }
    const int ok = time_calls(
        [&] {
            return convert::build_compressed_transpose_raw(cDim, uDim, nnz, d_ptr, d_idx,
                                                           reinterpret_cast<const __half *>(d_val), d_out_ptr, heads,
                                                           d_out_idx, reinterpret_cast<__half *>(d_out_val), scratch,
                                                           bytes, (cudaStream_t) 0);
        },
        (cudaStream_t) 0, warmup, reps, ms_per_call);
    cudaFree(heads);
    cudaFree(scratch);
    return ok;
}

int csrefgpu_major_nnz_plan_timed(const uint32_t *d_major_ptr, uint32_t major_dim, uint32_t *d_major_nnz,
                                  uint32_t *d_sorted, uint32_t *d_order_in, uint32_t *d_order_out,
                                  uint32_t *d_offsets, uint32_t requested, int warmup, int reps, float *ms_per_call) {
    std::size_t bytes = 0;
    if (!bucket::major_nnz_bucket_sort_scratch_bytes(major_dim, &bytes)) return 0;
    void *tmp = nullptr;
    if (cudaMalloc(&tmp, bytes < 256u ? 256u : bytes) != cudaSuccess) return 0;
    const int ok = time_calls(
        [&] {
            return bucket::build_major_nnz_bucket_plan_raw(d_major_ptr, major_dim, d_major_nnz, d_sorted, d_order_in,
                                                           d_order_out, d_offsets, requested, tmp, bytes,
                                                           (cudaStream_t) 0);
        },
        (cudaStream_t) 0, warmup, reps, ms_per_call);
    cudaFree(tmp);
    return ok;
}

int csrefgpu_group_reduce_blocked_ell_timed(const cs_blocked_ell_view *src, const uint32_t *d_masks,
                                            uint32_t group_count, const cs_row_feature_mask_view *m,
                                            const cs_group_filter_params *f, int warmup, int reps,
                                            float *ms_per_call) {
    runtime::sparse_group_reduce_workspace ws;
    runtime::init(&ws);
    if (!runtime::setup(&ws, 0)) return 0;
    runtime::group_mask_config_view groups{group_count, nullptr, d_masks};
    runtime::row_feature_mask_view mv = masks_of(m);
    runtime::sparse_group_filter_params filter{f->min_total, f->min_detected_features, f->max_group_fraction,
                                               f->fraction_group_index};
    runtime::sparse_group_reduce_result res{};
    const device::blocked_ell_view *v = reinterpret_cast<const device::blocked_ell_view *>(src);
    const int ok = time_calls([&] { return runtime::compute_sparse_group_reduce(v, &ws, &groups, &mv, &filter, &res); },
                              ws.stream, warmup, reps, ms_per_call);
    runtime::clear(&ws);
    return ok;
}


int csrefgpu_group_reduce_sliced_ell_timed(const cs_sliced_ell_view *src, const uint32_t *d_masks,
                                           uint32_t group_count, const cs_row_feature_mask_view *m,
                                           const cs_group_filter_params *f, int warmup, int reps, float *ms_per_call) {
    runtime::sparse_group_reduce_workspace ws;
    runtime::init(&ws);
    if (!runtime::setup(&ws, 0)) return 0;
    runtime::group_mask_config_view groups{group_count, nullptr, d_masks};
    runtime::row_feature_mask_view mv = masks_of(m);
    runtime::sparse_group_filter_params filter{f->min_total, f->min_detected_features, f->max_group_fraction,
                                               f->fraction_group_index};
    runtime::sparse_group_reduce_result res{};
    const device::sliced_ell_view *v = reinterpret_cast<const device::sliced_ell_view *>(src);
    const int ok = time_calls([&] { return runtime::compute_sparse_group_reduce(v, &ws, &groups, &mv, &filter, &res); },
                              ws.stream, warmup, reps, ms_per_call);
    runtime::clear(&ws);
    return ok;
}

int csrefgpu_group_reduce_compressed_timed(const cs_compressed_view *src, const uint32_t *d_masks,
                                           uint32_t group_count, const cs_row_feature_mask_view *m,
                                           const cs_group_filter_params *f, int warmup, int reps, float *ms_per_call) {
    runtime::sparse_group_reduce_workspace ws;
    runtime::init(&ws);
    if (!runtime::setup(&ws, 0)) return 0;
    runtime::group_mask_config_view groups{group_count, nullptr, d_masks};
    runtime::row_feature_mask_view mv = masks_of(m);
    runtime::sparse_group_filter_params filter{f->min_total, f->min_detected_features, f->max_group_fraction,
                                               f->fraction_group_index};
    runtime::sparse_group_reduce_result res{};
    const device::compressed_view *v = reinterpret_cast<const device::compressed_view *>(src);
    const int ok = time_calls(
        [&] { return runtime::compute_sparse_group_reduce_compressed_fallback(v, &ws, &groups, &mv, &filter, &res); },
        ws.stream, warmup, reps, ms_per_call);
    runtime::clear(&ws);
    return ok;
}

// convert::blocked_ell_from_coo_cuda / choose_blocked_ell_block_size_from_coo_cuda
// (src/convert/blocked_ell_from_coo_cuda.cuh:666,604): host COO in, host Blocked-ELL out
int csrefgpu_blocked_ell_from_coo_cuda(const cs_host_coo *src, uint32_t cols, const uint32_t *feature_to_global,
                                       unsigned int block_size, cs_host_blocked_ell *dst) {
    sparse::coo s;
    std::memcpy(&s, src, sizeof(s));
    s.storage = nullptr;
    sparse::blocked_ell d;
    sparse::init(&d);
    const int ok = convert::blocked_ell_from_coo_cuda(&s, cols, feature_to_global, block_size, &d, 0);
    std::memcpy(dst, &d, sizeof(d));
    return ok;
}

int csrefgpu_choose_blocked_ell_block_size_from_coo_cuda(const cs_host_coo *src, uint32_t cols,
                                                         const uint32_t *feature_to_global,
                                                         const unsigned int *candidates, unsigned int count,
                                                         cs_blocked_ell_tune_result *out) {
    sparse::coo s;
    std::memcpy(&s, src, sizeof(s));
    s.storage = nullptr;
    convert::blocked_ell_tune_result r{};
    const int ok =
        convert::choose_blocked_ell_block_size_from_coo_cuda(&s, cols, feature_to_global, candidates, count, 0, &r);
    out->block_size = r.block_size;
    out->fill_ratio = r.fill_ratio;
    out->padded_bytes = r.padded_bytes;
    return ok;
}

void csrefgpu_free(void *p) { std::free(p); }

} // extern "C"
