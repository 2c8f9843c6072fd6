// mask_groups runtime: masked per-row feature-group reductions and the masked
// Blocked-ELL -> CSR reoptimization.
//
// Semantics follow src/runtime/mask_groups.cu of the reference:
//   - rows whose row_keep is 0 emit zeros and keep = 0 (emit_empty_row, :81-105);
//   - a stored value counts when its column is < cols, it is nonzero and its
//     feature_keep is set (:155, :255, :338);
//   - per row: total, max, detected count, and sums over the <= 32 feature
//     groups of each column's bitmask; keep = total >= min_total and
//     detected >= min_detected and group[fraction_idx] / total <= max_fraction;
//     percentages 100 * group / total (:171-194).
// Layout of the work differs: one warp per row reads 16-byte vectors of the
// row's fp16 values (Blocked-ELL) and keeps the group sums in lane-private
// shared-memory columns (no atomics; one 32-way column sum per group at the
// end of the row) instead of shared-memory float atomics.
#include "common.cuh"

namespace csb {
namespace {

constexpr unsigned kRowWarps = 8;
constexpr unsigned kRowThreads = kRowWarps * 32;
constexpr uint32_t kStagePairs = 128; // per-warp (feature, value) staging in the Blocked-ELL reduce

struct row_acc {
    float sum;
    float vmax;
    uint32_t detected;
};

__device__ __forceinline__ bool feature_kept(const uint8_t *feature_keep, uint32_t c) {
    return feature_keep == nullptr || feature_keep[c] != 0u;
}

// Adds one participating value.  acc_col is this lane's column of the warp's
// [32 groups x 32 lanes] accumulator, or null when there are no groups.
__device__ __forceinline__ void add_value(row_acc &a, float v, uint32_t gene, const uint32_t *group_masks,
                                          uint32_t group_count, float *acc_col) {
    a.sum += v;
    a.vmax = fmaxf(a.vmax, v);
    a.detected += 1u;
    if (acc_col != nullptr) {
        uint32_t m = group_masks[gene];
        while (m != 0u) {
            const uint32_t g = __ffs(m) - 1u;
            if (g < group_count) acc_col[g * 32u] += v;
            m &= m - 1u;
        }
    }
}

// Bit q set when fp16 value q of the 8 packed in v (low half first) is
// nonzero (either sign of zero counts as zero).
__device__ __forceinline__ uint32_t nonzero_bits(const uint4 &v) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint32_t b = 0u;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t m = __vsetne2(w[i] & 0x7fff7fffu, 0u); // 1 in each nonzero half
        b |= ((m & 1u) | ((m >> 15) & 2u)) << (2 * i);
    }
    return b;
}

// add_value with the column's group mask already loaded.
__device__ __forceinline__ void add_value_masked(row_acc &a, float v, uint32_t m, uint32_t group_count,
                                                 float *acc_col) {
    a.sum += v;
    a.vmax = fmaxf(a.vmax, v);
    a.detected += 1u;
    if (acc_col != nullptr) {
        while (m != 0u) {
            const uint32_t g = __ffs(m) - 1u;
            if (g < group_count) acc_col[g * 32u] += v;
            m &= m - 1u;
        }
    }
}

// Warp epilogue shared by the three formats (mask_groups.cu:171-194).
__device__ __forceinline__ void finish_row(uint32_t row, row_acc a, float *acc_col, uint32_t group_count,
                                           const cs_group_filter_params &filter, const cs_group_reduce_out &out) {
    const unsigned lane = threadIdx.x & 31u;
    float sum = a.sum;
    float vmax = a.vmax;
    uint32_t det = a.detected;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    det = __reduce_add_sync(0xffffffffu, det);
    __syncwarp();
    float gsum = 0.0f;
    if (acc_col != nullptr && lane < group_count) {
        const float *grow = acc_col - lane + lane * 32u; // row `lane` of the accumulator
#pragma unroll 8
        for (unsigned k = 0; k < 32u; ++k) gsum += grow[(k + lane) & 31u];
    }
    float frac_num = 0.0f;
    if (filter.fraction_group_index < group_count)
        frac_num = __shfl_sync(0xffffffffu, gsum, filter.fraction_group_index & 31u);
    if (lane == 0u) {
        out.row_totals[row] = sum;
        out.max_values[row] = vmax;
        out.detected_features[row] = det;
        const float frac = sum > 0.0f ? __fdiv_rn(frac_num, sum) : 0.0f;
        out.row_keep[row] = (uint8_t) (sum >= filter.min_total && det >= filter.min_detected_features &&
                                       frac <= filter.max_group_fraction);
    }
    if (out.group_counts != nullptr && out.group_percentages != nullptr && lane < group_count) {
        const std::size_t o = (std::size_t) row * group_count + lane;
        out.group_counts[o] = gsum;
        out.group_percentages[o] = sum > 0.0f ? __fdiv_rn(__fmul_rn(100.0f, gsum), sum) : 0.0f;
    }
    __syncwarp();
}

__device__ __forceinline__ void empty_row(uint32_t row, uint32_t group_count, const cs_group_reduce_out &out) {
    const unsigned lane = threadIdx.x & 31u;
    if (lane == 0u) {
        out.row_totals[row] = 0.0f;
        out.detected_features[row] = 0u;
        out.max_values[row] = 0.0f;
        out.row_keep[row] = 0u;
    }
    if (out.group_counts != nullptr && out.group_percentages != nullptr) {
        for (uint32_t g = lane; g < group_count; g += 32u) {
            const std::size_t o = (std::size_t) row * group_count + g;
            out.group_counts[o] = 0.0f;
            out.group_percentages[o] = 0.0f;
        }
    }
}

__device__ __forceinline__ float *warp_acc_column(float *smem, bool groups) {
    if (!groups) return nullptr;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    return smem + (std::size_t) warp * 1024u + lane; // [group][lane] -> g * 32 + lane
}

__device__ __forceinline__ void zero_acc(float *acc_col) {
    if (acc_col == nullptr) return;
#pragma unroll 8
    for (unsigned g = 0; g < 32u; ++g) acc_col[g * 32u] = 0.0f;
    __syncwarp();
}

template <bool VEC>
__global__ void __launch_bounds__(kRowThreads) group_reduce_bell_kernel(cs_blocked_ell_view src,
                                                                         const uint32_t *__restrict__ group_masks,
                                                                         uint32_t group_count,
                                                                         cs_row_feature_mask_view masks,
                                                                         cs_group_filter_params filter,
                                                                         cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    const bool groups = group_masks != nullptr && group_count != 0u;
    float *acc_col = warp_acc_column(gr_smem, groups);
    // staging pairs follow the accumulator columns (if any)
    uint2 *stage = reinterpret_cast<uint2 *>(gr_smem + (groups ? kRowWarps * 1024u : 0u)) +
                   (threadIdx.x >> 5) * kStagePairs;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t B = src.block_size;
    const uint32_t W = B != 0u ? src.ell_cols / B : 0u;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        zero_acc(acc_col);
        row_acc a{0.0f, 0.0f, 0u};
        const uint32_t rb = B != 0u ? row / B : 0u;
        const uint32_t *bci = src.blockColIdx + (std::size_t) rb * W;
        const uint16_t *vrow = src.val + (std::size_t) row * src.ell_cols;
        if (VEC) {
            // U 16-byte vectors of values in flight per lane, loaded whether or
            // not their slot is padding (they lie inside the row) so no value
            // load waits for its block column.  The lane's nonzero values of
            // the U vectors become a 32-bit mask; the warp compacts them
            // (exclusive scan of the lanes' counts) into a per-warp staging
            // buffer of (value, feature) pairs and then works through the pairs
            // 32 at a time with every lane busy, instead of every lane stepping
            // through all its slots while most of them hold zeros.
            constexpr unsigned U = 4;
            for (uint32_t base = lane * 8u; base < src.ell_cols; base += 256u * U) {
                uint4 v[U];
                uint32_t bc[U], gene0[U];
#pragma unroll
                for (unsigned u = 0; u < U; ++u) {
                    const uint32_t e0 = base + u * 256u;
                    const bool in = e0 < src.ell_cols;
                    v[u] = in ? ld_stream_v4(vrow + e0) : make_uint4(0u, 0u, 0u, 0u);
                    bc[u] = in ? __ldg(bci + e0 / B) : CS_INVALID_COL;
                }
                // the feature flags are checked per staged value, not per vector
                uint32_t nzall = 0u;
#pragma unroll
                for (unsigned u = 0; u < U; ++u) {
                    const uint32_t e0 = base + u * 256u;
                    gene0[u] = bc[u] * B + (e0 % B);
                    if (bc[u] == CS_INVALID_COL) continue;
                    uint32_t nz = nonzero_bits(v[u]);
                    if (nz != 0u && gene0[u] + 8u > src.cols) {
                        const uint32_t lim = gene0[u] < src.cols ? src.cols - gene0[u] : 0u; // < 8 here
                        nz &= (1u << lim) - 1u;
                    }
                    nzall |= nz << (8u * u);
                }
                const uint32_t cnt = __popc(nzall);
                const uint32_t incl = warp_inclusive_scan(cnt);
                const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                const uint32_t excl = incl - cnt;
                for (uint32_t p0 = 0; p0 < total; p0 += kStagePairs) {
                    uint32_t bits = nzall, k = excl;
                    while (bits != 0u && k < p0 + kStagePairs) {
                        const uint32_t bitpos = __ffs(bits) - 1u;
                        bits &= bits - 1u;
                        if (k >= p0) {
                            const uint32_t u = bitpos >> 3, q = bitpos & 7u;
                            const uint4 vu = u < 2u ? (u == 0u ? v[0] : v[1]) : (u == 2u ? v[2] : v[3]);
                            const uint32_t g0 = u < 2u ? (u == 0u ? gene0[0] : gene0[1])
                                                       : (u == 2u ? gene0[2] : gene0[3]);
                            const uint32_t wq = q < 4u ? (q < 2u ? vu.x : vu.y) : (q < 6u ? vu.z : vu.w);
                            stage[k - p0] = make_uint2(g0 + q, (wq >> ((q & 1u) * 16u)) & 0xffffu);
                        }
                        ++k;
                    }
                    __syncwarp();
                    const uint32_t n = min(kStagePairs, total - p0);
                    for (uint32_t i = lane; i < n; i += 32u) {
                        const uint2 pr = stage[i];
                        if (!feature_kept(masks.feature_keep, pr.x)) continue;
                        const uint32_t m = acc_col != nullptr ? __ldg(group_masks + pr.x) : 0u;
                        add_value_masked(a, h2f((uint16_t) pr.y), m, group_count, acc_col);
                    }
                    __syncwarp();
                }
            }
        } else {
            for (uint32_t e = lane; e < src.ell_cols; e += 32u) {
                const uint32_t slot = e / B;
                const uint32_t bc = W != 0u ? bci[slot] : CS_INVALID_COL;
                const uint32_t gene = bc != CS_INVALID_COL ? bc * B + (e - slot * B) : src.cols;
                const uint16_t h = vrow[e];
                if (half_nonzero(h) && gene < src.cols && feature_kept(masks.feature_keep, gene))
                    add_value(a, h2f(h), gene, group_masks, group_count, acc_col);
            }
        }
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

__device__ __forceinline__ uint32_t find_slice(const cs_sliced_ell_view &src, uint32_t row) {
    if (src.slice_rows == 32u) return min(row >> 5, src.slice_count - 1u);
    if (src.slice_rows != 0u) return min(row / src.slice_rows, src.slice_count - 1u);
    // last slice whose start is <= row (the reference's linear walk, as a search)
    uint32_t lo = 0u, hi = src.slice_count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (row >= src.slice_row_offsets[mid])
            lo = mid;
        else
            hi = mid - 1u;
    }
    return lo;
}

__global__ void __launch_bounds__(kRowThreads) group_reduce_sell_kernel(cs_sliced_ell_view src,
                                                                         const uint32_t *__restrict__ group_masks,
                                                                         uint32_t group_count,
                                                                         cs_row_feature_mask_view masks,
                                                                         cs_group_filter_params filter,
                                                                         cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    const bool groups = group_masks != nullptr && group_count != 0u;
    float *acc_col = warp_acc_column(gr_smem, groups);
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        zero_acc(acc_col);
        row_acc a{0.0f, 0.0f, 0u};
        uint32_t width = 0u;
        std::size_t slot_base = 0u;
        if (src.slice_count != 0u) {
            const uint32_t slice = find_slice(src, row);
            width = src.slice_widths[slice];
            slot_base = (std::size_t) src.slice_slot_offsets[slice] +
                        (std::size_t) (row - src.slice_row_offsets[slice]) * width;
        }
        for (uint32_t k = lane; k < width; k += 32u) {
            const uint32_t col = src.col_idx[slot_base + k];
            const uint16_t h = src.val[slot_base + k];
            if (col < src.cols && half_nonzero(h) && feature_kept(masks.feature_keep, col))
                add_value(a, h2f(h), col, group_masks, group_count, acc_col);
        }
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

__global__ void __launch_bounds__(kRowThreads) group_reduce_csr_kernel(cs_compressed_view src,
                                                                        const uint32_t *__restrict__ group_masks,
                                                                        uint32_t group_count,
                                                                        cs_row_feature_mask_view masks,
                                                                        cs_group_filter_params filter,
                                                                        cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    const bool groups = group_masks != nullptr && group_count != 0u;
    float *acc_col = warp_acc_column(gr_smem, groups);
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        zero_acc(acc_col);
        row_acc a{0.0f, 0.0f, 0u};
        const uint32_t b = src.majorPtr[row], e = src.majorPtr[row + 1u];
        for (uint32_t i = b + lane; i < e; i += 32u) {
            const uint32_t col = src.minorIdx[i];
            const uint16_t h = src.val[i];
            if (col < src.cols && half_nonzero(h) && feature_kept(masks.feature_keep, col))
                add_value(a, h2f(h), col, group_masks, group_count, acc_col);
        }
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

unsigned row_grid(uint32_t rows) {
    uint32_t g = (rows + kRowWarps - 1u) / kRowWarps;
    const uint32_t cap = (uint32_t) sm_count() * 16u;
    if (g > cap) g = cap;
    return g == 0u ? 1u : g;
}

int check_common(uint32_t group_count, const cs_group_filter_params *filter, const cs_group_reduce_out *out,
                 const char *who) {
    if (filter == nullptr || out == nullptr) {
        set_error("%s: null filter or output", who);
        return 0;
    }
    if (group_count > CS_MAX_MASK_GROUPS) {
        set_error("%s: group_count %u exceeds %u", who, group_count, CS_MAX_MASK_GROUPS);
        return 0;
    }
    if (out->row_totals == nullptr || out->detected_features == nullptr || out->max_values == nullptr ||
        out->row_keep == nullptr) {
        set_error("%s: per-row outputs are required", who);
        return 0;
    }
    return 1;
}

std::size_t group_smem(const uint32_t *masks, uint32_t group_count) {
    return (masks != nullptr && group_count != 0u) ? kRowWarps * 1024u * sizeof(float) : 0u;
}

// ---------------------------------------------------------------------------
// Reoptimize: masked Blocked-ELL -> CSR.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool reopt_keep(const cs_blocked_ell_view &src, const cs_row_feature_mask_view &masks,
                                           uint32_t output_cols, uint16_t h, uint32_t gene, uint32_t *out_col) {
    if (!(half_nonzero(h) && gene < src.cols && feature_kept(masks.feature_keep, gene))) return false;
    const uint32_t oc = masks.feature_remap != nullptr ? masks.feature_remap[gene] : gene;
    *out_col = oc;
    return oc < output_cols;
}

template <bool EMIT>
__global__ void __launch_bounds__(kRowThreads) reopt_kernel(cs_blocked_ell_view src, cs_row_feature_mask_view masks,
                                                            uint32_t output_rows, uint32_t output_cols,
                                                            uint32_t *__restrict__ major_ptr,
                                                            uint32_t *__restrict__ claims,
                                                            uint32_t *__restrict__ minor_idx,
                                                            uint16_t *__restrict__ out_val, uint32_t *status) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t B = src.block_size;
    const uint32_t W = B != 0u ? src.ell_cols / B : 0u;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) continue;
        const uint32_t out_row = masks.row_remap != nullptr ? masks.row_remap[row] : row;
        if (out_row >= output_rows) continue;
        const uint32_t rb = B != 0u ? row / B : 0u;
        const uint32_t *bci = src.blockColIdx + (std::size_t) rb * W;
        const uint16_t *vrow = src.val + (std::size_t) row * src.ell_cols;
        uint32_t run = EMIT ? major_ptr[out_row] : 0u;
        // entries past the row's end (only possible when two rows remap to one
        // output row, which the count pass flags) are dropped, never written
        const uint32_t end = EMIT ? major_ptr[out_row + 1u] : 0u;
        for (uint32_t e0 = 0; e0 < src.ell_cols; e0 += 32u) {
            const uint32_t e = e0 + lane;
            uint32_t oc = 0u;
            uint16_t h = 0u;
            bool k = false;
            if (e < src.ell_cols) {
                const uint32_t slot = e / B;
                const uint32_t bc = bci[slot];
                if (bc != CS_INVALID_COL) {
                    h = vrow[e];
                    k = reopt_keep(src, masks, output_cols, h, bc * B + (e - slot * B), &oc);
                }
            }
            const uint32_t ballot = __ballot_sync(0xffffffffu, k);
            if (EMIT && k) {
                const uint32_t pos = run + __popc(ballot & ((1u << lane) - 1u));
                if (pos < end) {
                    minor_idx[pos] = oc;
                    out_val[pos] = h;
                }
            }
            run += __popc(ballot);
        }
        if (!EMIT && lane == 0u) {
            major_ptr[out_row] = run;
            if (atomicAdd(claims + out_row, 1u) != 0u) status_or(status, CS_STATUS_REMAP_COLLISION);
        }
    }
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_group_reduce_blocked_ell(const cs_blocked_ell_view *src, const uint32_t *d_feature_group_masks,
                                                uint32_t group_count, const cs_row_feature_mask_view *masks,
                                                const cs_group_filter_params *filter, const cs_group_reduce_out *out,
                                                cs_stream_t s) {
    if (src == nullptr || !check_common(group_count, filter, out, "group_reduce_blocked_ell")) {
        if (src == nullptr) set_error("group_reduce_blocked_ell: null view");
        return 0;
    }
    if (src->rows == 0u) return 1;
    if (src->block_size == 0u && src->ell_cols != 0u) {
        set_error("group_reduce_blocked_ell: zero block size");
        return 0;
    }
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    const bool vec = src->block_size != 0u && src->block_size % 8u == 0u &&
                     (reinterpret_cast<uintptr_t>(src->val) & 15u) == 0u;
    const std::size_t smem = group_smem(d_feature_group_masks, group_count) +
                             (vec ? (std::size_t) kRowWarps * kStagePairs * sizeof(uint2) : 0u);
    if (vec)
        group_reduce_bell_kernel<true><<<row_grid(src->rows), kRowThreads, smem, as_stream(s)>>>(
            *src, d_feature_group_masks, group_count, m, *filter, *out);
    else
        group_reduce_bell_kernel<false><<<row_grid(src->rows), kRowThreads, smem, as_stream(s)>>>(
            *src, d_feature_group_masks, group_count, m, *filter, *out);
    return launch_ok("group_reduce_bell_kernel");
}

extern "C" int cs_b200_group_reduce_sliced_ell(const cs_sliced_ell_view *src, const uint32_t *d_feature_group_masks,
                                               uint32_t group_count, const cs_row_feature_mask_view *masks,
                                               const cs_group_filter_params *filter, const cs_group_reduce_out *out,
                                               cs_stream_t s) {
    if (src == nullptr || !check_common(group_count, filter, out, "group_reduce_sliced_ell")) {
        if (src == nullptr) set_error("group_reduce_sliced_ell: null view");
        return 0;
    }
    if (src->rows == 0u) return 1;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    group_reduce_sell_kernel<<<row_grid(src->rows), kRowThreads, group_smem(d_feature_group_masks, group_count),
                               as_stream(s)>>>(*src, d_feature_group_masks, group_count, m, *filter, *out);
    return launch_ok("group_reduce_sell_kernel");
}

extern "C" int cs_b200_group_reduce_compressed(const cs_compressed_view *src, const uint32_t *d_feature_group_masks,
                                               uint32_t group_count, const cs_row_feature_mask_view *masks,
                                               const cs_group_filter_params *filter, const cs_group_reduce_out *out,
                                               cs_stream_t s) {
    if (src == nullptr || !check_common(group_count, filter, out, "group_reduce_compressed")) {
        if (src == nullptr) set_error("group_reduce_compressed: null view");
        return 0;
    }
    if (src->axis != CS_COMPRESSED_BY_ROW) {
        set_error("group_reduce_compressed: source must be compressed by row");
        return 0;
    }
    if (src->rows == 0u) return 1;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    group_reduce_csr_kernel<<<row_grid(src->rows), kRowThreads, group_smem(d_feature_group_masks, group_count),
                              as_stream(s)>>>(*src, d_feature_group_masks, group_count, m, *filter, *out);
    return launch_ok("group_reduce_csr_kernel");
}

extern "C" int cs_b200_reoptimize_scratch_bytes(uint32_t src_rows, uint32_t output_rows, size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("reoptimize_scratch_bytes: null output");
        return 0;
    }
    (void) src_rows;
    *out_bytes = align_up((std::size_t) output_rows * sizeof(uint32_t) + 16u, 256) +
                 scan_u32_scratch_bytes((std::size_t) output_rows);
    return 1;
}

extern "C" int cs_b200_reoptimize_count(const cs_blocked_ell_view *src, const cs_row_feature_mask_view *masks,
                                        uint32_t output_rows, uint32_t output_cols, uint32_t *d_major_ptr,
                                        void *d_scratch, size_t scratch_bytes, uint32_t *d_status, cs_stream_t s) {
    if (src == nullptr || d_major_ptr == nullptr) {
        set_error("reoptimize_count: null view or major_ptr");
        return 0;
    }
    if (src->block_size == 0u && src->ell_cols != 0u) {
        set_error("reoptimize_count: zero block size");
        return 0;
    }
    size_t need = 0;
    cs_b200_reoptimize_scratch_bytes(src->rows, output_rows, &need);
    if (d_scratch == nullptr || scratch_bytes < need) {
        set_error("reoptimize_count: scratch %zu < %zu", scratch_bytes, need);
        return 0;
    }
    cudaStream_t stream = as_stream(s);
    uint32_t *claims = (uint32_t *) d_scratch;
    void *scan_scratch = (char *) d_scratch + align_up((std::size_t) output_rows * sizeof(uint32_t) + 16u, 256);
    if (!cuda_ok(cudaMemsetAsync(d_major_ptr, 0, ((std::size_t) output_rows + 1u) * sizeof(uint32_t), stream),
                 "memset major_ptr") ||
        !cuda_ok(cudaMemsetAsync(claims, 0, (std::size_t) output_rows * sizeof(uint32_t) + 4u, stream),
                 "memset claims"))
        return 0;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    if (src->rows != 0u && output_rows != 0u) {
        reopt_kernel<false><<<row_grid(src->rows), kRowThreads, 0, stream>>>(*src, m, output_rows, output_cols,
                                                                            d_major_ptr, claims, nullptr, nullptr,
                                                                            d_status);
        if (!launch_ok("reopt_count_kernel")) return 0;
    }
    return scan_exclusive_u32(d_major_ptr, d_major_ptr, output_rows, true, scan_scratch,
                              scan_u32_scratch_bytes(output_rows), stream);
}

extern "C" int cs_b200_reoptimize_emit(const cs_blocked_ell_view *src, const cs_row_feature_mask_view *masks,
                                       uint32_t output_rows, uint32_t output_cols, const uint32_t *d_major_ptr,
                                       uint32_t *d_minor_idx, uint16_t *d_val, cs_stream_t s) {
    if (src == nullptr || d_major_ptr == nullptr) {
        set_error("reoptimize_emit: null view or major_ptr");
        return 0;
    }
    if (src->rows == 0u || output_rows == 0u) return 1;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    reopt_kernel<true><<<row_grid(src->rows), kRowThreads, 0, as_stream(s)>>>(
        *src, m, output_rows, output_cols, const_cast<uint32_t *>(d_major_ptr), nullptr, d_minor_idx, d_val, nullptr);
    return launch_ok("reopt_emit_kernel");
}
