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
#include "bell_vec.cuh"

#include <cstring>
#include <type_traits>

namespace csb {
namespace {

constexpr unsigned kRowWarps = 8;
constexpr unsigned kRowThreads = kRowWarps * 32;
constexpr uint32_t kStagePairs = 128; // per-warp (feature, value) staging in the Blocked-ELL reduce
#ifndef PIPE_WIDE_WARPS
#define PIPE_WIDE_WARPS 24u // warps of the many-warp Blocked-ELL-16 pipe
#endif

// Per-lane running values of one row.  The group sums live in registers:
// GR (8, 16 or 32, or 0 without groups) accumulators updated with one
// predicated add per group for every value, so lanes whose masks have
// different numbers of bits do not serialise the warp on a per-bit loop.
// They reach shared memory once per row (finish_row).
template <unsigned GR>
struct row_acc {
    float sum;
    float vmax;
    uint32_t detected;
    float g[GR != 0u ? GR : 1u];
};

template <unsigned GR>
__device__ __forceinline__ void init_acc(row_acc<GR> &a) {
    a.sum = 0.0f;
    a.vmax = 0.0f;
    a.detected = 0u;
#pragma unroll
    for (unsigned k = 0; k < (GR != 0u ? GR : 1u); ++k) a.g[k] = 0.0f;
}

__device__ __forceinline__ bool feature_kept(const uint8_t *feature_keep, uint32_t c) {
    return feature_keep == nullptr || feature_keep[c] != 0u;
}

// Adds one participating value whose column has group mask m.  Bits at or
// above the call's group count land in accumulators that are never written
// out, so they are ignored as the reference ignores them.
template <unsigned GR>
__device__ __forceinline__ void add_value_masked(row_acc<GR> &a, float v, uint32_t m) {
    a.sum += v;
    a.vmax = fmaxf(a.vmax, v);
    a.detected += 1u;
    if constexpr (GR != 0u) {
#pragma unroll
        for (unsigned k = 0; k < GR; ++k)
            if ((m >> k) & 1u) a.g[k] += v;
    }
}

template <unsigned GR>
__device__ __forceinline__ void add_value(row_acc<GR> &a, float v, uint32_t gene, const uint32_t *group_masks) {
    add_value_masked(a, v, GR != 0u ? __ldg(group_masks + gene) : 0u);
}

// Warp epilogue shared by the three formats (mask_groups.cu:171-194).
// acc_col is this lane's column of the warp's [group_count x 32 lanes]
// shared block (null without groups): the lanes' group sums are written
// there and each group's 32 partial sums are added by lane `group`.
template <unsigned GR>
__device__ __forceinline__ void finish_row(uint32_t row, const row_acc<GR> &a, float *acc_col,
                                           uint32_t group_count, const cs_group_filter_params &filter,
                                           const cs_group_reduce_out &out) {
    const unsigned lane = threadIdx.x & 31u;
    if constexpr (GR != 0u) {
#pragma unroll
        for (unsigned k = 0; k < GR; ++k)
            if (k < group_count) acc_col[k * 32u] = a.g[k];
    }
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

// Each warp owns group_count rows of 32 lane columns (group_count <= 32), so
// a call with few groups leaves most of the SM's shared memory to L1, where
// the column mask and feature tables are gathered from.
__device__ __forceinline__ float *warp_acc_column(float *smem, bool groups, uint32_t group_count) {
    if (!groups) return nullptr;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    return smem + (std::size_t) warp * group_count * 32u + lane; // [group][lane] -> g * 32 + lane
}

// One stored (column, value) pair of a compressed or Sliced-ELL row.
template <unsigned GR>
__device__ __forceinline__ void add_entry(row_acc<GR> &a, uint32_t col, uint32_t h, uint32_t cols,
                                          const uint8_t *feature_keep, const uint32_t *group_masks) {
    if (col < cols && (h & 0x7fffu) != 0u && feature_kept(feature_keep, col))
        add_value(a, h2f((uint16_t) h), col, group_masks);
}

// Reduces the entries [b, e) of one row held as parallel column / fp16 arrays
// (a CSR row, or one Sliced-ELL row's slots).  The body moves through aligned
// quads: per lane U 16-byte column vectors and U 8-byte value vectors are in
// flight before any is used, and the column flags and group masks of all 4U
// entries are gathered before the accumulation.  The unaligned head (< 4
// entries) runs on lanes 0-2 and the tail (< 4) on lanes 3-5.  Requires idx
// 16-byte and val 8-byte aligned.
template <unsigned U, unsigned GR>
__device__ __forceinline__ void reduce_span(const uint32_t *__restrict__ idx, const uint16_t *__restrict__ val,
                                            std::size_t b, std::size_t e, uint32_t cols,
                                            const uint8_t *__restrict__ feature_keep,
                                            const uint32_t *__restrict__ group_masks, row_acc<GR> &a) {
    const unsigned lane = threadIdx.x & 31u;
    const std::size_t a4 = min(e, (b + 3u) & ~(std::size_t) 3u);
    const std::size_t e4 = max(a4, e & ~(std::size_t) 3u);
    {
        const std::size_t i = lane < 3u ? b + lane : e4 + (lane - 3u);
        if (lane < 3u ? i < a4 : (lane < 6u && i < e))
            add_entry(a, __ldg(idx + i), __ldg(val + i), cols, feature_keep, group_masks);
    }
    const std::size_t q_end = e4 >> 2;
    for (std::size_t q = (a4 >> 2) + lane; q < q_end; q += 32u * U) {
        uint4 c[U];
        uint2 h[U];
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const std::size_t qi = q + 32u * u;
            const bool in = qi < q_end;
            c[u] = in ? ld_stream_v4(idx + qi * 4u) : make_uint4(cols, cols, cols, cols);
            h[u] = in ? ld_stream_v2(val + qi * 4u) : make_uint2(0u, 0u);
        }
        uint32_t col[4 * U], hv[4 * U], m[4 * U];
        bool ok[4 * U];
        bool any = false;
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            col[4 * u + 0] = c[u].x;
            col[4 * u + 1] = c[u].y;
            col[4 * u + 2] = c[u].z;
            col[4 * u + 3] = c[u].w;
            hv[4 * u + 0] = h[u].x & 0xffffu;
            hv[4 * u + 1] = h[u].x >> 16;
            hv[4 * u + 2] = h[u].y & 0xffffu;
            hv[4 * u + 3] = h[u].y >> 16;
            any = any || ((h[u].x | h[u].y) & 0x7fff7fffu) != 0u;
        }
        // quads of zeros (Sliced-ELL padding past a row's end) skip the gathers
        if (!any) continue;
#pragma unroll
        for (unsigned j = 0; j < 4 * U; ++j) {
            ok[j] = col[j] < cols && (hv[j] & 0x7fffu) != 0u;
            ok[j] = ok[j] && (feature_keep == nullptr || __ldg(feature_keep + col[j]) != 0u);
            m[j] = ok[j] && GR != 0u ? __ldg(group_masks + col[j]) : 0u;
        }
#pragma unroll
        for (unsigned j = 0; j < 4 * U; ++j)
            if (ok[j]) add_value_masked(a, h2f((uint16_t) hv[j]), m[j]);
    }
}

// Column codes in shared memory for the compressed reduce with at most 15
// groups: bit 15 = the column is kept, bits 0..14 its groups
// (bits at or above the group count cleared).  One 2-byte shared read per
// entry replaces two global gathers (the feature flag and the group mask) that
// touch ~32 distinct cache lines per warp for a row's sorted columns.
__device__ __forceinline__ void build_col_codes(uint16_t *tbl, uint32_t cols, const uint8_t *__restrict__ feature_keep,
                                                const uint32_t *__restrict__ group_masks, uint32_t gmask) {
    for (uint32_t c = threadIdx.x; c < cols; c += blockDim.x) {
        uint32_t e = 0u;
        if (feature_kept(feature_keep, c)) e = 0x8000u | (group_masks != nullptr ? __ldg(group_masks + c) & gmask : 0u);
        tbl[c] = (uint16_t) e;
    }
    __syncthreads();
}

// reduce_span with the column codes: same quads, loads in flight and
// head / tail handling.
template <unsigned U, unsigned GR>
__device__ __forceinline__ void reduce_span_codes(const uint32_t *__restrict__ idx, const uint16_t *__restrict__ val,
                                                  std::size_t b, std::size_t e, uint32_t cols,
                                                  const uint16_t *__restrict__ tbl, row_acc<GR> &a) {
    const unsigned lane = threadIdx.x & 31u;
    const std::size_t a4 = min(e, (b + 3u) & ~(std::size_t) 3u);
    const std::size_t e4 = max(a4, e & ~(std::size_t) 3u);
    {
        const std::size_t i = lane < 3u ? b + lane : e4 + (lane - 3u);
        if (lane < 3u ? i < a4 : (lane < 6u && i < e)) {
            const uint32_t col = __ldg(idx + i);
            const uint32_t h = __ldg(val + i);
            if (col < cols && (h & 0x7fffu) != 0u) {
                const uint32_t code = tbl[col];
                if (code & 0x8000u) add_value_masked(a, h2f((uint16_t) h), code & 0x7fffu);
            }
        }
    }
    const std::size_t q_end = e4 >> 2;
    for (std::size_t q = (a4 >> 2) + lane; q < q_end; q += 32u * U) {
        uint4 c[U];
        uint2 h[U];
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const std::size_t qi = q + 32u * u;
            const bool in = qi < q_end;
            c[u] = in ? ld_stream_v4(idx + qi * 4u) : make_uint4(cols, cols, cols, cols);
            h[u] = in ? ld_stream_v2(val + qi * 4u) : make_uint2(0u, 0u);
        }
        uint32_t col[4 * U], hv[4 * U], code[4 * U];
        bool any = false;
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            col[4 * u + 0] = c[u].x;
            col[4 * u + 1] = c[u].y;
            col[4 * u + 2] = c[u].z;
            col[4 * u + 3] = c[u].w;
            hv[4 * u + 0] = h[u].x & 0xffffu;
            hv[4 * u + 1] = h[u].x >> 16;
            hv[4 * u + 2] = h[u].y & 0xffffu;
            hv[4 * u + 3] = h[u].y >> 16;
            any = any || ((h[u].x | h[u].y) & 0x7fff7fffu) != 0u;
        }
        if (!any) continue;
#pragma unroll
        for (unsigned j = 0; j < 4 * U; ++j)
            code[j] = (col[j] < cols && (hv[j] & 0x7fffu) != 0u) ? (uint32_t) tbl[col[j]] : 0u;
#pragma unroll
        for (unsigned j = 0; j < 4 * U; ++j)
            if (code[j] & 0x8000u) add_value_masked(a, h2f((uint16_t) hv[j]), code[j] & 0x7fffu);
    }
}

// One Blocked-ELL row, warp-wide (reads, accumulation and outputs).
template <bool VEC, unsigned GR>
__device__ __forceinline__ void bell_row(const cs_blocked_ell_view &src, uint32_t row,
                                         const uint32_t *__restrict__ group_masks, uint32_t group_count,
                                         const cs_row_feature_mask_view &masks, const cs_group_filter_params &filter,
                                         const cs_group_reduce_out &out, float *acc_col, uint2 *stage) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t B = src.block_size;
    const uint32_t W = B != 0u ? src.ell_cols / B : 0u;
    if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
        empty_row(row, group_count, out);
        return;
    }
    row_acc<GR> a;
    init_acc(a);
    const uint32_t rb = B != 0u ? row / B : 0u;
    const block_div bd(B);
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
                bc[u] = in ? __ldg(bci + bd.div(e0)) : CS_INVALID_COL;
            }
            // the feature flags are checked per staged value, not per vector
            uint32_t nzall = 0u;
    #pragma unroll
            for (unsigned u = 0; u < U; ++u) {
                const uint32_t e0 = base + u * 256u;
                gene0[u] = bc[u] * B + bd.mod(e0);
                if (bc[u] == CS_INVALID_COL) continue;
                uint32_t nz = live_bits8(v[u]);
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
                    const uint32_t m = GR != 0u ? __ldg(group_masks + pr.x) : 0u;
                    add_value_masked(a, h2f((uint16_t) pr.y), m);
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
                add_value(a, h2f(h), gene, group_masks);
        }
    }
    __syncwarp();
    finish_row(row, a, acc_col, group_count, filter, out);
}

template <bool VEC, unsigned GR>
__global__ void __launch_bounds__(kRowThreads) group_reduce_bell_kernel(cs_blocked_ell_view src,
                                                                         const uint32_t *__restrict__ group_masks,
                                                                         uint32_t group_count,
                                                                         cs_row_feature_mask_view masks,
                                                                         cs_group_filter_params filter,
                                                                         cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    float *acc_col = warp_acc_column(gr_smem, GR != 0u, group_count);
    // staging pairs follow the accumulator columns (if any)
    uint2 *stage = reinterpret_cast<uint2 *>(gr_smem + (GR != 0u ? kRowWarps * group_count * 32u : 0u)) +
                   (threadIdx.x >> 5) * kStagePairs;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps)
        bell_row<VEC, GR>(src, row, group_masks, group_count, masks, filter, out, acc_col, stage);
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

// VEC: col_idx 16-byte and val 8-byte aligned; the row's slots go through
// reduce_span.  Padding slots hold a column >= cols and are skipped there.
template <bool VEC, unsigned GR, unsigned U = 2>
__global__ void __launch_bounds__(kRowThreads) group_reduce_sell_kernel(cs_sliced_ell_view src,
                                                                         const uint32_t *__restrict__ group_masks,
                                                                         uint32_t group_count,
                                                                         cs_row_feature_mask_view masks,
                                                                         cs_group_filter_params filter,
                                                                         cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    float *acc_col = warp_acc_column(gr_smem, GR != 0u, group_count);
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        row_acc<GR> a;
        init_acc(a);
        uint32_t width = 0u;
        std::size_t slot_base = 0u;
        if (src.slice_count != 0u) {
            const uint32_t slice = find_slice(src, row);
            width = src.slice_widths[slice];
            slot_base = (std::size_t) src.slice_slot_offsets[slice] +
                        (std::size_t) (row - src.slice_row_offsets[slice]) * width;
        }
        if (VEC) {
            reduce_span<U>(src.col_idx, src.val, slot_base, slot_base + width, src.cols, masks.feature_keep,
                           group_masks, a);
        } else {
            for (uint32_t k = lane; k < width; k += 32u)
                add_entry(a, src.col_idx[slot_base + k], src.val[slot_base + k], src.cols, masks.feature_keep,
                          group_masks);
        }
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

template <bool VEC, unsigned GR, unsigned U = 2>
__global__ void __launch_bounds__(kRowThreads) group_reduce_csr_kernel(cs_compressed_view src,
                                                                        const uint32_t *__restrict__ group_masks,
                                                                        uint32_t group_count,
                                                                        cs_row_feature_mask_view masks,
                                                                        cs_group_filter_params filter,
                                                                        cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    float *acc_col = warp_acc_column(gr_smem, GR != 0u, group_count);
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        row_acc<GR> a;
        init_acc(a);
        const uint32_t b = src.majorPtr[row], e = src.majorPtr[row + 1u];
        if (VEC) {
            reduce_span<U>(src.minorIdx, src.val, b, e, src.cols, masks.feature_keep, group_masks, a);
        } else {
            for (uint32_t i = b + lane; i < e; i += 32u)
                add_entry(a, src.minorIdx[i], src.val[i], src.cols, masks.feature_keep, group_masks);
        }
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

// The compressed reduce over shared-memory column codes (at most 15 groups,
// the code table in shared memory after the accumulators; minorIdx 16-byte
// and val 8-byte aligned).  A CTA of kCodesWarps warps shares one table:
// 32 warps per SM instead of the 24 that 8-warp CTAs with a table each allow
// (CSR on 500,000 x 32,768: 0.86 ms against 1.18 ms).
constexpr unsigned kCodesWarps = 32; // warps of a code-table CTA (they share one table)

template <unsigned GR, unsigned U = 4>
__global__ void __launch_bounds__(kCodesWarps * 32) group_reduce_csr_codes_kernel(cs_compressed_view src,
                                                                              const uint32_t *__restrict__ group_masks,
                                                                              uint32_t group_count,
                                                                              cs_row_feature_mask_view masks,
                                                                              cs_group_filter_params filter,
                                                                              cs_group_reduce_out out) {
    extern __shared__ __align__(16) float gr_smem[];
    float *acc_col = warp_acc_column(gr_smem, GR != 0u, group_count);
    uint16_t *tbl = reinterpret_cast<uint16_t *>(gr_smem + (GR != 0u ? kCodesWarps * group_count * 32u : 0u));
    build_col_codes(tbl, src.cols, masks.feature_keep, GR != 0u ? group_masks : nullptr,
                    GR != 0u ? (1u << group_count) - 1u : 0u);
    for (uint32_t row = blockIdx.x * kCodesWarps + (threadIdx.x >> 5); row < src.rows;
         row += gridDim.x * kCodesWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        row_acc<GR> a;
        init_acc(a);
        reduce_span_codes<U>(src.minorIdx, src.val, src.majorPtr[row], src.majorPtr[row + 1u], src.cols, tbl, a);
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

// The Sliced-ELL twin (slots of the row's slice; padding quads skip the table).
template <unsigned GR, unsigned U = 2>
__global__ void __launch_bounds__(kCodesWarps * 32) group_reduce_sell_codes_kernel(cs_sliced_ell_view src,
                                                                               const uint32_t *__restrict__ group_masks,
                                                                               uint32_t group_count,
                                                                               cs_row_feature_mask_view masks,
                                                                               cs_group_filter_params filter,
                                                                               cs_group_reduce_out out) {
    extern __shared__ __align__(16) float gr_smem[];
    float *acc_col = warp_acc_column(gr_smem, GR != 0u, group_count);
    uint16_t *tbl = reinterpret_cast<uint16_t *>(gr_smem + (GR != 0u ? kCodesWarps * group_count * 32u : 0u));
    build_col_codes(tbl, src.cols, masks.feature_keep, GR != 0u ? group_masks : nullptr,
                    GR != 0u ? (1u << group_count) - 1u : 0u);
    for (uint32_t row = blockIdx.x * kCodesWarps + (threadIdx.x >> 5); row < src.rows;
         row += gridDim.x * kCodesWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            empty_row(row, group_count, out);
            continue;
        }
        row_acc<GR> a;
        init_acc(a);
        uint32_t width = 0u;
        std::size_t slot_base = 0u;
        if (src.slice_count != 0u) {
            const uint32_t slice = find_slice(src, row);
            width = src.slice_widths[slice];
            slot_base = (std::size_t) src.slice_slot_offsets[slice] +
                        (std::size_t) (row - src.slice_row_offsets[slice]) * width;
        }
        reduce_span_codes<U>(src.col_idx, src.val, slot_base, slot_base + width, src.cols, tbl, a);
        __syncwarp();
        finish_row(row, a, acc_col, group_count, filter, out);
    }
}

#ifndef SELL_CODES
#define SELL_CODES 1
#endif
constexpr bool kSellCodes = SELL_CODES != 0; // the Sliced-ELL reduce over the shared code table

std::size_t group_smem(const uint32_t *masks, uint32_t group_count);

// Shared bytes of the code-table kernels, 0 when they do not apply (more than
// 15 groups, or a table above 96 KB).
std::size_t codes_smem(const uint32_t *masks, uint32_t group_count, uint32_t cols) {
    const bool groups = masks != nullptr && group_count != 0u;
    if (groups && group_count > 15u) return 0u;
    if ((std::size_t) cols * 2u > 96u * 1024u) return 0u;
    const std::size_t acc = groups ? (std::size_t) kCodesWarps * group_count * 32u * sizeof(float) : 0u;
    return align_up(acc, 16u) + align_up((std::size_t) cols * 2u, 16u);
}

template <typename View>
using reduce_codes_kernel_t = void (*)(View, const uint32_t *, uint32_t, cs_row_feature_mask_view,
                                       cs_group_filter_params, cs_group_reduce_out);

template <typename View>
int launch_codes(reduce_codes_kernel_t<View> k, const View &src, const uint32_t *masks, uint32_t group_count,
                 const cs_row_feature_mask_view &m, const cs_group_filter_params &filter,
                 const cs_group_reduce_out &out, std::size_t smem, cudaStream_t stream, const char *name) {
    if (smem > 48u * 1024u &&
        !cuda_ok(cudaFuncSetAttribute(reinterpret_cast<const void *>(k), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) smem),
                 name))
        return 0;
    const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kCodesWarps * 32u, smem,
                                        (src.rows + kCodesWarps - 1u) / kCodesWarps);
    k<<<grid, kCodesWarps * 32u, smem, stream>>>(src, masks, group_count, m, filter, out);
    return launch_ok(name);
}

// ---------------------------------------------------------------------------
// Blocked-ELL-16 reduce on the tensor cores.
//
// For one 16-row block and one 16-column slot, the block rows' group sums are
// a small product
//     D[n][grp] += sum_c V[n][c] * M[c][grp]
// with V[n][c] the slot's fp16 value of block row n, column c, and
// M[c][grp] = 1 when column c is inside the matrix, kept by the feature mask
// and in group grp.  One warp owns one row block and issues, per slot, one
// mma.m16n8k16 (fp16 operands, fp32 accumulators) per 8 groups, one whose B
// is the kept-column indicator (column 0 of D = the row totals) and one
// whose A is the nonzero indicator of the values (column 0 of D = the
// detected counts).  Products are v * 1 or v * 0, so the sums are fp32 sums
// of the values, as in the per-row path (addition order differs; integer data
// gives identical results).  The slot's 16 columns are dealt to the lanes as
// 4 consecutive columns per lane (lane = 4g + t reads columns 4t..4t+3 of
// block rows g and g + 8), the fragments' k order permuted: physical column
// 4t + {0,1,2,3} stands for k = 2t, 2t+1, 2t+8, 2t+9 in both operands.
// Maxima come from the same values with packed-half max.  A non-finite value
// turns its row total non-finite (0 * inf and 1 * inf alike), and such row
// blocks are redone by the per-row path.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                          uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t hmax2_bits(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// 0xffff in each half whose bit 15 is set, 0 in the others (prmt with the
// sign-replicating selector: each byte takes the sign of the half's high byte).
__device__ __forceinline__ uint32_t half_sign_mask(uint32_t x) {
    uint32_t d;
    asm("prmt.b32 %0, %1, 0, 0xbb99;" : "=r"(d) : "r"(x));
    return d;
}

// (without groups, G is the constant 0 and its comparisons fold away)
#pragma nv_diag_suppress 186
// NT: tiles of 8 groups (0 without groups); GR: accumulators of the per-row
// path that takes row blocks with non-finite values.
template <unsigned NT, unsigned GR, unsigned U>
__global__ void __launch_bounds__(kRowThreads) group_reduce_bell16_mma_kernel(
    cs_blocked_ell_view src, const uint32_t *__restrict__ group_masks, uint32_t group_count,
    cs_row_feature_mask_view masks, cs_group_filter_params filter, cs_group_reduce_out out) {
    extern __shared__ float gr_smem[];
    const bool groups = GR != 0u;
    const uint32_t G = groups ? group_count : 0u;
    float *acc_col = warp_acc_column(gr_smem, groups, group_count);
    uint2 *stage = reinterpret_cast<uint2 *>(gr_smem + (groups ? kRowWarps * group_count * 32u : 0u)) +
                   (threadIdx.x >> 5) * kStagePairs;
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    const uint32_t W = src.ell_cols >> 4;
    const uint32_t row_blocks = (src.rows + 15u) >> 4;
    const uint32_t gmask = G >= 32u ? 0xffffffffu : (1u << G) - 1u;
    const uint32_t unit_n0 = g == 0u ? 0x3c00u : 0u; // B column 0 only
    for (uint32_t rb = blockIdx.x * kRowWarps + (threadIdx.x >> 5); rb < row_blocks; rb += gridDim.x * kRowWarps) {
        uint32_t rowh[2];
        bool kept[2];
#pragma unroll
        for (unsigned h = 0; h < 2u; ++h) {
            rowh[h] = rb * 16u + 8u * h + g;
            kept[h] = rowh[h] < src.rows && (masks.row_keep == nullptr || masks.row_keep[rowh[h]] != 0u);
        }
        float dg[NT > 0u ? NT : 1u][4], dt[4] = {0.0f, 0.0f, 0.0f, 0.0f}, dd[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (unsigned nt = 0; nt < (NT > 0u ? NT : 1u); ++nt)
#pragma unroll
            for (unsigned q = 0; q < 4u; ++q) dg[nt][q] = 0.0f;
        uint32_t mx[2] = {0u, 0u};
        if (__any_sync(0xffffffffu, kept[0] || kept[1])) {
            const uint32_t *bci = src.blockColIdx + (std::size_t) rb * W;
            const uint16_t *vr[2];
#pragma unroll
            for (unsigned h = 0; h < 2u; ++h)
                vr[h] = src.val + (std::size_t) (kept[h] ? rowh[h] : 0u) * src.ell_cols + 4u * t;
            for (uint32_t s0 = 0; s0 < W; s0 += 32u) {
                const uint32_t n = min(32u, W - s0);
                const uint32_t my_bc = lane < n ? __ldg(bci + s0 + lane) : CS_INVALID_COL;
                for (uint32_t j0 = 0; j0 < n; j0 += U) {
                    uint2 x[U][2];
                    uint32_t bc[U];
#pragma unroll
                    for (unsigned u = 0; u < U; ++u) {
                        bc[u] = __shfl_sync(0xffffffffu, my_bc, (j0 + u) & 31u);
                        if (j0 + u >= n) bc[u] = CS_INVALID_COL;
                        const std::size_t off = (std::size_t) (s0 + j0 + u) * 16u;
#pragma unroll
                        for (unsigned h = 0; h < 2u; ++h)
                            x[u][h] = bc[u] != CS_INVALID_COL && kept[h] ? ld_stream_v2(vr[h] + off)
                                                                        : make_uint2(0u, 0u);
                    }
#pragma unroll
                    for (unsigned u = 0; u < U; ++u) {
                        if (bc[u] == CS_INVALID_COL) continue; // warp-uniform
                        // this lane's 4 columns: in range and kept (kw bytes), group bits
                        const uint32_t c0 = bc[u] * 16u + 4u * t;
                        uint32_t mk[4], kw;
                        if (c0 + 4u <= src.cols) {
                            const uint4 m4 = NT > 0u ? __ldg(reinterpret_cast<const uint4 *>(group_masks + c0))
                                                     : make_uint4(0u, 0u, 0u, 0u);
                            mk[0] = m4.x, mk[1] = m4.y, mk[2] = m4.z, mk[3] = m4.w;
                            kw = masks.feature_keep != nullptr
                                     ? __ldg(reinterpret_cast<const uint32_t *>(masks.feature_keep + c0))
                                     : 0x01010101u;
                        } else {
                            kw = 0u;
#pragma unroll
                            for (unsigned j = 0; j < 4u; ++j) {
                                const bool in = c0 + j < src.cols;
                                mk[j] = in && NT > 0u ? __ldg(group_masks + c0 + j) : 0u;
                                kw |= (in && feature_kept(masks.feature_keep, c0 + j) ? 1u : 0u) << (8u * j);
                            }
                        }
                        const uint32_t kv = __vsetne4(kw, 0u);                  // 1 per kept column byte
                        const uint32_t kb_lo = __byte_perm(kv, 0u, 0x4140u);     // columns 4t, 4t+1 -> bits 0, 16
                        const uint32_t kb_hi = __byte_perm(kv, 0u, 0x4342u);     // columns 4t+2, 4t+3
                        const uint32_t km_lo = kb_lo * 0xffffu, km_hi = kb_hi * 0xffffu;
                        const uint32_t a0 = x[u][0].x, a1 = x[u][1].x, a2 = x[u][0].y, a3 = x[u][1].y;
                        mma_16816(dt, a0, a1, a2, a3, kb_lo * unit_n0, kb_hi * unit_n0);
                        mma_16816(dd, nonzero_halves(a0), nonzero_halves(a1), nonzero_halves(a2),
                                  nonzero_halves(a3), kb_lo * unit_n0, kb_hi * unit_n0);
#pragma unroll
                        for (unsigned nt = 0; nt < NT; ++nt) {
                            // group 8nt + g of columns (4t, 4t+1) and (4t+2, 4t+3), as bits 0 and 16
                            const uint32_t sh = (8u * nt + g) & 15u;
                            const uint32_t sel = nt < 2u ? 0x5410u : 0x7632u;
                            const uint32_t p01 = __byte_perm(mk[0] & gmask, mk[1] & gmask, sel);
                            const uint32_t p23 = __byte_perm(mk[2] & gmask, mk[3] & gmask, sel);
                            mma_16816(dg[nt], a0, a1, a2, a3, ((p01 >> sh) & kb_lo) * 0x3c00u,
                                      ((p23 >> sh) & kb_hi) * 0x3c00u);
                        }
                        mx[0] = hmax2_bits(mx[0], hmax2_bits(a0 & km_lo, a2 & km_hi));
                        mx[1] = hmax2_bits(mx[1], hmax2_bits(a1 & km_lo, a3 & km_hi));
                    }
                }
            }
        }
        // D fragments of lane (g, t): [0] = D[g][2t], [1] = D[g][2t+1],
        // [2] = D[g+8][2t], [3] = D[g+8][2t+1]; totals and counts are column 0.
        const unsigned quad0 = lane & ~3u;
        float tot[2], cnt[2];
        tot[0] = __shfl_sync(0xffffffffu, dt[0], quad0);
        tot[1] = __shfl_sync(0xffffffffu, dt[2], quad0);
        cnt[0] = __shfl_sync(0xffffffffu, dd[0], quad0);
        cnt[1] = __shfl_sync(0xffffffffu, dd[2], quad0);
        if (__any_sync(0xffffffffu, !isfinite(tot[0]) || !isfinite(tot[1]))) {
            for (uint32_t r = 0; r < 16u; ++r)
                if (rb * 16u + r < src.rows)
                    bell_row<true, GR>(src, rb * 16u + r, group_masks, group_count, masks, filter, out, acc_col,
                                       stage);
            continue;
        }
        // fraction numerator: group F of rows g, g + 8 sits in lane (g, (F & 7) >> 1)
        const uint32_t F = filter.fraction_group_index;
        float fr[2] = {0.0f, 0.0f};
#pragma unroll
        for (unsigned nt = 0; nt < NT; ++nt)
            if (F < G && (F >> 3) == nt) {
                fr[0] = (F & 1u) ? dg[nt][1] : dg[nt][0];
                fr[1] = (F & 1u) ? dg[nt][3] : dg[nt][2];
            }
        const unsigned src_f = quad0 | ((F & 7u) >> 1);
        fr[0] = __shfl_sync(0xffffffffu, fr[0], src_f);
        fr[1] = __shfl_sync(0xffffffffu, fr[1], src_f);
#pragma unroll
        for (unsigned h = 0; h < 2u; ++h) {
            float vmax = fmaxf(h2f((uint16_t) (mx[h] & 0xffffu)), h2f((uint16_t) (mx[h] >> 16)));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, 1));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, 2));
            const uint32_t row = rowh[h];
            if (t == h && row < src.rows) {
                const float sum = tot[h];
                const uint32_t det = (uint32_t) cnt[h];
                out.row_totals[row] = sum;
                out.max_values[row] = vmax + 0.0f;
                out.detected_features[row] = det;
                const float frac = sum > 0.0f ? __fdiv_rn(F < G ? fr[h] : 0.0f, sum) : 0.0f;
                out.row_keep[row] = (uint8_t) (kept[h] && sum >= filter.min_total &&
                                               det >= filter.min_detected_features &&
                                               frac <= filter.max_group_fraction);
            }
            if (groups && out.group_counts != nullptr && out.group_percentages != nullptr && row < src.rows) {
#pragma unroll
                for (unsigned nt = 0; nt < NT; ++nt) {
#pragma unroll
                    for (unsigned q = 0; q < 2u; ++q) {
                        const uint32_t grp = 8u * nt + 2u * t + q;
                        if (grp < G) {
                            const float gs = dg[nt][2u * h + q];
                            const std::size_t o = (std::size_t) row * G + grp;
                            out.group_counts[o] = gs;
                            out.group_percentages[o] = tot[h] > 0.0f ? __fdiv_rn(__fmul_rn(100.0f, gs), tot[h])
                                                                     : 0.0f;
                        }
                    }
                }
            }
        }
    }
}

// Pipelined form for up to 15 groups and a column table that fits shared
// memory.  Each CTA first builds a u16 entry per column in shared memory
// (bit 15: in the matrix and kept; bits 0..G-1: the column's groups if
// kept), so the per-slot column lookups are shared-memory reads.  The values
// reach shared memory through 16-byte asynchronous copies, STAGES stages of
// SLOTS slots (16 rows x 32 * SLOTS bytes) per warp, so the bytes in flight do
// not depend on registers; rows the row mask drops are not copied.  A stage
// row is padded by 32 bytes, which puts the 8-byte fragment reads of a
// half-warp on distinct banks.  Row blocks with non-finite values use the
// per-row path, its shared memory taken from the warp's (then idle) stage
// buffers.  Stages of 4 slots, so more warps fit beside the table and hide
// the copies' latency (24 warps: 5.34 ms against 5.75 ms for 16 warps of
// 8-slot stages on 500,000 x 32,768); 16 warps where the table of a wider
// matrix leaves less room.
template <unsigned SLOTS, unsigned WARPS, unsigned STAGES>
struct pipe_cfg {
    static constexpr unsigned slots = SLOTS, warps = WARPS, stages = STAGES;
    static constexpr unsigned row_stride = SLOTS * 32u + 32u;
    static constexpr unsigned stage_bytes = 16u * row_stride;
    static constexpr unsigned pieces = SLOTS * 2u;            // 16-byte pieces of one row of a stage
    static constexpr unsigned rows_per_copy = 32u / pieces;   // stage rows one copy instruction covers
    static constexpr unsigned stages_per_window = 32u / SLOTS; // stages per 32-slot window of block columns
    static constexpr std::size_t warp_bytes = (std::size_t) STAGES * stage_bytes;
    static_assert(SLOTS >= 2u && SLOTS <= 16u && (SLOTS & (SLOTS - 1u)) == 0u, "a stage holds 2, 4, 8 or 16 slots");
    static_assert(warp_bytes >= 16u * 32u * sizeof(float) + kStagePairs * 8u,
                  "the per-row fallback's accumulators and pairs fit in a warp's stage buffers");
};
using pipe_wide = pipe_cfg<4u, PIPE_WIDE_WARPS, 2u>;
using pipe_narrow = pipe_cfg<4u, 16u, 2u>; // a column table of up to ~75,000 columns

std::size_t pipe_table_bytes(uint32_t cols) { return align_up(((std::size_t) cols + 15u) / 16u * 32u, 16u); }

template <class CFG>
std::size_t pipe_smem_bytes(uint32_t cols) { return CFG::warps * CFG::warp_bytes + pipe_table_bytes(cols); }

template <unsigned NT, unsigned GR, class CFG>
__global__ void __launch_bounds__(CFG::warps * 32, 1) group_reduce_bell16_pipe_kernel(
    cs_blocked_ell_view src, const uint32_t *__restrict__ group_masks, uint32_t group_count,
    cs_row_feature_mask_view masks, cs_group_filter_params filter, cs_group_reduce_out out) {
    extern __shared__ __align__(16) unsigned char pipe_smem[];
    constexpr unsigned STAGES = CFG::stages, kPipeSlots = CFG::slots, kPipeWarps = CFG::warps;
    constexpr unsigned kPipeStageBytes = CFG::stage_bytes, kPipePieces = CFG::pieces;
    constexpr unsigned kPipeRowsPerCopy = CFG::rows_per_copy, kPipeStagesPerWindow = CFG::stages_per_window;
    constexpr unsigned RS = CFG::row_stride;
    const bool groups = GR != 0u;
    const uint32_t G = groups ? group_count : 0u;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    unsigned char *buf = pipe_smem + (std::size_t) warp * CFG::warp_bytes;
    uint16_t *table = reinterpret_cast<uint16_t *>(pipe_smem + kPipeWarps * CFG::warp_bytes);
    // per-row fallback: accumulator block and pair staging inside this warp's stage buffers
    float *acc_col = groups ? reinterpret_cast<float *>(buf) + lane : nullptr;
    uint2 *stage = reinterpret_cast<uint2 *>(buf + (std::size_t) G * 32u * sizeof(float));
    const uint32_t col_blocks = (src.cols + 15u) >> 4;
    const uint32_t gmask = (1u << G) - 1u;
    for (uint32_t c = threadIdx.x; c < col_blocks * 16u; c += blockDim.x) {
        uint32_t e = 0u;
        if (c < src.cols && feature_kept(masks.feature_keep, c))
            e = 0x8000u | (NT > 0u ? __ldg(group_masks + c) & gmask : 0u);
        table[c] = (uint16_t) e;
    }
    __syncthreads();
    const uint32_t W = src.ell_cols >> 4;
    const uint32_t nstages = (W + kPipeSlots - 1u) / kPipeSlots;
    const uint32_t row_blocks = (src.rows + 15u) >> 4;
    const uint32_t unit_n0 = g == 0u ? 0x3c003c00u : 0u; // 1.0 pairs in B column 0 only
    // group g's bit of two table entries times 0x3c00 >> g is 1.0 (0x3c00) per
    // member half: 0x3c00 = 15 << 10, so the shift is exact for g < 8
    const uint32_t gsel = 0x00010001u << g, gmul = 0x3c00u >> g;
    for (uint32_t rb = blockIdx.x * kPipeWarps + warp; rb < row_blocks; rb += gridDim.x * kPipeWarps) {
        // rows of the block the row mask keeps (bit r = block row r)
        const uint32_t r16 = rb * 16u + (lane & 15u);
        const bool lane_keep = lane < 16u && r16 < src.rows && (masks.row_keep == nullptr || masks.row_keep[r16] != 0u);
        const uint32_t keep16 = __ballot_sync(0xffffffffu, lane_keep);
        const bool kept[2] = {((keep16 >> g) & 1u) != 0u, ((keep16 >> (g + 8u)) & 1u) != 0u};
        float dg[NT > 0u ? NT : 1u][4], dt[4] = {0.0f, 0.0f, 0.0f, 0.0f}, dd[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (unsigned nt = 0; nt < (NT > 0u ? NT : 1u); ++nt)
#pragma unroll
            for (unsigned q = 0; q < 4u; ++q) dg[nt][q] = 0.0f;
        uint32_t mx[2] = {0u, 0u};
        if (keep16 != 0u) {
            const uint32_t *bci = src.blockColIdx + (std::size_t) rb * W;
            // rows the mask drops are never copied: zero them in every stage once
            for (unsigned i = lane; i < STAGES * 16u * kPipePieces; i += 32u) {
                const unsigned r = (i / kPipePieces) % 16u;
                if (!((keep16 >> r) & 1u))
                    *reinterpret_cast<uint4 *>(buf + (i / (16u * kPipePieces)) * kPipeStageBytes + r * RS +
                                               (i % kPipePieces) * 16u) = make_uint4(0u, 0u, 0u, 0u);
            }
            // this lane's copies: 16-byte piece (lane % kPipePieces) of stage rows
            // lane / kPipePieces + kPipeRowsPerCopy * i
            const unsigned piece = lane % kPipePieces;
            const uint16_t *gsrc = src.val + (std::size_t) rb * 16u * src.ell_cols + piece * 8u;
            auto issue = [&](uint32_t k) {
                if (k < nstages && k * kPipeSlots + piece / 2u < W) {
                    unsigned char *dst = buf + (k % STAGES) * kPipeStageBytes + piece * 16u;
                    const uint16_t *from = gsrc + (std::size_t) k * kPipeSlots * 16u;
#pragma unroll
                    for (unsigned i = 0; i < 16u / kPipeRowsPerCopy; ++i) {
                        const unsigned r = lane / kPipePieces + kPipeRowsPerCopy * i;
                        if ((keep16 >> r) & 1u) cp_async_16(dst + r * RS, from + (std::size_t) r * src.ell_cols);
                    }
                }
                cp_async_commit();
            };
#pragma unroll
            for (unsigned p = 0; p + 1u < STAGES; ++p) issue(p);
            // block columns of slots [32w, 32w + 32) one per lane, the next window loaded ahead
            uint32_t my_bc = lane < W ? __ldg(bci + lane) : CS_INVALID_COL;
            uint32_t next_bc = 32u + lane < W ? __ldg(bci + 32u + lane) : CS_INVALID_COL;
            // slots of the window whose block column lies inside the table (bit = slot)
            uint32_t valid_bc = __ballot_sync(0xffffffffu, my_bc < col_blocks);
            for (uint32_t k = 0; k < nstages; ++k) {
                issue(k + STAGES - 1u);
                cp_async_wait<STAGES - 1>();
                __syncwarp();
                const unsigned char *sb = buf + (k % STAGES) * kPipeStageBytes + 8u * t;
                const uint32_t nslots = min(kPipeSlots, W - k * kPipeSlots);
                if (k % kPipeStagesPerWindow == 0u && k != 0u) {
                    my_bc = next_bc;
                    const uint32_t s = k * kPipeSlots + 32u + lane;
                    next_bc = s < W ? __ldg(bci + s) : CS_INVALID_COL;
                    valid_bc = __ballot_sync(0xffffffffu, my_bc < col_blocks);
                }
                const uint32_t wbase = (k % kPipeStagesPerWindow) * kPipeSlots;
                // one slot: the values of the columns the table does not keep are
                // zeroed once (the masked fragments give the totals, the detected
                // counts and the maxima against a constant B; the group bits of a
                // dropped column are zero in the table already)
                auto slot = [&](unsigned j, auto check) {
                    const uint32_t bc = __shfl_sync(0xffffffffu, my_bc, (wbase + j) & 31u);
                    if constexpr (decltype(check)::value)
                        if (bc >= col_blocks) return; // warp-uniform (padding or outside)
                    // this lane's 4 columns: two u16 entries per word (columns 4t, 4t+1 and 4t+2, 4t+3)
                    const uint2 te = *reinterpret_cast<const uint2 *>(table + bc * 16u + 4u * t);
                    const uint32_t km_lo = half_sign_mask(te.x), km_hi = half_sign_mask(te.y);
                    const uint2 lo = *reinterpret_cast<const uint2 *>(sb + g * RS + j * 32u);
                    const uint2 hi = *reinterpret_cast<const uint2 *>(sb + (g + 8u) * RS + j * 32u);
                    const uint32_t a0 = lo.x & km_lo, a1 = hi.x & km_lo, a2 = lo.y & km_hi, a3 = hi.y & km_hi;
                    mma_16816(dt, a0, a1, a2, a3, unit_n0, unit_n0);
                    mma_16816(dd, nonzero_halves(a0), nonzero_halves(a1), nonzero_halves(a2),
                              nonzero_halves(a3), unit_n0, unit_n0);
                    if constexpr (NT > 0u)
                        mma_16816(dg[0], a0, a1, a2, a3, (te.x & gsel) * gmul, (te.y & gsel) * gmul);
                    if constexpr (NT > 1u)
                        mma_16816(dg[NT - 1u], a0, a1, a2, a3, ((te.x >> (g + 8u)) & 0x00010001u) * 0x3c00u,
                                  ((te.y >> (g + 8u)) & 0x00010001u) * 0x3c00u);
                    mx[0] = hmax2_bits(mx[0], hmax2_bits(a0, a2));
                    mx[1] = hmax2_bits(mx[1], hmax2_bits(a1, a3));
                };
                constexpr uint32_t kStageSlotsMask = (1u << kPipeSlots) - 1u;
                if (nslots == kPipeSlots && ((valid_bc >> wbase) & kStageSlotsMask) == kStageSlotsMask) {
#pragma unroll
                    for (unsigned j = 0; j < kPipeSlots; ++j) slot(j, std::false_type{});
                } else {
                    for (unsigned j = 0; j < nslots; ++j) slot(j, std::true_type{});
                }
                __syncwarp();
            }
            cp_async_wait<0>();
            __syncwarp();
        }
        const unsigned quad0 = lane & ~3u;
        float tot[2], cnt[2];
        tot[0] = __shfl_sync(0xffffffffu, dt[0], quad0);
        tot[1] = __shfl_sync(0xffffffffu, dt[2], quad0);
        cnt[0] = __shfl_sync(0xffffffffu, dd[0], quad0);
        cnt[1] = __shfl_sync(0xffffffffu, dd[2], quad0);
        if (__any_sync(0xffffffffu, !isfinite(tot[0]) || !isfinite(tot[1]))) {
            for (uint32_t r = 0; r < 16u; ++r)
                if (rb * 16u + r < src.rows)
                    bell_row<true, GR>(src, rb * 16u + r, group_masks, group_count, masks, filter, out, acc_col,
                                       stage);
            __syncwarp();
            continue;
        }
        const uint32_t F = filter.fraction_group_index;
        float fr[2] = {0.0f, 0.0f};
#pragma unroll
        for (unsigned nt = 0; nt < NT; ++nt)
            if (F < G && (F >> 3) == nt) {
                fr[0] = (F & 1u) ? dg[nt][1] : dg[nt][0];
                fr[1] = (F & 1u) ? dg[nt][3] : dg[nt][2];
            }
        const unsigned src_f = quad0 | ((F & 7u) >> 1);
        fr[0] = __shfl_sync(0xffffffffu, fr[0], src_f);
        fr[1] = __shfl_sync(0xffffffffu, fr[1], src_f);
#pragma unroll
        for (unsigned h = 0; h < 2u; ++h) {
            float vmax = fmaxf(h2f((uint16_t) (mx[h] & 0xffffu)), h2f((uint16_t) (mx[h] >> 16)));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, 1));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, 2));
            const uint32_t row = rb * 16u + 8u * h + g;
            if (t == h && row < src.rows) {
                const float sum = tot[h];
                const uint32_t det = (uint32_t) cnt[h];
                out.row_totals[row] = sum;
                out.max_values[row] = vmax + 0.0f;
                out.detected_features[row] = det;
                const float frac = sum > 0.0f ? __fdiv_rn(F < G ? fr[h] : 0.0f, sum) : 0.0f;
                out.row_keep[row] = (uint8_t) (kept[h] && sum >= filter.min_total &&
                                               det >= filter.min_detected_features &&
                                               frac <= filter.max_group_fraction);
            }
            if (groups && out.group_counts != nullptr && out.group_percentages != nullptr && row < src.rows) {
#pragma unroll
                for (unsigned nt = 0; nt < NT; ++nt) {
#pragma unroll
                    for (unsigned q = 0; q < 2u; ++q) {
                        const uint32_t grp = 8u * nt + 2u * t + q;
                        if (grp < G) {
                            const float gs = dg[nt][2u * h + q];
                            const std::size_t o = (std::size_t) row * G + grp;
                            out.group_counts[o] = gs;
                            out.group_percentages[o] = tot[h] > 0.0f ? __fdiv_rn(__fmul_rn(100.0f, gs), tot[h])
                                                                     : 0.0f;
                        }
                    }
                }
            }
        }
    }
}

#pragma nv_diag_default 186

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
    return (masks != nullptr && group_count != 0u) ? kRowWarps * group_count * 32u * sizeof(float) : 0u;
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

// The Blocked-ELL partitions of one shard, rows concatenated in order (the
// reference's part_views / part_row_offsets, repack/kernels/sharded_blocked_ell.cuh:
// 13-21); a single view is a one-part table.
struct reopt_parts {
    cs_blocked_ell_view v[CS_MAX_REPACK_PARTS];
    uint32_t row_off[CS_MAX_REPACK_PARTS + 1];
    uint32_t count;
};

__device__ __forceinline__ uint32_t part_of_row(const reopt_parts &p, uint32_t row) {
    uint32_t lo = 0u, hi = p.count - 1u; // last part whose first row is <= row
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (p.row_off[mid] <= row)
            lo = mid;
        else
            hi = mid - 1u;
    }
    return lo;
}

// Count (EMIT false: per output row its kept entries, a claim per output row,
// and when kept != null the kept rows and their slots) or scatter (EMIT true).
template <bool EMIT>
__global__ void __launch_bounds__(kRowThreads) reopt_kernel(const __grid_constant__ reopt_parts parts,
                                                            cs_row_feature_mask_view masks, uint32_t output_rows,
                                                            uint32_t output_cols, uint32_t *__restrict__ major_ptr,
                                                            uint32_t *__restrict__ claims,
                                                            uint32_t *__restrict__ minor_idx,
                                                            uint16_t *__restrict__ out_val, uint32_t *status,
                                                            unsigned long long *__restrict__ kept,
                                                            uint32_t keep_words) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t rows = parts.row_off[parts.count];
    // keep_words != 0: the feature flags as a bitmap in shared memory (bit c of
    // word c / 32), so a vector's 8 consecutive columns are checked at once
    extern __shared__ uint32_t reopt_keep_bits[];
    const uint32_t *kbits = keep_words != 0u ? reopt_keep_bits : nullptr;
    uint32_t kcols = 0u; // columns the flags cover: the widest part
    for (uint32_t k = 0; k < parts.count; ++k) kcols = max(kcols, parts.v[k].cols);
    for (uint32_t w = threadIdx.x; w < keep_words; w += blockDim.x) {
        uint32_t word = 0u;
        const uint32_t c0 = w * 32u;
#pragma unroll 4
        for (uint32_t k = 0; k < 32u; ++k)
            if (c0 + k < kcols) word |= (masks.feature_keep[c0 + k] != 0u ? 1u : 0u) << k;
        reopt_keep_bits[w] = word;
    }
    if (keep_words != 0u) __syncthreads();
    uint32_t warp_kept_rows = 0u;       // count pass: kept rows of this warp and their slots,
    unsigned long long warp_kept_slots = 0u; // added to the totals once at the end
    for (uint32_t row = blockIdx.x * kRowWarps + (threadIdx.x >> 5); row < rows; row += gridDim.x * kRowWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) continue;
        const uint32_t part = part_of_row(parts, row);
        const cs_blocked_ell_view &src = parts.v[part];
        const uint32_t local = row - parts.row_off[part];
        if (!EMIT) {
            warp_kept_rows += 1u;
            warp_kept_slots += src.ell_cols;
        }
        const uint32_t out_row = masks.row_remap != nullptr ? masks.row_remap[row] : row;
        if (out_row >= output_rows) continue;
        const uint32_t B = src.block_size;
        const uint32_t W = B != 0u ? src.ell_cols / B : 0u;
        const uint32_t rb = B != 0u ? local / B : 0u;
        const block_div bd(B);
        const uint32_t *bci = src.blockColIdx + (std::size_t) rb * W;
        const uint16_t *vrow = src.val + (std::size_t) local * src.ell_cols;
        uint32_t run = EMIT ? major_ptr[out_row] : 0u;
        // entries past the row's end (only possible when two rows remap to one
        // output row, which the count pass flags) are dropped, never written
        const uint32_t end = EMIT ? major_ptr[out_row + 1u] : 0u;
        if (B % 8u == 0u && B != 0u && (reinterpret_cast<uintptr_t>(src.val) & 15u) == 0u) {
            // a 16-byte value vector per lane, four 256-value steps in flight; the
            // feature flag and remap are read only for the live values, and a warp
            // scan of the kept counts ranks them in slot order
            constexpr unsigned kRs = 4;
            uint32_t lane_count = 0u;
            for (uint32_t b0 = lane * 8u; b0 - lane * 8u < src.ell_cols; b0 += 256u * kRs) {
                uint4 v[kRs];
                uint32_t bcs[kRs];
                load_steps(vrow, bci, bd, src.ell_cols, b0, v, bcs);
#pragma unroll
                for (unsigned u = 0; u < kRs; ++u) {
                    const uint32_t gene0 = bcs[u] * B + bd.mod(b0 + u * 256u);
                    uint32_t live = live_bits8(v[u]) & in_range8(bcs[u], gene0, src.cols);
                    // gene0 is a multiple of 8: its 8 flags sit in one bitmap word
                    if (kbits != nullptr && live != 0u) live &= kbits[gene0 >> 5] >> (gene0 & 31u);
                    uint32_t keep = 0u;
                    if (masks.feature_remap == nullptr && (kbits != nullptr || masks.feature_keep == nullptr)) {
                        keep = live & in_range8(bcs[u], gene0, output_cols);
                    } else {
                        for (uint32_t bb = live; bb != 0u; bb &= bb - 1u) {
                            const uint32_t q = __ffs(bb) - 1u, c = gene0 + q;
                            if (kbits == nullptr && !feature_kept(masks.feature_keep, c)) continue;
                            const uint32_t oc = masks.feature_remap != nullptr ? masks.feature_remap[c] : c;
                            if (oc < output_cols) keep |= 1u << q;
                        }
                    }
                    const uint32_t cnt = __popc(keep);
                    if constexpr (EMIT) {
                        const uint32_t incl = warp_inclusive_scan(cnt);
                        uint32_t pos = run + incl - cnt;
                        for (uint32_t bb = keep; bb != 0u; bb &= bb - 1u, ++pos) {
                            const uint32_t q = __ffs(bb) - 1u, c = gene0 + q;
                            if (pos < end) {
                                minor_idx[pos] = masks.feature_remap != nullptr ? masks.feature_remap[c] : c;
                                out_val[pos] = half_of(v[u], q);
                            }
                        }
                        run += __shfl_sync(0xffffffffu, incl, 31);
                    } else {
                        lane_count += cnt; // the count pass needs only the row total
                    }
                }
            }
            if constexpr (!EMIT) run = __reduce_add_sync(0xffffffffu, lane_count);
        } else
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
            if constexpr (EMIT) {
                const uint32_t pos = run + __popc(ballot & ((1u << lane) - 1u));
                if (k && pos < end) {
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
    if (!EMIT && kept != nullptr && lane == 0u && warp_kept_rows != 0u) {
        atomicAdd(kept, (unsigned long long) warp_kept_rows);
        atomicAdd(kept + 1, warp_kept_slots);
    }
}

// ---------------------------------------------------------------------------
// One-pass filter: count, decoupled look-back over rows, emit while the row's
// values are still in L2.  Rows are claimed in order from a global counter by
// resident CTAs, so every row a CTA waits for is held by a running CTA.
// row_state[r]: (flag << 32) | value, flag 1 = the row's count, 2 = the
// inclusive prefix through the row.  The state word is all a reader needs, so
// it is published and read with relaxed 64-bit accesses (no fence).  A row the
// mask drops is published as count 0 by the thread that claims it, which then
// claims the next row; the kept row before it writes its row pointer.
// ---------------------------------------------------------------------------
constexpr unsigned long long kLbCount = 1ull << 32, kLbPrefix = 2ull << 32;
constexpr uint32_t kLbSpinLimit = 1u << 22; // ~0.3 s of 64 ns sleeps

__device__ __forceinline__ unsigned long long lb_load(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void lb_store(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// 16-byte value loads with an L2 eviction priority (createpolicy): the count
// pass marks a row's values evict_last so they stay in L2 for the emit's
// re-read, which marks them evict_first again.
__device__ __forceinline__ unsigned long long l2_evict_last_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ unsigned long long l2_evict_first_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ uint4 ld_policy_v4(const void *p, unsigned long long pol) {
    uint4 r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p), "l"(pol));
    return r;
}

// Kept entries among the 8 values of one vector (no feature remap).
// lim = min(cols, output_cols): the columns that exist and have an output slot.
__device__ __forceinline__ uint32_t onepass_keep(const uint4 &v, uint32_t bc, uint32_t gene0, uint32_t lim,
                                                 const uint32_t *kbits) {
    uint32_t live = live_bits8(v) & in_range8(bc, gene0, lim);
    if (kbits != nullptr && live != 0u) live &= kbits[gene0 >> 5] >> (gene0 & 31u);
    return live;
}

// One CTA per row at a time (rows claimed in order): the row's values are read
// once to count, and read again from L2 to emit -- the count's loads mark them
// evict_last, and the rows in flight (a few CTAs per SM) stay well inside L2.  Each thread owns kOpVecs consecutive
// 16-byte vectors of a 256 x kOpVecs-vector step, so one block scan per step
// gives every thread its output position in slot order.
// Block-wide exclusive scan of 64-bit values (the packed per-step counts);
// every thread calls it; smem holds 33 words.
__device__ __forceinline__ unsigned long long block_exclusive_scan_u64(unsigned long long v,
                                                                       unsigned long long *smem,
                                                                       unsigned long long &total) {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned long long incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned) o) incl += t;
    }
    if (lane == 31u) smem[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const unsigned long long w = lane < nw ? smem[lane] : 0ull;
        unsigned long long wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (unsigned) o) wi += t;
        }
        if (lane < nw) smem[lane] = wi - w;
        if (lane == 31u) smem[32] = wi;
    }
    __syncthreads();
    const unsigned long long r = smem[warp] + incl - v;
    total = smem[32];
    __syncthreads();
    return r;
}

constexpr unsigned kOpThreads = 256;
constexpr unsigned kOpVecs = 4;
constexpr uint32_t kOpPackedSteps = 4; // rows of up to 4 steps keep their per-step counts for one scan
constexpr unsigned kOpCtasPerSm = 5;
constexpr bool kOpPrefetch = false; // the next step's loads issued before this step's work

__global__ void __launch_bounds__(kOpThreads, kOpCtasPerSm) filter_onepass_kernel(
    const __grid_constant__ reopt_parts parts, cs_row_feature_mask_view masks, uint32_t output_cols,
    uint32_t *__restrict__ major_ptr, uint32_t *__restrict__ minor_idx, uint16_t *__restrict__ out_val,
    unsigned long long capacity, unsigned long long *__restrict__ row_state, uint32_t *__restrict__ row_counter,
    uint32_t *status, unsigned long long *__restrict__ kept, uint32_t keep_words) {
    const uint32_t rows = parts.row_off[parts.count];
    extern __shared__ uint32_t onepass_keep_bits[];
    // after the feature bitmap: the keep bits of this thread's 4 vectors of each
    // step of the current row (packed rows), read back by the same thread
    uint32_t *row_keep32 = onepass_keep_bits + ((keep_words + 3u) & ~3u) + threadIdx.x;
    __shared__ uint32_t s_row, s_excl, s_stop, scan33[33];
    __shared__ unsigned long long scan33w[33];
    const uint32_t *kbits = keep_words != 0u ? onepass_keep_bits : nullptr;
    uint32_t kcols = 0u;
    for (uint32_t k = 0; k < parts.count; ++k) kcols = max(kcols, parts.v[k].cols);
    for (uint32_t w = threadIdx.x; w < keep_words; w += blockDim.x) {
        uint32_t word = 0u;
        const uint32_t c0 = w * 32u;
#pragma unroll 4
        for (uint32_t k = 0; k < 32u; ++k)
            if (c0 + k < kcols) word |= (masks.feature_keep[c0 + k] != 0u ? 1u : 0u) << k;
        onepass_keep_bits[w] = word;
    }
    uint32_t cta_kept_rows = 0u;
    unsigned long long cta_kept_slots = 0u;
    constexpr uint32_t kStep = kOpThreads * kOpVecs * 8u; // values per step
    for (;;) {
        if (threadIdx.x == 0u) {
            // rows the mask drops are published as empty at once (their row
            // pointers come from the kept row before them) and not worked on
            uint32_t r;
            for (;;) {
                r = atomicAdd(row_counter, 1u);
                if (r >= rows || masks.row_keep == nullptr || masks.row_keep[r] != 0u) break;
                lb_store(row_state + r, kLbCount);
            }
            s_row = r;
            s_stop = 0u;
        }
        __syncthreads();
        const uint32_t row = s_row;
        if (row >= rows) break;
        const uint32_t part = part_of_row(parts, row);
        const cs_blocked_ell_view &src = parts.v[part];
        const uint32_t local = row - parts.row_off[part];
        const uint32_t B = src.block_size, W = src.ell_cols / B;
        const block_div bd(B);
        const uint32_t *bci = src.blockColIdx + (std::size_t) (local / B) * W;
        const uint16_t *vrow = src.val + (std::size_t) local * src.ell_cols;
        // this thread's vectors of one step, and their keep bits
        auto load_vecs = [&](uint32_t base, uint4 (&v)[kOpVecs], unsigned long long pol) {
#pragma unroll
            for (unsigned u = 0; u < kOpVecs; ++u) {
                const uint32_t e0 = base + (threadIdx.x * kOpVecs + u) * 8u;
                v[u] = e0 < src.ell_cols ? ld_policy_v4(vrow + e0, pol) : make_uint4(0u, 0u, 0u, 0u);
            }
        };
        auto keep_of = [&](uint32_t base, const uint4 (&v)[kOpVecs], uint32_t (&keep)[kOpVecs],
                           uint32_t (&gene0)[kOpVecs]) {
#pragma unroll
            for (unsigned u = 0; u < kOpVecs; ++u) {
                const uint32_t e0 = base + (threadIdx.x * kOpVecs + u) * 8u;
                const bool in = e0 < src.ell_cols;
                const uint32_t bc = in ? __ldg(bci + bd.div(e0)) : CS_INVALID_COL;
                gene0[u] = bc * B + bd.mod(e0);
                keep[u] = in ? onepass_keep(v[u], bc, gene0[u], min(src.cols, output_cols), kbits) : 0u;
            }
        };
        // the next step's loads go out before this step's work (kOpPrefetch) or after it
        auto next_step = [&](uint32_t base, uint4 (&v)[kOpVecs], uint4 (&nv)[kOpVecs], unsigned long long pol) {
            if (base + kStep >= src.ell_cols) return;
            if (kOpPrefetch) {
#pragma unroll
                for (unsigned u = 0; u < kOpVecs; ++u) v[u] = nv[u];
            } else {
                load_vecs(base + kStep, v, pol);
            }
        };
        // count (a row of at most kOpPackedSteps steps keeps each step's count,
        // 16 bits per step, so one scan orders the whole emit)
        const bool packed = src.ell_cols <= kOpPackedSteps * kStep;
        uint32_t my = 0u;
        unsigned long long my_steps = 0ull;
        {
            if (threadIdx.x == 0u) {
                cta_kept_rows += 1u;
                cta_kept_slots += src.ell_cols;
            }
            const unsigned long long pol = l2_evict_last_policy();
            uint4 v[kOpVecs], nv[kOpVecs];
            load_vecs(0u, v, pol);
            for (uint32_t base = 0u, st = 0u; base < src.ell_cols; base += kStep, ++st) {
                if (kOpPrefetch && base + kStep < src.ell_cols) load_vecs(base + kStep, nv, pol);
                uint32_t keep[kOpVecs], gene0[kOpVecs];
                keep_of(base, v, keep, gene0);
                uint32_t n = 0u;
#pragma unroll
                for (unsigned u = 0; u < kOpVecs; ++u) n += __popc(keep[u]);
                my += n;
                if (packed) {
                    my_steps += (unsigned long long) n << (16u * st);
                    row_keep32[st * kOpThreads] = keep[0] | (keep[1] << 8) | (keep[2] << 16) | (keep[3] << 24);
                }
                next_step(base, v, nv, pol);
            }
        }
        uint32_t count;
        unsigned long long step_excl = 0ull, step_tot = 0ull;
        if (packed) {
            step_excl = block_exclusive_scan_u64(my_steps, scan33w, step_tot);
            count = (uint32_t) (step_tot & 0xffffu) + (uint32_t) ((step_tot >> 16) & 0xffffu) +
                    (uint32_t) ((step_tot >> 32) & 0xffffu) + (uint32_t) (step_tot >> 48);
        } else {
            (void) block_exclusive_scan(my, scan33, count);
        }
        // publish the count, then the prefix once the rows before it are known:
        // warp 0 reads the states of the 32 rows before row j at once and stops
        // at the nearest one that holds its prefix (rows before row 0 count as
        // a zero prefix)
        if (threadIdx.x < 32u) {
            const unsigned lane = threadIdx.x;
            if (lane == 0u) lb_store(row_state + row, kLbCount | count);
            uint32_t excl = 0u, j = row;
            bool gave_up = false;
            while (j > 0u) {
                const bool real = lane < j;
                const uint32_t q = real ? j - 1u - lane : 0u;
                unsigned long long st = real ? lb_load(row_state + q) : kLbPrefix;
                for (uint32_t spins = 0; !__all_sync(0xffffffffu, (st >> 32) != 0ull);) {
                    if (++spins > kLbSpinLimit) {
                        gave_up = true;
                        break;
                    }
                    __nanosleep(64);
                    if ((st >> 32) == 0ull) st = lb_load(row_state + q);
                }
                if (gave_up) break;
                const uint32_t pm = __ballot_sync(0xffffffffu, (st & ~0xffffffffull) == kLbPrefix);
                const uint32_t first = pm != 0u ? (uint32_t) __ffs(pm) - 1u : 31u;
                excl += __reduce_add_sync(0xffffffffu, lane <= first ? (uint32_t) st : 0u);
                if (pm != 0u) break;
                j -= 32u; // pm == 0 means all 32 rows before j are real
            }
            if (lane == 0u) {
                if (gave_up) {
                    s_stop = 1u;
                    status_or(status, CS_STATUS_WAIT_LIMIT);
                } else {
                    lb_store(row_state + row, kLbPrefix | (excl + count));
                    major_ptr[row] = excl;
                    if (count != 0u && (unsigned long long) excl + count > capacity) {
                        s_stop = 2u; // this row does not fit: skip its emission
                        status_or(status, CS_STATUS_CAPACITY);
                    }
                }
                s_excl = excl;
            }
            // the row pointers of the dropped rows after this one (up to the
            // next kept row, or the shard's end: then major_ptr[rows]) are this
            // row's inclusive prefix; 32 rows per step
            if (!gave_up) {
                const uint32_t incl = excl + count;
                for (uint32_t k0 = row + 1u;; k0 += 32u) {
                    const uint32_t k = k0 + lane;
                    const bool dropped = k < rows && masks.row_keep != nullptr && masks.row_keep[k] == 0u;
                    const uint32_t stop = __ballot_sync(0xffffffffu, !dropped);
                    const uint32_t first = stop != 0u ? (uint32_t) __ffs(stop) - 1u : 32u;
                    if (lane < first) major_ptr[k] = incl;
                    if (stop != 0u) {
                        if (lane == 0u && k0 + first >= rows) major_ptr[rows] = incl;
                        break;
                    }
                }
            }
        }
        __syncthreads();
        if (s_stop == 1u) break;
        if (packed && my != 0u && s_stop == 0u) {
            // emit, re-reading the row (now in L2) in slot order: step st's
            // entries of this thread start after the earlier steps' entries and
            // the earlier threads' entries of step st -- no further barrier
            const unsigned long long pol = l2_evict_first_policy();
            uint32_t step_base = s_excl;
            for (uint32_t base = 0u, st = 0u; base < src.ell_cols; base += kStep, ++st) {
                const uint32_t sh = 16u * st;
                // only the vectors the count found kept entries in are re-read
                const uint32_t kw4 = row_keep32[st * kOpThreads];
                if (kw4 != 0u) {
                    uint32_t pos = step_base + (uint32_t) ((step_excl >> sh) & 0xffffull);
#pragma unroll
                    for (unsigned u = 0; u < kOpVecs; ++u) {
                        const uint32_t kb = (kw4 >> (8u * u)) & 0xffu;
                        if (kb == 0u) continue;
                        const uint32_t e0 = base + (threadIdx.x * kOpVecs + u) * 8u;
                        const uint4 v = ld_policy_v4(vrow + e0, pol);
                        const uint32_t gene0 = __ldg(bci + bd.div(e0)) * B + bd.mod(e0);
                        for (uint32_t bb = kb; bb != 0u; bb &= bb - 1u, ++pos) {
                            const uint32_t q = __ffs(bb) - 1u;
                            minor_idx[pos] = gene0 + q;
                            out_val[pos] = half_of(v, q);
                        }
                    }
                }
                step_base += (uint32_t) ((step_tot >> sh) & 0xffffull);
            }
        }
        if (!packed && count != 0u && s_stop == 0u) {
            // emit, re-reading the row (now in L2) in slot order
            uint32_t run = s_excl;
            const unsigned long long pol = l2_evict_first_policy();
            uint4 v[kOpVecs], nv[kOpVecs];
            load_vecs(0u, v, pol);
            for (uint32_t base = 0u; base < src.ell_cols; base += kStep) {
                if (kOpPrefetch && base + kStep < src.ell_cols) load_vecs(base + kStep, nv, pol);
                uint32_t keep[kOpVecs], gene0[kOpVecs];
                keep_of(base, v, keep, gene0);
                uint32_t n = 0u;
#pragma unroll
                for (unsigned u = 0; u < kOpVecs; ++u) n += __popc(keep[u]);
                uint32_t total;
                uint32_t pos = run + block_exclusive_scan(n, scan33, total);
#pragma unroll
                for (unsigned u = 0; u < kOpVecs; ++u)
                    for (uint32_t bb = keep[u]; bb != 0u; bb &= bb - 1u, ++pos) {
                        const uint32_t q = __ffs(bb) - 1u;
                        minor_idx[pos] = gene0[u] + q;
                        out_val[pos] = half_of(v[u], q);
                    }
                run += total;
                next_step(base, v, nv, pol);
            }
        }
        __syncthreads(); // s_row / s_excl are rewritten by the next claim
    }
    if (threadIdx.x == 0u && kept != nullptr && cta_kept_rows != 0u) {
        atomicAdd(kept, (unsigned long long) cta_kept_rows);
        atomicAdd(kept + 1, cta_kept_slots);
    }
}

// major_ptr[r] for r in (rows, output_rows]: the total, major_ptr[rows] (the
// last kept row's inclusive prefix, or the zero set before the kernel).
__global__ void filter_onepass_tail_kernel(uint32_t rows, uint32_t output_rows, uint32_t *__restrict__ major_ptr) {
    const uint32_t total = major_ptr[rows];
    for (uint32_t r = rows + 1u + blockIdx.x * blockDim.x + threadIdx.x; r <= output_rows;
         r += gridDim.x * blockDim.x)
        major_ptr[r] = total;
}

// ---------------------------------------------------------------------------
// Marked filter, two passes with no waits between CTAs.  Pass 1: one warp per
// kept row counts its kept entries (eight 16-byte value loads per lane in
// flight) and marks, one bit per 8-value vector, the vectors that hold any; a
// device scan turns the counts (0 for dropped rows) into the row pointers.
// Pass 2: one warp per kept row compacts the indices of its marked vectors
// into shared memory (slot order), reads only those vectors again and writes
// their entries, a warp scan ranking each round.  The values cross HBM once,
// the marked vectors (those holding kept entries) a second time.
// ---------------------------------------------------------------------------
constexpr unsigned kMkWarps = 8;
constexpr unsigned kMkSteps = 4;        // 256-value steps per lane per group; two groups in flight
constexpr uint32_t kMkChunkWords = 64;  // mark words compacted per list fill (2,048 vectors)
constexpr unsigned kMkRound = 4;        // marked vectors per lane in flight in pass 2
constexpr unsigned kMkCtasPerSm = 4;    // pass 1 at <= 64 registers: four CTAs per SM

__device__ __forceinline__ void fill_keep_bitmap(uint32_t *bits, uint32_t words, const reopt_parts &parts,
                                                 const cs_row_feature_mask_view &masks) {
    uint32_t kcols = 0u;
    for (uint32_t k = 0; k < parts.count; ++k) kcols = max(kcols, parts.v[k].cols);
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
        uint32_t word = 0u;
        const uint32_t c0 = w * 32u;
#pragma unroll 4
        for (uint32_t k = 0; k < 32u; ++k)
            if (c0 + k < kcols) word |= (masks.feature_keep[c0 + k] != 0u ? 1u : 0u) << k;
        bits[w] = word;
    }
}

__global__ void __launch_bounds__(kMkWarps * 32, kMkCtasPerSm) filter_mark_kernel(
    const __grid_constant__ reopt_parts parts, cs_row_feature_mask_view masks, uint32_t output_cols,
    uint32_t *__restrict__ counts, uint32_t *__restrict__ marks, uint32_t mark_words,
    unsigned long long *__restrict__ kept, uint32_t keep_words) {
    extern __shared__ __align__(16) uint32_t mark_smem[];
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t rows = parts.row_off[parts.count];
    const uint32_t *kbits = keep_words != 0u ? mark_smem : nullptr;
    fill_keep_bitmap(mark_smem, keep_words, parts, masks);
    __syncthreads();
    uint32_t warp_kept_rows = 0u;
    unsigned long long warp_kept_slots = 0u;
    for (uint32_t row = blockIdx.x * kMkWarps + (threadIdx.x >> 5); row < rows; row += gridDim.x * kMkWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) {
            if (lane == 0u) counts[row] = 0u;
            continue;
        }
        const uint32_t part = part_of_row(parts, row);
        const cs_blocked_ell_view &src = parts.v[part];
        const uint32_t local = row - parts.row_off[part];
        warp_kept_rows += 1u;
        warp_kept_slots += src.ell_cols;
        const uint32_t B = src.block_size, W = src.ell_cols / B;
        const block_div bd(B);
        const uint32_t *bci = src.blockColIdx + (std::size_t) (local / B) * W;
        const uint16_t *vrow = src.val + (std::size_t) local * src.ell_cols;
        uint32_t *mrow = marks + (std::size_t) row * mark_words;
        const uint32_t lim = min(src.cols, output_cols);
        uint32_t n = 0u;
        uint4 v[kMkSteps], vn[kMkSteps];
        uint32_t bc[kMkSteps], bcn[kMkSteps];
        load_steps(vrow, bci, bd, src.ell_cols, lane * 8u, v, bc);
        for (uint32_t s0 = 0u; s0 * 256u < src.ell_cols; s0 += kMkSteps) {
            load_steps(vrow, bci, bd, src.ell_cols, (s0 + kMkSteps) * 256u + lane * 8u, vn, bcn);
            uint32_t word = 0u; // lane u keeps step s0 + u's mark word
#pragma unroll
            for (unsigned u = 0; u < kMkSteps; ++u) {
                // a vector past the row is zeros in an invalid slot: no kept entries
                const uint32_t e0 = (s0 + u) * 256u + lane * 8u;
                const uint32_t keep = onepass_keep(v[u], bc[u], bc[u] * B + bd.mod(e0), lim, kbits);
                n += __popc(keep);
                const uint32_t m = __ballot_sync(0xffffffffu, keep != 0u);
                if (lane == u) word = m;
                v[u] = vn[u];
                bc[u] = bcn[u];
            }
            if (lane < kMkSteps && s0 + lane < mark_words) mrow[s0 + lane] = word;
        }
        n = __reduce_add_sync(0xffffffffu, n);
        if (lane == 0u) counts[row] = n;
    }
    if (kept != nullptr && lane == 0u && warp_kept_rows != 0u) {
        atomicAdd(kept, (unsigned long long) warp_kept_rows);
        atomicAdd(kept + 1, warp_kept_slots);
    }
}

// 16-byte load of a scattered vector: no L1 line and no L2 prefetch beyond
// its own sector (the streaming loads ask for 256-byte L2 fills).
__device__ __forceinline__ uint4 ld_gather_v4(const void *p) {
    uint4 r;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p));
    return r;
}

__global__ void __launch_bounds__(kMkWarps * 32) filter_marked_emit_kernel(
    const __grid_constant__ reopt_parts parts, cs_row_feature_mask_view masks, uint32_t output_cols,
    const uint32_t *__restrict__ major_ptr, const uint32_t *__restrict__ marks, uint32_t mark_words,
    uint32_t *__restrict__ minor_idx, uint16_t *__restrict__ out_val, unsigned long long capacity,
    uint32_t *status, uint32_t keep_words) {
    extern __shared__ __align__(16) uint32_t mark_smem[];
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t rows = parts.row_off[parts.count];
    const uint32_t *kbits = keep_words != 0u ? mark_smem : nullptr;
    // after the feature bitmap: each warp's list of marked vectors (offsets in
    // the current chunk of kMkChunkWords mark words)
    uint16_t *list = reinterpret_cast<uint16_t *>(mark_smem + ((keep_words + 3u) & ~3u)) +
                     (threadIdx.x >> 5) * (kMkChunkWords * 32u);
    fill_keep_bitmap(mark_smem, keep_words, parts, masks);
    __syncthreads();
    if (blockIdx.x == 0u && threadIdx.x == 0u && major_ptr[rows] > capacity) status_or(status, CS_STATUS_CAPACITY);
    for (uint32_t row = blockIdx.x * kMkWarps + (threadIdx.x >> 5); row < rows; row += gridDim.x * kMkWarps) {
        if (masks.row_keep != nullptr && masks.row_keep[row] == 0u) continue;
        uint32_t run = major_ptr[row];
        if (major_ptr[row + 1u] == run || run >= capacity) continue; // nothing kept, or nothing that fits
        const uint32_t part = part_of_row(parts, row);
        const cs_blocked_ell_view &src = parts.v[part];
        const uint32_t local = row - parts.row_off[part];
        const uint32_t B = src.block_size, W = src.ell_cols / B;
        const block_div bd(B);
        const uint32_t *bci = src.blockColIdx + (std::size_t) (local / B) * W;
        const uint16_t *vrow = src.val + (std::size_t) local * src.ell_cols;
        const uint32_t *mrow = marks + (std::size_t) row * mark_words;
        const uint32_t lim = min(src.cols, output_cols);
        const uint32_t nwords = (src.ell_cols + 255u) / 256u;
        for (uint32_t w0 = 0u; w0 < nwords; w0 += kMkChunkWords) {
            // two mark words per lane; their set bits, in order, fill the list
            const uint32_t wa = w0 + 2u * lane;
            const uint32_t m0 = wa < nwords ? mrow[wa] : 0u;
            const uint32_t m1 = wa + 1u < nwords ? mrow[wa + 1u] : 0u;
            const uint32_t c = __popc(m0) + __popc(m1);
            const uint32_t incl = warp_inclusive_scan(c);
            const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
            uint32_t at = incl - c;
            for (uint32_t bb = m0; bb != 0u; bb &= bb - 1u) list[at++] = (uint16_t) (64u * lane + __ffs(bb) - 1u);
            for (uint32_t bb = m1; bb != 0u; bb &= bb - 1u) list[at++] = (uint16_t) (64u * lane + 31u + __ffs(bb));
            __syncwarp();
            for (uint32_t i0 = 0u; i0 < total; i0 += 32u * kMkRound) {
                uint4 v[kMkRound];
                uint32_t bc[kMkRound], e0[kMkRound];
#pragma unroll
                for (unsigned k = 0; k < kMkRound; ++k) {
                    const uint32_t i = i0 + k * 32u + lane;
                    const bool in = i < total;
                    e0[k] = (w0 * 32u + (in ? (uint32_t) list[i] : 0u)) * 8u;
                    v[k] = in ? ld_gather_v4(vrow + e0[k]) : make_uint4(0u, 0u, 0u, 0u);
                    bc[k] = in ? __ldg(bci + bd.div(e0[k])) : CS_INVALID_COL;
                }
#pragma unroll
                for (unsigned k = 0; k < kMkRound; ++k) {
                    const uint32_t gene0 = bc[k] * B + bd.mod(e0[k]);
                    const uint32_t keep = onepass_keep(v[k], bc[k], gene0, lim, kbits);
                    const uint32_t cnt = __popc(keep);
                    const uint32_t inc = warp_inclusive_scan(cnt);
                    uint32_t pos = run + inc - cnt;
                    for (uint32_t bb = keep; bb != 0u; bb &= bb - 1u, ++pos) {
                        const uint32_t q = __ffs(bb) - 1u;
                        if (pos < capacity) {
                            minor_idx[pos] = gene0 + q;
                            out_val[pos] = half_of(v[k], q);
                        }
                    }
                    run += __shfl_sync(0xffffffffu, inc, 31);
                }
            }
            __syncwarp(); // the list is refilled by the next chunk
        }
    }
}

// Group accumulator registers a call needs: none, 8, 16 or 32.
unsigned group_regs(const uint32_t *masks, uint32_t group_count) {
    if (masks == nullptr || group_count == 0u) return 0u;
    return group_count <= 8u ? 8u : group_count <= 16u ? 16u : 32u;
}

template <typename View>
using reduce_kernel_t = void (*)(View, const uint32_t *, uint32_t, cs_row_feature_mask_view, cs_group_filter_params,
                                 cs_group_reduce_out);

// Tensor-core Blocked-ELL-16 kernel for a group count: tiles of 8 groups and
// the per-row fallback's accumulators.
template <unsigned U>
reduce_kernel_t<cs_blocked_ell_view> bell16_mma_kernel(uint32_t groups) {
    switch ((groups + 7u) / 8u) {
    case 0: return group_reduce_bell16_mma_kernel<0u, 0u, U>;
    case 1: return group_reduce_bell16_mma_kernel<1u, 8u, U>;
    case 2: return group_reduce_bell16_mma_kernel<2u, 16u, U>;
    case 3: return group_reduce_bell16_mma_kernel<3u, 32u, U>;
    default: return group_reduce_bell16_mma_kernel<4u, 32u, U>;
    }
}

#define CS_PICK_REDUCE(KERNEL, VEC, GR)                                                                          \
    ((GR) == 0u ? KERNEL<VEC, 0u> : (GR) == 8u ? KERNEL<VEC, 8u> : (GR) == 16u ? KERNEL<VEC, 16u> : KERNEL<VEC, 32u>)

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
    const unsigned gr = group_regs(d_feature_group_masks, group_count);
    const bool mma = vec && src->block_size == 16u &&
                     (gr == 0u || (reinterpret_cast<uintptr_t>(d_feature_group_masks) & 15u) == 0u) &&
                     (m.feature_keep == nullptr || (reinterpret_cast<uintptr_t>(m.feature_keep) & 3u) == 0u);
    const uint32_t G = gr != 0u ? group_count : 0u;
    if (vec && src->block_size == 16u && G <= 15u) {
        // pipelined tensor-core kernel when the column table fits shared memory
        int dev = 0, optin = 0;
        if (cuda_ok(cudaGetDevice(&dev), "group_reduce_blocked_ell device") &&
            cuda_ok(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                    "group_reduce_blocked_ell shared memory limit")) {
            auto launch = [&](auto cfg) -> int {
                using CFG = decltype(cfg);
                const std::size_t psmem = pipe_smem_bytes<CFG>(src->cols);
                const reduce_kernel_t<cs_blocked_ell_view> k =
                    G == 0u ? group_reduce_bell16_pipe_kernel<0u, 0u, CFG>
                            : G <= 8u ? group_reduce_bell16_pipe_kernel<1u, 8u, CFG>
                                      : group_reduce_bell16_pipe_kernel<2u, 16u, CFG>;
                if (!cuda_ok(cudaFuncSetAttribute(reinterpret_cast<const void *>(k),
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int) psmem),
                             "group_reduce_bell16_pipe_kernel shared memory"))
                    return 0;
                const uint32_t row_blocks = (src->rows + 15u) / 16u;
                const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), CFG::warps * 32u, psmem,
                                                    (row_blocks + CFG::warps - 1u) / CFG::warps);
                k<<<grid, CFG::warps * 32u, psmem, as_stream(s)>>>(*src, d_feature_group_masks, group_count, m,
                                                                    *filter, *out);
                return launch_ok("group_reduce_bell16_pipe_kernel");
            };
            if (pipe_smem_bytes<pipe_wide>(src->cols) <= (std::size_t) optin) return launch(pipe_wide{});
            if (pipe_smem_bytes<pipe_narrow>(src->cols) <= (std::size_t) optin) return launch(pipe_narrow{});
        }
    }
    if (mma) {
        const reduce_kernel_t<cs_blocked_ell_view> k = bell16_mma_kernel<4u>(G);
        const uint32_t row_blocks = (src->rows + 15u) / 16u;
        const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kRowThreads, smem,
                                            (row_blocks + kRowWarps - 1u) / kRowWarps);
        k<<<grid, kRowThreads, smem, as_stream(s)>>>(*src, d_feature_group_masks, group_count, m, *filter, *out);
        return launch_ok("group_reduce_bell16_mma_kernel");
    }
    const reduce_kernel_t<cs_blocked_ell_view> k = vec ? CS_PICK_REDUCE(group_reduce_bell_kernel, true, gr)
                                                       : CS_PICK_REDUCE(group_reduce_bell_kernel, false, gr);
    const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kRowThreads, smem,
                                        (src->rows + kRowWarps - 1u) / kRowWarps);
    k<<<grid, kRowThreads, smem, as_stream(s)>>>(*src, d_feature_group_masks, group_count, m, *filter, *out);
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
    const bool vec = (reinterpret_cast<uintptr_t>(src->col_idx) & 15u) == 0u &&
                     (reinterpret_cast<uintptr_t>(src->val) & 7u) == 0u;
    const std::size_t csmem = kSellCodes && vec ? codes_smem(d_feature_group_masks, group_count, src->cols) : 0u;
    if (csmem != 0u) {
        const unsigned g = group_regs(d_feature_group_masks, group_count);
        return launch_codes<cs_sliced_ell_view>(g == 0u ? group_reduce_sell_codes_kernel<0u>
                                                        : g == 8u ? group_reduce_sell_codes_kernel<8u>
                                                                  : group_reduce_sell_codes_kernel<16u>,
                                                *src, d_feature_group_masks, group_count, m, *filter, *out, csmem,
                                                as_stream(s), "group_reduce_sell_codes_kernel");
    }
    const std::size_t smem = group_smem(d_feature_group_masks, group_count);
    const unsigned gr = group_regs(d_feature_group_masks, group_count);
    const reduce_kernel_t<cs_sliced_ell_view> k = vec ? CS_PICK_REDUCE(group_reduce_sell_kernel, true, gr)
                                                      : CS_PICK_REDUCE(group_reduce_sell_kernel, false, gr);
    const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kRowThreads, smem,
                                        (src->rows + kRowWarps - 1u) / kRowWarps);
    k<<<grid, kRowThreads, smem, as_stream(s)>>>(*src, d_feature_group_masks, group_count, m, *filter, *out);
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
    const bool vec = (reinterpret_cast<uintptr_t>(src->minorIdx) & 15u) == 0u &&
                     (reinterpret_cast<uintptr_t>(src->val) & 7u) == 0u;
    const std::size_t csmem = vec ? codes_smem(d_feature_group_masks, group_count, src->cols) : 0u;
    if (csmem != 0u) {
        const unsigned g = group_regs(d_feature_group_masks, group_count);
        return launch_codes<cs_compressed_view>(g == 0u ? group_reduce_csr_codes_kernel<0u>
                                                        : g == 8u ? group_reduce_csr_codes_kernel<8u>
                                                                  : group_reduce_csr_codes_kernel<16u>,
                                                *src, d_feature_group_masks, group_count, m, *filter, *out, csmem,
                                                as_stream(s), "group_reduce_csr_codes_kernel");
    }
    const std::size_t smem = group_smem(d_feature_group_masks, group_count);
    const unsigned gr = group_regs(d_feature_group_masks, group_count);
    const reduce_kernel_t<cs_compressed_view> k = vec ? CS_PICK_REDUCE(group_reduce_csr_kernel, true, gr)
                                                      : CS_PICK_REDUCE(group_reduce_csr_kernel, false, gr);
    const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kRowThreads, smem,
                                        (src->rows + kRowWarps - 1u) / kRowWarps);
    k<<<grid, kRowThreads, smem, as_stream(s)>>>(*src, d_feature_group_masks, group_count, m, *filter, *out);
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

namespace csb {
namespace {

bool make_parts(const cs_blocked_ell_view *views, uint32_t count, reopt_parts *p, const char *who) {
    if (views == nullptr || count == 0u || count > CS_MAX_REPACK_PARTS) {
        set_error("%s: 1..%u partition views required", who, CS_MAX_REPACK_PARTS);
        return false;
    }
    std::memset(p, 0, sizeof(*p));
    uint64_t rows = 0u;
    for (uint32_t k = 0; k < count; ++k) {
        if (views[k].block_size == 0u && views[k].ell_cols != 0u) {
            set_error("%s: partition %u has a zero block size", who, k);
            return false;
        }
        p->v[k] = views[k];
        p->row_off[k] = (uint32_t) rows;
        rows += views[k].rows;
    }
    if (rows > 0xffffffffull) {
        set_error("%s: shard rows overflow 32 bits", who);
        return false;
    }
    p->row_off[count] = (uint32_t) rows;
    p->count = count;
    return true;
}

// Words of the shared feature bitmap: the flags of every column of every part
// (up to 12,288 words = 48 KB of dynamic shared memory), 0 without flags or
// beyond that width (the kernel then reads the flags per column).
uint32_t keep_bitmap_words(const reopt_parts &parts, const cs_row_feature_mask_view &m) {
    if (m.feature_keep == nullptr) return 0u;
    uint32_t cols = 0u;
    for (uint32_t k = 0; k < parts.count; ++k) cols = parts.v[k].cols > cols ? parts.v[k].cols : cols;
    const uint32_t words = (cols + 31u) / 32u;
    return words <= 12288u ? words : 0u;
}

// The vector filters (one pass, marked): no remaps, output_rows >= the
// shard's rows, block sizes multiples of 8 with 16-byte aligned values, and a
// feature bitmap that fits in shared memory (*kw words).
int vector_filter_qualifies(const reopt_parts &p, const cs_row_feature_mask_view &m, uint32_t output_rows,
                            uint32_t *kw, const char *who) {
    const uint32_t rows = p.row_off[p.count];
    if (m.row_remap != nullptr || m.feature_remap != nullptr) {
        set_error("%s: row or feature remaps need the count + emit path", who);
        return 0;
    }
    if (output_rows < rows) {
        set_error("%s: output_rows %u below the shard's %u rows", who, output_rows, rows);
        return 0;
    }
    for (uint32_t k = 0; k < p.count; ++k) {
        const cs_blocked_ell_view &v = p.v[k];
        if (v.rows == 0u || v.ell_cols == 0u) continue;
        if (v.block_size % 8u != 0u || (reinterpret_cast<uintptr_t>(v.val) & 15u) != 0u || v.val == nullptr ||
            v.blockColIdx == nullptr) {
            set_error("%s: partition %u needs a block size that is a multiple of 8 and 16-byte aligned values", who,
                      k);
            return 0;
        }
    }
    *kw = keep_bitmap_words(p, m);
    if (m.feature_keep != nullptr && *kw == 0u) {
        set_error("%s: too many columns for the shared feature bitmap", who);
        return 0;
    }
    return 1;
}

int reopt_count_launch(const reopt_parts &parts, const cs_row_feature_mask_view *masks, uint32_t output_rows,
                       uint32_t output_cols, uint32_t *d_major_ptr, uint64_t *d_kept, void *d_scratch,
                       std::size_t scratch_bytes, uint32_t *d_status, cudaStream_t stream, const char *who) {
    const uint32_t rows = parts.row_off[parts.count];
    size_t need = 0;
    cs_b200_reoptimize_scratch_bytes(rows, output_rows, &need);
    if (d_scratch == nullptr || scratch_bytes < need) {
        set_error("%s: scratch %zu < %zu", who, scratch_bytes, need);
        return 0;
    }
    uint32_t *claims = (uint32_t *) d_scratch;
    void *scan_scratch = (char *) d_scratch + align_up((std::size_t) output_rows * sizeof(uint32_t) + 16u, 256);
    if (!cuda_ok(cudaMemsetAsync(d_major_ptr, 0, ((std::size_t) output_rows + 1u) * sizeof(uint32_t), stream),
                 "memset major_ptr") ||
        !cuda_ok(cudaMemsetAsync(claims, 0, (std::size_t) output_rows * sizeof(uint32_t) + 4u, stream),
                 "memset claims") ||
        (d_kept != nullptr && !cuda_ok(cudaMemsetAsync(d_kept, 0, 16, stream), "memset kept")))
        return 0;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    if (rows != 0u && (output_rows != 0u || d_kept != nullptr)) {
        const uint32_t kw = keep_bitmap_words(parts, m);
        const auto k = reopt_kernel<false>;
        const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kRowThreads, kw * 4u,
                                            (rows + kRowWarps - 1u) / kRowWarps);
        k<<<grid, kRowThreads, kw * 4u, stream>>>(parts, m, output_rows, output_cols, d_major_ptr, claims, nullptr,
                                                 nullptr, d_status, reinterpret_cast<unsigned long long *>(d_kept),
                                                 kw);
        if (!launch_ok("reopt_count_kernel")) return 0;
    }
    return scan_exclusive_u32(d_major_ptr, d_major_ptr, output_rows, true, scan_scratch,
                              scan_u32_scratch_bytes(output_rows), stream);
}

int reopt_emit_launch(const reopt_parts &parts, const cs_row_feature_mask_view *masks, uint32_t output_rows,
                      uint32_t output_cols, const uint32_t *d_major_ptr, uint32_t *d_minor_idx, uint16_t *d_val,
                      cudaStream_t stream) {
    const uint32_t rows = parts.row_off[parts.count];
    if (rows == 0u || output_rows == 0u) return 1;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    const uint32_t kw = keep_bitmap_words(parts, m);
    const auto k = reopt_kernel<true>;
    const unsigned grid = resident_grid(reinterpret_cast<const void *>(k), kRowThreads, kw * 4u,
                                        (rows + kRowWarps - 1u) / kRowWarps);
    k<<<grid, kRowThreads, kw * 4u, stream>>>(parts, m, output_rows, output_cols, const_cast<uint32_t *>(d_major_ptr),
                                             nullptr, d_minor_idx, d_val, nullptr, nullptr, kw);
    return launch_ok("reopt_emit_kernel");
}

} // namespace
} // namespace csb

extern "C" int cs_b200_reoptimize_count(const cs_blocked_ell_view *src, const cs_row_feature_mask_view *masks,
                                        uint32_t output_rows, uint32_t output_cols, uint32_t *d_major_ptr,
                                        void *d_scratch, size_t scratch_bytes, uint32_t *d_status, cs_stream_t s) {
    if (src == nullptr || d_major_ptr == nullptr) {
        set_error("reoptimize_count: null view or major_ptr");
        return 0;
    }
    reopt_parts parts;
    if (!make_parts(src, 1u, &parts, "reoptimize_count")) return 0;
    return reopt_count_launch(parts, masks, output_rows, output_cols, d_major_ptr, nullptr, d_scratch, scratch_bytes,
                              d_status, as_stream(s), "reoptimize_count");
}

extern "C" int cs_b200_reoptimize_emit(const cs_blocked_ell_view *src, const cs_row_feature_mask_view *masks,
                                       uint32_t output_rows, uint32_t output_cols, const uint32_t *d_major_ptr,
                                       uint32_t *d_minor_idx, uint16_t *d_val, cs_stream_t s) {
    if (src == nullptr || d_major_ptr == nullptr) {
        set_error("reoptimize_emit: null view or major_ptr");
        return 0;
    }
    reopt_parts parts;
    if (!make_parts(src, 1u, &parts, "reoptimize_emit")) return 0;
    return reopt_emit_launch(parts, masks, output_rows, output_cols, d_major_ptr, d_minor_idx, d_val, as_stream(s));
}

extern "C" int cs_b200_filter_blocked_ell_scratch_bytes(uint32_t shard_rows, uint32_t output_rows, size_t *out_bytes) {
    return cs_b200_reoptimize_scratch_bytes(shard_rows, output_rows, out_bytes);
}

extern "C" int cs_b200_filter_blocked_ell_count(const cs_blocked_ell_view *parts, uint32_t part_count,
                                                const cs_row_feature_mask_view *masks, uint32_t output_rows,
                                                uint32_t output_cols, uint32_t *d_major_ptr, uint64_t *d_kept,
                                                void *d_scratch, size_t scratch_bytes, uint32_t *d_status,
                                                cs_stream_t s) {
    if (d_major_ptr == nullptr) {
        set_error("filter_blocked_ell_count: null major_ptr");
        return 0;
    }
    reopt_parts p;
    if (!make_parts(parts, part_count, &p, "filter_blocked_ell_count")) return 0;
    return reopt_count_launch(p, masks, output_rows, output_cols, d_major_ptr, d_kept, d_scratch, scratch_bytes,
                              d_status, as_stream(s), "filter_blocked_ell_count");
}

extern "C" int cs_b200_filter_blocked_ell_emit(const cs_blocked_ell_view *parts, uint32_t part_count,
                                               const cs_row_feature_mask_view *masks, uint32_t output_rows,
                                               uint32_t output_cols, const uint32_t *d_major_ptr,
                                               uint32_t *d_minor_idx, uint16_t *d_val, cs_stream_t s) {
    if (d_major_ptr == nullptr) {
        set_error("filter_blocked_ell_emit: null major_ptr");
        return 0;
    }
    reopt_parts p;
    if (!make_parts(parts, part_count, &p, "filter_blocked_ell_emit")) return 0;
    return reopt_emit_launch(p, masks, output_rows, output_cols, d_major_ptr, d_minor_idx, d_val, as_stream(s));
}

extern "C" int cs_b200_filter_blocked_ell_onepass_scratch_bytes(const cs_blocked_ell_view *parts, uint32_t part_count,
                                                                size_t *out_bytes) {
    static const char *who = "filter_blocked_ell_onepass_scratch_bytes";
    if (out_bytes == nullptr) {
        set_error("%s: null output", who);
        return 0;
    }
    reopt_parts p;
    if (!make_parts(parts, part_count, &p, who)) return 0;
    *out_bytes = align_up(((std::size_t) p.row_off[p.count] + 1u) * 8u + 16u, 256);
    return 1;
}

extern "C" int cs_b200_filter_blocked_ell_onepass(const cs_blocked_ell_view *parts, uint32_t part_count,
                                                  const cs_row_feature_mask_view *masks, uint32_t output_rows,
                                                  uint32_t output_cols, uint32_t *d_major_ptr, uint32_t *d_minor_idx,
                                                  uint16_t *d_val, uint64_t capacity, uint64_t *d_kept,
                                                  void *d_scratch, size_t scratch_bytes, uint32_t *d_status,
                                                  cs_stream_t s) {
    static const char *who = "filter_blocked_ell_onepass";
    if (d_major_ptr == nullptr || (capacity != 0u && (d_minor_idx == nullptr || d_val == nullptr))) {
        set_error("%s: null output array", who);
        return 0;
    }
    reopt_parts p;
    if (!make_parts(parts, part_count, &p, who)) return 0;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    const uint32_t rows = p.row_off[p.count];
    uint32_t kw = 0u;
    if (!vector_filter_qualifies(p, m, output_rows, &kw, who)) return 0;
    const std::size_t need = align_up(((std::size_t) rows + 1u) * 8u + 16u, 256);
    if (d_scratch == nullptr || scratch_bytes < need) {
        set_error("%s: scratch %zu < %zu", who, scratch_bytes, need);
        return 0;
    }
    cudaStream_t stream = as_stream(s);
    auto *state = static_cast<unsigned long long *>(d_scratch);
    auto *counter = reinterpret_cast<uint32_t *>(state + rows + 1u);
    // row pointers start at zero: dropped rows before the first kept row keep it
    if (!cuda_ok(cudaMemsetAsync(d_scratch, 0, need, stream), "onepass scratch memset") ||
        !cuda_ok(cudaMemsetAsync(d_major_ptr, 0, ((std::size_t) rows + 1u) * 4u, stream), "onepass row pointers") ||
        (d_kept != nullptr && !cuda_ok(cudaMemsetAsync(d_kept, 0, 16, stream), "memset kept")))
        return 0;
    if (rows != 0u) {
        const auto k = filter_onepass_kernel;
        // a few CTAs per SM: enough bytes in flight, few enough rows in flight to stay in L2
        unsigned grid = (unsigned) sm_count() * kOpCtasPerSm;
        if (grid > rows) grid = rows;
        const std::size_t smem = ((std::size_t) ((kw + 3u) & ~3u) + kOpPackedSteps * kOpThreads) * 4u;
        if (smem > 48u * 1024u &&
            !cuda_ok(cudaFuncSetAttribute(reinterpret_cast<const void *>(k),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                     "onepass shared memory"))
            return 0;
        k<<<grid, kOpThreads, smem, stream>>>(p, m, output_cols, d_major_ptr, d_minor_idx, d_val, capacity, state,
                                                 counter, d_status, reinterpret_cast<unsigned long long *>(d_kept),
                                                 kw);
        if (!launch_ok("filter_onepass_kernel")) return 0;
    }
    const uint32_t tail = output_rows - rows + 1u;
    filter_onepass_tail_kernel<<<(tail + 255u) / 256u > 1024u ? 1024u : (tail + 255u) / 256u, 256, 0, stream>>>(
        rows, output_rows, d_major_ptr);
    return launch_ok("filter_onepass_tail_kernel");
}

namespace {
// Mark words per row: one per 256 values of the widest partition.
uint32_t mark_words_of(const csb::reopt_parts &p) {
    uint32_t w = 0u;
    for (uint32_t k = 0; k < p.count; ++k) w = std::max(w, (p.v[k].ell_cols + 255u) / 256u);
    return w;
}
std::size_t marked_scan_bytes(uint32_t rows) { return align_up(scan_u32_scratch_bytes(rows), 256); }
} // namespace

extern "C" int cs_b200_filter_blocked_ell_marked_scratch_bytes(const cs_blocked_ell_view *parts, uint32_t part_count,
                                                               size_t *out_bytes) {
    static const char *who = "filter_blocked_ell_marked_scratch_bytes";
    if (out_bytes == nullptr) {
        set_error("%s: null output", who);
        return 0;
    }
    reopt_parts p;
    if (!make_parts(parts, part_count, &p, who)) return 0;
    const uint32_t rows = p.row_off[p.count];
    *out_bytes = marked_scan_bytes(rows) + align_up((std::size_t) rows * mark_words_of(p) * 4u + 4u, 256);
    return 1;
}

extern "C" int cs_b200_filter_blocked_ell_marked(const cs_blocked_ell_view *parts, uint32_t part_count,
                                                 const cs_row_feature_mask_view *masks, uint32_t output_rows,
                                                 uint32_t output_cols, uint32_t *d_major_ptr, uint32_t *d_minor_idx,
                                                 uint16_t *d_val, uint64_t capacity, uint64_t *d_kept,
                                                 void *d_scratch, size_t scratch_bytes, uint32_t *d_status,
                                                 cs_stream_t s) {
    static const char *who = "filter_blocked_ell_marked";
    if (d_major_ptr == nullptr || (capacity != 0u && (d_minor_idx == nullptr || d_val == nullptr))) {
        set_error("%s: null output array", who);
        return 0;
    }
    reopt_parts p;
    if (!make_parts(parts, part_count, &p, who)) return 0;
    const cs_row_feature_mask_view m = masks != nullptr ? *masks : cs_row_feature_mask_view{};
    const uint32_t rows = p.row_off[p.count];
    uint32_t kw = 0u;
    if (!vector_filter_qualifies(p, m, output_rows, &kw, who)) return 0;
    const uint32_t mw = mark_words_of(p);
    std::size_t need = 0;
    if (!cs_b200_filter_blocked_ell_marked_scratch_bytes(parts, part_count, &need)) return 0;
    if (d_scratch == nullptr || scratch_bytes < need) {
        set_error("%s: scratch %zu < %zu", who, scratch_bytes, need);
        return 0;
    }
    cudaStream_t stream = as_stream(s);
    void *scan_tmp = d_scratch;
    auto *marks = reinterpret_cast<uint32_t *>(static_cast<char *>(d_scratch) + marked_scan_bytes(rows));
    if (d_kept != nullptr && !cuda_ok(cudaMemsetAsync(d_kept, 0, 16, stream), "memset kept")) return 0;
    const std::size_t smem_mark = (std::size_t) kw * 4u;
    const std::size_t smem_emit = (std::size_t) ((kw + 3u) & ~3u) * 4u + (std::size_t) kMkWarps * kMkChunkWords * 32u * 2u;
    if (rows != 0u) {
        unsigned grid = (rows + kMkWarps - 1u) / kMkWarps;
        const unsigned cap = (unsigned) sm_count() * 16u;
        if (grid > cap) grid = cap;
        if (smem_mark > 48u * 1024u &&
            !cuda_ok(cudaFuncSetAttribute(reinterpret_cast<const void *>(filter_mark_kernel),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_mark),
                     "mark shared memory"))
            return 0;
        filter_mark_kernel<<<grid, kMkWarps * 32, smem_mark, stream>>>(
            p, m, output_cols, d_major_ptr, marks, mw, reinterpret_cast<unsigned long long *>(d_kept), kw);
        if (!launch_ok("filter_mark_kernel")) return 0;
        if (!scan_exclusive_u32(d_major_ptr, d_major_ptr, rows, true, scan_tmp, marked_scan_bytes(rows), stream))
            return 0;
        if (smem_emit > 48u * 1024u &&
            !cuda_ok(cudaFuncSetAttribute(reinterpret_cast<const void *>(filter_marked_emit_kernel),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_emit),
                     "marked emit shared memory"))
            return 0;
        filter_marked_emit_kernel<<<grid, kMkWarps * 32, smem_emit, stream>>>(
            p, m, output_cols, d_major_ptr, marks, mw, d_minor_idx, d_val, capacity, d_status, kw);
        if (!launch_ok("filter_marked_emit_kernel")) return 0;
    } else if (!cuda_ok(cudaMemsetAsync(d_major_ptr, 0, 4, stream), "marked row pointer")) {
        return 0;
    }
    const uint32_t tail = output_rows - rows + 1u;
    filter_onepass_tail_kernel<<<(tail + 255u) / 256u > 1024u ? 1024u : (tail + 255u) / 256u, 256, 0, stream>>>(
        rows, output_rows, d_major_ptr);
    return launch_ok("filter_onepass_tail_kernel");
}
