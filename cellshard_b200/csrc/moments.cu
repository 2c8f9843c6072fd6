// Row-label grouped per-feature moments over Blocked-ELL.
//
// For every kept row r with label g and every feature f:
//     sum[g][f] += x,  sumsq[g][f] += x*x   (x = fp16 value widened to fp32)
//
// Plan (all stream-ordered, no host synchronisation):
//   1. index     one warp per row block turns its ascending blockColIdx row
//                into a bitmap over column blocks plus per-32-block prefix
//                counts, so slot(rb, b) = prefix + popc(word & below(b)).
//   2. sort      stable counting sort of kept rows by label (tile histograms,
//                one-CTA group scan that also cuts each group's rows into
//                chunks, tile-local ranked scatter).
//   3. accumulate  grid (chunk, feature tile): each thread owns L consecutive
//                features of one column block and streams its chunk's rows
//                (all of one group), keeping its sums in registers; fp32 batch
//                sums of kBatch rows are folded into hi/lo two-sum pairs.
//                One partial (hi, lo) per (chunk, feature) goes to scratch.
//   4. combine   per (group, feature): add the group's chunk partials (fp64 or
//                fp32 by scheme), apply the feature mask, emit sum, sumsq,
//                mean and variance.
#include "common.cuh"
#include "moments_device.cuh"

#include <cstring>

namespace csb {
namespace {

constexpr unsigned kTileRows = 1024;   // rows per sort tile
constexpr unsigned kSortThreads = 256; // 8 warps x 128 rows
constexpr unsigned kSortWarps = kSortThreads / 32;
constexpr unsigned kAccThreads = 256;
constexpr unsigned kBatch = 8;         // rows per fp32 batch sum
constexpr unsigned kDefaultChunkRows = 2048;
constexpr unsigned kMaxChunkRows = 8192;
constexpr unsigned kIndexWarps = 4;
constexpr unsigned kMaxIndexWords = 2048; // column blocks / 32 per row block

struct chunk_desc {
    uint32_t group;
    uint32_t begin;
    uint32_t end;
    uint32_t pad;
};

struct moments_layout {
    uint2 *index;              // [row_blocks * words]
    uint32_t *tile_counts;     // [tiles * G]
    uint32_t *group_offsets;   // [G + 1]
    uint32_t *group_rows;      // [G]
    uint32_t *chunk_first;     // [G + 1]
    uint32_t *num_chunks;      // [1]
    chunk_desc *chunks;        // [max_chunks]
    uint32_t *sorted_rows;     // [rows]
    float *partials;           // [max_chunks * 4 * cols]
    std::size_t bytes;
    uint32_t row_blocks, words, tiles, max_chunks, chunk_rows, col_blocks;
};

bool make_layout(const cs_blocked_ell_view *src, const cs_group_moments_params *p, void *base, std::size_t cap,
                 moments_layout *lay) {
    const uint32_t B = src->block_size;
    lay->row_blocks = (src->rows + B - 1u) / B;
    lay->col_blocks = (src->cols + B - 1u) / B;
    lay->words = (lay->col_blocks + 31u) / 32u;
    lay->tiles = (src->rows + kTileRows - 1u) / kTileRows;
    lay->chunk_rows = p->chunk_rows == 0u ? kDefaultChunkRows : p->chunk_rows;
    const std::size_t G = p->group_count;
    lay->max_chunks = (uint32_t) ((src->rows + lay->chunk_rows - 1u) / lay->chunk_rows + G);
    scratch_carver c(base, cap);
    lay->index = c.take<uint2>((std::size_t) lay->row_blocks * lay->words + 1);
    lay->tile_counts = c.take<uint32_t>((std::size_t) lay->tiles * G + 1);
    lay->group_offsets = c.take<uint32_t>(G + 1);
    lay->group_rows = c.take<uint32_t>(G);
    lay->chunk_first = c.take<uint32_t>(G + 1);
    lay->num_chunks = c.take<uint32_t>(1);
    lay->chunks = c.take<chunk_desc>(lay->max_chunks);
    lay->sorted_rows = c.take<uint32_t>((std::size_t) src->rows + 1);
    lay->partials = c.take<float>((std::size_t) lay->max_chunks * 4u * src->cols + 1);
    lay->bytes = c.used;
    return c.fits();
}

// ---------------------------------------------------------------------------
// 1. Column-block index per row block.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kIndexWarps * 32) moments_index_kernel(const uint32_t *__restrict__ block_col_idx,
                                                                         uint32_t row_blocks, uint32_t width,
                                                                         uint32_t col_blocks, uint32_t words,
                                                                         uint2 *__restrict__ index,
                                                                         uint32_t *status, bool vec4) {
    extern __shared__ uint32_t bitmap_smem[];
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t *bits = bitmap_smem + (std::size_t) warp * words;
    for (uint32_t rb = blockIdx.x * kIndexWarps + warp; rb < row_blocks; rb += gridDim.x * kIndexWarps) {
        for (uint32_t w = lane; w < words; w += 32u) bits[w] = 0u;
        __syncwarp();
        const uint32_t *row = block_col_idx + (std::size_t) rb * width;
        uint32_t bad = 0u;
        auto mark = [&](uint32_t bc, uint32_t prev, bool has_prev) {
            if (bc == CS_INVALID_COL) return;
            if (bc >= col_blocks)
                bad |= CS_STATUS_INDEX_RANGE;
            else
                atomicOr(bits + (bc >> 5), 1u << (bc & 31u));
            if (has_prev && (prev == CS_INVALID_COL || prev >= bc)) bad |= CS_STATUS_BLOCK_COL_ORDER;
        };
        if (vec4) {
            // 4 entries per lane per step; the entry before a lane's first one is
            // the previous lane's last (or the previous step's lane 31)
            uint32_t carry = CS_INVALID_COL;
            for (uint32_t s0 = 0; s0 < width; s0 += 128u) {
                const uint32_t s = s0 + lane * 4u;
                uint4 q = make_uint4(CS_INVALID_COL, CS_INVALID_COL, CS_INVALID_COL, CS_INVALID_COL);
                if (s < width) q = __ldg(reinterpret_cast<const uint4 *>(row + s));
                uint32_t before = __shfl_up_sync(0xffffffffu, q.w, 1);
                if (lane == 0u) before = carry;
                if (s < width) {
                    mark(q.x, before, s > 0u);
                    mark(q.y, q.x, true);
                    mark(q.z, q.y, true);
                    mark(q.w, q.z, true);
                }
                carry = __shfl_sync(0xffffffffu, q.w, 31);
            }
        } else {
            for (uint32_t s = lane; s < width; s += 32u) mark(row[s], s > 0u ? row[s - 1u] : 0u, s > 0u);
        }
        bad = __reduce_or_sync(0xffffffffu, bad);
        if (lane == 0u) status_or(status, bad);
        __syncwarp();
        uint32_t carry = 0u;
        for (uint32_t w0 = 0; w0 < words; w0 += 32u) {
            const uint32_t w = w0 + lane;
            const uint32_t word = w < words ? bits[w] : 0u;
            const uint32_t cnt = __popc(word);
            uint32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (unsigned) o) incl += t;
            }
            if (w < words) index[(std::size_t) rb * words + w] = make_uint2(word, carry + incl - cnt);
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 2. Stable counting sort of kept rows by label.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t row_group(uint32_t r, uint32_t rows, const uint8_t *keep, const uint32_t *labels,
                                              uint32_t G) {
    if (r >= rows) return G;
    if (keep != nullptr && keep[r] == 0u) return G;
    const uint32_t g = labels != nullptr ? labels[r] : 0u;
    return g < G ? g : G;
}

__global__ void __launch_bounds__(kSortThreads) moments_tile_hist_kernel(uint32_t rows, const uint8_t *__restrict__ keep,
                                                                         const uint32_t *__restrict__ labels, uint32_t G,
                                                                         uint32_t *__restrict__ tile_counts) {
    extern __shared__ uint32_t hist[];
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) hist[g] = 0u;
    __syncthreads();
    const uint32_t base = blockIdx.x * kTileRows;
    for (uint32_t i = threadIdx.x; i < kTileRows; i += blockDim.x) {
        const uint32_t g = row_group(base + i, rows, keep, labels, G);
        if (g < G) atomicAdd(hist + g, 1u);
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x)
        tile_counts[(std::size_t) blockIdx.x * G + g] = hist[g];
}

// One warp per group: exclusive scan of the group's per-tile counts (in
// place, group-relative) and the group's row total.
__global__ void __launch_bounds__(256) moments_group_tiles_kernel(uint32_t tiles, uint32_t G,
                                                                  uint32_t *__restrict__ tile_counts,
                                                                  uint32_t *__restrict__ group_rows) {
    const uint32_t g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const unsigned lane = threadIdx.x & 31u;
    if (g >= G) return;
    uint32_t carry = 0u;
    for (uint32_t t0 = 0; t0 < tiles; t0 += 32u) {
        const uint32_t t = t0 + lane;
        const std::size_t k = (std::size_t) t * G + g;
        const uint32_t c = t < tiles ? tile_counts[k] : 0u;
        const uint32_t incl = warp_inclusive_scan(c);
        if (t < tiles) tile_counts[k] = carry + incl - c;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0u) group_rows[g] = carry;
}

// One CTA: group offsets, chunk cutting (each chunk holds rows of one group).
__global__ void __launch_bounds__(1024) moments_group_scan_kernel(uint32_t G, uint32_t chunk_rows, uint32_t max_chunks,
                                                                  const uint32_t *__restrict__ group_rows,
                                                                  uint32_t *__restrict__ group_offsets,
                                                                  uint32_t *__restrict__ chunk_first,
                                                                  uint32_t *__restrict__ num_chunks,
                                                                  chunk_desc *__restrict__ chunks) {
    __shared__ uint32_t smem[33];
    uint32_t carry_rows = 0u, carry_chunks = 0u;
    for (uint32_t g0 = 0; g0 < G; g0 += blockDim.x) {
        const uint32_t g = g0 + threadIdx.x;
        const uint32_t n = g < G ? group_rows[g] : 0u;
        const uint32_t nc = g < G ? (n + chunk_rows - 1u) / chunk_rows : 0u;
        uint32_t tot_n, tot_c;
        const uint32_t ex_n = block_exclusive_scan(n, smem, tot_n);
        const uint32_t ex_c = block_exclusive_scan(nc, smem, tot_c);
        if (g < G) {
            const uint32_t off = carry_rows + ex_n;
            const uint32_t cf = carry_chunks + ex_c;
            group_offsets[g] = off;
            chunk_first[g] = cf;
            for (uint32_t c = 0; c < nc; ++c) {
                const uint32_t b = off + c * chunk_rows;
                const uint32_t e = (c + 1u == nc) ? off + n : b + chunk_rows;
                if (cf + c < max_chunks) chunks[cf + c] = chunk_desc{g, b, e, 0u};
            }
        }
        carry_rows += tot_n;
        carry_chunks += tot_c;
    }
    if (threadIdx.x == 0) {
        group_offsets[G] = carry_rows;
        chunk_first[G] = carry_chunks;
        *num_chunks = carry_chunks;
    }
}

__global__ void __launch_bounds__(kSortThreads) moments_tile_scatter_kernel(uint32_t rows,
                                                                            const uint8_t *__restrict__ keep,
                                                                            const uint32_t *__restrict__ labels,
                                                                            uint32_t G,
                                                                            const uint32_t *__restrict__ tile_base,
                                                                            const uint32_t *__restrict__ group_offsets,
                                                                            uint32_t *__restrict__ sorted_rows) {
    extern __shared__ uint32_t warp_counts[]; // [kSortWarps][G]
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t i = threadIdx.x; i < kSortWarps * G; i += blockDim.x) warp_counts[i] = 0u;
    __syncthreads();
    constexpr uint32_t rows_per_warp = kTileRows / kSortWarps;
    const uint32_t wbase = blockIdx.x * kTileRows + warp * rows_per_warp;
    uint32_t *my = warp_counts + (std::size_t) warp * G;
    for (uint32_t b = 0; b < rows_per_warp; b += 32u) {
        const uint32_t r = wbase + b + lane;
        const uint32_t g = row_group(r, rows, keep, labels, G);
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        if (g < G && lane == (unsigned) (__ffs(peers) - 1)) my[g] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
        uint32_t run = tile_base[(std::size_t) blockIdx.x * G + g] + group_offsets[g];
        for (unsigned w = 0; w < kSortWarps; ++w) {
            const uint32_t c = warp_counts[(std::size_t) w * G + g];
            warp_counts[(std::size_t) w * G + g] = run;
            run += c;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t b = 0; b < rows_per_warp; b += 32u) {
        const uint32_t r = wbase + b + lane;
        const uint32_t g = row_group(r, rows, keep, labels, G);
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        uint32_t base = 0u;
        if (g < G) base = my[g];
        __syncwarp();
        if (g < G) {
            sorted_rows[base + __popc(peers & lt)] = r;
            if (lane == (unsigned) (__ffs(peers) - 1)) my[g] = base + __popc(peers);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 3. Accumulation.
// ---------------------------------------------------------------------------
// Where a sorted row's values and index entries live.  One partition: the
// row id and its row block's index offset, kept in shared memory as a uint2.
struct one_partition_rows {
    using entry = uint2;
    const uint16_t *__restrict__ val;
    const uint2 *__restrict__ index;
    const uint32_t *__restrict__ sorted_rows;
    uint32_t ell_cols, block_size, words;
    __device__ __forceinline__ entry fetch(uint32_t pos) const {
        const uint32_t r = sorted_rows[pos];
        return make_uint2(r, (r / block_size) * words);
    }
    __device__ __forceinline__ uint2 index_entry(const entry &e, uint32_t w) const { return __ldg(index + e.y + w); }
    __device__ __forceinline__ const uint16_t *row(const entry &e) const {
        return val + (std::size_t) e.x * ell_cols;
    }
};

// Several partitions (a shard): each sorted row's value row and index row
// addresses, precomputed by moments_row_ptrs_kernel.
struct many_partition_rows {
    using entry = ulonglong2;
    const ulonglong2 *__restrict__ row_ptrs;
    __device__ __forceinline__ entry fetch(uint32_t pos) const { return row_ptrs[pos]; }
    __device__ __forceinline__ uint2 index_entry(const entry &e, uint32_t w) const {
        return __ldg(reinterpret_cast<const uint2 *>(e.y) + w);
    }
    __device__ __forceinline__ const uint16_t *row(const entry &e) const {
        return reinterpret_cast<const uint16_t *>(e.x);
    }
};

template <int L, bool COMP, typename Rows>
__global__ void __launch_bounds__(kAccThreads, 2) moments_accumulate_kernel(
    Rows rows_of, uint32_t block_size, uint32_t col_blocks, uint32_t cols, const chunk_desc *__restrict__ chunks,
    const uint32_t *__restrict__ num_chunks, float *__restrict__ partials, const uint32_t *__restrict__ chunk_first,
    uint32_t g_lo, uint32_t g_hi) {
    using entry = typename Rows::entry;
    extern __shared__ __align__(16) unsigned char acc_smem[];
    entry *chunk_rows_smem = reinterpret_cast<entry *>(acc_smem);
    const uint32_t c = blockIdx.x;
    if (c >= *num_chunks) return;
    // with chunk_first: only the chunks of groups [g_lo, g_hi)
    if (chunk_first != nullptr && (c < chunk_first[g_lo] || c >= chunk_first[g_hi])) return;
    const chunk_desc d = chunks[c];
    const uint32_t n = d.end - d.begin;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) chunk_rows_smem[i] = rows_of.fetch(d.begin + i);
    __syncthreads();

    const uint32_t segs_per_block = block_size / L;
    const uint32_t seg = blockIdx.y * kAccThreads + threadIdx.x;
    const uint32_t b = seg / segs_per_block;
    const uint32_t part = seg - b * segs_per_block;
    if (b >= col_blocks) return;
    const uint32_t w = b >> 5;
    const uint32_t below = (1u << (b & 31u)) - 1u;
    const uint32_t bitmask = 1u << (b & 31u);
    const std::size_t lane_off = (std::size_t) part * L;

    float s_hi[L], s_lo[L], q_hi[L], q_lo[L];
#pragma unroll
    for (int j = 0; j < L; ++j) s_hi[j] = s_lo[j] = q_hi[j] = q_lo[j] = 0.0f;

    // two-stage software pipeline: the index entries of batch i+1 are in
    // flight while batch i's value loads are outstanding
    uint2 e_next[kBatch];
#pragma unroll
    for (unsigned u = 0; u < kBatch; ++u)
        e_next[u] = u < n ? rows_of.index_entry(chunk_rows_smem[u], w) : make_uint2(0u, 0u);
    uint32_t i = 0;
    for (; i + kBatch <= n; i += kBatch) {
        raw_vec<L> raw[kBatch];
#pragma unroll
        for (unsigned u = 0; u < kBatch; ++u) {
            const uint2 e = e_next[u];
            if (e.x & bitmask) {
                const uint32_t slot = e.y + __popc(e.x & below);
                load_raw<L>(rows_of.row(chunk_rows_smem[i + u]) + (std::size_t) slot * block_size + lane_off,
                            raw[u]);
            } else {
                zero_raw<L>(raw[u]);
            }
        }
#pragma unroll
        for (unsigned u = 0; u < kBatch; ++u) {
            const uint32_t k = i + kBatch + u;
            e_next[u] = k < n ? rows_of.index_entry(chunk_rows_smem[k], w) : make_uint2(0u, 0u);
        }
        if (COMP) {
            float bs[L], bq[L];
#pragma unroll
            for (int j = 0; j < L; ++j) bs[j] = bq[j] = 0.0f;
#pragma unroll
            for (unsigned u = 0; u < kBatch; ++u) {
                float x[L];
                unpack<L>(raw[u], x);
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    bs[j] = __fadd_rn(bs[j], x[j]);
                    bq[j] = __fmaf_rn(x[j], x[j], bq[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < L; ++j) {
                two_sum_acc(s_hi[j], s_lo[j], bs[j]);
                two_sum_acc(q_hi[j], q_lo[j], bq[j]);
            }
        } else {
#pragma unroll
            for (unsigned u = 0; u < kBatch; ++u) {
                float x[L];
                unpack<L>(raw[u], x);
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    s_hi[j] = __fadd_rn(s_hi[j], x[j]);
                    q_hi[j] = __fmaf_rn(x[j], x[j], q_hi[j]);
                }
            }
        }
    }
    // tail rows (fewer than a batch); their index entries are in e_next
#pragma unroll
    for (unsigned u = 0; u < kBatch; ++u) {
        if (i + u < n) {
            const uint2 e = e_next[u];
            if (e.x & bitmask) {
                raw_vec<L> raw;
                const uint32_t slot = e.y + __popc(e.x & below);
                load_raw<L>(rows_of.row(chunk_rows_smem[i + u]) + (std::size_t) slot * block_size + lane_off,
                            raw);
                float x[L];
                unpack<L>(raw, x);
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    if (COMP) {
                        two_sum_acc(s_hi[j], s_lo[j], x[j]);
                        two_sum_acc(q_hi[j], q_lo[j], __fmul_rn(x[j], x[j]));
                    } else {
                        s_hi[j] = __fadd_rn(s_hi[j], x[j]);
                        q_hi[j] = __fmaf_rn(x[j], x[j], q_hi[j]);
                    }
                }
            }
        }
    }
    const std::size_t f0 = (std::size_t) b * block_size + lane_off;
    float *p = partials + (std::size_t) c * 4u * cols;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const std::size_t f = f0 + j;
        if (f < cols) {
            p[f] = s_hi[j];
            p[cols + f] = s_lo[j];
            p[2u * (std::size_t) cols + f] = q_hi[j];
            p[3u * (std::size_t) cols + f] = q_lo[j];
        }
    }
}

// ---------------------------------------------------------------------------
// 4. Combine.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) moments_combine_kernel(
    uint32_t cols, uint32_t G, uint32_t scheme, uint32_t ddof, const uint32_t *__restrict__ chunk_first,
    const uint32_t *__restrict__ group_rows, const float *__restrict__ partials, const uint8_t *__restrict__ feature_keep,
    float *__restrict__ out_sum, float *__restrict__ out_sumsq, float *__restrict__ out_mean, float *__restrict__ out_var,
    double *__restrict__ out_mean64, double *__restrict__ out_var64, uint32_t *__restrict__ out_group_rows,
    uint32_t g_base) {
    const uint32_t g = g_base + blockIdx.y;
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    if (f == 0 && out_group_rows != nullptr) out_group_rows[g] = group_rows[g];
    if (f >= cols) return;
    const uint32_t c0 = chunk_first[g], c1 = chunk_first[g + 1];
    const uint32_t n = group_rows[g];
    const bool kept = feature_keep == nullptr || feature_keep[f] != 0u;
    const std::size_t o = (std::size_t) g * cols + f;
    float rs = 0.0f, rq = 0.0f, rm = 0.0f, rv = 0.0f;
    double dm = 0.0, dv = 0.0;
    if (kept) {
        if (scheme == CS_MOMENTS_TWOSUM_F64_COMBINE) {
            double s = 0.0, q = 0.0;
            for (uint32_t c = c0; c < c1; ++c) {
                const float *p = partials + (std::size_t) c * 4u * cols;
                s += (double) p[f] + (double) p[cols + f];
                q += (double) p[2u * (std::size_t) cols + f] + (double) p[3u * (std::size_t) cols + f];
            }
            rs = (float) s;
            rq = (float) q;
            if (n > 0u) {
                dm = s / (double) n;
                if (n > ddof) {
                    double m2 = q - s * dm;
                    if (m2 < 0.0) m2 = 0.0;
                    dv = m2 / (double) (n - ddof);
                }
            }
            rm = (float) dm;
            rv = (float) dv;
        } else {
            float s_hi = 0.0f, s_lo = 0.0f, q_hi = 0.0f, q_lo = 0.0f;
            for (uint32_t c = c0; c < c1; ++c) {
                const float *p = partials + (std::size_t) c * 4u * cols;
                if (scheme == CS_MOMENTS_TWOSUM_F32) {
                    two_sum_acc(s_hi, s_lo, p[f]);
                    s_lo = __fadd_rn(s_lo, p[cols + f]);
                    two_sum_acc(q_hi, q_lo, p[2u * (std::size_t) cols + f]);
                    q_lo = __fadd_rn(q_lo, p[3u * (std::size_t) cols + f]);
                } else {
                    s_hi = __fadd_rn(s_hi, p[f]);
                    q_hi = __fadd_rn(q_hi, p[2u * (std::size_t) cols + f]);
                }
            }
            rs = __fadd_rn(s_hi, s_lo);
            rq = __fadd_rn(q_hi, q_lo);
            if (n > 0u) {
                rm = __fdiv_rn(rs, (float) n);
                if (n > ddof) {
                    float m2 = __fsub_rn(rq, __fmul_rn(rs, rm));
                    if (m2 < 0.0f) m2 = 0.0f;
                    rv = __fdiv_rn(m2, (float) (n - ddof));
                }
            }
            dm = rm;
            dv = rv;
        }
    }
    out_sum[o] = rs;
    out_sumsq[o] = rq;
    if (out_mean != nullptr) out_mean[o] = rm;
    if (out_var != nullptr) out_var[o] = rv;
    if (out_mean64 != nullptr) out_mean64[o] = dm;
    if (out_var64 != nullptr) out_var64[o] = dv;
}

template <int L, bool COMP, typename Rows>
int launch_accumulate_rows(const Rows &rows_of, uint32_t block_size, uint32_t cols, const moments_layout &lay,
                           const uint32_t *chunk_first, uint32_t g_lo, uint32_t g_hi, cudaStream_t stream) {
    const uint32_t segs = lay.col_blocks * (block_size / L);
    dim3 grid(lay.max_chunks, (segs + kAccThreads - 1u) / kAccThreads);
    const std::size_t smem = (std::size_t) lay.chunk_rows * sizeof(typename Rows::entry);
    auto kern = moments_accumulate_kernel<L, COMP, Rows>;
    if (smem > 48u * 1024u &&
        !cuda_ok(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "moments smem attribute"))
        return 0;
    kern<<<grid, kAccThreads, smem, stream>>>(rows_of, block_size, lay.col_blocks, cols, lay.chunks, lay.num_chunks,
                                              lay.partials, chunk_first, g_lo, g_hi);
    return launch_ok("moments_accumulate_kernel");
}

template <int L, bool COMP>
int launch_accumulate(const cs_blocked_ell_view *src, const moments_layout &lay, const uint32_t *chunk_first,
                      uint32_t g_lo, uint32_t g_hi, cudaStream_t stream) {
    const one_partition_rows rows_of{reinterpret_cast<const uint16_t *>(src->val), lay.index, lay.sorted_rows,
                                     src->ell_cols, src->block_size, lay.words};
    return launch_accumulate_rows<L, COMP>(rows_of, src->block_size, src->cols, lay, chunk_first, g_lo, g_hi, stream);
}

int validate(const cs_blocked_ell_view *src, const cs_group_moments_params *p) {
    if (src == nullptr || p == nullptr) {
        set_error("group_moments: null view or params");
        return 0;
    }
    if (src->block_size == 0u || src->ell_cols % src->block_size != 0u) {
        set_error("group_moments: block_size %u does not divide ell_cols %u", src->block_size, src->ell_cols);
        return 0;
    }
    if (p->group_count == 0u || p->group_count > CS_MAX_MOMENT_GROUPS) {
        set_error("group_moments: group_count %u outside [1, %u]", p->group_count, CS_MAX_MOMENT_GROUPS);
        return 0;
    }
    if (p->scheme > CS_MOMENTS_TWOSUM_F64_COMBINE) {
        set_error("group_moments: unknown scheme %u", p->scheme);
        return 0;
    }
    if (p->chunk_rows > kMaxChunkRows) {
        set_error("group_moments: chunk_rows %u above %u", p->chunk_rows, kMaxChunkRows);
        return 0;
    }
    const uint32_t col_blocks = (src->cols + src->block_size - 1u) / src->block_size;
    if ((col_blocks + 31u) / 32u > kMaxIndexWords) {
        set_error("group_moments: %u column blocks exceed the index limit", col_blocks);
        return 0;
    }
    return 1;
}

// A shard's partitions, passed to moments_row_ptrs_kernel by value (the
// table travels in the launch, so nothing of the host call outlives it).
struct moment_part {
    const uint16_t *val;
    const uint2 *index;
    uint32_t row0;     // first global row of the partition
    uint32_t ell_cols;
};
struct moment_part_table {
    moment_part p[CS_MOMENTS_MAX_PARTS];
    uint32_t count, block_size, words, pad;
};

// row_ptrs[i] = (address of sorted row i's values, address of its row
// block's index entries) for the kept rows of all groups.
__global__ void __launch_bounds__(256) moments_row_ptrs_kernel(moment_part_table T,
                                                              const uint32_t *__restrict__ sorted_rows,
                                                              const uint32_t *__restrict__ group_offsets, uint32_t G,
                                                              ulonglong2 *__restrict__ row_ptrs) {
    __shared__ uint32_t row0[CS_MOMENTS_MAX_PARTS];
    for (uint32_t k = threadIdx.x; k < T.count; k += blockDim.x) row0[k] = T.p[k].row0;
    __syncthreads();
    const uint32_t total = group_offsets[G];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t r = sorted_rows[i];
        uint32_t lo = 0u, hi = T.count - 1u; // last partition whose first row is <= r
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (row0[mid] <= r)
                lo = mid;
            else
                hi = mid - 1u;
        }
        const uint32_t local = r - row0[lo];
        const uint16_t *v = T.p[lo].val + (std::size_t) local * T.p[lo].ell_cols;
        const uint2 *x = T.p[lo].index + (std::size_t) (local / T.block_size) * T.words;
        row_ptrs[i] = make_ulonglong2((unsigned long long) v, (unsigned long long) x);
    }
}

// Stable sort of the kept rows [0, rows) by label into lay.sorted_rows, with
// each group's rows cut into chunks (prepare phase, after the index).
int sort_rows_by_label(const moments_layout &lay, uint32_t rows, const uint8_t *d_row_keep,
                       const uint32_t *d_row_labels, uint32_t G, cudaStream_t stream) {
    const std::size_t sort_smem = (std::size_t) kSortWarps * G * sizeof(uint32_t);
    if (lay.tiles != 0u) {
        const std::size_t hist_smem = (std::size_t) G * sizeof(uint32_t);
        moments_tile_hist_kernel<<<lay.tiles, kSortThreads, hist_smem, stream>>>(rows, d_row_keep, d_row_labels, G,
                                                                                lay.tile_counts);
        if (!launch_ok("moments_tile_hist_kernel")) return 0;
        moments_group_tiles_kernel<<<(G + 7u) / 8u, 256, 0, stream>>>(lay.tiles, G, lay.tile_counts, lay.group_rows);
        if (!launch_ok("moments_group_tiles_kernel")) return 0;
    } else if (!cuda_ok(cudaMemsetAsync(lay.group_rows, 0, (std::size_t) G * sizeof(uint32_t), stream),
                        "group rows memset")) {
        return 0;
    }
    moments_group_scan_kernel<<<1, 1024, 0, stream>>>(G, lay.chunk_rows, lay.max_chunks, lay.group_rows,
                                                      lay.group_offsets, lay.chunk_first, lay.num_chunks, lay.chunks);
    if (!launch_ok("moments_group_scan_kernel")) return 0;
    if (lay.tiles != 0u) {
        if (sort_smem > 48u * 1024u &&
            !cuda_ok(cudaFuncSetAttribute(moments_tile_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) sort_smem),
                     "scatter smem attribute"))
            return 0;
        moments_tile_scatter_kernel<<<lay.tiles, kSortThreads, sort_smem, stream>>>(
            rows, d_row_keep, d_row_labels, G, lay.tile_counts, lay.group_offsets, lay.sorted_rows);
        if (!launch_ok("moments_tile_scatter_kernel")) return 0;
    }
    return 1;
}

// Combine phase for groups [g_lo, g_hi).
int combine_groups(const moments_layout &lay, uint32_t cols, const cs_group_moments_params *params,
                   const uint8_t *d_feature_keep, const cs_group_moments_out *out, uint32_t g_lo, uint32_t g_hi,
                   cudaStream_t stream) {
    dim3 grid((cols + 255u) / 256u == 0u ? 1u : (cols + 255u) / 256u, g_hi - g_lo);
    moments_combine_kernel<<<grid, 256, 0, stream>>>(cols, params->group_count, params->scheme, params->ddof,
                                                     lay.chunk_first, lay.group_rows, lay.partials, d_feature_keep,
                                                     out->sum, out->sumsq, out->mean, out->var, out->mean64,
                                                     out->var64, out->group_rows, g_lo);
    return launch_ok("moments_combine_kernel");
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_group_moments_scratch_bytes(const cs_blocked_ell_view *src, const cs_group_moments_params *params,
                                                   size_t *out_bytes) {
    if (!validate(src, params) || out_bytes == nullptr) {
        if (out_bytes == nullptr) set_error("group_moments_scratch_bytes: null output");
        return 0;
    }
    moments_layout lay;
    make_layout(src, params, nullptr, 0, &lay);
    *out_bytes = lay.bytes;
    return 1;
}

static int moments_run(const cs_blocked_ell_view *src, const uint8_t *d_row_keep, const uint8_t *d_feature_keep,
                       const uint32_t *d_row_labels, const cs_group_moments_params *params,
                       const cs_group_moments_out *out, void *d_scratch, size_t scratch_bytes, cs_stream_t s,
                       uint32_t phases, uint32_t g_lo = 0u, uint32_t g_hi = 0xffffffffu) {
    if (!validate(src, params)) return 0;
    if (out == nullptr || out->sum == nullptr || out->sumsq == nullptr) {
        set_error("group_moments: sum and sumsq outputs are required");
        return 0;
    }
    moments_layout lay;
    if (!make_layout(src, params, d_scratch, scratch_bytes, &lay) || d_scratch == nullptr) {
        set_error("group_moments: scratch too small (%zu bytes, need %zu)", scratch_bytes, lay.bytes);
        return 0;
    }
    if (src->rows != 0u && src->ell_cols != 0u && (src->val == nullptr || src->blockColIdx == nullptr)) {
        set_error("group_moments: null view arrays");
        return 0;
    }
    cudaStream_t stream = as_stream(s);
    const uint32_t G = params->group_count;
    const uint32_t width = src->ell_cols / src->block_size;
    // a column-block index the caller built once for this partition replaces the scratch one
    const bool prebuilt = params->index != nullptr;
    if (prebuilt) lay.index = static_cast<uint2 *>(const_cast<void *>(params->index));
    // accumulate and combine may be restricted to groups [g_lo, g_hi)
    if (g_hi > G) g_hi = G;
    const bool all_groups = g_lo == 0u && g_hi == G;
    if (g_lo >= g_hi) return 1;
    const uint32_t *range_first = all_groups ? nullptr : lay.chunk_first;

    if ((phases & CS_MOMENTS_PHASE_PREPARE) && !prebuilt && lay.row_blocks != 0u && lay.words != 0u) {
        if (width != 0u) {
            const uint32_t blocks = (lay.row_blocks + kIndexWarps - 1u) / kIndexWarps;
            const std::size_t smem = (std::size_t) kIndexWarps * lay.words * sizeof(uint32_t);
            if (smem > 48u * 1024u &&
                !cuda_ok(cudaFuncSetAttribute(moments_index_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int) smem),
                         "index smem attribute"))
                return 0;
            moments_index_kernel<<<blocks, kIndexWarps * 32, smem, stream>>>(
                src->blockColIdx, lay.row_blocks, width, lay.col_blocks, lay.words, lay.index, out->status,
                (width % 4u) == 0u && (reinterpret_cast<uintptr_t>(src->blockColIdx) & 15u) == 0u);
            if (!launch_ok("moments_index_kernel")) return 0;
        } else if (!cuda_ok(cudaMemsetAsync(lay.index, 0, (std::size_t) lay.row_blocks * lay.words * sizeof(uint2),
                                            stream),
                            "index memset")) {
            return 0;
        }
    }

    if ((phases & CS_MOMENTS_PHASE_PREPARE) && !sort_rows_by_label(lay, src->rows, d_row_keep, d_row_labels, G, stream))
        return 0;

    if ((phases & CS_MOMENTS_PHASE_ACCUMULATE) && lay.col_blocks != 0u && lay.max_chunks != 0u && src->cols != 0u) {
        const bool comp = params->scheme != CS_MOMENTS_PLAIN_F32;
        const uint32_t B = src->block_size;
        const bool aligned16 = (reinterpret_cast<uintptr_t>(src->val) & 15u) == 0u;
        int ok;
#define CS_ACC(L_)                                                                                     \
    (comp ? launch_accumulate<L_, true>(src, lay, range_first, g_lo, g_hi, stream)                      \
          : launch_accumulate<L_, false>(src, lay, range_first, g_lo, g_hi, stream))
        if (B % 8u == 0u && aligned16)
            ok = CS_ACC(8);
        else if (B % 4u == 0u && (reinterpret_cast<uintptr_t>(src->val) & 7u) == 0u)
            ok = CS_ACC(4);
        else if (B % 2u == 0u && (reinterpret_cast<uintptr_t>(src->val) & 3u) == 0u)
            ok = CS_ACC(2);
        else
            ok = CS_ACC(1);
#undef CS_ACC
        if (!ok) return 0;
    }

    if ((phases & CS_MOMENTS_PHASE_COMBINE) && (src->cols != 0u || out->group_rows != nullptr) &&
        !combine_groups(lay, src->cols, params, d_feature_keep, out, g_lo, g_hi, stream))
        return 0;
    return 1;
}

namespace csb {

// Column-block index of a Blocked-ELL partition (index[rb * words + w] =
// (occupancy bits of column blocks 32w..32w+31, slots before them)), as the
// moments prepare phase builds it; used by the serving loop, which keeps one
// per staged partition.  words = ceil(ceil(cols / block_size) / 32).
int build_column_block_index(const cs_blocked_ell_view *src, uint2 *index, uint32_t *status, cudaStream_t stream) {
    const uint32_t B = src->block_size;
    const uint32_t row_blocks = (src->rows + B - 1u) / B;
    const uint32_t col_blocks = (src->cols + B - 1u) / B;
    const uint32_t words = (col_blocks + 31u) / 32u;
    if (row_blocks == 0u || words == 0u) return 1;
    const uint32_t width = src->ell_cols / B;
    if (width == 0u)
        return cuda_ok(cudaMemsetAsync(index, 0, (std::size_t) row_blocks * words * sizeof(uint2), stream),
                       "index memset");
    const uint32_t blocks = (row_blocks + kIndexWarps - 1u) / kIndexWarps;
    const std::size_t smem = (std::size_t) kIndexWarps * words * sizeof(uint32_t);
    if (smem > 48u * 1024u &&
        !cuda_ok(cudaFuncSetAttribute(moments_index_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "index smem attribute"))
        return 0;
    moments_index_kernel<<<blocks, kIndexWarps * 32, smem, stream>>>(
        src->blockColIdx, row_blocks, width, col_blocks, words, index, status,
        (width % 4u) == 0u && (reinterpret_cast<uintptr_t>(src->blockColIdx) & 15u) == 0u);
    return launch_ok("moments_index_kernel");
}

std::size_t column_block_index_bytes(const cs_blocked_ell_view *src) {
    const uint32_t B = src->block_size;
    const std::size_t row_blocks = (src->rows + B - 1u) / B;
    const std::size_t words = (((std::size_t) src->cols + B - 1u) / B + 31u) / 32u;
    return (row_blocks * words + 1u) * sizeof(uint2);
}

// Scratch bytes the moments reduction needs for (src, params); 0 when the
// arguments are invalid (the error message is set).
std::size_t group_moments_scratch_needed(const cs_blocked_ell_view *src, const cs_group_moments_params *params) {
    if (!validate(src, params)) return 0;
    moments_layout lay;
    make_layout(src, params, nullptr, 0, &lay);
    return lay.bytes;
}

// The full reduction over caller-provided scratch (used by the entry points
// in this file and by the static-scratch entry point).
int group_moments_launch(const cs_blocked_ell_view *src, const uint8_t *d_row_keep, const uint8_t *d_feature_keep,
                         const uint32_t *d_row_labels, const cs_group_moments_params *params,
                         const cs_group_moments_out *out, void *d_scratch, size_t scratch_bytes, cs_stream_t s) {
    return moments_run(src, d_row_keep, d_feature_keep, d_row_labels, params, out, d_scratch, scratch_bytes, s,
                       CS_MOMENTS_PHASE_ALL);
}

} // namespace csb

extern "C" int cs_b200_group_moments_blocked_ell(const cs_blocked_ell_view *src, const uint8_t *d_row_keep,
                                                  const uint8_t *d_feature_keep, const uint32_t *d_row_labels,
                                                  const cs_group_moments_params *params,
                                                  const cs_group_moments_out *out, void *d_scratch,
                                                  size_t scratch_bytes, cs_stream_t s) {
    return moments_run(src, d_row_keep, d_feature_keep, d_row_labels, params, out, d_scratch, scratch_bytes, s,
                       CS_MOMENTS_PHASE_ALL);
}

extern "C" int cs_b200_group_moments_index_bytes(const cs_blocked_ell_view *src, size_t *out_bytes) {
    if (src == nullptr || out_bytes == nullptr || src->block_size == 0u) {
        set_error("group_moments_index_bytes: null argument or zero block size");
        return 0;
    }
    *out_bytes = column_block_index_bytes(src);
    return 1;
}

extern "C" int cs_b200_group_moments_build_index(const cs_blocked_ell_view *src, void *d_index, uint32_t *d_status,
                                                  cs_stream_t s) {
    if (src == nullptr || d_index == nullptr || src->block_size == 0u || src->ell_cols % src->block_size != 0u ||
        (src->rows != 0u && src->ell_cols != 0u && src->blockColIdx == nullptr)) {
        set_error("group_moments_build_index: null argument, zero block size or block size not dividing ell_cols");
        return 0;
    }
    const uint32_t col_blocks = (src->cols + src->block_size - 1u) / src->block_size;
    if ((col_blocks + 31u) / 32u > kMaxIndexWords) {
        set_error("group_moments_build_index: %u column blocks exceed the index limit", col_blocks);
        return 0;
    }
    return build_column_block_index(src, static_cast<uint2 *>(d_index), d_status, as_stream(s));
}

extern "C" int cs_b200_group_moments_phases(const cs_blocked_ell_view *src, const uint8_t *d_row_keep,
                                            const uint8_t *d_feature_keep, const uint32_t *d_row_labels,
                                            const cs_group_moments_params *params, const cs_group_moments_out *out,
                                            void *d_scratch, size_t scratch_bytes, uint32_t phases, cs_stream_t s) {
    if ((phases & ~(uint32_t) CS_MOMENTS_PHASE_ALL) != 0u) {
        set_error("group_moments_phases: unknown phase bits 0x%x", phases);
        return 0;
    }
    return moments_run(src, d_row_keep, d_feature_keep, d_row_labels, params, out, d_scratch, scratch_bytes, s,
                       phases);
}

// ---------------------------------------------------------------------------
// The reduction over a shard given as its partitions' views, in one call.
// ---------------------------------------------------------------------------
namespace {

struct parts_layout {
    moments_layout base;    // over all rows of the shard
    uint2 *part_index;      // per-partition column-block indexes built by the call
    ulonglong2 *row_ptrs;   // [rows]
    std::size_t bytes;
    uint32_t rows;
};

int validate_parts(const cs_blocked_ell_view *parts, uint32_t count, const cs_group_moments_params *params,
                   cs_blocked_ell_view *whole) {
    if (parts == nullptr || count == 0u || count > CS_MOMENTS_MAX_PARTS) {
        set_error("group_moments_parts: %u partitions (need 1..%u)", count, CS_MOMENTS_MAX_PARTS);
        return 0;
    }
    uint64_t rows = 0;
    for (uint32_t k = 0; k < count; ++k) {
        if (!validate(&parts[k], params)) return 0;
        if (parts[k].cols != parts[0].cols || parts[k].block_size != parts[0].block_size) {
            set_error("group_moments_parts: partition %u has cols %u / block size %u, partition 0 %u / %u", k,
                      parts[k].cols, parts[k].block_size, parts[0].cols, parts[0].block_size);
            return 0;
        }
        if (parts[k].rows != 0u && parts[k].ell_cols != 0u &&
            (parts[k].val == nullptr || parts[k].blockColIdx == nullptr)) {
            set_error("group_moments_parts: partition %u has null arrays", k);
            return 0;
        }
        rows += parts[k].rows;
    }
    if (rows >= 0xffffffffull) {
        set_error("group_moments_parts: %llu rows exceed the u32 row ids", (unsigned long long) rows);
        return 0;
    }
    *whole = parts[0];
    whole->rows = (uint32_t) rows;
    return 1;
}

bool make_parts_layout(const cs_blocked_ell_view *parts, uint32_t count, const cs_blocked_ell_view &whole,
                       const cs_group_moments_params *params, void *base, std::size_t cap, parts_layout *pl) {
    make_layout(&whole, params, base, cap, &pl->base);
    const uint32_t B = whole.block_size;
    std::size_t blocks = 0;
    for (uint32_t k = 0; k < count; ++k) blocks += (parts[k].rows + B - 1u) / B;
    scratch_carver c(base, cap);
    c.used = pl->base.bytes;
    pl->part_index = c.take<uint2>(blocks * pl->base.words + 1u);
    pl->row_ptrs = c.take<ulonglong2>((std::size_t) whole.rows + 1u);
    pl->bytes = c.used;
    pl->rows = whole.rows;
    return c.fits();
}

} // namespace

extern "C" int cs_b200_group_moments_parts_scratch_bytes(const cs_blocked_ell_view *parts, uint32_t count,
                                                          const cs_group_moments_params *params, size_t *out_bytes) {
    cs_blocked_ell_view whole;
    if (out_bytes == nullptr) {
        set_error("group_moments_parts_scratch_bytes: null output");
        return 0;
    }
    if (!validate_parts(parts, count, params, &whole)) return 0;
    parts_layout pl;
    make_parts_layout(parts, count, whole, params, nullptr, 0, &pl);
    *out_bytes = pl.bytes;
    return 1;
}

extern "C" int cs_b200_group_moments_blocked_ell_parts(const cs_blocked_ell_view *parts, uint32_t count,
                                                       const void *const *d_indexes, const uint8_t *d_row_keep,
                                                       const uint8_t *d_feature_keep, const uint32_t *d_row_labels,
                                                       const cs_group_moments_params *params,
                                                       const cs_group_moments_out *out, void *d_scratch,
                                                       size_t scratch_bytes, cs_stream_t s) {
    cs_blocked_ell_view whole;
    if (!validate_parts(parts, count, params, &whole)) return 0;
    if (out == nullptr || out->sum == nullptr || out->sumsq == nullptr) {
        set_error("group_moments_parts: sum and sumsq outputs are required");
        return 0;
    }
    parts_layout pl;
    if (!make_parts_layout(parts, count, whole, params, d_scratch, scratch_bytes, &pl) || d_scratch == nullptr) {
        set_error("group_moments_parts: scratch too small (%zu bytes, need %zu)", scratch_bytes, pl.bytes);
        return 0;
    }
    cudaStream_t stream = as_stream(s);
    const moments_layout &lay = pl.base;
    const uint32_t G = params->group_count, B = whole.block_size;
    moment_part_table T{};
    T.count = count;
    T.block_size = B;
    T.words = lay.words;
    uint32_t row0 = 0u;
    std::size_t built = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const uint2 *idx = d_indexes != nullptr ? static_cast<const uint2 *>(d_indexes[k]) : nullptr;
        if (idx == nullptr) {
            uint2 *mine = pl.part_index + built * lay.words;
            built += (parts[k].rows + B - 1u) / B;
            if (!build_column_block_index(&parts[k], mine, out->status, stream)) return 0;
            idx = mine;
        }
        T.p[k] = moment_part{reinterpret_cast<const uint16_t *>(parts[k].val), idx, row0, parts[k].ell_cols};
        row0 += parts[k].rows;
    }
    if (!sort_rows_by_label(lay, whole.rows, d_row_keep, d_row_labels, G, stream)) return 0;
    if (whole.rows != 0u) {
        const unsigned grid = resident_grid(reinterpret_cast<const void *>(moments_row_ptrs_kernel), 256, 0,
                                            (whole.rows + 255u) / 256u);
        moments_row_ptrs_kernel<<<grid, 256, 0, stream>>>(T, lay.sorted_rows, lay.group_offsets, G, pl.row_ptrs);
        if (!launch_ok("moments_row_ptrs_kernel")) return 0;
    }
    if (lay.col_blocks != 0u && lay.max_chunks != 0u && whole.cols != 0u) {
        const bool comp = params->scheme != CS_MOMENTS_PLAIN_F32;
        bool a16 = true, a8 = true, a4 = true;
        for (uint32_t k = 0; k < count; ++k) {
            const uintptr_t v = reinterpret_cast<uintptr_t>(parts[k].val);
            const uint32_t rowb = parts[k].ell_cols * 2u; // a row's bytes: every row start keeps the base alignment
            a16 = a16 && (v & 15u) == 0u && rowb % 16u == 0u;
            a8 = a8 && (v & 7u) == 0u && rowb % 8u == 0u;
            a4 = a4 && (v & 3u) == 0u && rowb % 4u == 0u;
        }
        const many_partition_rows rows_of{pl.row_ptrs};
        int ok;
#define CS_ACCM(L_)                                                                                       \
    (comp ? launch_accumulate_rows<L_, true>(rows_of, B, whole.cols, lay, nullptr, 0u, G, stream)         \
          : launch_accumulate_rows<L_, false>(rows_of, B, whole.cols, lay, nullptr, 0u, G, stream))
        if (B % 8u == 0u && a16)
            ok = CS_ACCM(8);
        else if (B % 4u == 0u && a8)
            ok = CS_ACCM(4);
        else if (B % 2u == 0u && a4)
            ok = CS_ACCM(2);
        else
            ok = CS_ACCM(1);
#undef CS_ACCM
        if (!ok) return 0;
    }
    if (whole.cols != 0u || out->group_rows != nullptr)
        return combine_groups(lay, whole.cols, params, d_feature_keep, out, 0u, G, stream);
    return 1;
}

namespace {

// Copy stream and events of the host-delivery entry point, one set per host
// thread and device ordinal (created on first use on that device, kept for the
// thread's lifetime, so a thread that moves between devices creates nothing
// new after its first call on each).
struct host_copy_ctx {
    cudaStream_t copy = nullptr;
    cudaEvent_t ready = nullptr, done = nullptr;
};

constexpr int kCopyDevices = 64;

host_copy_ctx *host_copy_setup() {
    thread_local host_copy_ctx ctxs[kCopyDevices];
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "get device")) return nullptr;
    if (dev < 0 || dev >= kCopyDevices) {
        set_error("group_moments_to_host: device ordinal %d outside the supported range", dev);
        return nullptr;
    }
    host_copy_ctx &c = ctxs[dev];
    if (c.copy != nullptr && c.ready != nullptr && c.done != nullptr) return &c;
    // a set-up that failed partway keeps what it created and completes it now
    if (c.copy == nullptr && !cuda_ok(cudaStreamCreateWithFlags(&c.copy, cudaStreamNonBlocking), "copy stream"))
        return nullptr;
    if (c.ready == nullptr && !cuda_ok(cudaEventCreateWithFlags(&c.ready, cudaEventDisableTiming), "copy event"))
        return nullptr;
    if (c.done == nullptr && !cuda_ok(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming), "copy event"))
        return nullptr;
    return &c;
}

template <typename T>
bool copy_rows(T *h, const T *d, uint32_t g0, uint32_t g1, std::size_t row_elems, cudaStream_t copy) {
    if (h == nullptr || d == nullptr || g1 <= g0) return true;
    return cuda_ok(cudaMemcpyAsync(h + (std::size_t) g0 * row_elems, d + (std::size_t) g0 * row_elems,
                                   (std::size_t) (g1 - g0) * row_elems * sizeof(T), cudaMemcpyDeviceToHost, copy),
                   "moments D2H") != 0;
}

} // namespace

extern "C" int cs_b200_group_moments_to_host(const cs_blocked_ell_view *src, const uint8_t *d_row_keep,
                                             const uint8_t *d_feature_keep, const uint32_t *d_row_labels,
                                             const cs_group_moments_params *params, const cs_group_moments_out *d_out,
                                             const cs_group_moments_out *h_out, void *d_scratch,
                                             size_t scratch_bytes, uint32_t parts, cs_stream_t s) {
    if (h_out == nullptr || d_out == nullptr) {
        set_error("group_moments_to_host: null outputs");
        return 0;
    }
    const struct {
        const void *h, *d;
        const char *name;
    } fields[] = {{h_out->sum, d_out->sum, "sum"},          {h_out->sumsq, d_out->sumsq, "sumsq"},
                  {h_out->mean, d_out->mean, "mean"},       {h_out->var, d_out->var, "var"},
                  {h_out->mean64, d_out->mean64, "mean64"}, {h_out->var64, d_out->var64, "var64"},
                  {h_out->group_rows, d_out->group_rows, "group_rows"}};
    for (const auto &f : fields)
        if (f.h != nullptr && f.d == nullptr) {
            set_error("group_moments_to_host: host %s given without its device array", f.name);
            return 0;
        }
    if (!validate(src, params)) return 0;
    const uint32_t G = params->group_count;
    if (parts == 0u) parts = 2u;
    if (parts > G) parts = G;
    cudaStream_t stream = as_stream(s);
    if (!moments_run(src, d_row_keep, d_feature_keep, d_row_labels, params, d_out, d_scratch, scratch_bytes, s,
                     CS_MOMENTS_PHASE_PREPARE))
        return 0;
    host_copy_ctx *cp = host_copy_setup();
    if (cp == nullptr) return 0;
    host_copy_ctx &ctx = *cp;
    const std::size_t cols = src->cols;
    for (uint32_t k = 0; k < parts; ++k) {
        const uint32_t g0 = (uint32_t) ((uint64_t) k * G / parts), g1 = (uint32_t) ((uint64_t) (k + 1u) * G / parts);
        if (g1 <= g0) continue;
        // groups [g0, g1) accumulated and combined; their rows copy while the next part computes
        if (!moments_run(src, d_row_keep, d_feature_keep, d_row_labels, params, d_out, d_scratch, scratch_bytes, s,
                         CS_MOMENTS_PHASE_ACCUMULATE | CS_MOMENTS_PHASE_COMBINE, g0, g1) ||
            !cuda_ok(cudaEventRecord(ctx.ready, stream), "part event") ||
            !cuda_ok(cudaStreamWaitEvent(ctx.copy, ctx.ready, 0), "copy wait") ||
            !copy_rows(h_out->sum, d_out->sum, g0, g1, cols, ctx.copy) ||
            !copy_rows(h_out->sumsq, d_out->sumsq, g0, g1, cols, ctx.copy) ||
            !copy_rows(h_out->mean, d_out->mean, g0, g1, cols, ctx.copy) ||
            !copy_rows(h_out->var, d_out->var, g0, g1, cols, ctx.copy) ||
            !copy_rows(h_out->mean64, d_out->mean64, g0, g1, cols, ctx.copy) ||
            !copy_rows(h_out->var64, d_out->var64, g0, g1, cols, ctx.copy) ||
            !copy_rows(h_out->group_rows, d_out->group_rows, g0, g1, 1u, ctx.copy))
            return 0;
    }
    if (h_out->status != nullptr && d_out->status != nullptr &&
        !cuda_ok(cudaMemcpyAsync(h_out->status, d_out->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx.copy),
                 "status D2H"))
        return 0;
    // the caller's stream waits for the copies, so a sync on it covers them
    return cuda_ok(cudaEventRecord(ctx.done, ctx.copy), "copy done event") &&
           cuda_ok(cudaStreamWaitEvent(stream, ctx.done, 0), "stream wait");
}
