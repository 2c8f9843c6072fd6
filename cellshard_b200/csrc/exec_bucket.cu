// Execution bucketing of one partition: the layout the reference persists
// for execution and reads back through its .cspack / .csh5 runtime.
//
// Blocked-ELL (build_bucketed_execution_partition and its helpers,
// src/io/csh5/execution_builders_part.hh:1011-1246):
//   widths[rb]  = valid block columns of row block rb              (one warp per row block)
//   order       = stable ascending sort of the row blocks by width; a partial
//                 last row block is left out of the sort and stays last
//   cuts        = bucket b spans sorted positions [b*RB/n, (b+1)*RB/n) (u32
//                 products, as written there), width = its widest row block;
//                 if every bucket has the same width they merge into one
//   fallback    = when more than one segment packs to no fewer bytes than the
//                 source (packed_blocked_ell_bytes, io/pack/packfile.cuh:110-116),
//                 the one-bucket layout is kept and its byte count reads as
//                 the source's
//   fill        = row block at sorted position p goes to its segment with its
//                 valid slots compacted to the front in slot order; padding is
//                 the invalid column with zero values; exec <-> canonical row
//                 maps; identity column maps.
//   choose_bucket_count_for_part (:1249-1272): counts 1..min(8, RB), fewest
//   bytes, ties to the smaller count.  The layout and the choice are computed
//   by one device thread from the sorted widths (O(segments) each: the sorted
//   widths give every segment's maximum directly).
// Sliced-ELL (build_bucketed_sliced_execution_partition, :1274-1570):
//   widths[row] = live slots of the row (one warp per row); stable ascending
//   sort of all rows; the split is the reference's dynamic programme (segments
//   of one slice, cost = fixed packed bytes + 6 bytes per slot, a segment as
//   wide as its last row, exactly `requested` non-empty segments before
//   equal-width neighbours merge) with its monotone convex-hull and its tie
//   rules.  The programme is sequential over the sorted widths: it runs on the
//   host over the widths copied back (4 bytes per row), as in the reference,
//   its levels pipelined over host threads; counting, sorting and copying run
//   on the device.  One programme of 8
//   levels serves all eight candidates of choose_bucket_count_for_sliced_part
//   (:1572-1596): level k's costs and cuts do not depend on how many levels
//   follow.
#include "common.cuh"

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace csb {
namespace {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr uint32_t kChooseMax = 8u;
constexpr unsigned kFillThreads = 256;
constexpr unsigned kFillWarps = kFillThreads / 32;
constexpr unsigned kSlotsPerThread = 8;
constexpr unsigned kChunk = kFillThreads * kSlotsPerThread;

// Head of the plan block the device writes and the host copies back.
struct plan_head {
    uint32_t S, bucket_count, units, block_size;
    uint64_t bytes, original_bytes, index_entries, value_entries;
    uint64_t pad[2];
};
static_assert(sizeof(plan_head) == 64, "plan head");

// One per segment plus an end record: offsets of segment s (units = sorted
// positions, exec rows, index entries, values), its width and its nnz field.
struct seg_rec {
    uint32_t unit_off, row_off, width, pad;
    uint64_t idx_off, val_off, nnz;
};

struct exec_scratch {
    uint32_t *widths, *order, *sorted;
    plan_head *head;
    seg_rec *rec;
    void *sort_tmp;
    std::size_t sort_bytes, bytes;
};

uint32_t plan_bound(uint32_t requested, uint32_t units) {
    const uint32_t b = requested == 0u ? kChooseMax : requested;
    const uint32_t u = units < 1u ? 1u : units;
    return b < u ? b : u;
}

// widths, order, sorted and the plan head sit at offsets that depend on the
// unit count only (the fill finds them from the part); records follow the
// head; the sort scratch comes last.
void carve(void *base, uint32_t units, uint32_t bound, exec_scratch *x) {
    scratch_carver c(base, ~std::size_t(0));
    x->widths = c.take<uint32_t>((std::size_t) units + 1u);
    x->order = c.take<uint32_t>((std::size_t) units + 1u);
    x->sorted = c.take<uint32_t>((std::size_t) units + 1u);
    char *block = c.take<char>(sizeof(plan_head) + ((std::size_t) bound + 1u) * sizeof(seg_rec));
    x->head = (plan_head *) block;
    x->rec = (seg_rec *) (block == nullptr ? nullptr : block + sizeof(plan_head));
    x->sort_bytes = sort_pairs_u32_scratch_bytes(units);
    x->sort_tmp = c.take<char>(x->sort_bytes);
    x->bytes = c.used;
}

__host__ __device__ inline uint64_t packed_bell_bytes(uint64_t rows, uint64_t ell_cols, uint32_t B) {
    // 16-byte disk header, two u32 words, block column indices, fp16 values
    const uint64_t rb = B == 0u ? 0u : (rows + B - 1u) / B;
    const uint64_t w = B == 0u ? 0u : ell_cols / B;
    return 16u + 8u + rb * w * 4u + rows * ell_cols * 2u;
}

inline uint64_t packed_sell_bytes(uint32_t slice_count, uint64_t total_slots) {
    // 13-byte header, one u32, slice offsets and widths, u32 columns, fp16 values
    return 13u + 4u + ((uint64_t) slice_count + 1u) * 4u + (uint64_t) slice_count * 4u + total_slots * 6u;
}

__device__ __forceinline__ uint32_t find_seg(const seg_rec *rec, uint32_t S, uint32_t pos) {
    uint32_t lo = 0u, hi = S;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (rec[mid].unit_off <= pos)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Blocked-ELL
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) bell_rb_width_kernel(const cs_blocked_ell_view src, uint32_t RB,
                                                            uint32_t *__restrict__ widths) {
    const uint32_t lane = threadIdx.x & 31u, W = src.ell_cols / src.block_size;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t rb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rb < RB; rb += warps) {
        const uint32_t *row = src.blockColIdx + (std::size_t) rb * W;
        uint32_t n = 0u;
        for (uint32_t k = lane; k < W; k += 32u) n += __ldg(row + k) != kInvalid;
        n = __reduce_add_sync(0xffffffffu, n);
        if (lane == 0u) widths[rb] = n;
    }
}

struct bell_geom {
    uint32_t rows, B, W, RB, sortable;
};

// Widest row block among sorted positions [lo, hi): positions below
// `sortable` ascend; the partial last row block sits at RB - 1.
__device__ __forceinline__ uint32_t bell_span_width(const bell_geom &g, const uint32_t *sorted, uint32_t lo,
                                                    uint32_t hi) {
    uint32_t m = 0u;
    const uint32_t sh = hi < g.sortable ? hi : g.sortable;
    if (lo < sh) m = sorted[sh - 1u];
    if (g.sortable < g.RB && hi == g.RB && lo < g.RB) m = max(m, sorted[g.RB - 1u]);
    return m;
}

__device__ __forceinline__ uint64_t bell_span_rows(const bell_geom &g, uint32_t lo, uint32_t hi) {
    uint64_t n = (uint64_t) (hi - lo) * g.B;
    if (hi == g.RB && lo < hi) n -= (uint64_t) g.RB * g.B - g.rows;
    return n;
}

// Segment cuts of build_execution_bucket_layout for `buckets` (before the
// fallback); returns S and writes lo/width per segment when rec != nullptr.
__device__ uint32_t bell_cuts(const bell_geom &g, const uint32_t *sorted, uint32_t buckets, uint64_t *bytes,
                              seg_rec *rec) {
    const uint32_t nb = buckets < 1u ? 1u : (buckets > g.RB ? g.RB : buckets);
    uint64_t total = 0u;
    uint32_t w0 = 0u;
    bool same = true;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t lo = (b * g.RB) / nb, hi = ((b + 1u) * g.RB) / nb;
        const uint32_t w = bell_span_width(g, sorted, lo, hi);
        if (b == 0u) w0 = w;
        same = same && w == w0;
        total += packed_bell_bytes(bell_span_rows(g, lo, hi), (uint64_t) w * g.B, g.B);
        if (rec != nullptr) {
            rec[b].unit_off = lo;
            rec[b].width = w;
        }
    }
    if (nb > 1u && same) {
        if (rec != nullptr) rec[0].width = w0;
        *bytes = packed_bell_bytes(g.rows, (uint64_t) w0 * g.B, g.B);
        return 1u;
    }
    *bytes = total;
    return nb;
}

// build_bucketed_execution_partition's byte rule: the kept layout's S.
__device__ uint32_t bell_kept(const bell_geom &g, const uint32_t *sorted, uint32_t buckets, uint64_t orig,
                              uint64_t *bytes, seg_rec *rec) {
    uint32_t S = bell_cuts(g, sorted, buckets, bytes, rec);
    if (S > 1u && *bytes >= orig) {
        uint64_t one = 0u;
        S = bell_cuts(g, sorted, 1u, &one, rec);
        *bytes = orig;
    }
    return S;
}

__global__ void bell_layout_kernel(bell_geom g, uint32_t requested, uint32_t *__restrict__ order,
                                   uint32_t *__restrict__ sorted, const uint32_t *__restrict__ widths,
                                   plan_head *__restrict__ head, seg_rec *__restrict__ rec) {
    if (threadIdx.x != 0u || blockIdx.x != 0u) return;
    plan_head h{};
    h.units = g.RB;
    h.block_size = g.B;
    h.original_bytes = packed_bell_bytes(g.rows, (uint64_t) g.W * g.B, g.B);
    if (g.RB == 0u) {
        h.bucket_count = requested == 0u ? 1u : requested;
        rec[0] = seg_rec{};
        *head = h;
        return;
    }
    if (g.sortable < g.RB) {
        order[g.RB - 1u] = g.RB - 1u;
        sorted[g.RB - 1u] = widths[g.RB - 1u];
    }
    uint32_t buckets = requested;
    if (requested == 0u) {
        const uint32_t top = g.RB < kChooseMax ? g.RB : kChooseMax;
        uint64_t best = ~0ull;
        for (uint32_t b = 1; b <= top; ++b) {
            uint64_t x = 0u;
            bell_kept(g, sorted, b, h.original_bytes, &x, nullptr);
            if (x < best) {
                best = x;
                buckets = b;
            }
        }
    }
    h.bucket_count = buckets;
    h.S = bell_kept(g, sorted, buckets, h.original_bytes, &h.bytes, rec);
    uint32_t row = 0u;
    uint64_t idx = 0u, val = 0u;
    for (uint32_t s = 0; s < h.S; ++s) {
        const uint32_t lo = rec[s].unit_off, hi = s + 1u < h.S ? rec[s + 1u].unit_off : g.RB;
        const uint64_t n = bell_span_rows(g, lo, hi);
        rec[s].row_off = row;
        rec[s].idx_off = idx;
        rec[s].val_off = val;
        rec[s].nnz = 0u;
        rec[s].pad = 0u;
        row += (uint32_t) n;
        idx += (uint64_t) (hi - lo) * rec[s].width;
        val += n * rec[s].width * g.B;
    }
    rec[h.S] = seg_rec{g.RB, row, 0u, 0u, idx, val, 0u};
    h.index_entries = idx;
    h.value_entries = val;
    *head = h;
}

// nnz field of each segment: sum over its row blocks of rows x own width x B
// (allocate_bucketed_execution_partition, :1121-1129), kept modulo 2^32 as
// the reference's u32 sum is.
__global__ void __launch_bounds__(256) bell_seg_nnz_kernel(bell_geom g, const uint32_t *__restrict__ order,
                                                           const uint32_t *__restrict__ widths,
                                                           const plan_head *__restrict__ head,
                                                           seg_rec *__restrict__ rec) {
    const uint32_t S = head->S, lane = threadIdx.x & 31u;
    // warp-uniform trips, so the whole warp meets the match and the reduction
    for (uint32_t p0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); p0 < g.RB; p0 += gridDim.x * blockDim.x) {
        const uint32_t p = p0 + lane;
        const bool on = p < g.RB;
        uint32_t s = kInvalid, v = 0u;
        if (on) {
            const uint32_t rb = order[p];
            s = find_seg(rec, S, p);
            v = min(g.B, g.rows - rb * g.B) * widths[rb] * g.B;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, s);
        const uint32_t sum = __reduce_add_sync(peers, v); // one atomic per segment per warp
        if (on && lane == (uint32_t) (__ffs(peers) - 1))
            atomicAdd((unsigned long long *) &rec[s].nnz, (unsigned long long) sum);
    }
}

// Block-wide exclusive scan of one count per thread; returns the prefix and
// the block total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *warp_sums, uint32_t *total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t) d) x += y;
    }
    if (lane == 31u) warp_sums[warp] = x;
    __syncthreads();
    uint32_t before = 0u, all = 0u;
#pragma unroll
    for (unsigned w = 0; w < kFillWarps; ++w) {
        const uint32_t t = warp_sums[w];
        before += w < warp ? t : 0u;
        all += t;
    }
    *total = all;
    return before + x - v;
}

// One column of a row block (16 bytes, or one half) for n rows: loads of 8
// rows are issued before their stores.
template <bool VEC>
__device__ __forceinline__ void copy_rows(const uint16_t *sp, std::size_t sstride, uint16_t *dp, std::size_t dstride,
                                          uint32_t n) {
    uint32_t rr = 0;
    if (VEC) {
        for (; rr + 8u <= n; rr += 8u) {
            uint4 x[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = __ldcs(reinterpret_cast<const uint4 *>(sp + (rr + k) * sstride));
#pragma unroll
            for (int k = 0; k < 8; ++k) __stcs(reinterpret_cast<uint4 *>(dp + (rr + k) * dstride), x[k]);
        }
        for (; rr < n; ++rr)
            __stcs(reinterpret_cast<uint4 *>(dp + rr * dstride), __ldcs(reinterpret_cast<const uint4 *>(sp + rr * sstride)));
    } else {
        for (; rr + 8u <= n; rr += 8u) {
            uint16_t x[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = sp[(rr + k) * sstride];
#pragma unroll
            for (int k = 0; k < 8; ++k) dp[(rr + k) * dstride] = x[k];
        }
        for (; rr < n; ++rr) dp[rr * dstride] = sp[rr * sstride];
    }
}

template <bool VEC>
__device__ __forceinline__ void zero_rows(uint16_t *dp, std::size_t dstride, uint32_t n) {
    for (uint32_t rr = 0; rr < n; ++rr) {
        if (VEC)
            __stcs(reinterpret_cast<uint4 *>(dp + rr * dstride), make_uint4(0, 0, 0, 0));
        else
            dp[rr * dstride] = 0u;
    }
}

// One CTA per destination row block (grid-stride).  Valid slots of the
// source row block are ranked chunk by chunk (8 slots per thread) and their
// values copied as 16-byte vectors when B is a multiple of 8 and the values
// are 16-byte aligned (VEC), else as halves.
template <bool VEC>
__global__ void __launch_bounds__(kFillThreads) bell_exec_fill_kernel(
    const cs_blocked_ell_view src, uint32_t RB, const uint32_t *__restrict__ order, const seg_rec *__restrict__ rec,
    const plan_head *__restrict__ head, uint32_t *__restrict__ dst_bci, uint16_t *__restrict__ dst_val,
    uint32_t *__restrict__ e2c, uint32_t *__restrict__ c2e, uint32_t *__restrict__ e2c_cols,
    uint32_t *__restrict__ c2e_cols) {
    __shared__ uint32_t list[kChunk];
    __shared__ uint32_t warp_sums[kFillWarps];
    const uint32_t B = src.block_size, W = src.ell_cols / B, ell = src.ell_cols, S = head->S;
    const uint32_t t = threadIdx.x;
    for (uint32_t c = blockIdx.x * blockDim.x + t; c < src.cols; c += gridDim.x * blockDim.x) {
        if (e2c_cols != nullptr) e2c_cols[c] = c;
        if (c2e_cols != nullptr) c2e_cols[c] = c;
    }
    constexpr uint32_t kVec = 8u; // halves per 16-byte vector
    const uint32_t vpb = VEC ? B / kVec : B;
    for (uint32_t pos = blockIdx.x; pos < RB; pos += gridDim.x) {
        const uint32_t s = find_seg(rec, S, pos);
        const seg_rec r = rec[s];
        const uint32_t w = r.width, dst_rb = pos - r.unit_off, src_rb = order[pos];
        const uint32_t n = min(B, src.rows - src_rb * B);
        const uint32_t exec0 = r.row_off + dst_rb * B;
        for (uint32_t rr = t; rr < n; rr += kFillThreads) {
            if (e2c != nullptr) e2c[exec0 + rr] = src_rb * B + rr;
            if (c2e != nullptr) c2e[src_rb * B + rr] = exec0 + rr;
        }
        const std::size_t dst_ell = (std::size_t) w * B;
        uint32_t *dbci = dst_bci + r.idx_off + (std::size_t) dst_rb * w;
        uint16_t *dval = dst_val + r.val_off + (std::size_t) dst_rb * B * dst_ell;
        const uint32_t *sbci = src.blockColIdx + (std::size_t) src_rb * W;
        const uint16_t *sval = src.val + (std::size_t) src_rb * B * ell;
        uint32_t off = 0u;
        for (uint32_t base = 0; base < W; base += kChunk) {
            uint32_t cols[kSlotsPerThread], mask = 0u;
#pragma unroll
            for (unsigned k = 0; k < kSlotsPerThread; ++k) {
                const uint32_t slot = base + t * kSlotsPerThread + k;
                cols[k] = slot < W ? __ldg(sbci + slot) : kInvalid;
                mask |= (cols[k] != kInvalid ? 1u : 0u) << k;
            }
            uint32_t total;
            uint32_t rank = block_excl_scan(__popc(mask), warp_sums, &total);
#pragma unroll
            for (unsigned k = 0; k < kSlotsPerThread; ++k) {
                if (mask >> k & 1u) {
                    dbci[off + rank] = cols[k];
                    list[rank] = base + t * kSlotsPerThread + k;
                    ++rank;
                }
            }
            __syncthreads();
            // each thread takes (slot, vector) pairs and copies that column of the
            // row block for all n rows, 8 rows' loads in flight at a time
            const uint32_t pairs = total * vpb;
            for (uint32_t q = t; q < pairs; q += kFillThreads) {
                const uint32_t j = q / vpb, v = q - j * vpb;
                const uint16_t *sp = sval + (std::size_t) list[j] * B + v * (VEC ? kVec : 1u);
                uint16_t *dp = dval + (std::size_t) (off + j) * B + v * (VEC ? kVec : 1u);
                copy_rows<VEC>(sp, ell, dp, dst_ell, n);
            }
            off += total;
            __syncthreads(); // list and warp_sums are rewritten by the next chunk
        }
        for (uint32_t j = off + t; j < w; j += kFillThreads) dbci[j] = kInvalid;
        const uint32_t pad_pairs = (w - off) * vpb;
        for (uint32_t q = t; q < pad_pairs; q += kFillThreads) {
            const uint32_t j = off + q / vpb, v = q % vpb;
            zero_rows<VEC>(dval + (std::size_t) j * B + v * (VEC ? kVec : 1u), dst_ell, n);
        }
    }
}

int bell_geometry(const cs_blocked_ell_view *part, bell_geom *g, bool need_values = true) {
    if (need_values) {
        if (!check_bell(part, "bucketed_blocked_ell")) return 0;
    } else if (part == nullptr || (part->rows != 0u && part->ell_cols != 0u &&
                                   (part->block_size == 0u || part->ell_cols % part->block_size != 0u ||
                                    part->blockColIdx == nullptr))) {
        set_error("blocked_ell_bucket_plan: block size must divide ell_cols and the block columns be set");
        return 0;
    }
    if (part->rows != 0u && part->block_size == 0u) {
        set_error("bucketed_blocked_ell: zero block size");
        return 0;
    }
    g->rows = part->rows;
    g->B = part->block_size;
    g->W = part->block_size == 0u ? 0u : part->ell_cols / part->block_size;
    g->RB = part->block_size == 0u ? 0u : (uint32_t) (((uint64_t) part->rows + part->block_size - 1u) / part->block_size);
    const uint32_t last = g->RB == 0u ? 0u : part->rows - (g->RB - 1u) * g->B;
    g->sortable = (g->RB != 0u && last != g->B) ? g->RB - 1u : g->RB;
    return 1;
}

void read_segments(const plan_head &h, const seg_rec *rec, cs_exec_bucket_plan *plan, cs_exec_bucket_segments *segs) {
    plan->segment_count = h.S;
    plan->bucket_count = h.bucket_count;
    plan->units = h.units;
    plan->block_size = h.block_size;
    plan->bytes = h.bytes;
    plan->original_bytes = h.original_bytes;
    plan->index_entries = h.index_entries;
    plan->value_entries = h.value_entries;
    if (segs == nullptr) return;
    for (uint32_t s = 0; s <= h.S; ++s) {
        if (segs->unit_offsets != nullptr) segs->unit_offsets[s] = rec[s].unit_off;
        if (segs->row_offsets != nullptr) segs->row_offsets[s] = rec[s].row_off;
        if (s < h.S && segs->widths != nullptr) segs->widths[s] = rec[s].width;
    }
}

int check_room(const cs_exec_bucket_segments *segs, uint32_t bound, const char *who) {
    if (segs != nullptr && segs->max_segments < bound) {
        set_error("%s: segment arrays hold %u segments, the plan may need %u", who, segs->max_segments, bound);
        return 0;
    }
    return 1;
}

int bell_plan(const cs_blocked_ell_view *part, uint32_t requested, void *scratch, std::size_t scratch_bytes,
              cs_exec_bucket_plan *plan, cs_exec_bucket_segments *segs, std::vector<seg_rec> *recs_out,
              cudaStream_t stream) {
    bell_geom g;
    if (plan == nullptr || !bell_geometry(part, &g)) {
        if (plan == nullptr) set_error("bucketed_blocked_ell_plan: null plan");
        return 0;
    }
    const uint32_t bound = plan_bound(requested, g.RB);
    if (!check_room(segs, bound, "bucketed_blocked_ell_plan")) return 0;
    exec_scratch x;
    carve(nullptr, g.RB, bound, &x);
    if (scratch == nullptr || scratch_bytes < x.bytes) {
        set_error("bucketed_blocked_ell_plan: scratch %zu < %zu bytes", scratch_bytes, x.bytes);
        return 0;
    }
    carve(scratch, g.RB, bound, &x);
    if (g.RB != 0u) {
        bell_rb_width_kernel<<<resident_grid((const void *) bell_rb_width_kernel, 256, 0, ((std::size_t) g.RB + 7u) / 8u),
                               256, 0, stream>>>(*part, g.RB, x.widths);
        if (!launch_ok("bell_rb_width_kernel")) return 0;
        if (!sort_pairs_u32(x.widths, nullptr, g.sortable, x.sorted, x.order, x.sort_tmp, x.sort_bytes, stream))
            return 0;
    }
    bell_layout_kernel<<<1, 32, 0, stream>>>(g, requested, x.order, x.sorted, x.widths, x.head, x.rec);
    if (!launch_ok("bell_layout_kernel")) return 0;
    if (g.RB != 0u) {
        bell_seg_nnz_kernel<<<resident_grid((const void *) bell_seg_nnz_kernel, 256, 0, g.RB), 256, 0, stream>>>(
            g, x.order, x.widths, x.head, x.rec);
        if (!launch_ok("bell_seg_nnz_kernel")) return 0;
    }
    std::vector<char> host(sizeof(plan_head) + ((std::size_t) bound + 1u) * sizeof(seg_rec));
    if (!cuda_ok(cudaMemcpyAsync(host.data(), x.head, host.size(), cudaMemcpyDeviceToHost, stream), "D2H plan") ||
        !cuda_ok(cudaStreamSynchronize(stream), "plan sync"))
        return 0;
    plan_head h;
    std::memcpy(&h, host.data(), sizeof(h));
    const seg_rec *rec = (const seg_rec *) (host.data() + sizeof(plan_head));
    read_segments(h, rec, plan, segs);
    if (recs_out != nullptr) recs_out->assign(rec, rec + h.S + 1u);
    return 1;
}

int bell_fill(const cs_blocked_ell_view *part, const void *scratch, const cs_exec_bucket_plan *plan,
              uint32_t *seg_bci, uint16_t *seg_val, uint32_t *e2c, uint32_t *c2e, uint32_t *e2c_cols,
              uint32_t *c2e_cols, cudaStream_t stream) {
    bell_geom g;
    if (plan == nullptr || scratch == nullptr || !bell_geometry(part, &g)) {
        if (plan == nullptr || scratch == nullptr) set_error("bucketed_blocked_ell_fill: null plan or scratch");
        return 0;
    }
    if (plan->units != g.RB || plan->block_size != g.B) {
        set_error("bucketed_blocked_ell_fill: the plan was made for another part");
        return 0;
    }
    if ((plan->index_entries != 0u && seg_bci == nullptr) || (plan->value_entries != 0u && seg_val == nullptr)) {
        set_error("bucketed_blocked_ell_fill: null segment arrays");
        return 0;
    }
    exec_scratch x;
    carve(const_cast<void *>(scratch), g.RB, 1u, &x);
    const bool vec = g.B % 8u == 0u && (reinterpret_cast<uintptr_t>(part->val) & 15u) == 0u &&
                     (reinterpret_cast<uintptr_t>(seg_val) & 15u) == 0u;
    // blocks: one per destination row block, and enough to write the column maps
    const std::size_t col_blocks = ((std::size_t) part->cols + kFillThreads - 1u) / kFillThreads;
    const std::size_t work = g.RB > col_blocks ? g.RB : col_blocks;
    if (work == 0u) return 1;
    const void *k = vec ? (const void *) bell_exec_fill_kernel<true> : (const void *) bell_exec_fill_kernel<false>;
    const unsigned grid = resident_grid(k, kFillThreads, 0, work);
    if (vec)
        bell_exec_fill_kernel<true><<<grid, kFillThreads, 0, stream>>>(*part, g.RB, x.order, x.rec, x.head, seg_bci,
                                                                      seg_val, e2c, c2e, e2c_cols, c2e_cols);
    else
        bell_exec_fill_kernel<false><<<grid, kFillThreads, 0, stream>>>(*part, g.RB, x.order, x.rec, x.head, seg_bci,
                                                                       seg_val, e2c, c2e, e2c_cols, c2e_cols);
    return launch_ok("bell_exec_fill_kernel");
}

// ---------------------------------------------------------------------------
// Sliced-ELL
// ---------------------------------------------------------------------------
// find_slice (formats/sliced_ell.cuh:80-87): the first slice whose end lies
// past the row.
__device__ __forceinline__ uint32_t slice_of(const cs_sliced_ell_view &v, uint32_t row) {
    // slices of one height h (all but possibly the last): slice row / h, checked
    // against the offsets; any other layout falls back to the binary search
    if (v.slice_count > 1u) {
        const uint32_t h = __ldg(v.slice_row_offsets + 1u) - __ldg(v.slice_row_offsets);
        const uint32_t g = h != 0u ? row / h : v.slice_count;
        if (g < v.slice_count && __ldg(v.slice_row_offsets + g) <= row && row < __ldg(v.slice_row_offsets + g + 1u))
            return g;
    }
    uint32_t lo = 0u, hi = v.slice_count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (row < v.slice_row_offsets[mid + 1u])
            hi = mid;
        else
            lo = mid + 1u;
    }
    return lo;
}

__global__ void __launch_bounds__(256) sell_row_width_kernel(const cs_sliced_ell_view src,
                                                             uint32_t *__restrict__ widths) {
    const uint32_t lane = threadIdx.x & 31u, warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < src.rows; row += warps) {
        const uint32_t s = slice_of(src, row);
        uint32_t n = 0u;
        if (s < src.slice_count) {
            const uint32_t w = src.slice_widths[s];
            const uint32_t *c = src.col_idx + src.slice_slot_offsets[s] + (std::size_t) (row - src.slice_row_offsets[s]) * w;
            for (uint32_t k = lane; k < w; k += 32u) n += __ldg(c + k) != kInvalid;
        }
        n = __reduce_add_sync(0xffffffffu, n);
        if (lane == 0u) widths[row] = n;
    }
}

// One warp per execution row: the row's live slots compacted by ballot rank,
// padding after them.
__global__ void __launch_bounds__(256) sell_exec_fill_kernel(const cs_sliced_ell_view src,
                                                             const uint32_t *__restrict__ order,
                                                             const seg_rec *__restrict__ rec,
                                                             const plan_head *__restrict__ head,
                                                             uint32_t *__restrict__ dst_col,
                                                             uint16_t *__restrict__ dst_val,
                                                             uint32_t *__restrict__ e2c, uint32_t *__restrict__ c2e) {
    const uint32_t lane = threadIdx.x & 31u, warps = (gridDim.x * blockDim.x) >> 5, S = head->S;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < src.rows; p += warps) {
        const seg_rec r = rec[find_seg(rec, S, p)];
        const uint32_t row = order[p], w = r.width;
        uint32_t *dc = dst_col + r.idx_off + (std::size_t) (p - r.unit_off) * w;
        uint16_t *dv = dst_val + r.val_off + (std::size_t) (p - r.unit_off) * w;
        const uint32_t s = slice_of(src, row);
        uint32_t off = 0u;
        if (s < src.slice_count) {
            const uint32_t sw = src.slice_widths[s];
            const std::size_t base = src.slice_slot_offsets[s] + (std::size_t) (row - src.slice_row_offsets[s]) * sw;
            // 128 slots per step: four column loads per lane; the live values of
            // a step are loaded together with the next step's columns, then four
            // ballot-ranked stores
            uint32_t cn[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t k = 32u * u + lane;
                cn[u] = k < sw ? __ldcs(src.col_idx + base + k) : kInvalid;
            }
            for (uint32_t k0 = 0; k0 < sw; k0 += 128u) {
                uint32_t c[4];
                uint16_t x[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) c[u] = cn[u];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    x[u] = c[u] != kInvalid ? __ldcs(src.val + base + k0 + 32u * u + lane) : (uint16_t) 0u;
                    const uint32_t k = k0 + 128u + 32u * u + lane;
                    cn[u] = k < sw ? __ldcs(src.col_idx + base + k) : kInvalid;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const unsigned m = __ballot_sync(0xffffffffu, c[u] != kInvalid);
                    if (c[u] != kInvalid) {
                        const uint32_t at = off + __popc(m & ((1u << lane) - 1u));
                        dc[at] = c[u];
                        dv[at] = x[u];
                    }
                    off += __popc(m);
                }
            }
        }
        for (uint32_t j = off + lane; j < w; j += 32u) {
            dc[j] = kInvalid;
            dv[j] = 0u;
        }
        if (lane == 0u) {
            if (e2c != nullptr) e2c[p] = row;
            if (c2e != nullptr) c2e[row] = p;
        }
    }
}

int check_sell(const cs_sliced_ell_view *part, const char *who) {
    if (part == nullptr) {
        set_error("%s: null view", who);
        return 0;
    }
    if (part->rows != 0u && part->slice_count != 0u &&
        (part->slice_row_offsets == nullptr || part->slice_widths == nullptr || part->slice_slot_offsets == nullptr)) {
        set_error("%s: slice offsets, widths and slot offsets must be set", who);
        return 0;
    }
    return 1;
}

// The split programme (build_sliced_execution_bucket_layout :1312-1412) for
// levels 1..K over ascending widths; cut(k, r) = first row of the last of k
// segments covering rows [0, r).
struct sliced_split {
    uint32_t rows = 0, K = 0;
    std::unique_ptr<uint32_t[]> cuts; // (K + 1) x (rows + 1)
    std::vector<uint64_t> cost_at_rows; // level k's cost of all rows

    static constexpr uint64_t kInf = ~0ull / 4u;
    static constexpr uint32_t kBlockRows = 4096u;

    struct line {
        int64_t slope, icpt;
        uint32_t cut;
    };

    // One level over rows k..rows: prev = level k-1's costs, curr = this
    // level's.  When `ready` is set, level k-1 runs in another thread and
    // `ready` holds the last row it has finished: rows are taken in blocks
    // once the previous level has passed them (bounded only by its progress,
    // which always advances).
    void level(uint32_t k, const std::vector<uint32_t> &w, const uint64_t *prev, uint64_t *curr,
               const std::atomic<uint32_t> *ready, std::atomic<uint32_t> *done) {
        const uint64_t fixed = packed_sell_bytes(1u, 0u), slot = 6u;
        auto at = [](const line &l, uint32_t x) { return l.icpt + l.slope * (int64_t) x; };
        auto redundant = [](const line &a, const line &m, const line &b) {
            const __int128 left = (__int128) (b.icpt - a.icpt) * (__int128) (a.slope - m.slope);
            const __int128 right = (__int128) (m.icpt - a.icpt) * (__int128) (a.slope - b.slope);
            return left <= right;
        };
        std::unique_ptr<line[]> hull(new line[(std::size_t) rows + 1u]); // written before read
        std::size_t n = 0u, h = 0u;
        uint32_t *cut = cuts.get() + (std::size_t) k * (rows + 1u);
        uint32_t avail = ready != nullptr ? ready->load(std::memory_order_acquire) : rows;
        while (avail < k - 1u) {
            std::this_thread::yield();
            avail = ready->load(std::memory_order_acquire);
        }
        if (prev[k - 1u] != kInf) hull[n++] = line{-(int64_t) slot * (int64_t) (k - 1u), (int64_t) prev[k - 1u], k - 1u};
        for (uint32_t r0 = k; r0 <= rows; r0 += kBlockRows) {
            const uint32_t r1 = r0 + kBlockRows - 1u < rows ? r0 + kBlockRows - 1u : rows;
            while (avail < r1) {
                std::this_thread::yield();
                avail = ready->load(std::memory_order_acquire);
            }
            for (uint32_t r = r0; r <= r1; ++r) {
                const uint32_t x = w[r - 1u];
                while (h + 1u < n && at(hull[h + 1u], x) < at(hull[h], x)) ++h;
                if (h < n) {
                    curr[r] = fixed + slot * (uint64_t) x * (uint64_t) r + (uint64_t) at(hull[h], x);
                    cut[r] = hull[h].cut;
                } else {
                    curr[r] = kInf;
                    cut[r] = 0u;
                }
                if (prev[r] != kInf) {
                    const line l{-(int64_t) slot * (int64_t) r, (int64_t) prev[r], r};
                    while (n >= h + 2u && redundant(hull[n - 2u], hull[n - 1u], l)) --n;
                    hull[n++] = l;
                }
            }
            if (done != nullptr) done->store(r1, std::memory_order_release);
        }
        if (done != nullptr) done->store(rows, std::memory_order_release);
    }

    // Levels 1..K.  Each level's loop is sequential (its hull depends on every
    // earlier row), but level k only needs level k-1's costs of rows up to the
    // one it is at, so the levels run as a pipeline, one thread each, level k
    // a block of rows behind level k-1; every cost and cut is the one the
    // sequential order computes.
    bool run(const std::vector<uint32_t> &w, uint32_t levels) {
        rows = (uint32_t) w.size();
        K = levels;
        // level 0: no rows cost 0, any row unreachable; a level k >= 1 writes
        // every entry r >= k, the only ones level k + 1 reads
        std::vector<std::unique_ptr<uint64_t[]>> cost((std::size_t) K + 1u);
        for (auto &c : cost) c.reset(new uint64_t[(std::size_t) rows + 1u]);
        for (uint32_t r = 0; r <= rows; ++r) cost[0][r] = r == 0u ? 0u : kInf;
        cuts.reset(new uint32_t[((std::size_t) K + 1u) * ((std::size_t) rows + 1u)]);
        cost_at_rows.assign((std::size_t) K + 1u, kInf);
        const unsigned hw = std::thread::hardware_concurrency();
        if (K <= 1u || rows < 2u * kBlockRows || K > 16u || hw < 2u) {
            for (uint32_t k = 1; k <= K; ++k) level(k, w, cost[k - 1u].get(), cost[k].get(), nullptr, nullptr);
        } else {
            std::vector<std::atomic<uint32_t>> progress((std::size_t) K + 1u);
            progress[0].store(rows);
            for (uint32_t k = 1; k <= K; ++k) progress[k].store(0u);
            std::vector<std::thread> th;
            th.reserve(K);
            uint32_t started = 0u;
            try {
                for (uint32_t k = 1; k <= K; ++k, ++started)
                    th.emplace_back([&, k] { level(k, w, cost[k - 1u].get(), cost[k].get(), &progress[k - 1u],
                                                   &progress[k]); });
            } catch (...) {
                // no thread for level `started + 1`: the remaining levels run here,
                // after the started ones (each still waits on its predecessor)
            }
            for (uint32_t k = started + 1u; k <= K; ++k)
                level(k, w, cost[k - 1u].get(), cost[k].get(), &progress[k - 1u], &progress[k]);
            for (auto &t : th) t.join();
        }
        for (uint32_t k = 1; k <= K; ++k) cost_at_rows[k] = cost[k][rows];
        return true;
    }
    // Segments of the k-level split after equal-width neighbours merge.
    bool layout(const std::vector<uint32_t> &w, uint32_t k, std::vector<uint32_t> *offs,
                std::vector<uint32_t> *widths) const {
        offs->assign(1, 0u);
        widths->clear();
        if (rows == 0u) return true;
        if (cost_at_rows[k] == kInf) return false;
        std::vector<uint32_t> raw_off((std::size_t) k + 1u), raw_w(k);
        uint32_t r = rows;
        raw_off[k] = rows;
        for (uint32_t j = k; j != 0u; --j) {
            const uint32_t begin = cuts.get()[(std::size_t) j * (rows + 1u) + r];
            raw_off[j - 1u] = begin;
            raw_w[j - 1u] = w[r - 1u];
            r = begin;
        }
        for (uint32_t j = 0; j < k; ++j) {
            if (!widths->empty() && widths->back() == raw_w[j]) {
                offs->back() = raw_off[j + 1u];
            } else {
                widths->push_back(raw_w[j]);
                offs->push_back(raw_off[j + 1u]);
            }
        }
        return true;
    }
};

uint64_t sliced_layout_bytes(const std::vector<uint32_t> &offs, const std::vector<uint32_t> &widths) {
    uint64_t b = 0u;
    for (std::size_t s = 0; s < widths.size(); ++s) {
        const uint32_t n = offs[s + 1] - offs[s];
        b += packed_sell_bytes(n != 0u ? 1u : 0u, (uint64_t) n * widths[s]);
    }
    return b;
}

int sell_plan(const cs_sliced_ell_view *part, uint32_t requested, void *scratch, std::size_t scratch_bytes,
              cs_exec_bucket_plan *plan, cs_exec_bucket_segments *segs, std::vector<seg_rec> *recs_out,
              cudaStream_t stream) {
    if (plan == nullptr) {
        set_error("bucketed_sliced_ell_plan: null plan");
        return 0;
    }
    if (!check_sell(part, "bucketed_sliced_ell_plan")) return 0;
    const uint32_t rows = part->rows;
    const uint32_t bound = plan_bound(requested, rows);
    if (!check_room(segs, bound, "bucketed_sliced_ell_plan")) return 0;
    exec_scratch x;
    carve(nullptr, rows, bound, &x);
    if (scratch == nullptr || scratch_bytes < x.bytes) {
        set_error("bucketed_sliced_ell_plan: scratch %zu < %zu bytes", scratch_bytes, x.bytes);
        return 0;
    }
    carve(scratch, rows, bound, &x);
    // source slots and packed bytes (partition_aux of the part: its slice
    // count and total slots, packfile.cuh:248-250)
    std::vector<uint32_t> src_offs((std::size_t) part->slice_count + 1u, 0u), src_w(part->slice_count);
    if (part->slice_count != 0u &&
        (!cuda_ok(cudaMemcpyAsync(src_offs.data(), part->slice_row_offsets, src_offs.size() * 4u,
                                  cudaMemcpyDeviceToHost, stream), "D2H slice offsets") ||
         !cuda_ok(cudaMemcpyAsync(src_w.data(), part->slice_widths, src_w.size() * 4u, cudaMemcpyDeviceToHost, stream),
                  "D2H slice widths") ||
         !cuda_ok(cudaStreamSynchronize(stream), "slice table sync")))
        return 0;
    uint64_t total = 0u;
    for (uint32_t s = 0; s < part->slice_count; ++s) total += (uint64_t) (src_offs[s + 1u] - src_offs[s]) * src_w[s];
    if (total != 0u && (part->col_idx == nullptr || part->val == nullptr)) {
        set_error("bucketed_sliced_ell_plan: %llu slots but null columns or values", (unsigned long long) total);
        return 0;
    }
    std::vector<uint32_t> w(rows);
    if (rows != 0u) {
        sell_row_width_kernel<<<resident_grid((const void *) sell_row_width_kernel, 256, 0, ((std::size_t) rows + 7u) / 8u),
                                256, 0, stream>>>(*part, x.widths);
        if (!launch_ok("sell_row_width_kernel")) return 0;
        if (!sort_pairs_u32(x.widths, nullptr, rows, x.sorted, x.order, x.sort_tmp, x.sort_bytes, stream)) return 0;
        if (!cuda_ok(cudaMemcpyAsync(w.data(), x.sorted, (std::size_t) rows * 4u, cudaMemcpyDeviceToHost, stream),
                     "D2H sorted widths") ||
            !cuda_ok(cudaStreamSynchronize(stream), "plan sync"))
            return 0;
    }
    plan_head h{};
    h.units = rows;
    h.block_size = 1u;
    h.original_bytes = packed_sell_bytes(part->slice_count, (uint32_t) total);
    std::vector<uint32_t> offs{0u}, widths;
    uint32_t buckets = requested == 0u ? 1u : requested;
    if (rows != 0u) {
        sliced_split dp;
        const uint32_t levels = bound;
        dp.run(w, levels);
        auto kept = [&](uint32_t b, std::vector<uint32_t> *o, std::vector<uint32_t> *wd, uint64_t *bytes) {
            if (!dp.layout(w, b, o, wd)) return false;
            *bytes = sliced_layout_bytes(*o, *wd);
            if (wd->size() > 1u && *bytes >= h.original_bytes) {
                if (!dp.layout(w, 1u, o, wd)) return false;
                *bytes = h.original_bytes;
            }
            return true;
        };
        if (requested == 0u) {
            uint64_t best = ~0ull;
            for (uint32_t b = 1; b <= levels; ++b) {
                std::vector<uint32_t> o, wd;
                uint64_t bytes = 0u;
                if (!kept(b, &o, &wd, &bytes)) {
                    set_error("bucketed_sliced_ell_plan: no split into %u segments", b);
                    return 0;
                }
                if (bytes < best) {
                    best = bytes;
                    buckets = b;
                }
            }
        }
        if (!kept(buckets < levels ? buckets : levels, &offs, &widths, &h.bytes)) {
            set_error("bucketed_sliced_ell_plan: no split into %u segments", buckets);
            return 0;
        }
    }
    h.bucket_count = buckets;
    h.S = (uint32_t) widths.size();
    std::vector<char> host(sizeof(plan_head) + ((std::size_t) h.S + 1u) * sizeof(seg_rec));
    seg_rec *rec = (seg_rec *) (host.data() + sizeof(plan_head));
    uint64_t slots = 0u;
    for (uint32_t s = 0; s < h.S; ++s) {
        uint32_t nnz = 0u; // the reference's u32 sum of the rows' live slots
        for (uint32_t p = offs[s]; p < offs[s + 1u]; ++p) nnz += w[p];
        rec[s] = seg_rec{offs[s], offs[s], widths[s], 0u, slots, slots, nnz};
        slots += (uint64_t) (offs[s + 1u] - offs[s]) * widths[s];
    }
    rec[h.S] = seg_rec{rows, rows, 0u, 0u, slots, slots, 0u};
    h.index_entries = slots;
    h.value_entries = slots;
    std::memcpy(host.data(), &h, sizeof(h));
    if (!cuda_ok(cudaMemcpyAsync(x.head, host.data(), host.size(), cudaMemcpyHostToDevice, stream), "H2D plan") ||
        !cuda_ok(cudaStreamSynchronize(stream), "plan upload"))
        return 0;
    read_segments(h, rec, plan, segs);
    if (recs_out != nullptr) recs_out->assign(rec, rec + h.S + 1u);
    return 1;
}

int sell_fill(const cs_sliced_ell_view *part, const void *scratch, const cs_exec_bucket_plan *plan, uint32_t *seg_col,
              uint16_t *seg_val, uint32_t *e2c, uint32_t *c2e, cudaStream_t stream) {
    if (plan == nullptr || scratch == nullptr) {
        set_error("bucketed_sliced_ell_fill: null plan or scratch");
        return 0;
    }
    if (!check_sell(part, "bucketed_sliced_ell_fill")) return 0;
    if (plan->units != part->rows || plan->block_size != 1u) {
        set_error("bucketed_sliced_ell_fill: the plan was made for another part");
        return 0;
    }
    if (plan->index_entries != 0u && (seg_col == nullptr || seg_val == nullptr)) {
        set_error("bucketed_sliced_ell_fill: null segment arrays");
        return 0;
    }
    if (part->rows == 0u) return 1;
    exec_scratch x;
    carve(const_cast<void *>(scratch), part->rows, 1u, &x);
    sell_exec_fill_kernel<<<resident_grid((const void *) sell_exec_fill_kernel, 256, 0, ((std::size_t) part->rows + 7u) / 8u),
                            256, 0, stream>>>(*part, x.order, x.rec, x.head, seg_col, seg_val, e2c, c2e);
    return launch_ok("sell_exec_fill_kernel");
}

// ---------------------------------------------------------------------------
// Ingest-time bucket-count choice
// ---------------------------------------------------------------------------
// Row-block key of bucket::build_plan (blocked_ell_bucket.cuh:78-95): the
// valid width, and a hash folded over the valid block columns in slot order
// (h ^= c + 0x9e3779b9 + (h << 6) + (h >> 2); h *= 16777619; from 2166136261).
// One warp per row block: the columns of each 32-slot step are broadcast by
// shuffle and every lane folds the same chain.
__global__ void __launch_bounds__(256) bell_rb_key_kernel(const cs_blocked_ell_view src, uint32_t RB,
                                                          uint32_t *__restrict__ widths,
                                                          uint32_t *__restrict__ hashes) {
    const uint32_t lane = threadIdx.x & 31u, W = src.ell_cols / src.block_size;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t rb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rb < RB; rb += warps) {
        const uint32_t *row = src.blockColIdx + (std::size_t) rb * W;
        uint32_t n = 0u, h = 2166136261u;
        for (uint32_t k0 = 0; k0 < W; k0 += 32u) {
            const uint32_t k = k0 + lane;
            const uint32_t c = k < W ? __ldg(row + k) : kInvalid;
            unsigned m = __ballot_sync(0xffffffffu, c != kInvalid);
            n += __popc(m);
            while (m != 0u) {
                const uint32_t x = __shfl_sync(0xffffffffu, c, __ffs(m) - 1);
                m &= m - 1u;
                h ^= x + 0x9e3779b9u + (h << 6) + (h >> 2);
                h *= 16777619u;
            }
        }
        if (lane == 0u) {
            widths[rb] = n;
            hashes[rb] = h;
        }
    }
}

__global__ void gather_u32_kernel(uint32_t n, const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx,
                                  uint32_t *__restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// choose_bucket_count_for_part of the ingest path (convert_layout_support_part.hh:
// 116-181): for 1..min(8, RB) buckets of equal row-block ranges over the plan
// order, idx + values of width = the range's last sorted width, plus both row
// maps and the offsets; a count must beat the source's packed bytes.
__global__ void __launch_bounds__(256) ingest_choose_kernel(uint32_t rows, uint32_t B, uint32_t W, uint32_t RB,
                                                            const uint32_t *__restrict__ order,
                                                            const uint32_t *__restrict__ width_sorted,
                                                            uint32_t *__restrict__ out_count,
                                                            unsigned long long *__restrict__ out_bytes) {
    __shared__ uint32_t partial_pos;
    const uint32_t last_rows = RB == 0u ? 0u : rows - (RB - 1u) * B;
    if (threadIdx.x == 0u) partial_pos = kInvalid;
    __syncthreads();
    if (RB > 1u && last_rows != B)
        for (uint32_t p = threadIdx.x; p < RB; p += blockDim.x)
            if (order[p] == RB - 1u) partial_pos = p;
    __syncthreads();
    if (threadIdx.x != 0u) return;
    uint64_t best = packed_bell_bytes(rows, (uint64_t) W * B, B);
    uint32_t best_b = 1u;
    if (RB > 1u) {
        const uint32_t top = RB < kChooseMax ? RB : kChooseMax;
        for (uint32_t nb = 1; nb <= top; ++nb) {
            uint64_t bytes = 0u;
            for (uint32_t b = 0; b < nb; ++b) {
                const uint32_t lo = (b * RB) / nb, hi = ((b + 1u) * RB) / nb;
                if (hi <= lo) continue;
                const uint32_t w = width_sorted[hi - 1u];
                uint32_t seg_rows = (hi - lo) * B;
                if (partial_pos >= lo && partial_pos < hi) seg_rows -= B - last_rows;
                bytes += (uint64_t) (hi - lo) * w * 4u;
                bytes += (uint64_t) seg_rows * w * B * 2u;
            }
            bytes += (uint64_t) rows * 8u + ((uint64_t) nb + 1u) * 4u;
            if (bytes < best) {
                best = bytes;
                best_b = nb;
            }
        }
    }
    *out_count = best_b;
    *out_bytes = best;
}

struct plan_scratch {
    uint32_t *widths, *hashes, *order1, *hash_sorted, *w1;
    void *sort_tmp;
    std::size_t sort_bytes, bytes;
};

void carve_plan(void *base, uint32_t RB, plan_scratch *x) {
    scratch_carver c(base, ~std::size_t(0));
    x->widths = c.take<uint32_t>((std::size_t) RB + 1u);
    x->hashes = c.take<uint32_t>((std::size_t) RB + 1u);
    x->order1 = c.take<uint32_t>((std::size_t) RB + 1u);
    x->hash_sorted = c.take<uint32_t>((std::size_t) RB + 1u);
    x->w1 = c.take<uint32_t>((std::size_t) RB + 1u);
    x->sort_bytes = sort_pairs_u32_scratch_bytes(RB);
    x->sort_tmp = c.take<char>(x->sort_bytes);
    x->bytes = c.used;
}

// bucket::build_plan: keys, then a stable sort by the 64-bit key as two
// stable 32-bit passes (hash, then width), which orders equal keys by row
// block as the reference's 64-bit radix sort does.
int bucket_plan(const cs_blocked_ell_view *part, uint32_t *order, uint32_t *width_sorted, void *scratch,
                std::size_t scratch_bytes, cudaStream_t stream) {
    bell_geom g;
    if (!bell_geometry(part, &g, false)) return 0;
    plan_scratch x;
    carve_plan(nullptr, g.RB, &x);
    if (scratch == nullptr || scratch_bytes < x.bytes) {
        set_error("blocked_ell_bucket_plan: scratch %zu < %zu bytes", scratch_bytes, x.bytes);
        return 0;
    }
    if (g.RB == 0u) return 1;
    if (order == nullptr || width_sorted == nullptr) {
        set_error("blocked_ell_bucket_plan: null outputs");
        return 0;
    }
    carve_plan(scratch, g.RB, &x);
    bell_rb_key_kernel<<<resident_grid((const void *) bell_rb_key_kernel, 256, 0, ((std::size_t) g.RB + 7u) / 8u), 256,
                         0, stream>>>(*part, g.RB, x.widths, x.hashes);
    if (!launch_ok("bell_rb_key_kernel")) return 0;
    if (!sort_pairs_u32(x.hashes, nullptr, g.RB, x.hash_sorted, x.order1, x.sort_tmp, x.sort_bytes, stream)) return 0;
    gather_u32_kernel<<<resident_grid((const void *) gather_u32_kernel, 256, 0, ((std::size_t) g.RB + 255u) / 256u), 256,
                        0, stream>>>(g.RB, x.widths, x.order1, x.w1);
    if (!launch_ok("gather_u32_kernel")) return 0;
    return sort_pairs_u32(x.w1, x.order1, g.RB, width_sorted, order, x.sort_tmp, x.sort_bytes, stream);
}

std::size_t scratch_for(uint32_t units, uint32_t max_segments) {
    exec_scratch x;
    const uint32_t b = max_segments > kChooseMax ? max_segments : kChooseMax;
    carve(nullptr, units, plan_bound(b, units), &x);
    return x.bytes;
}

uint32_t *host_u32(std::size_t n) { return n == 0u ? nullptr : (uint32_t *) std::malloc(n * 4u); }

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_bucketed_blocked_ell_scratch_bytes(uint32_t rows, uint32_t block_size, uint32_t max_segments,
                                                          size_t *out_bytes) {
    if (out_bytes == nullptr || (rows != 0u && block_size == 0u)) {
        set_error("bucketed_blocked_ell_scratch_bytes: null output or zero block size");
        return 0;
    }
    const uint32_t RB = rows == 0u ? 0u : (uint32_t) (((uint64_t) rows + block_size - 1u) / block_size);
    *out_bytes = scratch_for(RB, max_segments);
    return 1;
}

extern "C" int cs_b200_bucketed_blocked_ell_plan(const cs_blocked_ell_view *part, uint32_t requested, void *d_scratch,
                                                 size_t scratch_bytes, cs_exec_bucket_plan *plan,
                                                 cs_exec_bucket_segments *segments, cs_stream_t s) {
    return bell_plan(part, requested, d_scratch, scratch_bytes, plan, segments, nullptr, as_stream(s));
}

extern "C" int cs_b200_bucketed_blocked_ell_fill(const cs_blocked_ell_view *part, const void *d_scratch,
                                                 const cs_exec_bucket_plan *plan, uint32_t *d_seg_block_col_idx,
                                                 uint16_t *d_seg_val, uint32_t *d_exec_to_canonical_rows,
                                                 uint32_t *d_canonical_to_exec_rows,
                                                 uint32_t *d_exec_to_canonical_cols,
                                                 uint32_t *d_canonical_to_exec_cols, cs_stream_t s) {
    return bell_fill(part, d_scratch, plan, d_seg_block_col_idx, d_seg_val, d_exec_to_canonical_rows,
                     d_canonical_to_exec_rows, d_exec_to_canonical_cols, d_canonical_to_exec_cols, as_stream(s));
}

extern "C" int cs_b200_bucketed_sliced_ell_scratch_bytes(uint32_t rows, uint32_t max_segments, size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("bucketed_sliced_ell_scratch_bytes: null output");
        return 0;
    }
    *out_bytes = scratch_for(rows, max_segments);
    return 1;
}

extern "C" int cs_b200_bucketed_sliced_ell_plan(const cs_sliced_ell_view *part, uint32_t requested, void *d_scratch,
                                                size_t scratch_bytes, cs_exec_bucket_plan *plan,
                                                cs_exec_bucket_segments *segments, cs_stream_t s) {
    return sell_plan(part, requested, d_scratch, scratch_bytes, plan, segments, nullptr, as_stream(s));
}

extern "C" int cs_b200_bucketed_sliced_ell_fill(const cs_sliced_ell_view *part, const void *d_scratch,
                                                const cs_exec_bucket_plan *plan, uint32_t *d_seg_col_idx,
                                                uint16_t *d_seg_val, uint32_t *d_exec_to_canonical_rows,
                                                uint32_t *d_canonical_to_exec_rows, cs_stream_t s) {
    return sell_fill(part, d_scratch, plan, d_seg_col_idx, d_seg_val, d_exec_to_canonical_rows,
                     d_canonical_to_exec_rows, as_stream(s));
}

extern "C" int cs_b200_blocked_ell_bucket_plan_scratch_bytes(uint32_t rows, uint32_t block_size, size_t *out_bytes) {
    if (out_bytes == nullptr || (rows != 0u && block_size == 0u)) {
        set_error("blocked_ell_bucket_plan_scratch_bytes: null output or zero block size");
        return 0;
    }
    plan_scratch x;
    carve_plan(nullptr, rows == 0u ? 0u : (uint32_t) (((uint64_t) rows + block_size - 1u) / block_size), &x);
    *out_bytes = x.bytes;
    return 1;
}

extern "C" int cs_b200_blocked_ell_bucket_plan(const cs_blocked_ell_view *part, uint32_t *d_row_block_order,
                                               uint32_t *d_row_block_width_sorted, void *d_scratch,
                                               size_t scratch_bytes, cs_stream_t s) {
    return bucket_plan(part, d_row_block_order, d_row_block_width_sorted, d_scratch, scratch_bytes, as_stream(s));
}

extern "C" int cs_b200_choose_bucket_count_from_plan(const cs_blocked_ell_view *part,
                                                     const uint32_t *d_row_block_order,
                                                     const uint32_t *d_row_block_width_sorted,
                                                     uint32_t *d_bucket_count, uint64_t *d_estimated_bytes,
                                                     cs_stream_t s) {
    bell_geom g;
    if (!bell_geometry(part, &g, false)) return 0;
    if (d_bucket_count == nullptr || d_estimated_bytes == nullptr ||
        (g.RB > 1u && (d_row_block_order == nullptr || d_row_block_width_sorted == nullptr))) {
        set_error("choose_bucket_count_from_plan: null argument");
        return 0;
    }
    ingest_choose_kernel<<<1, 256, 0, as_stream(s)>>>(g.rows, g.B, g.W, g.RB, d_row_block_order,
                                                     d_row_block_width_sorted, d_bucket_count,
                                                     (unsigned long long *) d_estimated_bytes);
    return launch_ok("ingest_choose_kernel");
}

extern "C" int cs_b200_choose_ingest_bucket_count_for_part(const cs_host_blocked_ell *part, int device,
                                                           uint32_t *bucket_count_out) {
    if (part == nullptr || bucket_count_out == nullptr || (part->rows != 0u && part->block_size == 0u)) {
        set_error("choose_ingest_bucket_count_for_part: null argument or zero block size");
        return 0;
    }
    const uint32_t B = part->block_size;
    const uint32_t RB = part->rows == 0u ? 0u : (uint32_t) (((uint64_t) part->rows + B - 1u) / B);
    if (RB <= 1u) {
        *bucket_count_out = 1u;
        return 1;
    }
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return 0;
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    // the plan reads the block column indices only (the reference uploads just those)
    const std::size_t idx_bytes = (std::size_t) RB * (part->ell_cols / B) * 4u;
    plan_scratch x;
    carve_plan(nullptr, RB, &x);
    dmem bci, scratch, out;
    if (!bci.alloc(idx_bytes, "bucket plan idx") || !scratch.alloc(x.bytes, "bucket plan scratch") ||
        !out.alloc(((std::size_t) RB * 2u + 4u) * 4u, "bucket plan out"))
        return 0;
    if (idx_bytes != 0u &&
        !cuda_ok(cudaMemcpyAsync(bci.p, part->blockColIdx, idx_bytes, cudaMemcpyHostToDevice, g.s), "H2D idx"))
        return 0;
    const cs_blocked_ell_view v{part->rows, part->cols, part->nnz, B, part->ell_cols, (uint32_t *) bci.p, nullptr};
    uint32_t *order = (uint32_t *) out.p, *ws = order + RB, *res = ws + RB;
    if (!bucket_plan(&v, order, ws, scratch.p, x.bytes, g.s)) return 0;
    ingest_choose_kernel<<<1, 256, 0, g.s>>>(v.rows, B, v.ell_cols / B, RB, order, ws, res,
                                            (unsigned long long *) (res + 2));
    if (!launch_ok("ingest_choose_kernel")) return 0;
    return cuda_ok(cudaMemcpyAsync(bucket_count_out, res, 4, cudaMemcpyDeviceToHost, g.s), "D2H count") &&
           cuda_ok(cudaStreamSynchronize(g.s), "sync choose");
}

// ---------------------------------------------------------------------------
// The reference's host signatures
// ---------------------------------------------------------------------------
extern "C" void cs_b200_host_bucketed_blocked_ell_clear(cs_host_bucketed_blocked_ell *p) {
    if (p == nullptr) return;
    if (p->segments != nullptr)
        for (uint32_t s = 0; s < p->segment_count; ++s) cs_b200_host_blocked_ell_clear(p->segments + s);
    std::free(p->segments);
    std::free(p->segment_row_offsets);
    std::free(p->exec_to_canonical_rows);
    std::free(p->canonical_to_exec_rows);
    std::free(p->exec_to_canonical_cols);
    std::free(p->canonical_to_exec_cols);
    std::memset(p, 0, sizeof(*p));
}

extern "C" void cs_b200_host_bucketed_sliced_ell_clear(cs_host_bucketed_sliced_ell *p) {
    if (p == nullptr) return;
    if (p->segments != nullptr)
        for (uint32_t s = 0; s < p->segment_count; ++s) cs_b200_host_sliced_ell_clear(p->segments + s);
    std::free(p->segments);
    std::free(p->segment_row_offsets);
    std::free(p->exec_to_canonical_rows);
    std::free(p->canonical_to_exec_rows);
    std::free(p->canonical_slice_row_offsets);
    std::free(p->canonical_slice_widths);
    std::memset(p, 0, sizeof(*p));
}

namespace {

int host_bell_bucketed(cs_host_bucketed_blocked_ell *out, const cs_host_blocked_ell *part, uint32_t requested,
                       uint64_t *bytes, uint32_t *chosen, bool plan_only) {
    if (out == nullptr || part == nullptr || (part->rows != 0u && part->block_size == 0u)) {
        set_error("build_bucketed_blocked_ell_partition: null argument or zero block size");
        return 0;
    }
    std::memset(out, 0, sizeof(*out));
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    staged_bell sb;
    if (!stage_bell(part, &sb, g.s)) return 0;
    const uint32_t B = part->block_size;
    const uint32_t RB = part->rows == 0u ? 0u : (uint32_t) (((uint64_t) part->rows + B - 1u) / B);
    dmem scratch;
    const std::size_t sb_bytes = scratch_for(RB, requested);
    if (!scratch.alloc(sb_bytes, "bucket scratch")) return 0;
    cs_exec_bucket_plan plan{};
    std::vector<seg_rec> rec;
    if (!bell_plan(&sb.view, requested, scratch.p, sb_bytes, &plan, nullptr, &rec, g.s)) return 0;
    if (chosen != nullptr) *chosen = plan.bucket_count;
    if (bytes != nullptr) *bytes = plan.bytes;
    if (plan_only) return 1;
    const uint32_t rows = part->rows, cols = part->cols, S = plan.segment_count;
    dmem d_bci, d_val, d_maps;
    if (!d_bci.alloc(plan.index_entries * 4u, "segment idx") || !d_val.alloc(plan.value_entries * 2u, "segment val") ||
        !d_maps.alloc(((std::size_t) rows * 2u + (std::size_t) cols * 2u) * 4u, "maps"))
        return 0;
    uint32_t *maps = (uint32_t *) d_maps.p;
    if (!bell_fill(&sb.view, scratch.p, &plan, (uint32_t *) d_bci.p, (uint16_t *) d_val.p, maps, maps + rows,
                   maps + 2u * (std::size_t) rows, maps + 2u * (std::size_t) rows + cols, g.s))
        return 0;
    out->rows = rows;
    out->cols = cols;
    out->nnz = part->nnz;
    out->segment_count = S;
    out->segments = S != 0u ? (cs_host_blocked_ell *) std::calloc(S, sizeof(cs_host_blocked_ell)) : nullptr;
    out->segment_row_offsets = host_u32((std::size_t) S + 1u);
    out->exec_to_canonical_rows = host_u32(rows);
    out->canonical_to_exec_rows = host_u32(rows);
    out->exec_to_canonical_cols = host_u32(cols);
    out->canonical_to_exec_cols = host_u32(cols);
    bool ok = (S == 0u || out->segments != nullptr) && out->segment_row_offsets != nullptr &&
              (rows == 0u || (out->exec_to_canonical_rows != nullptr && out->canonical_to_exec_rows != nullptr)) &&
              (cols == 0u || (out->exec_to_canonical_cols != nullptr && out->canonical_to_exec_cols != nullptr));
    for (uint32_t s = 0; ok && s < S; ++s) {
        cs_host_blocked_ell *m = out->segments + s;
        m->rows = rec[s + 1u].row_off - rec[s].row_off;
        m->cols = cols;
        m->nnz = (uint32_t) rec[s].nnz;
        m->block_size = B;
        m->ell_cols = rec[s].width * B;
        ok = host_blocked_ell_allocate(m) != 0;
        const std::size_t ni = rec[s + 1u].idx_off - rec[s].idx_off, nv = rec[s + 1u].val_off - rec[s].val_off;
        ok = ok && (ni == 0u || cuda_ok(cudaMemcpyAsync(m->blockColIdx, (uint32_t *) d_bci.p + rec[s].idx_off, ni * 4u,
                                                        cudaMemcpyDeviceToHost, g.s), "D2H segment idx"));
        ok = ok && (nv == 0u || cuda_ok(cudaMemcpyAsync(m->val, (uint16_t *) d_val.p + rec[s].val_off, nv * 2u,
                                                        cudaMemcpyDeviceToHost, g.s), "D2H segment val"));
    }
    if (ok) {
        for (uint32_t s = 0; s <= S; ++s) out->segment_row_offsets[s] = rec[s].row_off;
        ok = (rows == 0u ||
              (cuda_ok(cudaMemcpyAsync(out->exec_to_canonical_rows, maps, (std::size_t) rows * 4u,
                                       cudaMemcpyDeviceToHost, g.s), "D2H maps") &&
               cuda_ok(cudaMemcpyAsync(out->canonical_to_exec_rows, maps + rows, (std::size_t) rows * 4u,
                                       cudaMemcpyDeviceToHost, g.s), "D2H maps"))) &&
             (cols == 0u ||
              (cuda_ok(cudaMemcpyAsync(out->exec_to_canonical_cols, maps + 2u * (std::size_t) rows,
                                       (std::size_t) cols * 4u, cudaMemcpyDeviceToHost, g.s), "D2H col maps") &&
               cuda_ok(cudaMemcpyAsync(out->canonical_to_exec_cols, maps + 2u * (std::size_t) rows + cols,
                                       (std::size_t) cols * 4u, cudaMemcpyDeviceToHost, g.s), "D2H col maps"))) &&
             cuda_ok(cudaStreamSynchronize(g.s), "sync bucketed");
    }
    if (!ok) {
        set_error("build_bucketed_blocked_ell_partition: host allocation or copy failed");
        cs_b200_host_bucketed_blocked_ell_clear(out);
        return 0;
    }
    return 1;
}

int host_sell_bucketed(cs_host_bucketed_sliced_ell *out, const cs_host_sliced_ell *part, uint32_t requested,
                       uint64_t *bytes, uint32_t *chosen, bool plan_only) {
    if (out == nullptr || part == nullptr) {
        set_error("build_bucketed_sliced_ell_partition: null argument");
        return 0;
    }
    std::memset(out, 0, sizeof(*out));
    const uint32_t rows = part->rows, S_src = part->slice_count;
    // slot offsets of the source slices (slice_slot_base, sliced_ell.cuh:70-78)
    std::vector<uint32_t> slot_offs(S_src);
    uint64_t total = 0u;
    for (uint32_t s = 0; s < S_src; ++s) {
        slot_offs[s] = (uint32_t) total;
        total += (uint64_t) (part->slice_row_offsets[s + 1u] - part->slice_row_offsets[s]) * part->slice_widths[s];
    }
    if (total > 0xffffffffull) {
        set_error("build_bucketed_sliced_ell_partition: %llu slots overflow the u32 slot index",
                  (unsigned long long) total);
        return 0;
    }
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    dmem d_offs, d_w, d_slots, d_col, d_val;
    if (!d_offs.alloc(((std::size_t) S_src + 1u) * 4u, "slice offsets") || !d_w.alloc((std::size_t) S_src * 4u, "widths") ||
        !d_slots.alloc((std::size_t) S_src * 4u, "slot offsets") || !d_col.alloc(total * 4u, "col") ||
        !d_val.alloc(total * 2u, "val"))
        return 0;
    bool ok = cuda_ok(cudaMemcpyAsync(d_offs.p, part->slice_row_offsets, ((std::size_t) S_src + 1u) * 4u,
                                      cudaMemcpyHostToDevice, g.s), "H2D offsets") &&
              (S_src == 0u ||
               (cuda_ok(cudaMemcpyAsync(d_w.p, part->slice_widths, (std::size_t) S_src * 4u, cudaMemcpyHostToDevice,
                                        g.s), "H2D widths") &&
                cuda_ok(cudaMemcpyAsync(d_slots.p, slot_offs.data(), (std::size_t) S_src * 4u, cudaMemcpyHostToDevice,
                                        g.s), "H2D slot offsets"))) &&
              (total == 0u ||
               (cuda_ok(cudaMemcpyAsync(d_col.p, part->col_idx, total * 4u, cudaMemcpyHostToDevice, g.s), "H2D col") &&
                cuda_ok(cudaMemcpyAsync(d_val.p, part->val, total * 2u, cudaMemcpyHostToDevice, g.s), "H2D val")));
    if (!ok) return 0;
    const cs_sliced_ell_view v{rows, part->cols, part->nnz, S_src, 0u, (uint32_t *) d_offs.p, (uint32_t *) d_w.p,
                               (uint32_t *) d_slots.p, (uint32_t *) d_col.p, (uint16_t *) d_val.p};
    dmem scratch;
    const std::size_t sb_bytes = scratch_for(rows, requested);
    if (!scratch.alloc(sb_bytes, "bucket scratch")) return 0;
    cs_exec_bucket_plan plan{};
    std::vector<seg_rec> rec;
    if (!sell_plan(&v, requested, scratch.p, sb_bytes, &plan, nullptr, &rec, g.s)) return 0;
    if (chosen != nullptr) *chosen = plan.bucket_count;
    if (bytes != nullptr) *bytes = plan.bytes;
    if (plan_only) return 1;
    const uint32_t S = plan.segment_count;
    dmem o_col, o_val, d_maps;
    if (!o_col.alloc(plan.index_entries * 4u, "segment col") || !o_val.alloc(plan.value_entries * 2u, "segment val") ||
        !d_maps.alloc((std::size_t) rows * 8u, "row maps"))
        return 0;
    uint32_t *maps = (uint32_t *) d_maps.p;
    if (!sell_fill(&v, scratch.p, &plan, (uint32_t *) o_col.p, (uint16_t *) o_val.p, maps, maps + rows, g.s)) return 0;
    out->rows = rows;
    out->cols = part->cols;
    out->nnz = part->nnz;
    out->segment_count = S;
    out->segments = S != 0u ? (cs_host_sliced_ell *) std::calloc(S, sizeof(cs_host_sliced_ell)) : nullptr;
    out->segment_row_offsets = host_u32((std::size_t) S + 1u);
    out->exec_to_canonical_rows = host_u32(rows);
    out->canonical_to_exec_rows = host_u32(rows);
    out->canonical_slice_count = S_src;
    out->canonical_slice_row_offsets = host_u32((std::size_t) S_src + 1u);
    out->canonical_slice_widths = host_u32(S_src);
    ok = (S == 0u || out->segments != nullptr) && out->segment_row_offsets != nullptr &&
         out->canonical_slice_row_offsets != nullptr && (S_src == 0u || out->canonical_slice_widths != nullptr) &&
         (rows == 0u || (out->exec_to_canonical_rows != nullptr && out->canonical_to_exec_rows != nullptr));
    for (uint32_t s = 0; ok && s < S; ++s) {
        cs_host_sliced_ell *m = out->segments + s;
        const uint32_t n = rec[s + 1u].unit_off - rec[s].unit_off;
        const uint64_t slots = (uint64_t) n * rec[s].width;
        ok = host_sliced_alloc(m, n, part->cols, (uint32_t) rec[s].nnz, n != 0u ? 1u : 0u, slots) != 0;
        if (!ok) break;
        m->slice_row_offsets[0] = 0u;
        if (n != 0u) {
            m->slice_row_offsets[1] = n;
            m->slice_widths[0] = rec[s].width;
        }
        ok = slots == 0u ||
             (cuda_ok(cudaMemcpyAsync(m->col_idx, (uint32_t *) o_col.p + rec[s].idx_off, slots * 4u,
                                      cudaMemcpyDeviceToHost, g.s), "D2H segment col") &&
              cuda_ok(cudaMemcpyAsync(m->val, (uint16_t *) o_val.p + rec[s].val_off, slots * 2u, cudaMemcpyDeviceToHost,
                                      g.s), "D2H segment val"));
    }
    if (ok) {
        for (uint32_t s = 0; s <= S; ++s) out->segment_row_offsets[s] = rec[s].row_off;
        std::memcpy(out->canonical_slice_row_offsets, part->slice_row_offsets, ((std::size_t) S_src + 1u) * 4u);
        if (S_src != 0u) std::memcpy(out->canonical_slice_widths, part->slice_widths, (std::size_t) S_src * 4u);
        ok = (rows == 0u ||
              (cuda_ok(cudaMemcpyAsync(out->exec_to_canonical_rows, maps, (std::size_t) rows * 4u,
                                       cudaMemcpyDeviceToHost, g.s), "D2H maps") &&
               cuda_ok(cudaMemcpyAsync(out->canonical_to_exec_rows, maps + rows, (std::size_t) rows * 4u,
                                       cudaMemcpyDeviceToHost, g.s), "D2H maps"))) &&
             cuda_ok(cudaStreamSynchronize(g.s), "sync bucketed");
    }
    if (!ok) {
        set_error("build_bucketed_sliced_ell_partition: host allocation or copy failed");
        cs_b200_host_bucketed_sliced_ell_clear(out);
        return 0;
    }
    return 1;
}

} // namespace

extern "C" int cs_b200_build_bucketed_blocked_ell_partition(cs_host_bucketed_blocked_ell *out,
                                                            const cs_host_blocked_ell *part,
                                                            uint32_t requested_bucket_count,
                                                            uint64_t *bucketed_bytes_out) {
    // a request of 0 behaves as 1 (max(1, min(requested, row blocks)))
    return host_bell_bucketed(out, part, requested_bucket_count == 0u ? 1u : requested_bucket_count,
                              bucketed_bytes_out, nullptr, false);
}

extern "C" int cs_b200_choose_bucket_count_for_part(const cs_host_blocked_ell *part, uint32_t *bucket_count_out,
                                                    uint64_t *bucketed_bytes_out) {
    if (bucket_count_out == nullptr || bucketed_bytes_out == nullptr) {
        set_error("choose_bucket_count_for_part: null output");
        return 0;
    }
    cs_host_bucketed_blocked_ell tmp;
    const int ok = host_bell_bucketed(&tmp, part, 0u, bucketed_bytes_out, bucket_count_out, true);
    cs_b200_host_bucketed_blocked_ell_clear(&tmp);
    return ok;
}

extern "C" int cs_b200_build_bucketed_sliced_ell_partition(cs_host_bucketed_sliced_ell *out,
                                                           const cs_host_sliced_ell *part,
                                                           uint32_t requested_bucket_count,
                                                           uint64_t *bucketed_bytes_out) {
    return host_sell_bucketed(out, part, requested_bucket_count == 0u ? 1u : requested_bucket_count,
                              bucketed_bytes_out, nullptr, false);
}

extern "C" int cs_b200_choose_bucket_count_for_sliced_part(const cs_host_sliced_ell *part,
                                                           uint32_t *bucket_count_out,
                                                           uint64_t *bucketed_bytes_out) {
    if (bucket_count_out == nullptr || bucketed_bytes_out == nullptr) {
        set_error("choose_bucket_count_for_sliced_part: null output");
        return 0;
    }
    cs_host_bucketed_sliced_ell tmp;
    const int ok = host_sell_bucketed(&tmp, part, 0u, bucketed_bytes_out, bucket_count_out, true);
    cs_b200_host_bucketed_sliced_ell_clear(&tmp);
    return ok;
}
