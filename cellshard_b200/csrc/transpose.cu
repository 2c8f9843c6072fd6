// Stable compressed transpose: CSR (cDim x uDim) -> CSC, row indices ascending
// inside every column -- the result of cusparseCsr2cscEx2 (ALG1), which the
// reference's build_compressed_transpose_raw uses as its primary path
// (src/convert/compressed_transpose_raw.cuh:43-81).  Its atomic fallback
// (:84-121) is order-nondeterministic and is not reproduced.
//
//   hist     rows are cut into T tiles; each CTA counts its tile's entries
//            per column in shared memory -> H[t][c].
//   colscan  per column, exclusive scan of H over tiles (in place) and the
//            column total; one device scan of the totals gives out_ptr.
//   scatter  each CTA replays its tile 16 rows at a time.  Round A sets, per
//            column, a 16-bit mask of which batch rows hold it (atomicOr in a
//            packed shared word: mask << 16 | running count); round B places
//            entry (r, c) at out_ptr[c] + H[t][c] + count + popc(mask below r);
//            round C advances the count.  Placement is therefore fixed by
//            (tile, row) order alone -- deterministic and stable.
// The one-pass path below is used only where the two-pass path (further down,
// the default) does not apply.  On the one-pass path a row that repeats a
// column sets CS_STATUS_DUPLICATE_COL in the status word at the start of the
// caller's scratch; the two-pass path keeps repeated entries, in row order.
#include "common.cuh"

namespace csb {
namespace {

constexpr unsigned kThreads = 512;
constexpr unsigned kBatchRows = 16;
constexpr uint32_t kColRange = 32768; // columns per shared-memory pass (128 KB)
constexpr uint32_t kMaxTileRows = 65535;

struct tr_layout {
    uint32_t *status;
    uint32_t *hist; // [tiles * uDim]
    void *scan_tmp;
    std::size_t scan_bytes;
    std::size_t bytes;
    uint32_t tiles, tile_rows, passes;
};

void make_layout(uint32_t cDim, uint32_t uDim, void *base, std::size_t cap, tr_layout *l) {
    const uint32_t sms = (uint32_t) sm_count();
    uint32_t tiles = cDim == 0u ? 1u : (cDim + 15u) / 16u;
    if (tiles > 2u * sms) tiles = 2u * sms;
    const uint32_t min_tiles = cDim == 0u ? 1u : (cDim + kMaxTileRows - 1u) / kMaxTileRows;
    if (tiles < min_tiles) tiles = min_tiles;
    if (tiles == 0u) tiles = 1u;
    l->tiles = tiles;
    l->tile_rows = cDim == 0u ? 0u : (cDim + tiles - 1u) / tiles;
    l->passes = uDim == 0u ? 0u : (uDim + kColRange - 1u) / kColRange;
    scratch_carver c(base, cap);
    l->status = c.take<uint32_t>(4);
    l->hist = c.take<uint32_t>((std::size_t) tiles * uDim + 1u);
    l->scan_bytes = scan_u32_scratch_bytes(uDim);
    l->scan_tmp = c.take<char>(l->scan_bytes);
    l->bytes = c.used;
}

__global__ void __launch_bounds__(kThreads) tr_hist_kernel(const uint32_t *__restrict__ ptr,
                                                          const uint32_t *__restrict__ idx, uint32_t cDim,
                                                          uint32_t uDim, uint32_t tile_rows,
                                                          uint32_t *__restrict__ hist, uint32_t *status) {
    extern __shared__ uint32_t tr_counts[];
    const uint32_t t = blockIdx.x;
    const uint32_t c0 = blockIdx.y * kColRange;
    const uint32_t cr = min(kColRange, uDim - c0);
    for (uint32_t k = threadIdx.x; k < cr; k += blockDim.x) tr_counts[k] = 0u;
    __syncthreads();
    const uint32_t r0 = t * tile_rows;
    const uint32_t r1 = min(cDim, r0 + tile_rows);
    uint32_t bad = 0u;
    if (r0 < r1) {
        const uint32_t a = ptr[r0], e = ptr[r1];
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c >= uDim) {
                bad |= CS_STATUS_INDEX_RANGE;
                continue;
            }
            if (c - c0 < cr) atomicAdd(tr_counts + (c - c0), 1u);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cr; k += blockDim.x) hist[(std::size_t) t * uDim + c0 + k] = tr_counts[k];
    if (bad) status_or(status, bad);
}

__global__ void __launch_bounds__(256) tr_colscan_kernel(uint32_t uDim, uint32_t tiles, uint32_t *__restrict__ hist,
                                                         uint32_t *__restrict__ totals) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= uDim) return;
    uint32_t run = 0u;
    for (uint32_t t = 0; t < tiles; ++t) {
        const std::size_t k = (std::size_t) t * uDim + c;
        const uint32_t v = hist[k];
        hist[k] = run;
        run += v;
    }
    totals[c] = run;
}

__global__ void __launch_bounds__(kThreads) tr_scatter_kernel(const uint32_t *__restrict__ ptr,
                                                             const uint32_t *__restrict__ idx,
                                                             const uint16_t *__restrict__ val, uint32_t cDim,
                                                             uint32_t uDim, uint32_t tile_rows,
                                                             const uint32_t *__restrict__ hist,
                                                             const uint32_t *__restrict__ out_ptr,
                                                             uint32_t *__restrict__ out_idx,
                                                             uint16_t *__restrict__ out_val, uint32_t *status) {
    extern __shared__ uint32_t tr_packed[]; // (mask << 16) | count per column of the pass
    __shared__ uint32_t rp[kBatchRows + 1];
    const uint32_t t = blockIdx.x;
    const uint32_t c0 = blockIdx.y * kColRange;
    const uint32_t cr = min(kColRange, uDim - c0);
    for (uint32_t k = threadIdx.x; k < cr; k += blockDim.x) tr_packed[k] = 0u;
    const uint32_t r0 = t * tile_rows;
    const uint32_t r1 = min(cDim, r0 + tile_rows);
    const uint32_t *hrow = hist + (std::size_t) t * uDim;
    uint32_t bad = 0u;
    for (uint32_t b0 = r0; b0 < r1; b0 += kBatchRows) {
        const uint32_t nb = min(kBatchRows, r1 - b0);
        __syncthreads();
        if (threadIdx.x <= nb) rp[threadIdx.x] = ptr[b0 + threadIdx.x];
        __syncthreads();
        const uint32_t a = rp[0], e = rp[nb];
        // round A: which batch rows hold each column
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c - c0 >= cr || c >= uDim) continue;
            uint32_t rl = 0u;
            while (rl + 1u < nb && rp[rl + 1u] <= i) ++rl;
            const uint32_t bit = 1u << (16u + rl);
            if (atomicOr(tr_packed + (c - c0), bit) & bit) bad |= CS_STATUS_DUPLICATE_COL;
        }
        __syncthreads();
        // round B: place
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c - c0 >= cr || c >= uDim) continue;
            uint32_t rl = 0u;
            while (rl + 1u < nb && rp[rl + 1u] <= i) ++rl;
            const uint32_t w = tr_packed[c - c0];
            const uint32_t mask = w >> 16;
            const uint32_t rank = (w & 0xffffu) + __popc(mask & ((1u << rl) - 1u));
            const uint32_t pos = out_ptr[c] + hrow[c] + rank;
            out_idx[pos] = b0 + rl;
            out_val[pos] = val[i];
        }
        __syncthreads();
        // round C: advance the per-column count, clear the mask
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c - c0 >= cr || c >= uDim) continue;
            uint32_t rl = 0u;
            while (rl + 1u < nb && rp[rl + 1u] <= i) ++rl;
            const uint32_t w = tr_packed[c - c0];
            const uint32_t mask = w >> 16;
            if (rl == (uint32_t) (__ffs(mask) - 1)) tr_packed[c - c0] = ((w & 0xffffu) + __popc(mask)) & 0xffffu;
        }
    }
    if (bad) status_or(status, bad);
}


// ---------------------------------------------------------------------------
// Two-pass stable transpose (default path).
//
// The one-pass scatter above appends to every column segment from every CTA
// at once; at 32,768 columns that leaves hundreds of MB of partially written
// sectors open, far beyond L2.  Here the column key is sorted in two stable
// counting-sort passes whose open write frontier is small:
//   pass 1  by bucket = column >> 8 (<= 1,024 buckets), tiles of 8,192
//           consecutive entries; entries become packed keys
//           (row << 8 | column & 255) + values.
//   pass 2  inside each bucket by column & 255, in chunks of <= 8,192 that
//           never cross a bucket, writing straight into the CSC.
// Each tile or chunk is reordered whole in shared memory and leaves as one
// run per digit, so global writes are long runs, not scattered entries.
// Both passes rank entries in input order (warp match on the digit plus
// per-warp running counts), so the result is the stable transpose.
// Needs cDim < 2^24 and uDim <= 262,144.
// ---------------------------------------------------------------------------
constexpr unsigned kTpThreads = 256;
constexpr unsigned kTpWarps = kTpThreads / 32;
constexpr uint32_t kTpBucketBits = 8;
constexpr uint32_t kTpMaxBuckets = 1024;
constexpr uint32_t kTpTile1 = 8192;  // entries per pass-1 tile (staged whole in shared memory)
constexpr uint32_t kTpChunk = 8192;  // entries per pass-2 chunk (staged whole in shared memory)
constexpr uint32_t kTpGran = 256;    // entries per warp per step; rows are looked up per granule

struct tp2_layout {
    uint32_t *status;
    uint32_t *hist1;       // [K * tiles1 + 1], bucket-major
    uint32_t *tmp_key;     // [nnz]
    uint16_t *tmp_val;     // [nnz]
    uint32_t *chunk_bucket; // [max_chunks]
    uint32_t *chunk_begin;  // [max_chunks]
    uint32_t *chunk_end;    // [max_chunks]
    uint32_t *chunk_first;  // [K + 1]
    uint32_t *gran_row;     // [nnz / kTpGran + 1] row holding entry j * kTpGran
    uint32_t *hist2;        // [256 * max_chunks + 1], digit-major
    void *scan_tmp;
    std::size_t scan_bytes, bytes;
    uint32_t K, tiles1, max_chunks;
};

bool tp2_applicable(uint32_t cDim, uint32_t uDim) {
    return cDim < (1u << 24) && uDim <= kTpMaxBuckets * 256u;
}

void tp2_make_layout(uint32_t cDim, uint32_t uDim, uint32_t nnz, void *base, std::size_t cap, tp2_layout *l) {
    l->K = (uDim + 255u) >> kTpBucketBits;
    if (l->K == 0u) l->K = 1u;
    l->tiles1 = nnz == 0u ? 1u : (uint32_t) (((std::size_t) nnz + kTpTile1 - 1u) / kTpTile1);
    l->max_chunks = nnz / kTpChunk + l->K + 1u;
    scratch_carver c(base, cap);
    l->status = c.take<uint32_t>(4);
    l->hist1 = c.take<uint32_t>((std::size_t) l->K * l->tiles1 + 1u);
    l->tmp_key = c.take<uint32_t>((std::size_t) nnz + 1u);
    l->tmp_val = c.take<uint16_t>((std::size_t) nnz + 8u);
    l->gran_row = c.take<uint32_t>((std::size_t) nnz / kTpGran + 1u);
    l->chunk_bucket = c.take<uint32_t>(l->max_chunks);
    l->chunk_begin = c.take<uint32_t>(l->max_chunks);
    l->chunk_end = c.take<uint32_t>(l->max_chunks);
    l->chunk_first = c.take<uint32_t>((std::size_t) l->K + 1u);
    l->hist2 = c.take<uint32_t>((std::size_t) 256u * l->max_chunks + 1u);
    std::size_t sb = scan_u32_scratch_bytes((std::size_t) l->K * l->tiles1);
    const std::size_t sb2 = scan_u32_scratch_bytes((std::size_t) 256u * l->max_chunks);
    const std::size_t sb3 = scan_u32_scratch_bytes(uDim);
    if (sb2 > sb) sb = sb2;
    if (sb3 > sb) sb = sb3;
    l->scan_bytes = sb;
    l->scan_tmp = c.take<char>(sb);
    l->bytes = c.used;
}

// gran_row[j] = the row holding entry j * kTpGran (rows own the granules that
// start inside them).
__global__ void __launch_bounds__(256) tp_gran_rows_kernel(const uint32_t *__restrict__ ptr, uint32_t cDim,
                                                          uint32_t *__restrict__ gran_row) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cDim) return;
    const uint32_t lo = ptr[r], hi = ptr[r + 1u];
    for (std::size_t j = ((std::size_t) lo + kTpGran - 1u) / kTpGran; j * kTpGran < hi; ++j) gran_row[j] = r;
}

// Pass-1 histogram: tile t is entries [t * kTpTile1, (t + 1) * kTpTile1).
__global__ void __launch_bounds__(kTpThreads) tp_hist1_kernel(const uint32_t *__restrict__ idx, uint32_t nnz,
                                                             uint32_t uDim, uint32_t K, uint32_t tiles1,
                                                             uint32_t *__restrict__ hist1, uint32_t *status) {
    extern __shared__ uint32_t tp_h[];
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) tp_h[k] = 0u;
    __syncthreads();
    const uint32_t a = blockIdx.x * kTpTile1, e = min(nnz, a + kTpTile1);
    uint32_t bad = 0u;
    constexpr unsigned U = 4;
    for (uint32_t i0 = a; i0 < e; i0 += U * blockDim.x) {
        uint32_t c[U];
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * blockDim.x + threadIdx.x;
            c[u] = i < e ? __ldg(idx + i) : uDim;
        }
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            if (c[u] < uDim)
                atomicAdd(tp_h + (c[u] >> kTpBucketBits), 1u);
            else if (i0 + u * blockDim.x + threadIdx.x < e)
                bad = CS_STATUS_INDEX_RANGE;
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) hist1[(std::size_t) k * tiles1 + blockIdx.x] = tp_h[k];
    if (bad) status_or(status, bad);
}

// Block-wide exclusive scan of n <= 4 * blockDim.x values in place (each
// thread scans up to 4 consecutive entries); out[n] receives the total.
__device__ __forceinline__ void block_scan_small(uint32_t *v, uint32_t n, uint32_t *smem33) {
    const uint32_t t = threadIdx.x;
    uint32_t loc[4], sum = 0u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t k = t * 4u + q;
        loc[q] = k < n ? v[k] : 0u;
        sum += loc[q];
    }
    uint32_t tot;
    uint32_t run = block_exclusive_scan(sum, smem33, tot);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t k = t * 4u + q;
        if (k < n) v[k] = run;
        run += loc[q];
    }
    if (t == 0) v[n] = tot;
    __syncthreads();
}

constexpr uint32_t kTpSub = 2048;                        // entries counted and placed per step
constexpr unsigned kTpBatches = kTpSub / kTpWarps / 32; // 32-entry batches per warp per step

// lanes of the warp holding the same digit (valid lanes only; 0 if invalid).
// match.any is cheaper than one ballot per digit bit when a batch holds few
// distinct digits (pass 1: consecutive entries of a row share a bucket); with
// ~30 distinct digits per batch (pass 2) the ballots win.
__device__ __forceinline__ uint32_t tp_peers(uint32_t d, bool valid) {
    const uint32_t m = __match_any_sync(0xffffffffu, valid ? d : 0xffffffffu);
    return valid ? m : 0u;
}

// last major r in [0, cDim) with ptr[r] <= i
__device__ __forceinline__ uint32_t major_of(const uint32_t *__restrict__ ptr, uint32_t cDim, uint32_t i) {
    uint32_t lo = 0u, hi = cDim - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (__ldg(ptr + mid) <= i)
            lo = mid;
        else
            hi = mid - 1u;
    }
    return lo;
}

// Stable in-CTA reorder shared by both passes.  The tile's per-digit counts
// are known up front (from the pass's histogram), so `lb` holds each digit's
// first staging slot.  Each step of kTpSub entries gives every warp
// kTpBatches batches of 32 held in registers: the warp counts them per digit
// (peer masks from warp_match_digit), the CTA turns the per-warp counts into
// staging slots (digit base + entries already placed + earlier warps), and
// the warp places its entries in order.  Counters are u16: one warp places at
// most kTpSub / kTpWarps entries per step and the stage holds <= 65535.
struct tp_stage {
    uint16_t *cnt;  // [kTpWarps][D]
    uint16_t *bas;  // [kTpWarps][D]
    uint32_t *lb;   // [D + 1]
    uint32_t *fill; // [D]
};

__device__ __forceinline__ void tp_stage_prefix(const tp_stage &sg, uint32_t D) {
    for (uint32_t d = threadIdx.x; d < D; d += blockDim.x) {
        uint32_t t = sg.lb[d] + sg.fill[d];
        const uint32_t t0 = t;
#pragma unroll
        for (unsigned w = 0; w < kTpWarps; ++w) {
            const uint32_t c = sg.cnt[w * D + d];
            sg.cnt[w * D + d] = 0u;
            sg.bas[w * D + d] = (uint16_t) t;
            t += c;
        }
        sg.fill[d] += t - t0;
    }
}

// Pass 1: tile t = entries [t * kTpTile1, ...) of the CSR, reordered by
// bucket (column >> 8) in shared memory, stable, then written out as one run
// per bucket.  Keys are (row << 8 | column & 255).
__global__ void __launch_bounds__(kTpThreads) tp_scatter1_kernel(const uint32_t *__restrict__ ptr,
                                                                const uint32_t *__restrict__ idx,
                                                                const uint16_t *__restrict__ val, uint32_t cDim,
                                                                uint32_t uDim, uint32_t nnz, uint32_t K,
                                                                uint32_t tiles1, const uint32_t *__restrict__ hist1,
                                                                const uint32_t *__restrict__ gran_row,
                                                                uint32_t *__restrict__ tmp_key,
                                                                uint16_t *__restrict__ tmp_val) {
    extern __shared__ __align__(16) uint32_t tp_s[];
    __shared__ uint32_t scan33[33];
    // staged entry: key | value << 32 | bucket << 48
    unsigned long long *st = reinterpret_cast<unsigned long long *>(tp_s); // [kTpTile1]
    uint32_t *run = reinterpret_cast<uint32_t *>(st + kTpTile1);           // [K] global base per bucket
    tp_stage sg;
    sg.lb = run + K;                                                       // [K + 1]
    sg.fill = sg.lb + K + 1u;                                              // [K]
    sg.cnt = reinterpret_cast<uint16_t *>(sg.fill + K);                    // [kTpWarps][K]
    sg.bas = sg.cnt + kTpWarps * K;                                        // [kTpWarps][K]
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t a = blockIdx.x * kTpTile1, e = min(nnz, a + kTpTile1);
    if (a >= e) return;
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
        const uint32_t h = hist1[(std::size_t) k * tiles1 + blockIdx.x];
        run[k] = h;
        sg.lb[k] = hist1[(std::size_t) k * tiles1 + blockIdx.x + 1u] - h;
        sg.fill[k] = 0u;
    }
    for (uint32_t k = threadIdx.x; k < kTpWarps * K; k += blockDim.x) sg.cnt[k] = 0u;
    __syncthreads();
    block_scan_small(sg.lb, K, scan33);
    const unsigned lt = (1u << lane) - 1u;
    uint16_t *my_cnt = sg.cnt + warp * K;
    uint16_t *my_bas = sg.bas + warp * K;
    static_assert(kTpSub / kTpWarps == kTpGran, "a warp's step range is one row granule");
    uint32_t ncc[kTpBatches], nrc;
    uint16_t nvv[kTpBatches];
    auto fetch = [&](uint32_t sc) {
        const uint32_t n = min(kTpSub, e - sc);
        const uint32_t wa = sc + min(n, warp * kTpGran), we = sc + min(n, (warp + 1u) * kTpGran);
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            const uint32_t i = wa + q * 32u + lane;
            const bool in = i < we;
            ncc[q] = in ? __ldg(idx + i) : uDim;
            nvv[q] = in ? __ldg(reinterpret_cast<const unsigned short *>(val) + i) : (uint16_t) 0u;
        }
        nrc = wa < we ? min(__ldg(gran_row + wa / kTpGran), cDim - 1u) : 0u;
    };
    fetch(a);
    for (uint32_t sc0 = a; sc0 < e; sc0 += kTpSub) {
        const uint32_t n = min(kTpSub, e - sc0);
        const uint32_t wa = sc0 + min(n, warp * kTpGran);
        const uint32_t we = sc0 + min(n, (warp + 1u) * kTpGran);
        uint32_t cc[kTpBatches], pk[kTpBatches], rl[kTpBatches];
        uint16_t vv[kTpBatches];
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            cc[q] = ncc[q];
            vv[q] = nvv[q];
        }
        uint32_t r_cur = nrc;
        if (sc0 + kTpSub < e) fetch(sc0 + kTpSub);
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            const uint32_t i = wa + q * 32u + lane;
            const bool in = i < we;
            // row of entry i: walk forward from the warp's current row; a
            // batch that spans many short rows finishes by binary search
            uint32_t r = r_cur;
            for (unsigned step = 0;; ++step) {
                const bool adv = in && r + 1u < cDim && __ldg(ptr + r + 1u) <= i;
                if (!__any_sync(0xffffffffu, adv)) break;
                if (step == 3u) {
                    if (adv) {
                        const uint32_t lo = r + 1u;
                        r = lo + major_of(ptr + lo, cDim - lo, i);
                    }
                    break;
                }
                r += adv ? 1u : 0u;
            }
            rl[q] = r;
            r_cur = __shfl_sync(0xffffffffu, r, 31);
            const bool ok = cc[q] < uDim;
            const uint32_t k = cc[q] >> kTpBucketBits;
            pk[q] = tp_peers(k, ok);
            if (ok && lane == (unsigned) (__ffs(pk[q]) - 1)) my_cnt[k] += (uint16_t) __popc(pk[q]);
            __syncwarp();
        }
        __syncthreads();
        tp_stage_prefix(sg, K);
        __syncthreads();
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            const bool ok = cc[q] < uDim;
            const uint32_t k = cc[q] >> kTpBucketBits;
            uint32_t lp = 0u;
            if (ok) lp = my_bas[k] + __popc(pk[q] & lt);
            __syncwarp();
            if (ok) {
                if (lp < kTpTile1)
                    st[lp] = (unsigned long long) ((rl[q] << kTpBucketBits) | (cc[q] & 255u)) |
                             ((unsigned long long) vv[q] << 32) | ((unsigned long long) k << 48);
                if (lane == (unsigned) (__ffs(pk[q]) - 1)) my_bas[k] += (uint16_t) __popc(pk[q]);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    const uint32_t placed = min(sg.lb[K], kTpTile1);
    // run[k] - lb[k]: the global slot of staging slot 0 for bucket k
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) run[k] -= sg.lb[k];
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < placed; j += blockDim.x) {
        const unsigned long long v = st[j];
        const uint32_t g = run[(uint32_t) (v >> 48)] + j;
        tmp_key[g] = (uint32_t) v;
        tmp_val[g] = (uint16_t) (v >> 32);
    }
}

std::size_t tp_scatter1_smem(uint32_t K) {
    return (std::size_t) kTpTile1 * 8u + ((std::size_t) 3u * K + 1u) * 4u + (std::size_t) 2u * kTpWarps * K * 2u;
}

// one CTA: cut every bucket's entry range into chunks of <= kTpChunk entries
__global__ void __launch_bounds__(1024) tp_chunks_kernel(const uint32_t *__restrict__ hist1, uint32_t tiles1,
                                                         uint32_t K, uint32_t max_chunks,
                                                         uint32_t *__restrict__ chunk_bucket,
                                                         uint32_t *__restrict__ chunk_begin,
                                                         uint32_t *__restrict__ chunk_end,
                                                         uint32_t *__restrict__ chunk_first) {
    __shared__ uint32_t smem[33];
    const uint32_t total = hist1[(std::size_t) K * tiles1];
    uint32_t carry = 0u;
    for (uint32_t k0 = 0; k0 < K; k0 += blockDim.x) {
        const uint32_t k = k0 + threadIdx.x;
        uint32_t b = 0u, n = 0u, nc = 0u;
        if (k < K) {
            b = hist1[(std::size_t) k * tiles1];
            const uint32_t e = k + 1u < K ? hist1[(std::size_t) (k + 1u) * tiles1] : total;
            n = e - b;
            nc = (n + kTpChunk - 1u) / kTpChunk;
        }
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(nc, smem, tot);
        if (k < K) {
            chunk_first[k] = carry + ex;
            for (uint32_t j = 0; j < nc; ++j) {
                const uint32_t id = carry + ex + j;
                if (id < max_chunks) {
                    chunk_bucket[id] = k;
                    chunk_begin[id] = b + j * kTpChunk;
                    chunk_end[id] = min(b + n, b + (j + 1u) * kTpChunk);
                }
            }
        }
        carry += tot;
    }
    if (threadIdx.x == 0) chunk_first[K] = carry;
    // unused chunk slots carry empty ranges so their histograms are zero
    for (uint32_t id = carry + threadIdx.x; id < max_chunks; id += blockDim.x) {
        chunk_bucket[id] = 0u;
        chunk_begin[id] = 0u;
        chunk_end[id] = 0u;
    }
}

__global__ void __launch_bounds__(kTpThreads) tp_hist2_kernel(const uint32_t *__restrict__ tmp_key,
                                                             const uint32_t *__restrict__ chunk_begin,
                                                             const uint32_t *__restrict__ chunk_end,
                                                             uint32_t max_chunks, uint32_t *__restrict__ hist2) {
    __shared__ uint32_t h[kTpWarps][256];
    const unsigned warp = threadIdx.x >> 5;
    for (uint32_t d = threadIdx.x; d < kTpWarps * 256u; d += blockDim.x) (&h[0][0])[d] = 0u;
    __syncthreads();
    const uint32_t b = chunk_begin[blockIdx.x], e = chunk_end[blockIdx.x];
    constexpr unsigned U = 4;
    for (uint32_t i0 = b; i0 < e; i0 += U * blockDim.x) {
        uint32_t kk[U];
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * blockDim.x + threadIdx.x;
            kk[u] = i < e ? __ldg(tmp_key + i) : 0xffffffffu;
        }
#pragma unroll
        for (unsigned u = 0; u < U; ++u)
            if (kk[u] != 0xffffffffu) atomicAdd(&h[warp][kk[u] & 255u], 1u);
    }
    __syncthreads();
    uint32_t t = 0u;
    for (unsigned w = 0; w < kTpWarps; ++w) t += h[w][threadIdx.x];
    hist2[(std::size_t) threadIdx.x * max_chunks + blockIdx.x] = t;
}

// column totals from the digit-major scan: count(k*256+d) = P[d][last] - P[d][first]
__global__ void __launch_bounds__(256) tp_colcount_kernel(const uint32_t *__restrict__ hist2, uint32_t max_chunks,
                                                          const uint32_t *__restrict__ chunk_first, uint32_t uDim,
                                                          uint32_t *__restrict__ counts) {
    const uint32_t k = blockIdx.x, d = threadIdx.x;
    const uint32_t c = k * 256u + d;
    if (c >= uDim) return;
    const uint32_t f = chunk_first[k], l = chunk_first[k + 1u];
    counts[c] = hist2[(std::size_t) d * max_chunks + l] - hist2[(std::size_t) d * max_chunks + f];
}

// Pass 2: a chunk of one bucket reordered by the low column byte in shared
// memory (stable), then written out as one run per column.
__global__ void __launch_bounds__(kTpThreads) tp_scatter2_kernel(const uint32_t *__restrict__ tmp_key,
                                                                const uint16_t *__restrict__ tmp_val,
                                                                const uint32_t *__restrict__ chunk_bucket,
                                                                const uint32_t *__restrict__ chunk_begin,
                                                                const uint32_t *__restrict__ chunk_end,
                                                                const uint32_t *__restrict__ chunk_first,
                                                                uint32_t max_chunks, const uint32_t *__restrict__ hist2,
                                                                const uint32_t *__restrict__ out_ptr, uint32_t uDim,
                                                                uint32_t *__restrict__ out_idx,
                                                                uint16_t *__restrict__ out_val) {
    extern __shared__ __align__(16) uint32_t tp_s2[];
    __shared__ uint32_t gbase[256];
    __shared__ uint32_t lb[257];
    __shared__ uint32_t fill[256];
    __shared__ uint32_t scan33[33];
    uint32_t *st_key = tp_s2;                                              // [kTpChunk]
    uint16_t *st_val = reinterpret_cast<uint16_t *>(st_key + kTpChunk);   // [kTpChunk]
    tp_stage sg;
    sg.cnt = st_val + kTpChunk;                                            // [kTpWarps][256]
    sg.bas = sg.cnt + kTpWarps * 256u;                                     // [kTpWarps][256]
    sg.lb = lb;
    sg.fill = fill;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t b = chunk_begin[blockIdx.x], e = chunk_end[blockIdx.x];
    if (b >= e) return;
    const uint32_t k = chunk_bucket[blockIdx.x];
    const uint32_t f = chunk_first[k];
    {
        const uint32_t d = threadIdx.x; // kTpThreads == 256
        const uint32_t c = k * 256u + d;
        const std::size_t row = (std::size_t) d * max_chunks;
        const uint32_t h = hist2[row + blockIdx.x];
        lb[d] = hist2[row + blockIdx.x + 1u] - h;
        gbase[d] = c < uDim ? out_ptr[c] + h - hist2[row + f] : 0u;
        fill[d] = 0u;
#pragma unroll
        for (unsigned w = 0; w < kTpWarps; ++w) sg.cnt[w * 256u + d] = 0u;
    }
    __syncthreads();
    block_scan_small(lb, 256u, scan33);
    const unsigned lt = (1u << lane) - 1u;
    uint16_t *my_cnt = sg.cnt + warp * 256u;
    uint16_t *my_bas = sg.bas + warp * 256u;
    uint32_t nkk[kTpBatches];
    uint16_t nvv[kTpBatches];
    auto fetch = [&](uint32_t sc) {
        const uint32_t n = min(kTpSub, e - sc);
        const uint32_t wa = sc + min(n, warp * kTpGran), we = sc + min(n, (warp + 1u) * kTpGran);
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            const uint32_t i = wa + q * 32u + lane;
            const bool in = i < we;
            nkk[q] = in ? __ldg(tmp_key + i) : 0u;
            nvv[q] = in ? __ldg(reinterpret_cast<const unsigned short *>(tmp_val) + i) : (uint16_t) 0u;
        }
    };
    fetch(b);
    for (uint32_t sc0 = b; sc0 < e; sc0 += kTpSub) {
        const uint32_t n = min(kTpSub, e - sc0);
        const uint32_t wa = sc0 + min(n, warp * kTpGran);
        const uint32_t we = sc0 + min(n, (warp + 1u) * kTpGran);
        uint32_t kk[kTpBatches], pk[kTpBatches];
        uint16_t vv[kTpBatches];
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            kk[q] = nkk[q];
            vv[q] = nvv[q];
        }
        if (sc0 + kTpSub < e) fetch(sc0 + kTpSub);
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            const bool in = wa + q * 32u + lane < we;
            const uint32_t d = kk[q] & 255u;
            pk[q] = warp_match_digit<8>(d, in);
            if (in && lane == (unsigned) (__ffs(pk[q]) - 1)) my_cnt[d] += (uint16_t) __popc(pk[q]);
            __syncwarp();
        }
        __syncthreads();
        tp_stage_prefix(sg, 256u);
        __syncthreads();
#pragma unroll
        for (unsigned q = 0; q < kTpBatches; ++q) {
            const bool in = wa + q * 32u + lane < we;
            const uint32_t d = kk[q] & 255u;
            uint32_t lp = 0u;
            if (in) lp = my_bas[d] + __popc(pk[q] & lt);
            __syncwarp();
            if (in) {
                if (lp < kTpChunk) {
                    st_key[lp] = kk[q];
                    st_val[lp] = vv[q];
                }
                if (lane == (unsigned) (__ffs(pk[q]) - 1)) my_bas[d] += (uint16_t) __popc(pk[q]);
            }
            __syncwarp();
        }
    }
    gbase[threadIdx.x] -= lb[threadIdx.x]; // global slot of staging slot 0 for digit d
    __syncthreads();
    const uint32_t n = min(e - b, kTpChunk);
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        const uint32_t key = st_key[j];
        const uint32_t g = gbase[key & 255u] + j;
        out_idx[g] = key >> kTpBucketBits;
        out_val[g] = st_val[j];
    }
}

constexpr std::size_t kTpScatter2Smem = (std::size_t) kTpChunk * 6u + (std::size_t) 2u * kTpWarps * 256u * 2u;

int transpose2_launch(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *ptr, const uint32_t *idx,
                      const uint16_t *val, uint32_t *out_ptr, uint32_t *out_idx, uint16_t *out_val,
                      const tp2_layout &l, cudaStream_t stream) {
    const std::size_t h1_smem = (std::size_t) l.K * 4u;
    const std::size_t s1_smem = tp_scatter1_smem(l.K);
    auto s1 = tp_scatter1_kernel;
    if (!cuda_ok(cudaFuncSetAttribute(s1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) s1_smem),
                 "scatter1 smem attribute") ||
        !cuda_ok(cudaFuncSetAttribute(tp_scatter2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) kTpScatter2Smem),
                 "scatter2 smem attribute"))
        return 0;
    tp_gran_rows_kernel<<<(cDim + 255u) / 256u, 256, 0, stream>>>(ptr, cDim, l.gran_row);
    if (!launch_ok("tp_gran_rows_kernel")) return 0;
    tp_hist1_kernel<<<l.tiles1, kTpThreads, h1_smem, stream>>>(idx, nnz, uDim, l.K, l.tiles1, l.hist1, l.status);
    if (!launch_ok("tp_hist1_kernel")) return 0;
    if (!scan_exclusive_u32(l.hist1, l.hist1, (std::size_t) l.K * l.tiles1, true, l.scan_tmp, l.scan_bytes, stream))
        return 0;
    s1<<<l.tiles1, kTpThreads, s1_smem, stream>>>(ptr, idx, val, cDim, uDim, nnz, l.K, l.tiles1, l.hist1,
                                                  l.gran_row, l.tmp_key, l.tmp_val);
    if (!launch_ok("tp_scatter1_kernel")) return 0;
    tp_chunks_kernel<<<1, 1024, 0, stream>>>(l.hist1, l.tiles1, l.K, l.max_chunks, l.chunk_bucket, l.chunk_begin,
                                             l.chunk_end, l.chunk_first);
    if (!launch_ok("tp_chunks_kernel")) return 0;
    tp_hist2_kernel<<<l.max_chunks, kTpThreads, 0, stream>>>(l.tmp_key, l.chunk_begin, l.chunk_end, l.max_chunks,
                                                             l.hist2);
    if (!launch_ok("tp_hist2_kernel")) return 0;
    if (!scan_exclusive_u32(l.hist2, l.hist2, (std::size_t) 256u * l.max_chunks, true, l.scan_tmp, l.scan_bytes,
                            stream))
        return 0;
    tp_colcount_kernel<<<l.K, 256, 0, stream>>>(l.hist2, l.max_chunks, l.chunk_first, uDim, out_ptr);
    if (!launch_ok("tp_colcount_kernel")) return 0;
    if (!scan_exclusive_u32(out_ptr, out_ptr, uDim, true, l.scan_tmp, l.scan_bytes, stream)) return 0;
    tp_scatter2_kernel<<<l.max_chunks, kTpThreads, kTpScatter2Smem, stream>>>(l.tmp_key, l.tmp_val, l.chunk_bucket, l.chunk_begin,
                                                                l.chunk_end, l.chunk_first, l.max_chunks, l.hist2,
                                                                out_ptr, uDim, out_idx, out_val);
    return launch_ok("tp_scatter2_kernel");
}

} // namespace

int transpose_launch(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *ptr, const uint32_t *idx,
                     const uint16_t *val, uint32_t *out_ptr, uint32_t *out_idx, uint16_t *out_val, void *scratch,
                     std::size_t scratch_bytes, cudaStream_t stream) {
    if (tp2_applicable(cDim, uDim)) {
        tp2_layout l2;
        tp2_make_layout(cDim, uDim, nnz, scratch, scratch_bytes, &l2);
        if (scratch == nullptr || l2.bytes > scratch_bytes) {
            set_error("compressed_transpose: scratch %zu < %zu bytes", scratch_bytes, l2.bytes);
            return 0;
        }
        if (!cuda_ok(cudaMemsetAsync(l2.status, 0, 16, stream), "transpose status memset") ||
            !cuda_ok(cudaMemsetAsync(out_ptr, 0, ((std::size_t) uDim + 1u) * 4u, stream), "transpose out_ptr memset"))
            return 0;
        if (nnz == 0u || cDim == 0u || uDim == 0u) return 1;
        return transpose2_launch(cDim, uDim, nnz, ptr, idx, val, out_ptr, out_idx, out_val, l2, stream);
    }
    tr_layout l;
    make_layout(cDim, uDim, scratch, scratch_bytes, &l);
    if (scratch == nullptr || l.bytes > scratch_bytes) {
        set_error("compressed_transpose: scratch %zu < %zu bytes", scratch_bytes, l.bytes);
        return 0;
    }
    if (!cuda_ok(cudaMemsetAsync(l.status, 0, 16, stream), "transpose status memset") ||
        !cuda_ok(cudaMemsetAsync(out_ptr, 0, ((std::size_t) uDim + 1u) * 4u, stream), "transpose out_ptr memset"))
        return 0;
    if (nnz == 0u || cDim == 0u || uDim == 0u) return 1;
    const std::size_t smem = (std::size_t) min(uDim, kColRange) * sizeof(uint32_t);
    if (!cuda_ok(cudaFuncSetAttribute(tr_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "hist smem attribute") ||
        !cuda_ok(cudaFuncSetAttribute(tr_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "scatter smem attribute"))
        return 0;
    dim3 grid(l.tiles, l.passes);
    tr_hist_kernel<<<grid, kThreads, smem, stream>>>(ptr, idx, cDim, uDim, l.tile_rows, l.hist, l.status);
    if (!launch_ok("tr_hist_kernel")) return 0;
    tr_colscan_kernel<<<(uDim + 255u) / 256u, 256, 0, stream>>>(uDim, l.tiles, l.hist, out_ptr);
    if (!launch_ok("tr_colscan_kernel")) return 0;
    if (!scan_exclusive_u32(out_ptr, out_ptr, uDim, true, l.scan_tmp, l.scan_bytes, stream)) return 0;
    tr_scatter_kernel<<<grid, kThreads, smem, stream>>>(ptr, idx, val, cDim, uDim, l.tile_rows, l.hist, out_ptr,
                                                        out_idx, out_val, l.status);
    return launch_ok("tr_scatter_kernel");
}

std::size_t transpose_scratch(uint32_t cDim, uint32_t uDim, uint32_t nnz) {
    if (tp2_applicable(cDim, uDim)) {
        tp2_layout l2;
        tp2_make_layout(cDim, uDim, nnz, nullptr, 0, &l2);
        return l2.bytes;
    }
    tr_layout l;
    make_layout(cDim, uDim, nullptr, 0, &l);
    return l.bytes;
}

// CSC (cols-major) -> CSR (rows-major) into fresh device buffers (used by the
// host conversion wrappers for column-compressed input).
int transpose_csc_to_csr_staged(const cs_compressed_view *src, uint32_t **d_ptr, uint32_t **d_idx, uint16_t **d_val,
                                cudaStream_t stream) {
    const uint32_t cDim = src->cols, uDim = src->rows;
    void *scratch = nullptr;
    const std::size_t sb = transpose_scratch(cDim, uDim, src->nnz);
    if (!cuda_ok(cudaMalloc((void **) d_ptr, ((std::size_t) uDim + 1u) * 4u), "transpose ptr") ||
        !cuda_ok(cudaMalloc((void **) d_idx, (std::size_t) src->nnz * 4u + 16u), "transpose idx") ||
        !cuda_ok(cudaMalloc((void **) d_val, (std::size_t) src->nnz * 2u + 16u), "transpose val") ||
        !cuda_ok(cudaMalloc(&scratch, sb), "transpose scratch"))
        return 0;
    int ok = transpose_launch(cDim, uDim, src->nnz, src->majorPtr, src->minorIdx, src->val, *d_ptr, *d_idx, *d_val,
                              scratch, sb, stream);
    uint32_t status = 0u;
    if (ok)
        ok = cuda_ok(cudaMemcpyAsync(&status, scratch, 4, cudaMemcpyDeviceToHost, stream), "transpose status") &&
             cuda_ok(cudaStreamSynchronize(stream), "transpose sync");
    cudaFree(scratch);
    if (ok && status != 0u) {
        set_error("column-compressed input rejected (status 0x%x)", status);
        ok = 0;
    }
    return ok;
}

} // namespace csb

using namespace csb;

extern "C" int cs_b200_compressed_transpose_scratch_bytes(uint32_t cDim, uint32_t uDim, uint32_t nnz,
                                                          size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("compressed_transpose_scratch_bytes: null output");
        return 0;
    }
    *out_bytes = transpose_scratch(cDim, uDim, nnz);
    return 1;
}

extern "C" int cs_b200_build_compressed_transpose(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *d_cAxPtr,
                                                  const uint32_t *d_uAxIdx, const uint16_t *d_val,
                                                  uint32_t *d_out_uAxPtr, uint32_t *d_heads, uint32_t *d_out_cAxIdx,
                                                  uint16_t *d_out_val, void *d_scan_tmp, size_t scan_bytes,
                                                  cs_stream_t s) {
    (void) d_heads;
    if (d_out_uAxPtr == nullptr || (nnz != 0u && (d_cAxPtr == nullptr || d_uAxIdx == nullptr || d_val == nullptr ||
                                                  d_out_cAxIdx == nullptr || d_out_val == nullptr))) {
        set_error("compressed_transpose: null device array");
        return 0;
    }
    return transpose_launch(cDim, uDim, nnz, d_cAxPtr, d_uAxIdx, d_val, d_out_uAxPtr, d_out_cAxIdx, d_out_val,
                            d_scan_tmp, scan_bytes, as_stream(s));
}
