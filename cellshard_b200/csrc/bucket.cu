// Major-axis nnz bucketing.
//
// Plan (bucket::build_major_nnz_bucket_plan_raw, src/bucket/major_nnz_raw.cuh:64-120):
//   major_nnz[i] = ptr[i+1] - ptr[i]; major_order_in = identity; a stable
//   ascending sort of the counts with row ids as values (the reference runs
//   CUB DeviceRadixSort::SortPairs over all 32 key bits) -> major_nnz_sorted,
//   major_order_out; equal-count bucket offsets where the first n % B buckets
//   take one extra row (fill_equal_count_bucket_offsets.cuh).
//   Here the sort is an LSD radix sort of 8-bit digit passes in the onesweep
//   style: the counting kernel also builds the global digit histograms of all
//   four passes (they depend only on the keys, not on their order) and the
//   largest count; each pass is one kernel whose CTAs take tiles in start
//   order, rank their keys stably (warp match on the digit + per-warp running
//   counts), find each digit's offset among earlier tiles by a decoupled
//   look-back over the tiles' published counts, and scatter.  Passes 3 and 4
//   return at once when every count is below 2^16 (the keys are then sorted
//   after two passes).  Look-back waits are bounded; one that runs out sets
//   word 0 of the sort scratch (a status word, CS_STATUS_* style; 1 = a wait
//   ran out).
// Power-of-two bins (no reference function): bin k >= 1 holds counts in
//   [2^k, 2^(k+1)), bin 0 holds 0 and 1; offsets are lower bounds in the sorted
//   counts, so they are pinned by the sort.
// Rebuild (rebuild_compressed_major_order_raw, major_nnz_raw.cuh:188-250): rows
//   copied into sorted order with one warp per destination row.  The reference
//   feeds counts already shifted by one slot into an exclusive scan, which
//   yields dst_major_ptr = [0, 0, c0, c0+c1, ...] and overlapping rows; the row
//   pointer here is the permuted CSR that rebuild is meant to produce.
// Shard variants take per-part pointer tables and locate a row's part by
// binary search over the part row offsets (find_offset_span semantics,
// include/CellShard/core/offset_span.cuh:12-24).
#include "common.cuh"

namespace csb {
namespace {

constexpr unsigned kSortThreads = 256;
constexpr unsigned kSortWarps = kSortThreads / 32;
constexpr unsigned kTileKeys = 4096; // 8 warps x 512 keys
constexpr unsigned kKeysPerWarp = kTileKeys / kSortWarps;
constexpr unsigned kRadix = 256;

__device__ __forceinline__ uint32_t find_part(uint32_t row, const uint32_t *offsets, uint32_t count) {
    uint32_t lo = 0u, hi = count;
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (row < offsets[mid])
            hi = mid;
        else if (row >= offsets[mid + 1u])
            lo = mid + 1u;
        else
            return mid;
    }
    return count;
}

// counts + identity + global digit histograms of the 4 passes + max count
__global__ void __launch_bounds__(256) count_hist_kernel(uint32_t n, const uint32_t *__restrict__ ptr,
                                                         const uint32_t *const *__restrict__ parts,
                                                         const uint32_t *__restrict__ part_offsets,
                                                         uint32_t part_count, uint32_t *__restrict__ nnz,
                                                         uint32_t *__restrict__ order_in, uint32_t *__restrict__ ghist,
                                                         uint32_t *__restrict__ max_key, uint32_t buckets,
                                                         uint32_t *__restrict__ offsets) {
    __shared__ uint32_t h[4][kRadix];
    // equal-count bucket offsets (fill_equal_count_bucket_offsets) by block 0
    if (blockIdx.x == 0u && offsets != nullptr) {
        const uint32_t size = n / buckets, rem = n % buckets;
        for (uint32_t b = threadIdx.x; b <= buckets; b += blockDim.x)
            offsets[b] = b == buckets ? n : b * size + min(b, rem);
    }
    for (uint32_t i = threadIdx.x; i < 4u * kRadix; i += blockDim.x) (&h[0][0])[i] = 0u;
    __syncthreads();
    uint32_t mx = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t c;
        if (parts == nullptr) {
            c = ptr[i + 1u] - ptr[i];
        } else {
            const uint32_t p = find_part(i, part_offsets, part_count);
            const uint32_t *pp = parts[p];
            const uint32_t local = i - part_offsets[p];
            c = pp[local + 1u] - pp[local];
        }
        nnz[i] = c;
        order_in[i] = i;
        mx = max(mx, c);
#pragma unroll
        for (int q = 0; q < 4; ++q) atomicAdd(&h[q][(c >> (8 * q)) & 0xffu], 1u);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31u) == 0u && mx != 0u) atomicMax(max_key, mx);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 4u * kRadix; i += blockDim.x) {
        const uint32_t v = (&h[0][0])[i];
        if (v != 0u) atomicAdd(ghist + i, v);
    }
}

constexpr unsigned long long kLookAggregate = 1ull << 62;
constexpr unsigned long long kLookInclusive = 2ull << 62;
constexpr unsigned long long kLookValue = (1ull << 62) - 1ull;
constexpr uint32_t kLookSpin = 1u << 22;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One stable counting-sort pass over digit (key >> shift) & 255.  vals ==
// nullptr means the identity (the row ids).  Tiles are taken in start order so
// every look-back target belongs to a CTA that is already running.  The tile
// is ranked in registers, placed in shared memory grouped by digit, and
// written from there: consecutive threads store consecutive positions of one
// digit's run, so the global stores come out as runs instead of one sector
// per key.
__global__ void __launch_bounds__(kSortThreads) onesweep_pass_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, uint32_t n, uint32_t shift,
    const uint32_t *__restrict__ ghist, unsigned long long *__restrict__ look, uint32_t *__restrict__ tile_counter,
    const uint32_t *__restrict__ max_key, uint32_t skip_below, uint32_t *__restrict__ out_keys,
    uint32_t *__restrict__ out_vals, uint32_t *__restrict__ status) {
    __shared__ uint32_t wc[kSortWarps][kRadix];
    __shared__ uint32_t scan33[33];
    __shared__ uint32_t tile_s;
    __shared__ uint32_t dg_global[kRadix], dg_local[kRadix];
    __shared__ uint32_t s_keys[kTileKeys], s_vals[kTileKeys];
    if (skip_below != 0u && *max_key < skip_below) return; // uniform: the pass changes nothing
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
    for (uint32_t d = lane; d < kRadix; d += 32u) wc[warp][d] = 0u;
    __syncthreads();
    const uint32_t t = tile_s;
    const uint32_t wbase = t * kTileKeys + warp * kKeysPerWarp;
    uint32_t kk[kKeysPerWarp / 32u], pk[kKeysPerWarp / 32u], vv[kKeysPerWarp / 32u];
    // keys and values of the tile are loaded up front (all in flight together)
#pragma unroll
    for (uint32_t b = 0; b < kKeysPerWarp / 32u; ++b) {
        const uint32_t k = wbase + b * 32u + lane;
        kk[b] = k < n ? __ldcs(keys + k) : 0u;
        vv[b] = vals != nullptr ? (k < n ? __ldcs(vals + k) : 0u) : k;
    }
#pragma unroll
    for (uint32_t b = 0; b < kKeysPerWarp / 32u; ++b) {
        const uint32_t k = wbase + b * 32u + lane;
        const uint32_t d = k < n ? (kk[b] >> shift) & 0xffu : kRadix;
        pk[b] = __match_any_sync(0xffffffffu, d);
        if (d < kRadix && lane == (unsigned) (__ffs(pk[b]) - 1)) wc[warp][d] += __popc(pk[b]);
        __syncwarp();
    }
    __syncthreads();
    {
        const uint32_t d = threadIdx.x; // kSortThreads == kRadix
        uint32_t cnt = 0u;
#pragma unroll
        for (unsigned w = 0; w < kSortWarps; ++w) cnt += wc[w][d];
        unsigned long long *mine = look + (std::size_t) t * kRadix + d;
        uint32_t excl = 0u;
        if (t == 0u) {
            st_release_u64(mine, kLookInclusive | cnt);
        } else {
            st_release_u64(mine, kLookAggregate | cnt);
            bool ok = true;
            for (uint32_t j = t; j-- > 0u;) {
                unsigned long long v = 0ull;
                uint32_t it = 0u;
                while (((v = ld_acquire_u64(look + (std::size_t) j * kRadix + d)) & ~kLookValue) == 0ull) {
                    if (++it >= kLookSpin) {
                        ok = false;
                        break;
                    }
                    __nanosleep(32);
                }
                if (!ok) break;
                excl += (uint32_t) (v & kLookValue);
                if (v & kLookInclusive) break;
            }
            if (!ok) atomicOr(status, 1u);
            st_release_u64(mine, kLookInclusive | (unsigned long long) (excl + cnt));
        }
        // global base of digit d: exclusive scan of the pass's digit totals;
        // tile-local base: exclusive scan of this tile's digit counts
        uint32_t tot, tile_tot;
        const uint32_t gbase = block_exclusive_scan(ghist[d], scan33, tot);
        const uint32_t lbase = block_exclusive_scan(cnt, scan33, tile_tot);
        dg_global[d] = gbase + excl;
        dg_local[d] = lbase;
        uint32_t run = lbase;
#pragma unroll
        for (unsigned w = 0; w < kSortWarps; ++w) {
            const uint32_t c = wc[w][d];
            wc[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (uint32_t b = 0; b < kKeysPerWarp / 32u; ++b) {
        const uint32_t k = wbase + b * 32u + lane;
        const uint32_t d = k < n ? (kk[b] >> shift) & 0xffu : kRadix;
        uint32_t pos = 0u;
        if (d < kRadix) pos = wc[warp][d] + __popc(pk[b] & lt);
        __syncwarp();
        if (d < kRadix) {
            s_keys[pos] = kk[b];
            s_vals[pos] = vv[b];
            if (lane == (unsigned) (__ffs(pk[b]) - 1)) wc[warp][d] += __popc(pk[b]);
        }
        __syncwarp();
    }
    __syncthreads();
    const uint32_t tile_n = n - t * kTileKeys < kTileKeys ? n - t * kTileKeys : kTileKeys;
    for (uint32_t i = threadIdx.x; i < tile_n; i += kSortThreads) {
        const uint32_t key = s_keys[i];
        const uint32_t d = (key >> shift) & 0xffu;
        const uint32_t g = dg_global[d] + (i - dg_local[d]);
        out_keys[g] = key;
        out_vals[g] = s_vals[i];
    }
}

__global__ void pow2_bins_kernel(const uint32_t *__restrict__ sorted, uint32_t n, uint32_t *__restrict__ bins) {
    const uint32_t k = threadIdx.x;
    if (k > 33u) return;
    if (k == 0u) {
        bins[0] = 0u;
        return;
    }
    if (k == 33u) {
        bins[33] = n;
        return;
    }
    const unsigned long long bound = 1ull << k;
    uint32_t lo = 0u, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if ((unsigned long long) sorted[mid] < bound)
            lo = mid + 1u;
        else
            hi = mid;
    }
    bins[k] = lo;
}

// dst counts in order (single matrix or shard)
__global__ void gather_counts_kernel(uint32_t n, const uint32_t *__restrict__ order, const uint32_t *__restrict__ ptr,
                                     const uint32_t *const *__restrict__ parts,
                                     const uint32_t *__restrict__ part_offsets, uint32_t part_count,
                                     uint32_t *__restrict__ counts, uint32_t *__restrict__ inverse) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = order[i];
        uint32_t c;
        if (parts == nullptr) {
            c = ptr[s + 1u] - ptr[s];
        } else {
            const uint32_t p = find_part(s, part_offsets, part_count);
            const uint32_t local = s - part_offsets[p];
            c = parts[p][local + 1u] - parts[p][local];
        }
        counts[i] = c;
        if (inverse != nullptr) inverse[s] = i;
    }
}

__global__ void __launch_bounds__(256) segment_copy_kernel(uint32_t n, const uint32_t *__restrict__ order,
                                                           const uint32_t *__restrict__ ptr,
                                                           const uint32_t *__restrict__ idx,
                                                           const uint16_t *__restrict__ val,
                                                           const uint32_t *const *__restrict__ part_ptr,
                                                           const uint32_t *const *__restrict__ part_idx,
                                                           const uint16_t *const *__restrict__ part_val,
                                                           const uint32_t *__restrict__ part_offsets,
                                                           uint32_t part_count, const uint32_t *__restrict__ dst_ptr,
                                                           uint32_t *__restrict__ dst_idx,
                                                           uint16_t *__restrict__ dst_val) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t step = gridDim.x * 8u;
    // a row's source arrays and bounds, from its source row id s and position i
    struct row_src {
        const uint32_t *si;
        const uint16_t *sv;
        uint32_t a, len, d;
    };
    auto locate = [&](uint32_t s, uint32_t i) {
        const uint32_t *sp = ptr;
        row_src r{idx, val, 0u, 0u, 0u};
        uint32_t local = s;
        if (part_ptr != nullptr) {
            const uint32_t p = find_part(s, part_offsets, part_count);
            local = s - part_offsets[p];
            sp = part_ptr[p];
            r.si = part_idx[p];
            r.sv = part_val[p];
        }
        r.a = sp[local];
        r.len = sp[local + 1u] - r.a;
        r.d = dst_ptr[i];
        return r;
    };
    // pipelined: row i's bounds and row i + step's source id are known when
    // row i is copied, so those lookups overlap the copy instead of preceding it
    uint32_t i = blockIdx.x * 8u + (threadIdx.x >> 5);
    if (i >= n) return;
    row_src cur = locate(order[i], i);
    uint32_t s_next = i + step > i && i + step < n ? order[i + step] : 0u;
    for (; i < n; i += step) {
        row_src nxt{idx, val, 0u, 0u, 0u};
        uint32_t s_after = 0u;
        if (i + step > i && i + step < n) {
            nxt = locate(s_next, i + step);
            if (i + 2u * step < n && i + 2u * step > i) s_after = order[i + 2u * step];
        }
        // eight coalesced loads per array in flight per lane before the stores
        constexpr unsigned U = 8;
        for (uint32_t j0 = 0; j0 < cur.len; j0 += 32u * U) {
            uint32_t iv[U];
            uint16_t vv[U];
#pragma unroll
            for (unsigned u = 0; u < U; ++u) {
                const uint32_t j = j0 + u * 32u + lane;
                if (j < cur.len) {
                    iv[u] = __ldcs(cur.si + cur.a + j);
                    vv[u] = __ldcs(reinterpret_cast<const unsigned short *>(cur.sv) + cur.a + j);
                }
            }
#pragma unroll
            for (unsigned u = 0; u < U; ++u) {
                const uint32_t j = j0 + u * 32u + lane;
                if (j < cur.len) {
                    dst_idx[cur.d + j] = iv[u];
                    dst_val[cur.d + j] = vv[u];
                }
            }
        }
        cur = nxt;
        s_next = s_after;
        if (i + step < i) break; // the next index would wrap past 2^32
    }
}

unsigned grid1d(uint32_t n, uint32_t threads) {
    uint32_t g = (n + threads - 1u) / threads;
    const uint32_t cap = (uint32_t) sm_count() * 16u;
    if (g > cap) g = cap;
    return g == 0u ? 1u : g;
}

uint32_t clamp_buckets(uint32_t n, uint32_t requested) {
    if (n == 0u) return 1u;
    if (requested < 1u) return 1u;
    return requested > n ? n : requested;
}

struct sort_layout {
    uint32_t *status;             // word 0 of the scratch
    uint32_t *max_key;
    uint32_t *tile_counters;      // [4]
    uint32_t *ghist;              // [4][256]
    unsigned long long *look;     // [4][tiles][256]
    uint32_t *tmp_keys, *tmp_vals;
    std::size_t clear_bytes, bytes;
    uint32_t tiles;
};

void make_sort_layout(uint32_t n, void *base, std::size_t cap, sort_layout *l) {
    l->tiles = (n + kTileKeys - 1u) / kTileKeys;
    scratch_carver c(base, cap);
    // status, max, counters and histograms first, then the look-back words:
    // one memset clears them all
    l->status = c.take<uint32_t>(8);
    l->max_key = l->status + 1;
    l->tile_counters = l->status + 2;
    l->ghist = c.take<uint32_t>(4u * kRadix);
    l->look = c.take<unsigned long long>((std::size_t) 4u * l->tiles * kRadix);
    l->clear_bytes = c.used;
    l->tmp_keys = c.take<uint32_t>((std::size_t) n + 1u);
    l->tmp_vals = c.take<uint32_t>((std::size_t) n + 1u);
    l->bytes = c.used;
}

// Digit histograms of the 4 passes and the largest key, for keys given as is
// (the sort_pairs_u32 entry below).
__global__ void __launch_bounds__(256) key_hist_kernel(uint32_t n, const uint32_t *__restrict__ keys,
                                                       uint32_t *__restrict__ ghist, uint32_t *__restrict__ max_key) {
    __shared__ uint32_t h[4][kRadix];
    for (uint32_t i = threadIdx.x; i < 4u * kRadix; i += blockDim.x) (&h[0][0])[i] = 0u;
    __syncthreads();
    uint32_t mx = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = keys[i];
        mx = max(mx, c);
#pragma unroll
        for (int q = 0; q < 4; ++q) atomicAdd(&h[q][(c >> (8 * q)) & 0xffu], 1u);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31u) == 0u && mx != 0u) atomicMax(max_key, mx);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 4u * kRadix; i += blockDim.x) {
        const uint32_t v = (&h[0][0])[i];
        if (v != 0u) atomicAdd(ghist + i, v);
    }
}

int run_passes(const uint32_t *keys, const uint32_t *vals, uint32_t n, uint32_t *out_keys, uint32_t *out_vals,
               const sort_layout &l, cudaStream_t stream) {
    // passes 0 and 1 always run (they leave the result in the output arrays);
    // passes 2 and 3 only when some key reaches 2^16
    const uint32_t *ik = keys, *iv = vals;
    for (uint32_t pass = 0; pass < 4u; ++pass) {
        uint32_t *ok = (pass % 2u == 0u) ? l.tmp_keys : out_keys;
        uint32_t *ov = (pass % 2u == 0u) ? l.tmp_vals : out_vals;
        onesweep_pass_kernel<<<l.tiles, kSortThreads, 0, stream>>>(
            ik, iv, n, 8u * pass, l.ghist + pass * kRadix, l.look + (std::size_t) pass * l.tiles * kRadix,
            l.tile_counters + pass, l.max_key, pass >= 2u ? (1u << 16) : 0u, ok, ov, l.status);
        if (!launch_ok("onesweep_pass_kernel")) return 0;
        ik = ok;
        iv = ov;
    }
    return 1;
}

int plan_common(uint32_t n, const uint32_t *ptr, const uint32_t *const *parts, const uint32_t *part_offsets,
                uint32_t part_count, uint32_t *d_nnz, uint32_t *d_sorted, uint32_t *d_order_in, uint32_t *d_order_out,
                uint32_t *d_offsets, uint32_t requested, void *tmp, std::size_t tmp_bytes, cudaStream_t stream) {
    if (n == 0u) {
        if (d_offsets != nullptr) return cuda_ok(cudaMemsetAsync(d_offsets, 0, 4, stream), "empty bucket offsets");
        return 1;
    }
    sort_layout l;
    make_sort_layout(n, tmp, tmp_bytes, &l);
    if (tmp == nullptr || l.bytes > tmp_bytes) {
        set_error("major_nnz_bucket_plan: sort scratch %zu < %zu bytes", tmp_bytes, l.bytes);
        return 0;
    }
    if (!cuda_ok(cudaMemsetAsync(l.status, 0, l.clear_bytes, stream), "plan scratch clear")) return 0;
    count_hist_kernel<<<grid1d(n, 256), 256, 0, stream>>>(n, ptr, parts, part_offsets, part_count, d_nnz, d_order_in,
                                                          l.ghist, l.max_key, clamp_buckets(n, requested), d_offsets);
    if (!launch_ok("count_hist_kernel")) return 0;
    return run_passes(d_nnz, nullptr, n, d_sorted, d_order_out, l, stream);
}

int rebuild_common(uint32_t n, const uint32_t *order, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                   const uint32_t *const *pp, const uint32_t *const *pi, const uint16_t *const *pv,
                   const uint32_t *part_offsets, uint32_t part_count, uint32_t *dst_ptr, uint32_t *dst_idx,
                   uint16_t *dst_val, uint32_t *inverse, void *tmp, std::size_t tmp_bytes, cudaStream_t stream) {
    if (n == 0u) return 1;
    if (tmp == nullptr || tmp_bytes < scan_u32_scratch_bytes(n)) {
        set_error("rebuild: scan scratch %zu < %zu bytes", tmp_bytes, scan_u32_scratch_bytes(n));
        return 0;
    }
    gather_counts_kernel<<<grid1d(n, 256), 256, 0, stream>>>(n, order, ptr, pp, part_offsets, part_count, dst_ptr,
                                                             inverse);
    if (!launch_ok("gather_counts_kernel")) return 0;
    if (!scan_exclusive_u32(dst_ptr, dst_ptr, n, true, tmp, tmp_bytes, stream)) return 0;
    segment_copy_kernel<<<grid1d(n, 8), 256, 0, stream>>>(n, order, ptr, idx, val, pp, pi, pv, part_offsets,
                                                          part_count, dst_ptr, dst_idx, dst_val);
    return launch_ok("segment_copy_kernel");
}

} // namespace

std::size_t sort_pairs_u32_scratch_bytes(uint32_t n) {
    sort_layout l;
    make_sort_layout(n, nullptr, 0, &l);
    return l.bytes;
}

int sort_pairs_u32(const uint32_t *keys, const uint32_t *vals, uint32_t n, uint32_t *out_keys, uint32_t *out_vals,
                   void *tmp, std::size_t tmp_bytes, cudaStream_t stream) {
    if (n == 0u) return 1;
    sort_layout l;
    make_sort_layout(n, tmp, tmp_bytes, &l);
    if (tmp == nullptr || l.bytes > tmp_bytes) {
        set_error("sort_pairs_u32: sort scratch %zu < %zu bytes", tmp_bytes, l.bytes);
        return 0;
    }
    if (!cuda_ok(cudaMemsetAsync(l.status, 0, l.clear_bytes, stream), "sort scratch clear")) return 0;
    key_hist_kernel<<<grid1d(n, 256), 256, 0, stream>>>(n, keys, l.ghist, l.max_key);
    if (!launch_ok("key_hist_kernel")) return 0;
    return run_passes(keys, vals, n, out_keys, out_vals, l, stream);
}

} // namespace csb

using namespace csb;

extern "C" int cs_b200_major_nnz_bucket_sort_scratch_bytes(uint32_t major_dim, size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("sort_scratch_bytes: null output");
        return 0;
    }
    sort_layout l;
    make_sort_layout(major_dim, nullptr, 0, &l);
    *out_bytes = l.bytes;
    return 1;
}

extern "C" int cs_b200_major_nnz_bucket_scan_scratch_bytes(uint32_t major_dim, size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("scan_scratch_bytes: null output");
        return 0;
    }
    *out_bytes = scan_u32_scratch_bytes(major_dim);
    return 1;
}

extern "C" int cs_b200_build_major_nnz_bucket_plan(const uint32_t *d_major_ptr, uint32_t major_dim,
                                                   uint32_t *d_major_nnz, uint32_t *d_major_nnz_sorted,
                                                   uint32_t *d_major_order_in, uint32_t *d_major_order_out,
                                                   uint32_t *d_bucket_offsets, uint32_t requested_bucket_count,
                                                   void *d_sort_tmp, size_t sort_tmp_bytes, cs_stream_t s) {
    if (d_major_ptr == nullptr || d_major_nnz == nullptr || d_major_nnz_sorted == nullptr ||
        d_major_order_in == nullptr || d_major_order_out == nullptr) {
        set_error("build_major_nnz_bucket_plan: null device array");
        return 0;
    }
    return plan_common(major_dim, d_major_ptr, nullptr, nullptr, 0u, d_major_nnz, d_major_nnz_sorted, d_major_order_in,
                       d_major_order_out, d_bucket_offsets, requested_bucket_count, d_sort_tmp, sort_tmp_bytes,
                       as_stream(s));
}

extern "C" int cs_b200_build_shard_major_nnz_bucket_plan(const uint32_t *const *d_part_major_ptr,
                                                         const uint32_t *d_part_row_offsets, uint32_t part_count,
                                                         uint32_t shard_rows, uint32_t *d_major_nnz,
                                                         uint32_t *d_major_nnz_sorted, uint32_t *d_major_order_in,
                                                         uint32_t *d_major_order_out, uint32_t *d_bucket_offsets,
                                                         uint32_t requested_bucket_count, void *d_sort_tmp,
                                                         size_t sort_tmp_bytes, cs_stream_t s) {
    if (d_part_major_ptr == nullptr || d_part_row_offsets == nullptr || d_major_nnz == nullptr ||
        d_major_nnz_sorted == nullptr || d_major_order_in == nullptr || d_major_order_out == nullptr) {
        set_error("build_shard_major_nnz_bucket_plan: null device array");
        return 0;
    }
    return plan_common(shard_rows, nullptr, d_part_major_ptr, d_part_row_offsets, part_count, d_major_nnz,
                       d_major_nnz_sorted, d_major_order_in, d_major_order_out, d_bucket_offsets,
                       requested_bucket_count, d_sort_tmp, sort_tmp_bytes, as_stream(s));
}

extern "C" int cs_b200_pow2_nnz_bin_offsets(const uint32_t *d_major_nnz_sorted, uint32_t major_dim,
                                            uint32_t *d_bin_offsets, cs_stream_t s) {
    if (d_bin_offsets == nullptr || (major_dim != 0u && d_major_nnz_sorted == nullptr)) {
        set_error("pow2_nnz_bin_offsets: null device array");
        return 0;
    }
    pow2_bins_kernel<<<1, 64, 0, as_stream(s)>>>(d_major_nnz_sorted, major_dim, d_bin_offsets);
    return launch_ok("pow2_bins_kernel");
}

extern "C" int cs_b200_rebuild_compressed_major_order(const uint32_t *d_src_major_ptr, const uint32_t *d_src_minor_idx,
                                                      const uint16_t *d_src_val, uint32_t major_dim,
                                                      const uint32_t *d_major_order, uint32_t *d_dst_major_ptr,
                                                      uint32_t *d_dst_minor_idx, uint16_t *d_dst_val,
                                                      uint32_t *d_inverse_major_order, void *d_scan_tmp,
                                                      size_t scan_tmp_bytes, cs_stream_t s) {
    if (d_src_major_ptr == nullptr || d_src_minor_idx == nullptr || d_src_val == nullptr || d_major_order == nullptr ||
        d_dst_major_ptr == nullptr || d_dst_minor_idx == nullptr || d_dst_val == nullptr) {
        set_error("rebuild_compressed_major_order: null device array");
        return 0;
    }
    return rebuild_common(major_dim, d_major_order, d_src_major_ptr, d_src_minor_idx, d_src_val, nullptr, nullptr,
                          nullptr, nullptr, 0u, d_dst_major_ptr, d_dst_minor_idx, d_dst_val, d_inverse_major_order,
                          d_scan_tmp, scan_tmp_bytes, as_stream(s));
}

extern "C" int cs_b200_rebuild_bucketed_shard_compressed(const uint32_t *const *d_part_major_ptr,
                                                         const uint32_t *const *d_part_minor_idx,
                                                         const uint16_t *const *d_part_val,
                                                         const uint32_t *d_part_row_offsets, uint32_t part_count,
                                                         uint32_t shard_rows, const uint32_t *d_major_order,
                                                         uint32_t *d_dst_major_ptr, uint32_t *d_dst_minor_idx,
                                                         uint16_t *d_dst_val, uint32_t *d_inverse_major_order,
                                                         void *d_scan_tmp, size_t scan_tmp_bytes, cs_stream_t s) {
    if (d_part_major_ptr == nullptr || d_part_minor_idx == nullptr || d_part_val == nullptr ||
        d_part_row_offsets == nullptr || d_major_order == nullptr || d_dst_major_ptr == nullptr ||
        d_dst_minor_idx == nullptr || d_dst_val == nullptr) {
        set_error("rebuild_bucketed_shard_compressed: null device array");
        return 0;
    }
    return rebuild_common(shard_rows, d_major_order, nullptr, nullptr, nullptr, d_part_major_ptr, d_part_minor_idx,
                          d_part_val, d_part_row_offsets, part_count, d_dst_major_ptr, d_dst_minor_idx, d_dst_val,
                          d_inverse_major_order, d_scan_tmp, scan_tmp_bytes, as_stream(s));
}
