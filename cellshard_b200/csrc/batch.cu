// Batched CSR -> Sliced-ELL conversion with nnz bucket plans for many uneven
// partitions: one persistent launch per wave, fed from a device work queue and
// replayed from a CUDA graph.
//
// Per partition the work is what convert::choose_sliced_ell_slice_rows_from_
// compressed + convert::sliced_ell_from_compressed
// (src/convert/sliced_ell_from_blocked_ell.cuh:64-142,196-221;
// src/convert/sliced_ell_from_compressed.cuh:20-164) and
// bucket::build_major_nnz_bucket_plan_raw (src/bucket/major_nnz_raw.cuh:64-120)
// compute, with the same results bit for bit.
//
// Work items, dequeued in this order by every resident CTA (atomic head):
//   LAYOUT (p, rows r0..r1)  row nnz (-> plan's major_nnz), per-candidate
//                            slice widths (segmented warp max + atomicMax),
//                            partition max nnz; then layout_done[p] += 1.
//   CHOOSE (p)               waits for p's layout items; padded slots per
//                            candidate, the reference score/tie-break in
//                            IEEE doubles, the chosen layout (row offsets,
//                            widths, u32 slot offsets) written into an arena
//                            block taken first-fit in wave order (a chain over
//                            the wave's partitions, so offsets are the same on
//                            every run); a partition that does not fit is
//                            deferred to the next wave.  choose_done[p] = 1.
//   PLAN (p)                 waits for p's layout items; stable LSD radix sort
//                            of (nnz, row) inside the CTA (8-bit digits, only
//                            as many passes as the max nnz needs), equal-count
//                            bucket offsets, power-of-two bin offsets.
//   EMIT (p, rows r0..r1)    waits for choose_done[p]; each group of GL lanes
//                            writes one row's slots with 16-byte stores.
// Every dependency points at an item earlier in the queue, which some running
// CTA has already dequeued, so the waits end; each wait is still bounded, and
// a wait that runs out sets CS_BATCH_WAIT_TIMEOUT and skips the item.
#include "common.cuh"
#include "emit_rows.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

struct cs_batch_plan {
    int device = 0;
    cudaStream_t cap_stream = nullptr;
    uint32_t count = 0;
    std::vector<cs_batch_part> parts;
    uint32_t ncand = 0;
    uint32_t cand[CS_BATCH_MAX_CANDIDATES] = {0, 0, 0, 0};
    cs_batch_tiles tiles{};
    unsigned char *arena = nullptr;
    uint64_t arena_bytes = 0;
    std::vector<uint32_t> wave; // partitions of the current wave, in chain order
    // device memory (owned)
    void *d_parts = nullptr;      // csb::bpart[count]
    void *d_items = nullptr;      // uint4[item_cap]
    std::size_t item_cap = 0;
    uint32_t n_items = 0;
    void *d_state = nullptr;      // zeroed per wave
    std::size_t state_bytes = 0;
    uint32_t *d_sort_tmp = nullptr;
    cs_batch_sliced_result *d_results = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int ctas_per_sm = 1;
    uint32_t grid = 0;
    uint64_t launches = 0;
};

namespace csb {
namespace {

constexpr unsigned kBThreads = 256;
constexpr unsigned kBWarps = kBThreads / 32;
constexpr uint32_t kSpinLimit = 1u << 22; // x up to 256 ns sleeps: about a second
constexpr uint32_t kPlanTile = kBThreads * 8u;

enum : uint32_t { ITEM_LAYOUT = 0u, ITEM_CHOOSE = 1u, ITEM_PLAN = 2u, ITEM_EMIT = 3u };

struct bpart {
    uint32_t rows, cols, nnz, bucket_count;
    const uint32_t *ptr;
    const uint32_t *idx;
    const uint16_t *val;
    uint32_t *major_nnz, *sorted_nnz, *order, *bucket_offsets, *pow2_offsets;
    uint32_t *sort_tmp;                           // 2 * rows
    uint32_t *widths;                             // per candidate, zeroed per wave
    uint32_t cand_h[CS_BATCH_MAX_CANDIDATES];     // clamped heights (0 = unused)
    uint32_t cand_off[CS_BATCH_MAX_CANDIDATES];   // offsets into widths
    uint32_t n_layout;                            // layout items this wave
    uint32_t wave_pos;                            // position in the allocation chain
};

struct bstate_ptrs {
    uint32_t *head;        // [1]
    uint32_t *error;       // [1]
    uint32_t *deferred;    // [1]
    uint32_t *layout_done; // [count]
    uint32_t *max_nnz;     // [count]
    uint32_t *choose_done; // [count]
    uint32_t *alloc_ready; // [count] by wave position
    unsigned long long *alloc_cursor; // [count] by wave position
    uint32_t *widths;      // all candidate widths
};

struct bparams {
    const uint4 *items;
    uint32_t n_items;
    uint32_t ncand;
    uint32_t cand[CS_BATCH_MAX_CANDIDATES];
    bpart *parts;
    bstate_ptrs st;
    cs_batch_sliced_result *results;
    unsigned char *arena;
    unsigned long long arena_bytes;
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// bounded wait for *p >= target (one thread)
__device__ bool wait_geq(const uint32_t *p, uint32_t target) {
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        if (ld_acquire(p) >= target) return true;
        __nanosleep(it < 256u ? 32u : 256u);
    }
    return false;
}

__device__ __forceinline__ bool is_pow2(uint32_t h) { return h != 0u && (h & (h - 1u)) == 0u; }

struct bsmem {
    uint4 item;
    uint32_t flag;
    uint32_t scan33[33];
    unsigned long long red[kBWarps][CS_BATCH_MAX_CANDIDATES];
    uint32_t u32s[8];
    unsigned long long u64s[2];
    uint32_t cnt[kBWarps][256];
    uint32_t bas[kBWarps][256];
    uint32_t dig[257];
};

// ---------------------------------------------------------------------------
// LAYOUT
// ---------------------------------------------------------------------------
__device__ void do_layout(const bparams &P, bsmem &sm, uint32_t pi, uint32_t r0, uint32_t r1) {
    const bpart &p = P.parts[pi];
    const unsigned lane = threadIdx.x & 31u;
    uint32_t mx = 0u;
    for (uint32_t base = r0; base < r1; base += kBThreads) {
        const uint32_t r = base + threadIdx.x;
        const bool in = r < r1;
        const uint32_t n = in ? __ldg(p.ptr + r + 1u) - __ldg(p.ptr + r) : 0u;
        if (in && p.major_nnz != nullptr) p.major_nnz[r] = n;
        mx = max(mx, n);
#pragma unroll
        for (uint32_t k = 0; k < CS_BATCH_MAX_CANDIDATES; ++k) {
            const uint32_t h = p.cand_h[k];
            if (h == 0u) continue;
            uint32_t *wk = p.widths + p.cand_off[k];
            if (is_pow2(h)) {
                const uint32_t span = h < 32u ? h : 32u;
                uint32_t v = n;
                for (uint32_t off = 1u; off < span; off <<= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
                if (in && (lane & (span - 1u)) == 0u && v != 0u) atomicMax(wk + r / h, v);
            } else if (in && n != 0u) {
                atomicMax(wk + r / h, n);
            }
        }
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane == 0u && mx != 0u) atomicMax(P.st.max_nnz + pi, mx);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(P.st.layout_done + pi, 1u);
    }
}

// ---------------------------------------------------------------------------
// CHOOSE + allocate + layout arrays
// ---------------------------------------------------------------------------
__device__ void block_scan_u32(uint32_t *v, uint32_t n, uint32_t *smem33, uint32_t carry_in,
                               uint32_t *total_out) {
    // exclusive scan of v[0..n) in place, in tiles of blockDim.x * 4
    uint32_t carry = carry_in;
    for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x * 4u) {
        uint32_t loc[4], sum = 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t k = t0 + threadIdx.x * 4u + q;
            loc[q] = k < n ? v[k] : 0u;
            sum += loc[q];
        }
        uint32_t tot;
        uint32_t run = block_exclusive_scan(sum, smem33, tot) + carry;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t k = t0 + threadIdx.x * 4u + q;
            if (k < n) v[k] = run;
            run += loc[q];
        }
        carry += tot;
        __syncthreads();
    }
    if (total_out != nullptr) *total_out = carry;
}

__device__ __forceinline__ std::size_t align_up(std::size_t x, std::size_t a) { return (x + a - 1u) / a * a; }

__device__ void do_choose(const bparams &P, bsmem &sm, uint32_t pi) {
    const bpart &p = P.parts[pi];
    cs_batch_sliced_result *res = P.results + pi;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) sm.flag = wait_geq(P.st.layout_done + pi, p.n_layout) ? 1u : 0u;
    __syncthreads();
    const bool ready = sm.flag != 0u;
    __syncthreads();
    const uint32_t rows = p.rows;
    // padded slots per candidate (per-warp partial sums)
    if (ready) {
#pragma unroll
        for (uint32_t k = 0; k < CS_BATCH_MAX_CANDIDATES; ++k) {
            const uint32_t h = p.cand_h[k];
            if (h == 0u) continue;
            const uint32_t S = (rows + h - 1u) / h;
            const uint32_t *wk = p.widths + p.cand_off[k];
            unsigned long long acc = 0ull;
            for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
                const uint32_t rin = min(rows, (s + 1u) * h) - s * h;
                acc += (unsigned long long) rin * __ldcg(wk + s);
            }
            for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
            if (lane == 0u) sm.red[warp][k] = acc;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t status = ready ? 0u : CS_BATCH_WAIT_TIMEOUT;
        uint32_t best_h = 0u, best_S = 0u;
        unsigned long long best_slots = 0ull, best_bytes = 0ull;
        double best_score = 0.0;
        bool have = false;
        if (ready && rows != 0u) {
            for (uint32_t k = 0; k < CS_BATCH_MAX_CANDIDATES; ++k) {
                const uint32_t h = p.cand_h[k];
                if (h == 0u) continue;
                unsigned long long slots = 0ull;
                for (unsigned w = 0; w < kBWarps; ++w) slots += sm.red[w][k];
                const uint32_t S = (rows + h - 1u) / h;
                const unsigned long long bytes = slots * 6ull + ((unsigned long long) S * 2ull + 1ull) * 4ull;
                // the reference's score in IEEE doubles, no contraction:
                // padded / nnz + 0.25 * (S / rows)
                const double ratio = p.nnz == 0u ? 1.0 : __ddiv_rn((double) slots, (double) p.nnz);
                const double pen = __dmul_rn(0.25, __ddiv_rn((double) S, (double) rows));
                const double score = __dadd_rn(ratio, pen);
                if (!have || __dadd_rn(score, 1.0e-12) < best_score ||
                    (score <= __dadd_rn(best_score, 1.0e-12) && bytes < best_bytes) ||
                    (score <= __dadd_rn(best_score, 1.0e-12) && bytes == best_bytes && h > best_h)) {
                    have = true;
                    best_h = h;
                    best_S = S;
                    best_slots = slots;
                    best_bytes = bytes;
                    best_score = score;
                }
            }
            if (!have) status |= CS_BATCH_NO_CANDIDATE;
            if (best_slots > 0xffffffffull) status |= CS_BATCH_TOO_LARGE;
        }
        // arena block: [row offsets S+1][widths S][slot offsets S] | col_idx | val
        const std::size_t hdr = align_up(((std::size_t) best_S * 3u + 1u) * 4u, 256u);
        const std::size_t cbytes = align_up((std::size_t) best_slots * 4u, 256u);
        const std::size_t vbytes = align_up((std::size_t) best_slots * 2u, 256u);
        const unsigned long long need = (status == 0u && rows != 0u) ? hdr + cbytes + vbytes : 0ull;
        // allocation chain over the wave, first fit in wave order
        unsigned long long cursor = 0ull;
        bool chain_ok = true;
        if (p.wave_pos > 0u) {
            chain_ok = wait_geq(P.st.alloc_ready + p.wave_pos - 1u, 1u);
            cursor = chain_ok ? __ldcg(P.st.alloc_cursor + p.wave_pos - 1u) : P.arena_bytes;
        }
        if (!chain_ok) status |= CS_BATCH_WAIT_TIMEOUT;
        unsigned long long off = ~0ull;
        if (need > P.arena_bytes) status |= CS_BATCH_EXCEEDS_ARENA;
        if (status == 0u && need != 0ull) {
            if (cursor + need <= P.arena_bytes) {
                off = cursor;
                cursor += need;
            } else {
                status |= CS_BATCH_DEFERRED;
            }
        }
        P.st.alloc_cursor[p.wave_pos] = cursor;
        __threadfence();
        st_release(P.st.alloc_ready + p.wave_pos, 1u);
        res->status = status;
        res->slice_rows = best_h;
        res->slice_count = best_S;
        res->total_slots = best_slots;
        res->arena_offset = off;
        res->arena_bytes = need;
        res->score = best_score;
        cs_sliced_ell_view v{};
        v.rows = rows;
        v.cols = p.cols;
        v.nnz = p.nnz;
        v.slice_count = best_S;
        v.slice_rows = best_h;
        if (off != ~0ull) {
            unsigned char *b = P.arena + off;
            v.slice_row_offsets = reinterpret_cast<uint32_t *>(b);
            v.slice_widths = v.slice_row_offsets + best_S + 1u;
            v.slice_slot_offsets = v.slice_widths + best_S;
            v.col_idx = reinterpret_cast<uint32_t *>(b + hdr);
            v.val = reinterpret_cast<uint16_t *>(b + hdr + cbytes);
        }
        res->view = v;
        if (status & CS_BATCH_DEFERRED) atomicAdd(P.st.deferred, 1u);
        if (status & (CS_BATCH_WAIT_TIMEOUT | CS_BATCH_TOO_LARGE | CS_BATCH_NO_CANDIDATE | CS_BATCH_EXCEEDS_ARENA))
            atomicOr(P.st.error, status);
        sm.u32s[0] = status;
        sm.u32s[1] = best_h;
        sm.u32s[2] = best_S;
        sm.u64s[0] = off;
        sm.u64s[1] = hdr;
        // candidate index of best_h for its widths
        uint32_t kb = 0u;
        for (uint32_t k = 0; k < CS_BATCH_MAX_CANDIDATES; ++k)
            if (p.cand_h[k] == best_h && best_h != 0u) {
                kb = k;
                break;
            }
        sm.u32s[3] = kb;
    }
    __syncthreads();
    const uint32_t status = sm.u32s[0], h = sm.u32s[1], S = sm.u32s[2], kb = sm.u32s[3];
    const unsigned long long off = sm.u64s[0];
    if (status == 0u && off != ~0ull && S != 0u) {
        uint32_t *ro = reinterpret_cast<uint32_t *>(P.arena + off);
        uint32_t *wd = ro + S + 1u;
        uint32_t *so = wd + S;
        const uint32_t *wk = p.widths + p.cand_off[kb];
        for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) ro[s] = min(rows, s * h);
        for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
            const uint32_t w = __ldcg(wk + s);
            wd[s] = w;
            so[s] = (min(rows, (s + 1u) * h) - s * h) * w;
        }
        __syncthreads();
        block_scan_u32(so, S, sm.scan33, 0u, nullptr);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(P.st.choose_done + pi, 1u);
    }
}

// ---------------------------------------------------------------------------
// PLAN: stable sort of (row nnz, row) inside one CTA
// ---------------------------------------------------------------------------
__device__ void do_plan(const bparams &P, bsmem &sm, uint32_t pi) {
    const bpart &p = P.parts[pi];
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) sm.flag = wait_geq(P.st.layout_done + pi, p.n_layout) ? 1u : 0u;
    __syncthreads();
    if (sm.flag == 0u) {
        if (threadIdx.x == 0) {
            atomicOr(P.st.error, CS_BATCH_WAIT_TIMEOUT);
            P.results[pi].plan_status = CS_BATCH_WAIT_TIMEOUT;
        }
        __syncthreads();
        return;
    }
    const uint32_t n = p.rows;
    if (n == 0u) {
        if (threadIdx.x == 0) {
            p.bucket_offsets[0] = 0u;
            if (p.pow2_offsets != nullptr)
                for (int k = 0; k < 34; ++k) p.pow2_offsets[k] = 0u;
        }
        __syncthreads();
        return;
    }
    const uint32_t mx = __ldcg(P.st.max_nnz + pi);
    const uint32_t passes = mx < 256u ? 1u : (mx < 65536u ? 2u : (mx < (1u << 24) ? 3u : 4u));
    const unsigned lt = (1u << lane) - 1u;
    uint32_t *tk = p.sort_tmp, *tv = p.sort_tmp + n;
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const uint32_t shift = 8u * pass;
        // destination: the last pass lands in (sorted_nnz, order)
        const bool to_out = ((passes - 1u - pass) & 1u) == 0u;
        uint32_t *dk = to_out ? p.sorted_nnz : tk, *dv = to_out ? p.order : tv;
        const uint32_t *sk = pass == 0u ? p.major_nnz : (to_out ? tk : p.sorted_nnz);
        const uint32_t *sv = pass == 0u ? nullptr : (to_out ? tv : p.order);
        // histogram
        for (uint32_t d = threadIdx.x; d < kBWarps * 256u; d += blockDim.x) (&sm.cnt[0][0])[d] = 0u;
        __syncthreads();
        for (uint32_t r = threadIdx.x; r < n; r += blockDim.x) atomicAdd(&sm.cnt[warp][(__ldcg(sk + r) >> shift) & 255u], 1u);
        __syncthreads();
        {
            const uint32_t d = threadIdx.x; // 256 threads == 256 digits
            uint32_t t = 0u;
#pragma unroll
            for (unsigned w = 0; w < kBWarps; ++w) {
                t += sm.cnt[w][d];
                sm.cnt[w][d] = 0u;
            }
            uint32_t tot;
            sm.dig[d] = block_exclusive_scan(t, sm.scan33, tot);
        }
        __syncthreads();
        for (uint32_t t0 = 0; t0 < n; t0 += kPlanTile) {
            const uint32_t wa = t0 + warp * 256u, we = min(n, wa + 256u);
            uint32_t kk[8], vv[8], pk[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t i = wa + 32u * q + lane;
                const bool in = i < we;
                kk[q] = in ? __ldcg(sk + i) : 0u;
                vv[q] = in ? (sv != nullptr ? __ldcg(sv + i) : i) : 0u;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool in = wa + 32u * q + lane < we;
                const uint32_t d = (kk[q] >> shift) & 255u;
                pk[q] = warp_match_digit<8>(d, in);
                if (in && lane == (unsigned) (__ffs(pk[q]) - 1)) sm.cnt[warp][d] += __popc(pk[q]);
                __syncwarp();
            }
            __syncthreads();
            {
                const uint32_t d = threadIdx.x;
                uint32_t t = sm.dig[d];
#pragma unroll
                for (unsigned w = 0; w < kBWarps; ++w) {
                    const uint32_t c = sm.cnt[w][d];
                    sm.cnt[w][d] = 0u;
                    sm.bas[w][d] = t;
                    t += c;
                }
                sm.dig[d] = t;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool in = wa + 32u * q + lane < we;
                const uint32_t d = (kk[q] >> shift) & 255u;
                uint32_t pos = 0u;
                if (in) pos = sm.bas[warp][d] + __popc(pk[q] & lt);
                __syncwarp();
                if (in) {
                    dk[pos] = kk[q];
                    dv[pos] = vv[q];
                    if (lane == (unsigned) (__ffs(pk[q]) - 1)) sm.bas[warp][d] += __popc(pk[q]);
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
    // equal-count bucket offsets (clamp(requested, 1, n) buckets)
    uint32_t B = p.bucket_count < 1u ? 1u : p.bucket_count;
    if (B > n) B = n;
    const uint32_t size = n / B, rem = n % B;
    for (uint32_t b = threadIdx.x; b <= B; b += blockDim.x) p.bucket_offsets[b] = b == B ? n : b * size + min(b, rem);
    // power-of-two bins: offsets[k] = lower_bound(sorted, 2^k), [0] = 0, [33] = n
    if (p.pow2_offsets != nullptr && threadIdx.x < 34u) {
        const uint32_t k = threadIdx.x;
        uint32_t o;
        if (k == 0u)
            o = 0u;
        else if (k == 33u)
            o = n;
        else {
            const unsigned long long bound = 1ull << k;
            uint32_t lo = 0u, hi = n;
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                if ((unsigned long long) __ldcg(p.sorted_nnz + mid) < bound)
                    lo = mid + 1u;
                else
                    hi = mid;
            }
            o = lo;
        }
        p.pow2_offsets[k] = o;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// EMIT
// ---------------------------------------------------------------------------
template <unsigned GL>
__device__ void do_emit(const bparams &P, bsmem &sm, uint32_t pi, uint32_t r0, uint32_t r1) {
    const bpart &p = P.parts[pi];
    if (threadIdx.x == 0) {
        const bool ok = wait_geq(P.st.choose_done + pi, 1u);
        if (!ok) atomicOr(P.st.error, CS_BATCH_WAIT_TIMEOUT);
        sm.flag = ok ? 1u : 0u;
    }
    __syncthreads();
    const cs_batch_sliced_result *res = P.results + pi;
    const unsigned long long aoff = __ldcg(&res->arena_offset);
    const bool go = sm.flag != 0u && __ldcg(&res->status) == 0u && aoff != ~0ull;
    if (go) {
        const uint32_t h = __ldcg(&res->slice_rows);
        const uint32_t S = __ldcg(&res->slice_count);
        const unsigned char *b = P.arena + aoff;
        const uint32_t *wd = reinterpret_cast<const uint32_t *>(b) + S + 1u;
        const uint32_t *so = wd + S;
        const std::size_t hdr = align_up(((std::size_t) S * 3u + 1u) * 4u, 256u);
        const std::size_t cbytes = align_up((std::size_t) __ldcg(&res->total_slots) * 4u, 256u);
        uint32_t *col = reinterpret_cast<uint32_t *>(P.arena + aoff + hdr);
        uint16_t *vo = reinterpret_cast<uint16_t *>(P.arena + aoff + hdr + cbytes);
        constexpr unsigned RPW = 32u / GL;
        const unsigned lane = threadIdx.x & 31u, gl = lane % GL;
        for (uint32_t r = r0 + (threadIdx.x >> 5) * RPW + lane / GL; r < r1; r += kBWarps * RPW) {
            const uint32_t s = r / h;
            const uint32_t w = __ldcg(wd + s);
            const std::size_t base = (std::size_t) __ldcg(so + s) + (std::size_t) (r - s * h) * w;
            const uint32_t a = __ldg(p.ptr + r);
            sell_emit_row_vec<GL>(p.idx, p.val, a, __ldg(p.ptr + r + 1u) - a, w, base, col, vo, gl);
        }
    }
    __syncthreads();
}

template <unsigned GL>
__global__ void __launch_bounds__(kBThreads) batch_sliced_kernel(bparams P) {
    __shared__ bsmem sm;
    while (true) {
        if (threadIdx.x == 0) {
            const uint32_t i = atomicAdd(P.st.head, 1u);
            sm.item = i < P.n_items ? P.items[i] : make_uint4(0xffffffffu, 0u, 0u, 0u);
        }
        __syncthreads();
        const uint4 it = sm.item;
        __syncthreads();
        if (it.x == 0xffffffffu) break;
        switch (it.x) {
        case ITEM_LAYOUT: do_layout(P, sm, it.y, it.z, it.w); break;
        case ITEM_CHOOSE: do_choose(P, sm, it.y); break;
        case ITEM_PLAN: do_plan(P, sm, it.y); break;
        default: do_emit<GL>(P, sm, it.y, it.z, it.w); break;
        }
        __syncthreads();
    }
}

using kernel_t = void (*)(bparams);

kernel_t kernel_for(uint32_t lanes) {
    switch (lanes) {
    case 4: return batch_sliced_kernel<4>;
    case 8: return batch_sliced_kernel<8>;
    case 16: return batch_sliced_kernel<16>;
    default: return batch_sliced_kernel<32>;
    }
}

uint32_t clamp_h(uint32_t rows, uint32_t h) { return rows == 0u ? 0u : (h < rows ? h : rows); }

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct state_layout {
    std::size_t head, error, deferred, layout_done, max_nnz, choose_done, alloc_ready, alloc_cursor, widths, bytes;
};

state_layout make_state_layout(uint32_t count, std::size_t width_words) {
    state_layout s{};
    std::size_t o = 0;
    auto take = [&](std::size_t bytes) {
        const std::size_t at = o;
        o = (o + bytes + 255u) / 256u * 256u;
        return at;
    };
    s.head = take(4);
    s.error = take(4);
    s.deferred = take(4);
    s.layout_done = take((std::size_t) count * 4u);
    s.max_nnz = take((std::size_t) count * 4u);
    s.choose_done = take((std::size_t) count * 4u);
    s.alloc_ready = take((std::size_t) count * 4u);
    s.alloc_cursor = take((std::size_t) count * 8u);
    s.widths = take(width_words * 4u);
    s.bytes = o;
    return s;
}

bool tiles_valid(const cs_batch_tiles &t) {
    return t.layout_rows >= 32u && t.layout_rows % 32u == 0u && t.emit_rows >= 1u &&
           (t.emit_lanes == 4u || t.emit_lanes == 8u || t.emit_lanes == 16u || t.emit_lanes == 32u) &&
           t.ctas_per_sm <= 8u;
}

cs_batch_tiles default_tiles(const std::vector<cs_batch_part> &parts) {
    cs_batch_tiles t{};
    t.layout_rows = 4096u;
    t.emit_rows = 512u;
    uint64_t rows = 0, nnz = 0;
    for (const auto &p : parts) {
        rows += p.src.rows;
        nnz += p.src.nnz;
    }
    const double mean = rows ? (double) nnz / (double) rows : 0.0;
    t.emit_lanes = mean >= 96.0 ? 32u : (mean >= 24.0 ? 16u : 8u);
    t.ctas_per_sm = 0u; // 0 = as many as fit
    return t;
}

// builds items, partition descriptors and the state layout for plan->wave;
// uploads them and (re)captures the graph
int build_wave(cs_batch_plan *pl) {
    const uint32_t count = pl->count;
    std::vector<bpart> dp(count);
    std::size_t width_words = 0;
    std::vector<uint32_t> pos(count, 0xffffffffu);
    for (uint32_t q = 0; q < (uint32_t) pl->wave.size(); ++q) pos[pl->wave[q]] = q;
    for (uint32_t i = 0; i < count; ++i) {
        const cs_batch_part &hp = pl->parts[i];
        bpart &b = dp[i];
        std::memset(&b, 0, sizeof(b));
        b.rows = hp.src.rows;
        b.cols = hp.src.cols;
        b.nnz = hp.src.nnz;
        b.bucket_count = hp.bucket_count;
        b.ptr = hp.src.majorPtr;
        b.idx = hp.src.minorIdx;
        b.val = hp.src.val;
        if (hp.d_major_nnz != nullptr) {
            b.major_nnz = hp.d_major_nnz;
            b.sorted_nnz = hp.d_sorted_nnz;
            b.order = hp.d_order;
            b.bucket_offsets = hp.d_bucket_offsets;
            b.pow2_offsets = hp.d_pow2_offsets;
        }
        for (uint32_t k = 0; k < CS_BATCH_MAX_CANDIDATES; ++k) {
            const uint32_t h = k < pl->ncand ? clamp_h(b.rows, pl->cand[k]) : 0u;
            // a candidate equal to an earlier one adds nothing (same score, same bytes)
            bool dup = false;
            for (uint32_t j = 0; j < k; ++j) dup = dup || (b.cand_h[j] == h);
            b.cand_h[k] = dup ? 0u : h;
            b.cand_off[k] = (uint32_t) width_words;
            if (b.cand_h[k] != 0u) width_words += (b.rows + h - 1u) / h;
        }
        b.n_layout = b.rows == 0u ? 0u : (b.rows + pl->tiles.layout_rows - 1u) / pl->tiles.layout_rows;
        b.wave_pos = pos[i] == 0xffffffffu ? 0u : pos[i];
    }
    const state_layout sl = make_state_layout(count, width_words);
    // items in dependency order
    std::vector<uint4> items;
    for (uint32_t q : pl->wave)
        for (uint32_t r = 0; r < dp[q].rows; r += pl->tiles.layout_rows)
            items.push_back(make_uint4(ITEM_LAYOUT, q, r, std::min(dp[q].rows, r + pl->tiles.layout_rows)));
    for (uint32_t q : pl->wave) items.push_back(make_uint4(ITEM_CHOOSE, q, 0u, 0u));
    for (uint32_t q : pl->wave)
        if (dp[q].major_nnz != nullptr) items.push_back(make_uint4(ITEM_PLAN, q, 0u, 0u));
    for (uint32_t q : pl->wave)
        for (uint32_t r = 0; r < dp[q].rows; r += pl->tiles.emit_rows)
            items.push_back(make_uint4(ITEM_EMIT, q, r, std::min(dp[q].rows, r + pl->tiles.emit_rows)));
    // device buffers
    if (items.size() > pl->item_cap) {
        if (pl->d_items) cudaFree(pl->d_items);
        pl->d_items = nullptr;
        pl->item_cap = items.size() + 64u;
        if (!cuda_ok(cudaMalloc(&pl->d_items, pl->item_cap * sizeof(uint4)), "batch items")) return 0;
    }
    if (sl.bytes > pl->state_bytes) {
        if (pl->d_state) cudaFree(pl->d_state);
        pl->d_state = nullptr;
        if (!cuda_ok(cudaMalloc(&pl->d_state, sl.bytes), "batch state")) return 0;
        pl->state_bytes = sl.bytes;
    }
    unsigned char *st = static_cast<unsigned char *>(pl->d_state);
    for (auto &b : dp) b.widths = reinterpret_cast<uint32_t *>(st + sl.widths);
    // sort scratch: 2 * rows per partition
    {
        std::size_t off = 0;
        for (uint32_t i = 0; i < count; ++i) {
            dp[i].sort_tmp = pl->d_sort_tmp + off;
            off += 2u * (std::size_t) dp[i].rows;
        }
    }
    pl->n_items = (uint32_t) items.size();
    if (!cuda_ok(cudaMemcpy(pl->d_parts, dp.data(), sizeof(bpart) * count, cudaMemcpyHostToDevice), "batch parts") ||
        (!items.empty() && !cuda_ok(cudaMemcpy(pl->d_items, items.data(), sizeof(uint4) * items.size(),
                                               cudaMemcpyHostToDevice),
                                    "batch items upload")))
        return 0;
    // kernel parameters
    bparams P{};
    P.items = static_cast<const uint4 *>(pl->d_items);
    P.n_items = pl->n_items;
    P.ncand = pl->ncand;
    for (uint32_t k = 0; k < CS_BATCH_MAX_CANDIDATES; ++k) P.cand[k] = pl->cand[k];
    P.parts = static_cast<bpart *>(pl->d_parts);
    P.st.head = reinterpret_cast<uint32_t *>(st + sl.head);
    P.st.error = reinterpret_cast<uint32_t *>(st + sl.error);
    P.st.deferred = reinterpret_cast<uint32_t *>(st + sl.deferred);
    P.st.layout_done = reinterpret_cast<uint32_t *>(st + sl.layout_done);
    P.st.max_nnz = reinterpret_cast<uint32_t *>(st + sl.max_nnz);
    P.st.choose_done = reinterpret_cast<uint32_t *>(st + sl.choose_done);
    P.st.alloc_ready = reinterpret_cast<uint32_t *>(st + sl.alloc_ready);
    P.st.alloc_cursor = reinterpret_cast<unsigned long long *>(st + sl.alloc_cursor);
    P.st.widths = reinterpret_cast<uint32_t *>(st + sl.widths);
    P.results = pl->d_results;
    P.arena = pl->arena;
    P.arena_bytes = pl->arena_bytes;
    kernel_t k = kernel_for(pl->tiles.emit_lanes);
    int occ = 0;
    if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kBThreads, 0), "batch occupancy")) return 0;
    if (occ < 1) occ = 1;
    if (pl->tiles.ctas_per_sm != 0u && (int) pl->tiles.ctas_per_sm < occ) occ = (int) pl->tiles.ctas_per_sm;
    pl->ctas_per_sm = occ;
    pl->grid = (uint32_t) (occ * sm_count());
    if (pl->grid > pl->n_items && pl->n_items > 0u) pl->grid = pl->n_items;
    if (pl->grid == 0u) pl->grid = 1u;
    // graph: zero the wave state, then the persistent kernel
    if (pl->exec) cudaGraphExecDestroy(pl->exec);
    if (pl->graph) cudaGraphDestroy(pl->graph);
    pl->exec = nullptr;
    pl->graph = nullptr;
    if (!cuda_ok(cudaStreamBeginCapture(pl->cap_stream, cudaStreamCaptureModeThreadLocal), "batch capture begin"))
        return 0;
    cudaMemsetAsync(pl->d_state, 0, sl.bytes, pl->cap_stream);
    if (pl->n_items > 0u) k<<<pl->grid, kBThreads, 0, pl->cap_stream>>>(P);
    const cudaError_t le = cudaGetLastError();
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(pl->cap_stream, &g);
    if (!cuda_ok(le, "batch kernel capture") || !cuda_ok(ce, "batch capture end")) {
        if (g) cudaGraphDestroy(g);
        return 0;
    }
    pl->graph = g;
    if (!cuda_ok(cudaGraphInstantiate(&pl->exec, g, 0), "batch graph instantiate")) return 0;
    return 1;
}

std::mutex g_tune_mu;
std::map<std::tuple<uint32_t, uint64_t, uint64_t, uint32_t>, cs_batch_tiles> g_tune_cache;

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_batch_sliced_create(const cs_batch_part *parts, uint32_t count, const uint32_t *candidates,
                                           uint32_t candidate_count, void *d_arena, uint64_t arena_bytes,
                                           const cs_batch_tiles *tiles, cs_batch_plan **out) {
    if (out == nullptr || (count != 0u && parts == nullptr) || candidates == nullptr || candidate_count == 0u ||
        candidate_count > CS_BATCH_MAX_CANDIDATES) {
        set_error("batch_sliced_create: null argument or 1..%d candidates required", CS_BATCH_MAX_CANDIDATES);
        return 0;
    }
    *out = nullptr;
    for (uint32_t i = 0; i < count; ++i) {
        const cs_batch_part &p = parts[i];
        if (p.src.axis != CS_COMPRESSED_BY_ROW) {
            set_error("batch_sliced_create: partition %u is not row-compressed", i);
            return 0;
        }
        if (p.src.rows != 0u && p.src.majorPtr == nullptr) {
            set_error("batch_sliced_create: partition %u has no row pointers", i);
            return 0;
        }
        if (p.src.nnz != 0u && (p.src.minorIdx == nullptr || p.src.val == nullptr)) {
            set_error("batch_sliced_create: partition %u has no entries", i);
            return 0;
        }
        if (p.d_major_nnz != nullptr &&
            (p.d_sorted_nnz == nullptr || p.d_order == nullptr || p.d_bucket_offsets == nullptr)) {
            set_error("batch_sliced_create: partition %u plan outputs incomplete", i);
            return 0;
        }
    }
    for (uint32_t k = 0; k < candidate_count; ++k)
        if (candidates[k] == 0u) {
            set_error("batch_sliced_create: zero slice height candidate");
            return 0;
        }
    if (d_arena == nullptr || ((uintptr_t) d_arena & 255u) != 0u) {
        set_error("batch_sliced_create: arena must be a 256-byte aligned device pointer");
        return 0;
    }
    auto *pl = new cs_batch_plan();
    pl->count = count;
    pl->parts.assign(parts, parts + count);
    pl->ncand = candidate_count;
    for (uint32_t k = 0; k < candidate_count; ++k) pl->cand[k] = candidates[k];
    pl->arena = static_cast<unsigned char *>(d_arena);
    pl->arena_bytes = arena_bytes;
    pl->tiles = tiles != nullptr ? *tiles : default_tiles(pl->parts);
    if (!tiles_valid(pl->tiles)) {
        set_error("batch_sliced_create: invalid tiles (layout_rows multiple of 32, emit_lanes 4/8/16/32)");
        delete pl;
        return 0;
    }
    for (uint32_t i = 0; i < count; ++i) pl->wave.push_back(i);
    std::size_t rows_total = 0;
    for (const auto &p : pl->parts) rows_total += p.src.rows;
    cudaGetDevice(&pl->device);
    int ok = cuda_ok(cudaStreamCreateWithFlags(&pl->cap_stream, cudaStreamNonBlocking), "batch stream") &&
             cuda_ok(cudaMalloc(&pl->d_parts, sizeof(bpart) * (count ? count : 1u)), "batch parts") &&
             cuda_ok(cudaMalloc((void **) &pl->d_sort_tmp, (2u * rows_total + 4u) * 4u), "batch sort scratch") &&
             cuda_ok(cudaMalloc((void **) &pl->d_results, sizeof(cs_batch_sliced_result) * (count ? count : 1u)),
                     "batch results") &&
             cuda_ok(cudaMemset(pl->d_results, 0, sizeof(cs_batch_sliced_result) * (count ? count : 1u)),
                     "batch results clear");
    if (ok) ok = build_wave(pl);
    if (!ok) {
        cs_b200_batch_sliced_destroy(pl);
        return 0;
    }
    *out = pl;
    return 1;
}

extern "C" int cs_b200_batch_sliced_run(cs_batch_plan *plan, cs_stream_t s) {
    if (plan == nullptr || plan->exec == nullptr) {
        set_error("batch_sliced_run: no plan");
        return 0;
    }
    if (plan->wave.empty()) return 1;
    if (!cuda_ok(cudaGraphLaunch(plan->exec, as_stream(s)), "batch graph launch")) return 0;
    ++plan->launches;
    return 1;
}

extern "C" int cs_b200_batch_sliced_results(cs_batch_plan *plan, cs_batch_sliced_result *h_results,
                                            uint32_t *deferred, uint32_t *error_bits, cs_stream_t s) {
    if (plan == nullptr || h_results == nullptr) {
        set_error("batch_sliced_results: null argument");
        return 0;
    }
    cudaStream_t st = as_stream(s);
    uint32_t hdr[3] = {0u, 0u, 0u};
    if (!cuda_ok(cudaMemcpyAsync(h_results, plan->d_results, sizeof(cs_batch_sliced_result) * plan->count,
                                 cudaMemcpyDeviceToHost, st),
                 "batch results copy") ||
        !cuda_ok(cudaMemcpyAsync(hdr, plan->d_state, sizeof(hdr), cudaMemcpyDeviceToHost, st), "batch state copy") ||
        !cuda_ok(cudaStreamSynchronize(st), "batch results sync"))
        return 0;
    const state_layout sl = make_state_layout(plan->count, 0);
    uint32_t err = 0u, def = 0u;
    if (!cuda_ok(cudaMemcpy(&err, static_cast<unsigned char *>(plan->d_state) + sl.error, 4, cudaMemcpyDeviceToHost),
                 "batch error copy") ||
        !cuda_ok(cudaMemcpy(&def, static_cast<unsigned char *>(plan->d_state) + sl.deferred, 4,
                            cudaMemcpyDeviceToHost),
                 "batch deferred copy"))
        return 0;
    if (deferred) *deferred = def;
    if (error_bits) *error_bits = err;
    return 1;
}

extern "C" int cs_b200_batch_sliced_next_wave(cs_batch_plan *plan, void *d_arena, uint64_t arena_bytes,
                                              uint32_t *wave_size) {
    if (plan == nullptr || d_arena == nullptr || ((uintptr_t) d_arena & 255u) != 0u) {
        set_error("batch_sliced_next_wave: null plan or unaligned arena");
        return 0;
    }
    std::vector<cs_batch_sliced_result> r(plan->count ? plan->count : 1u);
    if (!cuda_ok(cudaMemcpy(r.data(), plan->d_results, sizeof(cs_batch_sliced_result) * plan->count,
                            cudaMemcpyDeviceToHost),
                 "batch results copy"))
        return 0;
    std::vector<uint32_t> next;
    for (uint32_t q : plan->wave)
        if (r[q].status & CS_BATCH_DEFERRED) next.push_back(q);
    plan->wave = next;
    plan->arena = static_cast<unsigned char *>(d_arena);
    plan->arena_bytes = arena_bytes;
    if (wave_size) *wave_size = (uint32_t) next.size();
    return build_wave(plan);
}

extern "C" int cs_b200_batch_sliced_reset(cs_batch_plan *plan, void *d_arena, uint64_t arena_bytes) {
    if (plan == nullptr || d_arena == nullptr || ((uintptr_t) d_arena & 255u) != 0u) {
        set_error("batch_sliced_reset: null plan or unaligned arena");
        return 0;
    }
    plan->wave.clear();
    for (uint32_t i = 0; i < plan->count; ++i) plan->wave.push_back(i);
    plan->arena = static_cast<unsigned char *>(d_arena);
    plan->arena_bytes = arena_bytes;
    return build_wave(plan);
}

extern "C" int cs_b200_batch_sliced_autotune(cs_batch_plan *plan, cs_stream_t s, cs_batch_tiles *chosen) {
    if (plan == nullptr) {
        set_error("batch_sliced_autotune: no plan");
        return 0;
    }
    uint64_t rows = 0, nnz = 0;
    for (const auto &p : plan->parts) {
        rows += p.src.rows;
        nnz += p.src.nnz;
    }
    const auto key = std::make_tuple(plan->count, rows, nnz, plan->cand[0]);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            plan->tiles = it->second;
            if (chosen) *chosen = plan->tiles;
            return build_wave(plan);
        }
    }
    cudaStream_t st = as_stream(s);
    const cs_batch_tiles base = default_tiles(plan->parts);
    std::vector<cs_batch_tiles> cands;
    const uint32_t lanes[3] = {32u, 16u, 8u};
    const uint32_t erows[3] = {128u, 512u, 2048u};
    for (uint32_t l : lanes)
        for (uint32_t e : erows) {
            cs_batch_tiles t = base;
            t.emit_lanes = l;
            t.emit_rows = e;
            cands.push_back(t);
        }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!cuda_ok(cudaEventCreate(&e0), "event") || !cuda_ok(cudaEventCreate(&e1), "event")) return 0;
    float best_ms = 0.0f;
    cs_batch_tiles best = base;
    bool have = false;
    int ok = 1;
    for (const auto &t : cands) {
        plan->tiles = t;
        if (!build_wave(plan)) {
            ok = 0;
            break;
        }
        // one warm-up, then the best of three
        float ms_min = 0.0f;
        for (int rep = 0; rep < 4 && ok; ++rep) {
            ok = cuda_ok(cudaEventRecord(e0, st), "event") && cuda_ok(cudaGraphLaunch(plan->exec, st), "tune launch") &&
                 cuda_ok(cudaEventRecord(e1, st), "event") && cuda_ok(cudaEventSynchronize(e1), "tune sync");
            float ms = 0.0f;
            if (ok) cudaEventElapsedTime(&ms, e0, e1);
            if (rep == 1 || (rep > 1 && ms < ms_min)) ms_min = ms;
        }
        if (!ok) break;
        if (!have || ms_min < best_ms) {
            have = true;
            best_ms = ms_min;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    plan->tiles = best;
    if (!ok) return 0;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = best;
    }
    if (chosen) *chosen = best;
    return build_wave(plan);
}

extern "C" int cs_b200_batch_sliced_tiles(const cs_batch_plan *plan, cs_batch_tiles *out, uint32_t *grid,
                                          uint32_t *items) {
    if (plan == nullptr || out == nullptr) {
        set_error("batch_sliced_tiles: null argument");
        return 0;
    }
    *out = plan->tiles;
    if (grid) *grid = plan->grid;
    if (items) *items = plan->n_items;
    return 1;
}

extern "C" void cs_b200_batch_sliced_destroy(cs_batch_plan *plan) {
    if (plan == nullptr) return;
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    if (plan->d_items) cudaFree(plan->d_items);
    if (plan->d_state) cudaFree(plan->d_state);
    if (plan->d_parts) cudaFree(plan->d_parts);
    if (plan->d_sort_tmp) cudaFree(plan->d_sort_tmp);
    if (plan->d_results) cudaFree(plan->d_results);
    if (plan->cap_stream) cudaStreamDestroy(plan->cap_stream);
    delete plan;
}
