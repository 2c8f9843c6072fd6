// Serving loop for masked grouped moments over staged Blocked-ELL partitions.
//
// A device-resident persistent kernel pulls work items from two rings in
// device memory: a device ring that the kernel itself appends to, and a host
// ring that the host scheduler appends request starts to with ordered copies
// (item, sequence word, tail) on a control stream.  Nothing the kernel polls
// lives in host memory: hundreds of resident CTAs polling over PCIe would
// starve the result copies.  Every
// request runs as a dataflow of items; the item that completes a stage
// appends the next stage's items, so no item ever waits for another:
//
//   START(q)            -> HIST(q, t) for every 8,192-row tile of the
//                          concatenated partitions
//   HIST(q, t)          per-group kept-row counts of the tile; the last one
//                          appends SCAN(q)
//   SCAN(q)             per group: scan over tiles, group offsets, chunks of
//                          <= chunk_rows rows of one group (a chunk may span
//                          partitions); appends SCATTER(q, t)
//   SCATTER(q, t)       stable placement of the tile's kept rows by group;
//                          the last one appends ACC(q, c, ft) for every chunk
//                          and feature tile
//   ACC(q, c, ft)       the chunk's rows, each from its own partition through
//                          that partition's column-block index, 8 features per
//                          thread, fp32 batch sums folded into two-sum pairs
//                          (as the single-partition moments kernel); feature
//                          groups the request masks out are not read
//   COMBINE(q, g, fb)   chunk partials of group g -> sum, sumsq, mean, var;
//                          the last one raises the request's done word
//
// Requests are admitted by the host scheduler when a slot and their scratch
// fit the HBM budget; the requests in flight share the persistent kernel, so
// their items interleave on the device.  A request's results depend only on
// its own masks and labels (chunking and summation orders are fixed by them),
// so a request gives the same bits alone and in any mix.
//
// The kernel exits after an idle period (bounded poll) or a stop request;
// the scheduler relaunches it when work is pending.  Queue waits are bounded.
#include "common.cuh"
#include "moments_device.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace csb {
int build_column_block_index(const cs_blocked_ell_view *src, uint2 *index, uint32_t *status, cudaStream_t stream);

namespace {

constexpr unsigned kSThreads = 256;
constexpr unsigned kSWarps = kSThreads / 32;
constexpr uint32_t kServeTile = 8192;        // rows per HIST / SCATTER tile
constexpr uint32_t kServeCombFeat = 2048;    // features per COMBINE item
constexpr uint32_t kServeMaxGroups = 1024;
constexpr uint32_t kServeMaxChunkRows = 2048;
constexpr uint32_t kServeBatch = 8;
constexpr uint32_t kSeqSpin = 1u << 22;
constexpr unsigned long long kDevRing = 1ull << 22;
constexpr unsigned long long kHostRing = 1ull << 14;
constexpr unsigned long long kOrphans = 1ull << 12;

enum : uint32_t { IT_START = 1u, IT_HIST, IT_SCAN, IT_SCATTER, IT_ACC, IT_COMBINE };

struct spart {
    uint32_t rows, ell_cols, row_base, pad;
    const uint16_t *val;
    const uint2 *index;
};

struct sreq {
    uint32_t G, scheme, ddof, chunk_rows;
    uint32_t max_chunks, pad0, pad1, pad2;
    const uint8_t *row_keep;
    const uint32_t *labels;
    const uint8_t *feature_keep;
    uint32_t *hist;          // [G * T] group-major
    uint32_t *group_rows;    // [G]
    uint32_t *group_offsets; // [G + 1]
    uint32_t *chunk_first;   // [G + 1]
    uint4 *chunks;           // [max_chunks] (group, begin, end, 0)
    uint32_t *n_chunks;      // [1]
    uint32_t *sorted_rows;   // [kept]
    float *partials;         // [max_chunks * 4 * cols]
    float *sum, *sumsq, *mean, *var;
    uint32_t *out_group_rows;
    uint32_t *counters;      // [4] hist, scatter, acc, combine
    uint32_t *done;          // mapped host word
};

struct squeue {
    unsigned long long *head; // device memory
    unsigned long long *tail; // device memory (device ring) or mapped host memory (host ring)
    uint4 *slots;
    unsigned long long *seq;
    unsigned long long mask;
};

struct sparams {
    const spart *parts;
    uint32_t nparts, total_rows, cols, block_size;
    uint32_t col_blocks, words, tiles, pad;
    sreq *reqs;
    squeue dq, hq;
    const volatile uint32_t *stop; // device memory, written by the host at close
    uint32_t *error;
    unsigned long long idle_ns;
    unsigned long long *prof; // [16]: items per kind [0..7], device ns per kind [8..15]
    unsigned long long *orph_head, *orph_tail; // tickets left by CTAs that exited on idle
    unsigned long long *orph, *orph_seq;       // [kOrphans]
    uint32_t *idle_ctas;                       // CTAs of this launch waiting for work
    uint32_t *closing;                         // set once every CTA was idle: all exit
};

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned long long ld_acq_gpu64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acq_sys64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_rel_gpu64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_rel_sys32(uint32_t *p, uint32_t v) {
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint4 ld_volatile_v4(const uint4 *p) {
    uint4 v;
    asm volatile("ld.volatile.global.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

// one thread: claim the next item of q, if any
__device__ bool try_pop(const squeue &q, bool host_ring, uint4 &item, uint32_t *error) {
    const unsigned long long h = ld_acq_gpu64(q.head);
    const unsigned long long t = host_ring ? ld_acq_sys64(q.tail) : ld_acq_gpu64(q.tail);
    if (h >= t) return false;
    if (atomicCAS(q.head, h, h + 1ull) != h) return false;
    const unsigned long long slot = h & q.mask;
    for (uint32_t it = 0; it < kSeqSpin; ++it) {
        const unsigned long long s = host_ring ? ld_acq_sys64(q.seq + slot) : ld_acq_gpu64(q.seq + slot);
        if (s == h + 1ull) {
            item = ld_volatile_v4(q.slots + slot);
            return true;
        }
        __nanosleep(64);
    }
    atomicOr(error, 1u); // the producer of a claimed slot never published it
    return false;
}

// cooperative append of n items produced by gen(i); all threads of the CTA
// call it; base reserved by thread 0
template <class Gen>
__device__ void push_items(const squeue &q, uint32_t n, Gen gen, unsigned long long *sbase) {
    if (n == 0u) return;
    if (threadIdx.x == 0) *sbase = atomicAdd(q.tail, (unsigned long long) n);
    __syncthreads();
    const unsigned long long base = *sbase;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long k = base + i;
        q.slots[k & q.mask] = gen(i);
        __threadfence();
        st_rel_gpu64(q.seq + (k & q.mask), k + 1ull);
    }
    __syncthreads();
}

// The kernel outlives requests and the scratch pool is reused, so request
// data (descriptors, masks, labels, intermediate arrays) is read through L2
// (ld.cg); only the staged partitions, fixed for the server's lifetime, use
// the read-only path.
struct ssmem {
    sreq req;
    uint4 item;
    uint32_t flag;
    uint32_t last;
    unsigned long long base;
    uint32_t scan33[33];
    uint32_t u[4];
};

__device__ __forceinline__ uint32_t req_group(const sreq &R, uint32_t r, uint32_t total_rows) {
    if (r >= total_rows) return 0xffffffffu;
    if (R.row_keep != nullptr && __ldcg(R.row_keep + r) == 0u) return 0xffffffffu;
    const uint32_t g = R.labels != nullptr ? __ldcg(R.labels + r) : 0u;
    return g < R.G ? g : 0xffffffffu;
}

// counter increment after the CTA's writes; returns (to all threads) whether
// this CTA completed the stage
__device__ bool stage_done(uint32_t *counter, uint32_t total, ssmem &sm) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t old = atomicAdd(counter, 1u);
        sm.last = (old + 1u == total) ? 1u : 0u;
        if (sm.last) __threadfence();
    }
    __syncthreads();
    return sm.last != 0u;
}

__device__ void do_start(const sparams &P, ssmem &sm, uint32_t q) {
    push_items(P.dq, P.tiles, [&](uint32_t t) { return make_uint4(IT_HIST | (q << 8), t, 0u, 0u); }, &sm.base);
}

__device__ void do_hist(const sparams &P, ssmem &sm, uint32_t *dyn, uint32_t q, uint32_t t) {
    const sreq &R = sm.req;
    const uint32_t G = R.G;
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) dyn[g] = 0u;
    __syncthreads();
    const uint32_t base = t * kServeTile;
    for (uint32_t i = threadIdx.x; i < kServeTile; i += blockDim.x) {
        const uint32_t g = req_group(R, base + i, P.total_rows);
        if (g != 0xffffffffu) atomicAdd(dyn + g, 1u);
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) R.hist[(std::size_t) g * P.tiles + t] = dyn[g];
    if (stage_done(R.counters + 0, P.tiles, sm))
        push_items(P.dq, 1u, [&](uint32_t) { return make_uint4(IT_SCAN | (q << 8), 0u, 0u, 0u); }, &sm.base);
}

__device__ void do_scan(const sparams &P, ssmem &sm, uint32_t q) {
    const sreq &R = sm.req;
    const uint32_t G = R.G, T = P.tiles;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t g = warp; g < G; g += kSWarps) {
        uint32_t carry = 0u;
        uint32_t *h = R.hist + (std::size_t) g * T;
        for (uint32_t t0 = 0; t0 < T; t0 += 32u) {
            const uint32_t t = t0 + lane;
            const uint32_t c = t < T ? __ldcg(h + t) : 0u;
            const uint32_t incl = warp_inclusive_scan(c);
            if (t < T) h[t] = carry + incl - c;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0u) R.group_rows[g] = carry;
    }
    __syncthreads();
    uint32_t carry_rows = 0u, carry_chunks = 0u;
    const uint32_t cr = R.chunk_rows;
    for (uint32_t g0 = 0; g0 < G; g0 += blockDim.x) {
        const uint32_t g = g0 + threadIdx.x;
        const uint32_t n = g < G ? __ldcg(R.group_rows + g) : 0u;
        const uint32_t nc = g < G ? (n + cr - 1u) / cr : 0u;
        uint32_t tot_n, tot_c;
        const uint32_t ex_n = block_exclusive_scan(n, sm.scan33, tot_n);
        const uint32_t ex_c = block_exclusive_scan(nc, sm.scan33, tot_c);
        if (g < G) {
            const uint32_t off = carry_rows + ex_n, cf = carry_chunks + ex_c;
            R.group_offsets[g] = off;
            R.chunk_first[g] = cf;
            for (uint32_t c = 0; c < nc; ++c) {
                const uint32_t b = off + c * cr;
                const uint32_t e = (c + 1u == nc) ? off + n : b + cr;
                if (cf + c < R.max_chunks) R.chunks[cf + c] = make_uint4(g, b, e, 0u);
            }
        }
        carry_rows += tot_n;
        carry_chunks += tot_c;
    }
    if (threadIdx.x == 0) {
        R.group_offsets[G] = carry_rows;
        R.chunk_first[G] = carry_chunks;
        *R.n_chunks = carry_chunks;
        if (carry_chunks > R.max_chunks) atomicOr(P.error, 2u);
        __threadfence();
    }
    __syncthreads();
    push_items(P.dq, T, [&](uint32_t t) { return make_uint4(IT_SCATTER | (q << 8), t, 0u, 0u); }, &sm.base);
}

__device__ void push_combine(const sparams &P, ssmem &sm, uint32_t q, const sreq &R) {
    const uint32_t fb = (P.cols + kServeCombFeat - 1u) / kServeCombFeat;
    const uint32_t n = R.G * (fb == 0u ? 1u : fb);
    push_items(P.dq, n, [&](uint32_t i) {
        return make_uint4(IT_COMBINE | (q << 8), i / (fb == 0u ? 1u : fb), i % (fb == 0u ? 1u : fb), 0u);
    }, &sm.base);
}

__device__ void do_scatter(const sparams &P, ssmem &sm, uint32_t *dyn, uint32_t q, uint32_t t) {
    const sreq &R = sm.req;
    const uint32_t G = R.G, T = P.tiles;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t i = threadIdx.x; i < kSWarps * G; i += blockDim.x) dyn[i] = 0u;
    __syncthreads();
    constexpr uint32_t per_warp = kServeTile / kSWarps;
    const uint32_t wbase = t * kServeTile + warp * per_warp;
    uint32_t *my = dyn + (std::size_t) warp * G;
    for (uint32_t b = 0; b < per_warp; b += 32u) {
        const uint32_t g = req_group(R, wbase + b + lane, P.total_rows);
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        if (g != 0xffffffffu && lane == (unsigned) (__ffs(peers) - 1)) my[g] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
        uint32_t run = __ldcg(R.hist + (std::size_t) g * T + t) + __ldcg(R.group_offsets + g);
        for (unsigned w = 0; w < kSWarps; ++w) {
            const uint32_t c = dyn[(std::size_t) w * G + g];
            dyn[(std::size_t) w * G + g] = run;
            run += c;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t b = 0; b < per_warp; b += 32u) {
        const uint32_t r = wbase + b + lane;
        const uint32_t g = req_group(R, r, P.total_rows);
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        uint32_t base = 0u;
        if (g != 0xffffffffu) base = my[g];
        __syncwarp();
        if (g != 0xffffffffu) {
            R.sorted_rows[base + __popc(peers & lt)] = r;
            if (lane == (unsigned) (__ffs(peers) - 1)) my[g] = base + __popc(peers);
        }
        __syncwarp();
    }
    if (stage_done(R.counters + 1, T, sm)) {
        const uint32_t nc = min(__ldcg(R.n_chunks), R.max_chunks);
        if (nc == 0u) {
            push_combine(P, sm, q, R);
        } else {
            const uint32_t segs = P.col_blocks * (P.block_size / 8u);
            const uint32_t ft = (segs + kSThreads - 1u) / kSThreads;
            push_items(P.dq, nc * ft, [&](uint32_t i) { return make_uint4(IT_ACC | (q << 8), i / ft, i % ft, 0u); },
                       &sm.base);
        }
    }
}

template <bool COMP>
__device__ void acc_body(const sparams &P, const ulonglong2 *rows, uint32_t n, uint32_t b, uint32_t part,
                         float *out, std::size_t cols) {
    constexpr int L = 8;
    const uint32_t B = P.block_size;
    const uint32_t w = b >> 5;
    const uint32_t below = (1u << (b & 31u)) - 1u;
    const uint32_t bitmask = 1u << (b & 31u);
    const std::size_t lane_off = (std::size_t) part * L;
    float s_hi[L], s_lo[L], q_hi[L], q_lo[L];
#pragma unroll
    for (int j = 0; j < L; ++j) s_hi[j] = s_lo[j] = q_hi[j] = q_lo[j] = 0.0f;
    uint2 e_next[kServeBatch];
#pragma unroll
    for (unsigned u = 0; u < kServeBatch; ++u)
        e_next[u] = u < n ? __ldg(reinterpret_cast<const uint2 *>(rows[u].y) + w) : make_uint2(0u, 0u);
    uint32_t i = 0;
    for (; i + kServeBatch <= n; i += kServeBatch) {
        raw_vec<L> raw[kServeBatch];
#pragma unroll
        for (unsigned u = 0; u < kServeBatch; ++u) {
            const uint2 e = e_next[u];
            if (e.x & bitmask) {
                const uint32_t slot = e.y + __popc(e.x & below);
                load_raw<L>(reinterpret_cast<const uint16_t *>(rows[i + u].x) + (std::size_t) slot * B + lane_off,
                            raw[u]);
            } else {
                zero_raw<L>(raw[u]);
            }
        }
#pragma unroll
        for (unsigned u = 0; u < kServeBatch; ++u) {
            const uint32_t k = i + kServeBatch + u;
            e_next[u] = k < n ? __ldg(reinterpret_cast<const uint2 *>(rows[k].y) + w) : make_uint2(0u, 0u);
        }
        if (COMP) {
            float bs[L], bq[L];
#pragma unroll
            for (int j = 0; j < L; ++j) bs[j] = bq[j] = 0.0f;
#pragma unroll
            for (unsigned u = 0; u < kServeBatch; ++u) {
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
            for (unsigned u = 0; u < kServeBatch; ++u) {
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
#pragma unroll
    for (unsigned u = 0; u < kServeBatch; ++u) {
        if (i + u < n) {
            const uint2 e = e_next[u];
            if (e.x & bitmask) {
                raw_vec<L> raw;
                const uint32_t slot = e.y + __popc(e.x & below);
                load_raw<L>(reinterpret_cast<const uint16_t *>(rows[i + u].x) + (std::size_t) slot * B + lane_off, raw);
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
    const std::size_t f0 = (std::size_t) b * B + lane_off;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const std::size_t f = f0 + j;
        if (f < cols) {
            out[f] = s_hi[j];
            out[cols + f] = s_lo[j];
            out[2u * cols + f] = q_hi[j];
            out[3u * cols + f] = q_lo[j];
        }
    }
}

__device__ void do_acc(const sparams &P, ssmem &sm, ulonglong2 *rows, uint32_t q, uint32_t c, uint32_t ft) {
    const sreq &R = sm.req;
    const uint4 d = __ldcg(R.chunks + c);
    const uint32_t n = min(d.z - d.y, kServeMaxChunkRows);
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t r = __ldcg(R.sorted_rows + d.y + i);
        // partition of global row r: last p with row_base <= r
        uint32_t lo = 0u, hi = P.nparts - 1u;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (P.parts[mid].row_base <= r)
                lo = mid;
            else
                hi = mid - 1u;
        }
        const spart &sp = P.parts[lo];
        const uint32_t lr = r - sp.row_base;
        rows[i] = make_ulonglong2((unsigned long long) (sp.val + (std::size_t) lr * sp.ell_cols),
                                  (unsigned long long) (sp.index + (std::size_t) (lr / P.block_size) * P.words));
    }
    __syncthreads();
    const uint32_t segs_per_block = P.block_size / 8u;
    const uint32_t seg = ft * kSThreads + threadIdx.x;
    const uint32_t b = seg / segs_per_block;
    const uint32_t part = seg - b * segs_per_block;
    float *out = R.partials + (std::size_t) c * 4u * P.cols;
    if (b < P.col_blocks) {
        bool any = true;
        if (R.feature_keep != nullptr) {
            any = false;
            const uint32_t f0 = b * P.block_size + part * 8u;
            for (uint32_t j = 0; j < 8u && f0 + j < P.cols; ++j) any |= __ldcg(R.feature_keep + f0 + j) != 0u;
        }
        if (any) {
            if (R.scheme != CS_MOMENTS_PLAIN_F32)
                acc_body<true>(P, rows, n, b, part, out, P.cols);
            else
                acc_body<false>(P, rows, n, b, part, out, P.cols);
        }
    }
    const uint32_t segs = P.col_blocks * segs_per_block;
    const uint32_t fts = (segs + kSThreads - 1u) / kSThreads;
    const uint32_t nc = min(__ldcg(R.n_chunks), R.max_chunks);
    if (stage_done(R.counters + 2, nc * fts, sm)) push_combine(P, sm, q, R);
}

__device__ void do_combine(const sparams &P, ssmem &sm, uint32_t q, uint32_t g, uint32_t fb) {
    const sreq &R = sm.req;
    const uint32_t cols = P.cols;
    const uint32_t c0 = min(__ldcg(R.chunk_first + g), R.max_chunks);
    const uint32_t c1 = min(__ldcg(R.chunk_first + g + 1u), R.max_chunks);
    const uint32_t n = __ldcg(R.group_rows + g);
    if (fb == 0u && threadIdx.x == 0 && R.out_group_rows != nullptr) R.out_group_rows[g] = n;
    for (uint32_t f = fb * kServeCombFeat + threadIdx.x; f < min(cols, (fb + 1u) * kServeCombFeat); f += blockDim.x) {
        const bool kept = R.feature_keep == nullptr || __ldcg(R.feature_keep + f) != 0u;
        const std::size_t o = (std::size_t) g * cols + f;
        float rs = 0.0f, rq = 0.0f, rm = 0.0f, rv = 0.0f;
        if (kept) {
            if (R.scheme == CS_MOMENTS_TWOSUM_F64_COMBINE) {
                double s = 0.0, qq = 0.0;
                for (uint32_t c = c0; c < c1; ++c) {
                    const float *p = R.partials + (std::size_t) c * 4u * cols;
                    s += (double) __ldcg(p + f) + (double) __ldcg(p + cols + f);
                    qq += (double) __ldcg(p + 2u * (std::size_t) cols + f) +
                          (double) __ldcg(p + 3u * (std::size_t) cols + f);
                }
                rs = (float) s;
                rq = (float) qq;
                if (n > 0u) {
                    const double dm = s / (double) n;
                    double dv = 0.0;
                    if (n > R.ddof) {
                        double m2 = qq - s * dm;
                        if (m2 < 0.0) m2 = 0.0;
                        dv = m2 / (double) (n - R.ddof);
                    }
                    rm = (float) dm;
                    rv = (float) dv;
                }
            } else {
                float s_hi = 0.0f, s_lo = 0.0f, q_hi = 0.0f, q_lo = 0.0f;
                for (uint32_t c = c0; c < c1; ++c) {
                    const float *p = R.partials + (std::size_t) c * 4u * cols;
                    if (R.scheme == CS_MOMENTS_TWOSUM_F32) {
                        two_sum_acc(s_hi, s_lo, __ldcg(p + f));
                        s_lo = __fadd_rn(s_lo, __ldcg(p + cols + f));
                        two_sum_acc(q_hi, q_lo, __ldcg(p + 2u * (std::size_t) cols + f));
                        q_lo = __fadd_rn(q_lo, __ldcg(p + 3u * (std::size_t) cols + f));
                    } else {
                        s_hi = __fadd_rn(s_hi, __ldcg(p + f));
                        q_hi = __fadd_rn(q_hi, __ldcg(p + 2u * (std::size_t) cols + f));
                    }
                }
                rs = __fadd_rn(s_hi, s_lo);
                rq = __fadd_rn(q_hi, q_lo);
                if (n > 0u) {
                    rm = __fdiv_rn(rs, (float) n);
                    if (n > R.ddof) {
                        float m2 = __fsub_rn(rq, __fmul_rn(rs, rm));
                        if (m2 < 0.0f) m2 = 0.0f;
                        rv = __fdiv_rn(m2, (float) (n - R.ddof));
                    }
                }
            }
        }
        R.sum[o] = rs;
        R.sumsq[o] = rq;
        if (R.mean != nullptr) R.mean[o] = rm;
        if (R.var != nullptr) R.var[o] = rv;
    }
    const uint32_t fbs = (cols + kServeCombFeat - 1u) / kServeCombFeat;
    if (stage_done(R.counters + 3, R.G * (fbs == 0u ? 1u : fbs), sm) && threadIdx.x == 0) {
        __threadfence_system();
        st_rel_sys32(R.done, 1u);
    }
}

// one thread: take a ticket left by an exited CTA, if any
__device__ bool claim_orphan(const sparams &P, unsigned long long &ticket) {
    // retry until one is taken or none is left, so a launch's CTAs hold every
    // orphaned ticket before any of them takes a fresh one
    unsigned long long h = ld_acq_gpu64(P.orph_head);
    while (true) {
        if (h >= ld_acq_gpu64(P.orph_tail)) return false;
        const unsigned long long seen = atomicCAS(P.orph_head, h, h + 1ull);
        if (seen == h) break;
        h = seen;
    }
    const unsigned long long slot = h & (kOrphans - 1ull);
    for (uint32_t it = 0; it < kSeqSpin; ++it) {
        if (ld_acq_gpu64(P.orph_seq + slot) == h + 1ull) {
            ticket = __ldcg(P.orph + slot);
            return true;
        }
        __nanosleep(64);
    }
    atomicOr(P.error, 8u); // an exiting CTA reserved an orphan slot and never filled it
    return false;
}

__global__ void __launch_bounds__(kSThreads, 2) serve_kernel(sparams P) {
    extern __shared__ __align__(16) unsigned char serve_dyn[];
    __shared__ ssmem sm;
    // Device-ring items are taken by ticket: a CTA takes the next ring index
    // with one atomicAdd (no compare-and-swap race between hundreds of CTAs)
    // and waits for that slot's sequence word; tickets may run ahead of the
    // tail, so waiting CTAs are served in order as items are appended.  The
    // host ring (request starts only) is polled by compare-and-swap while a
    // CTA waits on its ticket.  Exit is all-or-nothing: a CTA leaves only
    // once every CTA of the launch has been idle for idle_ns (then it raises
    // `closing` and the others follow), or on stop, or after a hard bound of
    // 8 x idle_ns; its unfilled ticket goes to the orphan ring, which the next
    // launch's CTAs drain before taking fresh tickets, so no item is lost.
    unsigned long long idle_since = 0ull, ticket = 0ull;
    bool have_ticket = false;
    while (true) {
        if (threadIdx.x == 0) {
            uint4 it = make_uint4(0u, 0u, 0u, 0u);
            bool got = false;
            if (!have_ticket) {
                if (!claim_orphan(P, ticket)) ticket = atomicAdd(P.dq.head, 1ull);
                have_ticket = true;
            }
            atomicAdd(P.idle_ctas, 1u);
            while (true) {
                const unsigned long long slot = ticket & P.dq.mask;
                if (ld_acq_gpu64(P.dq.seq + slot) == ticket + 1ull) {
                    it = ld_volatile_v4(P.dq.slots + slot);
                    have_ticket = false;
                    got = true;
                    break;
                }
                if (try_pop(P.hq, true, it, P.error)) {
                    got = true;
                    break;
                }
                const unsigned long long now = globaltimer();
                if (idle_since == 0ull) idle_since = now;
                const unsigned long long idle = now - idle_since;
                bool leave = *P.stop != 0u || *reinterpret_cast<volatile uint32_t *>(P.closing) != 0u ||
                             idle > 8ull * P.idle_ns;
                if (!leave && idle > P.idle_ns &&
                    *reinterpret_cast<volatile uint32_t *>(P.idle_ctas) >= gridDim.x) {
                    atomicExch(P.closing, 1u);
                    leave = true;
                }
                if (leave) {
                    const unsigned long long k = atomicAdd(P.orph_tail, 1ull);
                    P.orph[k & (kOrphans - 1ull)] = ticket;
                    __threadfence();
                    st_rel_gpu64(P.orph_seq + (k & (kOrphans - 1ull)), k + 1ull);
                    have_ticket = false;
                    break;
                }
                __nanosleep(200);
            }
            if (got) {
                atomicSub(P.idle_ctas, 1u);
                idle_since = 0ull;
            }
            sm.item = got ? it : make_uint4(0u, 0u, 0u, 0u);
        }
        __syncthreads();
        const uint4 it = sm.item;
        __syncthreads();
        const uint32_t kind = it.x & 255u, q = it.x >> 8;
        if (kind == 0u) break;
        static_assert(sizeof(sreq) % 16u == 0u, "sreq copies as uint4");
        if (threadIdx.x < sizeof(sreq) / 16u)
            reinterpret_cast<uint4 *>(&sm.req)[threadIdx.x] = __ldcg(reinterpret_cast<const uint4 *>(P.reqs + q) +
                                                                       threadIdx.x);
        __syncthreads();
        const unsigned long long t_item = threadIdx.x == 0 ? globaltimer() : 0ull;
        switch (kind) {
        case IT_START: do_start(P, sm, q); break;
        case IT_HIST: do_hist(P, sm, reinterpret_cast<uint32_t *>(serve_dyn), q, it.y); break;
        case IT_SCAN: do_scan(P, sm, q); break;
        case IT_SCATTER: do_scatter(P, sm, reinterpret_cast<uint32_t *>(serve_dyn), q, it.y); break;
        case IT_ACC: do_acc(P, sm, reinterpret_cast<ulonglong2 *>(serve_dyn), q, it.y, it.z); break;
        case IT_COMBINE: do_combine(P, sm, q, it.y, it.z); break;
        default: atomicOr(P.error, 4u); break;
        }
        __syncthreads();
        if (threadIdx.x == 0 && kind < 8u) {
            atomicAdd(P.prof + kind, 1ull);
            atomicAdd(P.prof + 8u + kind, globaltimer() - t_item);
        }
    }
}

constexpr std::size_t kServeDynSmem =
    (kSWarps * kServeMaxGroups * 4u > kServeMaxChunkRows * 16u) ? kSWarps * kServeMaxGroups * 4u
                                                               : kServeMaxChunkRows * 16u;

std::size_t align256(std::size_t x) { return (x + 255u) / 256u * 256u; }

} // namespace
} // namespace csb

using namespace csb;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

using clk = std::chrono::steady_clock;

enum slot_state { SLOT_FREE = 0, SLOT_COPY_IN, SLOT_RUNNING, SLOT_COPY_OUT };

struct ticket_rec {
    cs_serve_request req;
    uint64_t need = 0;
    uint32_t max_chunks = 0;
    uint32_t state = CS_SERVE_QUEUED;
    uint32_t status = 0;
    clk::time_point t_submit, t_admit, t_start, t_device_done, t_done;
};

struct slot_rec {
    slot_state state = SLOT_FREE;
    uint64_t ticket = 0;
    uint64_t off = 0, bytes = 0;
    cudaEvent_t ev = nullptr;
    float *d_sum = nullptr, *d_sumsq = nullptr, *d_mean = nullptr, *d_var = nullptr;
    uint32_t *d_group_rows = nullptr;
};

} // namespace

struct cs_server {
    int device = 0;
    cs_serve_config cfg{};
    uint32_t nparts = 0, total_rows = 0, cols = 0, block_size = 0, col_blocks = 0, words = 0, tiles = 0;
    std::vector<spart> hparts;
    spart *d_parts = nullptr;
    std::vector<uint2 *> d_index;
    cudaStream_t kstream = nullptr, cstream = nullptr;
    cudaEvent_t kdone = nullptr;
    bool kernel_launched = false;
    uint32_t grid = 0;
    // pool
    unsigned char *pool = nullptr;
    uint64_t pool_bytes = 0;
    std::map<uint64_t, uint64_t> free_blocks; // offset -> size
    uint64_t pool_used = 0;
    // slots
    std::vector<slot_rec> slots;
    sreq *d_reqs = nullptr;
    sreq *h_reqs = nullptr;       // pinned staging
    uint32_t *h_done = nullptr;   // mapped
    uint32_t *d_done = nullptr;
    uint32_t *h_zero = nullptr;   // pinned zeros
    // rings
    unsigned long long *d_heads = nullptr; // [0] device ring head, [1] tail, [2] host ring head, [3..4] orphans,
                                           // [5] idle CTAs, [6] closing
    uint4 *d_dslots = nullptr;
    unsigned long long *d_dseq = nullptr;
    uint4 *d_hslots = nullptr;             // host ring in device memory
    unsigned long long *d_hseq = nullptr;
    unsigned long long *d_htail = nullptr; // [0] tail, [1] stop word
    unsigned char *h_push = nullptr;       // pinned staging of host-ring writes (32 B per slot)
    cudaStream_t pstream = nullptr;        // control stream for host-ring writes
    unsigned long long *d_prof = nullptr;
    unsigned long long *d_orph = nullptr; // [2 * kOrphans]: tickets, sequence words
    uint32_t *d_error = nullptr;
    unsigned long long host_tail = 0;
    // requests
    std::mutex mu;
    std::condition_variable cv;
    std::deque<uint64_t> pending;
    std::map<uint64_t, ticket_rec> tickets;
    uint64_t next_ticket = 1;
    uint64_t completed = 0, admitted = 0, kernel_launches = 0;
    uint64_t outstanding_items = 0;
    std::thread sched;
    std::atomic<bool> quit{false};
    std::string sched_error;
};

namespace {

bool pool_alloc(cs_server *s, uint64_t bytes, uint64_t *off) {
    for (auto it = s->free_blocks.begin(); it != s->free_blocks.end(); ++it) {
        if (it->second >= bytes) {
            *off = it->first;
            const uint64_t rest = it->second - bytes;
            const uint64_t roff = it->first + bytes;
            s->free_blocks.erase(it);
            if (rest) s->free_blocks[roff] = rest;
            s->pool_used += bytes;
            return true;
        }
    }
    return false;
}

void pool_free(cs_server *s, uint64_t off, uint64_t bytes) {
    s->pool_used -= bytes;
    auto it = s->free_blocks.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != s->free_blocks.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        s->free_blocks.erase(nx);
    }
    if (it != s->free_blocks.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            s->free_blocks.erase(it);
        }
    }
}

struct req_layout {
    uint64_t in_keep, in_labels, in_fk, hist, group_rows, group_offsets, chunk_first, chunks, n_chunks, sorted,
        partials, out_sum, out_sumsq, out_mean, out_var, out_group_rows, counters, bytes;
};

req_layout layout_for(const cs_server *s, const cs_serve_request &r, uint32_t max_chunks, uint64_t kept) {
    req_layout L{};
    uint64_t o = 0;
    auto take = [&](uint64_t bytes) {
        const uint64_t at = o;
        o = align256(o + (bytes ? bytes : 1));
        return at;
    };
    const bool host_in = (r.flags & CS_SERVE_DEVICE_INPUTS) == 0u;
    const uint64_t G = r.group_count, C = s->cols, R = s->total_rows;
    L.in_keep = host_in && r.row_keep ? take(R) : 0;
    L.in_labels = host_in && r.row_labels ? take(R * 4u) : 0;
    L.in_fk = host_in && r.feature_keep ? take(C) : 0;
    L.hist = take(G * s->tiles * 4u);
    L.group_rows = take(G * 4u);
    L.group_offsets = take((G + 1u) * 4u);
    L.chunk_first = take((G + 1u) * 4u);
    L.chunks = take((uint64_t) max_chunks * 16u);
    L.n_chunks = take(4);
    L.sorted = take((kept + 1u) * 4u);
    L.partials = take((uint64_t) max_chunks * 4u * C * 4u);
    L.out_sum = take(G * C * 4u);
    L.out_sumsq = take(G * C * 4u);
    L.out_mean = r.mean ? take(G * C * 4u) : 0;
    L.out_var = r.var ? take(G * C * 4u) : 0;
    L.out_group_rows = take(G * 4u);
    L.counters = take(16);
    L.bytes = o;
    return L;
}

uint64_t items_for(const cs_server *s, uint32_t G, uint32_t max_chunks) {
    const uint64_t segs = (uint64_t) s->col_blocks * (s->block_size / 8u);
    const uint64_t ft = (segs + kSThreads - 1u) / kSThreads;
    const uint64_t fb = (s->cols + kServeCombFeat - 1u) / kServeCombFeat;
    return 2u * s->tiles + 2u + (uint64_t) max_chunks * ft + (uint64_t) G * (fb ? fb : 1u);
}

bool launch_kernel(cs_server *s) {
    sparams P{};
    P.parts = s->d_parts;
    P.nparts = s->nparts;
    P.total_rows = s->total_rows;
    P.cols = s->cols;
    P.block_size = s->block_size;
    P.col_blocks = s->col_blocks;
    P.words = s->words;
    P.tiles = s->tiles;
    P.reqs = s->d_reqs;
    P.dq = squeue{s->d_heads + 0, s->d_heads + 1, s->d_dslots, s->d_dseq, kDevRing - 1ull};
    P.hq = squeue{s->d_heads + 2, s->d_htail, s->d_hslots, s->d_hseq, kHostRing - 1ull};
    P.stop = reinterpret_cast<const volatile uint32_t *>(s->d_htail + 1);
    P.prof = s->d_prof;
    P.orph_head = s->d_heads + 3;
    P.orph_tail = s->d_heads + 4;
    P.orph = s->d_orph;
    P.orph_seq = s->d_orph + kOrphans;
    P.idle_ctas = reinterpret_cast<uint32_t *>(s->d_heads + 5);
    P.closing = reinterpret_cast<uint32_t *>(s->d_heads + 6);
    // a new launch starts with no idle CTAs and no exit in progress
    cudaMemcpyAsync(s->d_heads + 5, s->h_zero, 16, cudaMemcpyHostToDevice, s->kstream);
    P.error = s->d_error;
    P.idle_ns = (unsigned long long) (s->cfg.idle_exit_us ? s->cfg.idle_exit_us : 20000u) * 1000ull;
    serve_kernel<<<s->grid, kSThreads, kServeDynSmem, s->kstream>>>(P);
    if (cudaGetLastError() != cudaSuccess) return false;
    cudaEventRecord(s->kdone, s->kstream);
    s->kernel_launched = true;
    ++s->kernel_launches;
    return true;
}

bool kernel_running(cs_server *s) { return s->kernel_launched && cudaEventQuery(s->kdone) == cudaErrorNotReady; }

// item, then its sequence word, then the tail: three copies in stream order,
// each complete before the next starts, so a consumer that sees the tail sees
// the item.  The staging slot is reused only kHostRing pushes later.
void push_host_item(cs_server *s, uint4 item) {
    const unsigned long long k = s->host_tail;
    const unsigned long long slot = k & (kHostRing - 1ull);
    unsigned char *st = s->h_push + slot * 32u;
    std::memcpy(st, &item, 16);
    const unsigned long long seq = k + 1ull;
    std::memcpy(st + 16, &seq, 8);
    std::memcpy(st + 24, &seq, 8);
    cudaMemcpyAsync(s->d_hslots + slot, st, 16, cudaMemcpyHostToDevice, s->pstream);
    cudaMemcpyAsync(s->d_hseq + slot, st + 16, 8, cudaMemcpyHostToDevice, s->pstream);
    cudaMemcpyAsync(s->d_htail, st + 24, 8, cudaMemcpyHostToDevice, s->pstream);
    s->host_tail = seq;
}

// admission of the queue head; returns false when it does not fit now
bool try_admit(cs_server *s, uint64_t ticket) {
    ticket_rec &t = s->tickets[ticket];
    int slot = -1;
    for (size_t i = 0; i < s->slots.size(); ++i)
        if (s->slots[i].state == SLOT_FREE) {
            slot = (int) i;
            break;
        }
    if (slot < 0) return false;
    if (s->outstanding_items + items_for(s, t.req.group_count, t.max_chunks) > kDevRing / 2) return false;
    uint64_t off = 0;
    if (!pool_alloc(s, t.need, &off)) return false;
    slot_rec &sr = s->slots[slot];
    sr.state = SLOT_COPY_IN;
    sr.ticket = ticket;
    sr.off = off;
    sr.bytes = t.need;
    s->outstanding_items += items_for(s, t.req.group_count, t.max_chunks);
    const cs_serve_request &r = t.req;
    uint64_t kept = s->total_rows;
    const req_layout L = layout_for(s, r, t.max_chunks, kept);
    unsigned char *b = s->pool + off;
    const bool host_in = (r.flags & CS_SERVE_DEVICE_INPUTS) == 0u;
    sreq &q = s->h_reqs[slot];
    std::memset(&q, 0, sizeof(q));
    q.G = r.group_count;
    q.scheme = r.scheme;
    q.ddof = r.ddof;
    q.chunk_rows = s->cfg.chunk_rows;
    q.max_chunks = t.max_chunks;
    q.row_keep = r.row_keep ? (host_in ? b + L.in_keep : r.row_keep) : nullptr;
    q.labels = r.row_labels ? (host_in ? reinterpret_cast<const uint32_t *>(b + L.in_labels) : r.row_labels) : nullptr;
    q.feature_keep = r.feature_keep ? (host_in ? b + L.in_fk : r.feature_keep) : nullptr;
    q.hist = reinterpret_cast<uint32_t *>(b + L.hist);
    q.group_rows = reinterpret_cast<uint32_t *>(b + L.group_rows);
    q.group_offsets = reinterpret_cast<uint32_t *>(b + L.group_offsets);
    q.chunk_first = reinterpret_cast<uint32_t *>(b + L.chunk_first);
    q.chunks = reinterpret_cast<uint4 *>(b + L.chunks);
    q.n_chunks = reinterpret_cast<uint32_t *>(b + L.n_chunks);
    q.sorted_rows = reinterpret_cast<uint32_t *>(b + L.sorted);
    q.partials = reinterpret_cast<float *>(b + L.partials);
    sr.d_sum = reinterpret_cast<float *>(b + L.out_sum);
    sr.d_sumsq = reinterpret_cast<float *>(b + L.out_sumsq);
    sr.d_mean = r.mean ? reinterpret_cast<float *>(b + L.out_mean) : nullptr;
    sr.d_var = r.var ? reinterpret_cast<float *>(b + L.out_var) : nullptr;
    sr.d_group_rows = reinterpret_cast<uint32_t *>(b + L.out_group_rows);
    const bool dev_out = (r.flags & CS_SERVE_DEVICE_OUTPUTS) != 0u;
    q.sum = dev_out ? r.sum : sr.d_sum;
    q.sumsq = dev_out ? r.sumsq : sr.d_sumsq;
    q.mean = dev_out ? r.mean : sr.d_mean;
    q.var = dev_out ? r.var : sr.d_var;
    q.out_group_rows = dev_out ? r.group_rows : sr.d_group_rows;
    q.counters = reinterpret_cast<uint32_t *>(b + L.counters);
    q.done = s->d_done + slot;
    s->h_done[slot] = 0u;
    cudaStream_t cs = s->cstream;
    const uint64_t R = s->total_rows;
    if (host_in && r.row_keep) cudaMemcpyAsync(b + L.in_keep, r.row_keep, R, cudaMemcpyHostToDevice, cs);
    if (host_in && r.row_labels) cudaMemcpyAsync(b + L.in_labels, r.row_labels, R * 4u, cudaMemcpyHostToDevice, cs);
    if (host_in && r.feature_keep) cudaMemcpyAsync(b + L.in_fk, r.feature_keep, s->cols, cudaMemcpyHostToDevice, cs);
    cudaMemcpyAsync(q.counters, s->h_zero, 16, cudaMemcpyHostToDevice, cs);
    cudaMemcpyAsync(s->d_reqs + slot, &q, sizeof(sreq), cudaMemcpyHostToDevice, cs);
    cudaEventRecord(sr.ev, cs);
    t.state = CS_SERVE_RUNNING;
    t.t_admit = clk::now();
    ++s->admitted;
    return true;
}

void finish_slot(cs_server *s, int i) {
    slot_rec &sr = s->slots[i];
    ticket_rec &t = s->tickets[sr.ticket];
    t.state = CS_SERVE_DONE;
    t.t_done = clk::now();
    s->outstanding_items -= items_for(s, t.req.group_count, t.max_chunks);
    pool_free(s, sr.off, sr.bytes);
    sr.state = SLOT_FREE;
    ++s->completed;
}

void sched_loop(cs_server *s) {
    cudaSetDevice(s->device);
    while (!s->quit.load()) {
        bool busy = false;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->pending.empty() && try_admit(s, s->pending.front())) s->pending.pop_front();
            for (size_t i = 0; i < s->slots.size(); ++i) {
                slot_rec &sr = s->slots[i];
                if (sr.state == SLOT_FREE) continue;
                busy = true;
                if (sr.state == SLOT_COPY_IN && cudaEventQuery(sr.ev) == cudaSuccess) {
                    push_host_item(s, make_uint4(IT_START | ((uint32_t) i << 8), 0u, 0u, 0u));
                    s->tickets[sr.ticket].t_start = clk::now();
                    sr.state = SLOT_RUNNING;
                } else if (sr.state == SLOT_RUNNING &&
                           reinterpret_cast<volatile uint32_t *>(s->h_done)[i] != 0u) {
                    ticket_rec &t = s->tickets[sr.ticket];
                    t.t_device_done = clk::now();
                    const cs_serve_request &r = t.req;
                    if ((r.flags & CS_SERVE_DEVICE_OUTPUTS) == 0u) {
                        const std::size_t gc = (std::size_t) r.group_count * s->cols * 4u;
                        cudaStream_t cs = s->cstream;
                        if (r.sum) cudaMemcpyAsync(r.sum, sr.d_sum, gc, cudaMemcpyDeviceToHost, cs);
                        if (r.sumsq) cudaMemcpyAsync(r.sumsq, sr.d_sumsq, gc, cudaMemcpyDeviceToHost, cs);
                        if (r.mean) cudaMemcpyAsync(r.mean, sr.d_mean, gc, cudaMemcpyDeviceToHost, cs);
                        if (r.var) cudaMemcpyAsync(r.var, sr.d_var, gc, cudaMemcpyDeviceToHost, cs);
                        if (r.group_rows)
                            cudaMemcpyAsync(r.group_rows, sr.d_group_rows, (std::size_t) r.group_count * 4u,
                                            cudaMemcpyDeviceToHost, cs);
                    }
                    cudaEventRecord(sr.ev, s->cstream);
                    sr.state = SLOT_COPY_OUT;
                } else if (sr.state == SLOT_COPY_OUT && cudaEventQuery(sr.ev) == cudaSuccess) {
                    finish_slot(s, (int) i);
                    s->cv.notify_all();
                }
            }
            bool running_work = false;
            for (auto &sr : s->slots) running_work |= (sr.state == SLOT_RUNNING);
            if (running_work && !kernel_running(s)) {
                if (!launch_kernel(s)) s->sched_error = "serve kernel launch failed";
            }
        }
        if (!busy) {
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(5));
        }
    }
}

} // namespace

extern "C" int cs_b200_serve_open(const cs_blocked_ell_view *parts, uint32_t count, const cs_serve_config *cfg,
                                  cs_server **out) {
    if (out == nullptr || parts == nullptr || count == 0u) {
        set_error("serve_open: null argument or no partitions");
        return 0;
    }
    *out = nullptr;
    const uint32_t B = parts[0].block_size, cols = parts[0].cols;
    uint64_t total = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const cs_blocked_ell_view &p = parts[i];
        if (p.block_size != B || p.cols != cols || B == 0u || B % 8u != 0u || p.ell_cols % B != 0u ||
            (p.rows != 0u && p.ell_cols != 0u && ((uintptr_t) p.val & 15u) != 0u)) {
            set_error("serve_open: partition %u: block size (multiple of 8), cols and 16-byte aligned values "
                      "must agree",
                      i);
            return 0;
        }
        total += p.rows;
    }
    if (total == 0u || total >= (1ull << 32)) {
        set_error("serve_open: total rows %llu outside [1, 2^32)", (unsigned long long) total);
        return 0;
    }
    auto *s = new cs_server();
    s->cfg = cfg ? *cfg : cs_serve_config{};
    if (s->cfg.scratch_budget_bytes == 0u) s->cfg.scratch_budget_bytes = 16ull << 30;
    if (s->cfg.max_inflight == 0u) s->cfg.max_inflight = 32u;
    if (s->cfg.max_inflight > 256u) s->cfg.max_inflight = 256u;
    if (s->cfg.chunk_rows == 0u || s->cfg.chunk_rows > kServeMaxChunkRows) s->cfg.chunk_rows = kServeMaxChunkRows;
    cudaGetDevice(&s->device);
    s->nparts = count;
    s->total_rows = (uint32_t) total;
    s->cols = cols;
    s->block_size = B;
    s->col_blocks = (cols + B - 1u) / B;
    s->words = (s->col_blocks + 31u) / 32u;
    s->tiles = (s->total_rows + kServeTile - 1u) / kServeTile;
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking), "serve stream") &&
              cuda_ok(cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking), "serve copy stream") &&
              cuda_ok(cudaEventCreateWithFlags(&s->kdone, cudaEventDisableTiming), "serve event");
    // partition table and per-partition column-block index
    uint32_t *d_status = nullptr;
    if (ok) ok = cuda_ok(cudaMalloc(&d_status, 4), "serve status") && cuda_ok(cudaMemset(d_status, 0, 4), "status");
    uint32_t base = 0;
    for (uint32_t i = 0; ok && i < count; ++i) {
        const cs_blocked_ell_view &p = parts[i];
        const uint32_t rb = (p.rows + B - 1u) / B;
        uint2 *idx = nullptr;
        ok = cuda_ok(cudaMalloc(&idx, ((std::size_t) rb * s->words + 1u) * sizeof(uint2)), "serve index");
        if (!ok) break;
        s->d_index.push_back(idx);
        if (p.rows) ok = build_column_block_index(&p, idx, d_status, s->kstream) != 0;
        spart sp{};
        sp.rows = p.rows;
        sp.ell_cols = p.ell_cols;
        sp.row_base = base;
        sp.val = p.val;
        sp.index = idx;
        s->hparts.push_back(sp);
        base += p.rows;
    }
    uint32_t status = 0u;
    if (ok)
        ok = cuda_ok(cudaStreamSynchronize(s->kstream), "serve index sync") &&
             cuda_ok(cudaMemcpy(&status, d_status, 4, cudaMemcpyDeviceToHost), "serve status copy");
    if (d_status) cudaFree(d_status);
    if (ok && status != 0u) {
        set_error("serve_open: Blocked-ELL input rejected (status 0x%x)", status);
        ok = false;
    }
    const uint32_t S = s->cfg.max_inflight;
    if (ok)
        ok = cuda_ok(cudaMalloc(&s->d_parts, sizeof(spart) * count), "serve parts") &&
             cuda_ok(cudaMemcpy(s->d_parts, s->hparts.data(), sizeof(spart) * count, cudaMemcpyHostToDevice),
                     "serve parts upload") &&
             cuda_ok(cudaMalloc(&s->d_reqs, sizeof(sreq) * S), "serve requests") &&
             cuda_ok(cudaHostAlloc(&s->h_reqs, sizeof(sreq) * S, cudaHostAllocDefault), "serve request staging") &&
             cuda_ok(cudaHostAlloc(&s->h_done, 4u * S, cudaHostAllocMapped), "serve done words") &&
             cuda_ok(cudaHostGetDevicePointer((void **) &s->d_done, s->h_done, 0), "serve done map") &&
             cuda_ok(cudaHostAlloc(&s->h_zero, 64, cudaHostAllocDefault), "serve zeros") &&
             cuda_ok(cudaMalloc(&s->d_heads, 64), "serve heads") && cuda_ok(cudaMemset(s->d_heads, 0, 64), "heads") &&
             cuda_ok(cudaMalloc(&s->d_dslots, sizeof(uint4) * kDevRing), "serve ring") &&
             cuda_ok(cudaMalloc(&s->d_dseq, 8u * kDevRing), "serve ring seq") &&
             cuda_ok(cudaMemset(s->d_dseq, 0, 8u * kDevRing), "ring seq clear") &&
             cuda_ok(cudaMalloc(&s->d_hslots, sizeof(uint4) * kHostRing), "host ring") &&
             cuda_ok(cudaMalloc(&s->d_hseq, 8u * kHostRing), "host ring seq") &&
             cuda_ok(cudaMemset(s->d_hseq, 0, 8u * kHostRing), "host ring seq clear") &&
             cuda_ok(cudaMalloc(&s->d_htail, 64), "host ring tail") &&
             cuda_ok(cudaMemset(s->d_htail, 0, 64), "host ring tail clear") &&
             cuda_ok(cudaHostAlloc(&s->h_push, 32u * kHostRing, cudaHostAllocDefault), "host ring staging") &&
             cuda_ok(cudaStreamCreateWithFlags(&s->pstream, cudaStreamNonBlocking), "serve control stream") &&
             cuda_ok(cudaMalloc(&s->d_prof, 16u * 8u), "serve profile") &&
             cuda_ok(cudaMalloc(&s->d_orph, 16u * kOrphans), "serve orphans") &&
             cuda_ok(cudaMemset(s->d_orph, 0, 16u * kOrphans), "serve orphans clear") &&
             cuda_ok(cudaMemset(s->d_prof, 0, 16u * 8u), "serve profile clear") &&
             cuda_ok(cudaMalloc(&s->d_error, 4), "serve error") && cuda_ok(cudaMemset(s->d_error, 0, 4), "error");
    if (ok) {
        std::memset(s->h_zero, 0, 64);
        std::memset(s->h_done, 0, 4u * S);
        s->pool_bytes = s->cfg.scratch_budget_bytes;
        ok = cuda_ok(cudaMalloc(&s->pool, s->pool_bytes), "serve scratch pool");
        if (ok) s->free_blocks[0] = s->pool_bytes;
    }
    if (ok) {
        ok = cuda_ok(cudaFuncSetAttribute(serve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) kServeDynSmem),
                     "serve smem attribute");
        int occ = 0;
        if (ok)
            ok = cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, serve_kernel, kSThreads, kServeDynSmem),
                         "serve occupancy");
        if (occ < 1) occ = 1;
        if (s->cfg.ctas_per_sm != 0u && (int) s->cfg.ctas_per_sm < occ) occ = (int) s->cfg.ctas_per_sm;
        s->grid = (uint32_t) (occ * sm_count());
    }
    if (ok) {
        s->slots.resize(S);
        for (auto &sr : s->slots)
            ok = ok && cuda_ok(cudaEventCreateWithFlags(&sr.ev, cudaEventDisableTiming), "slot event");
    }
    if (!ok) {
        cs_b200_serve_close(s);
        return 0;
    }
    s->sched = std::thread(sched_loop, s);
    *out = s;
    return 1;
}

extern "C" int cs_b200_serve_submit(cs_server *s, const cs_serve_request *req, uint64_t *ticket) {
    if (s == nullptr || req == nullptr || ticket == nullptr) {
        set_error("serve_submit: null argument");
        return 0;
    }
    if (req->group_count == 0u || req->group_count > kServeMaxGroups || req->scheme > CS_MOMENTS_TWOSUM_F64_COMBINE ||
        req->sum == nullptr || req->sumsq == nullptr) {
        set_error("serve_submit: group_count in [1, %u], a known scheme and sum/sumsq outputs are required",
                  kServeMaxGroups);
        return 0;
    }
    // kept rows bound the sorted list and the chunk count
    uint64_t kept = s->total_rows;
    if (req->row_keep != nullptr && (req->flags & CS_SERVE_DEVICE_INPUTS) == 0u) {
        kept = 0;
        for (uint32_t r = 0; r < s->total_rows; ++r) kept += req->row_keep[r] != 0u;
    }
    ticket_rec t;
    t.req = *req;
    t.max_chunks = (uint32_t) ((kept + s->cfg.chunk_rows - 1u) / s->cfg.chunk_rows + req->group_count);
    t.need = layout_for(s, *req, t.max_chunks, s->total_rows).bytes;
    t.t_submit = clk::now();
    if (t.need > s->pool_bytes) {
        set_error("serve_submit: request needs %llu scratch bytes, budget is %llu", (unsigned long long) t.need,
                  (unsigned long long) s->pool_bytes);
        return 0;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t id = s->next_ticket++;
    s->tickets[id] = t;
    s->pending.push_back(id);
    *ticket = id;
    return 1;
}

extern "C" int cs_b200_serve_poll(cs_server *s, uint64_t ticket, uint32_t *state, double *latency_ms) {
    if (s == nullptr || state == nullptr) {
        set_error("serve_poll: null argument");
        return 0;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) {
        set_error("serve_poll: unknown ticket %llu", (unsigned long long) ticket);
        return 0;
    }
    *state = it->second.state;
    if (latency_ms && it->second.state == CS_SERVE_DONE)
        *latency_ms = std::chrono::duration<double, std::milli>(it->second.t_done - it->second.t_submit).count();
    return 1;
}

extern "C" int cs_b200_serve_wait(cs_server *s, uint64_t ticket, uint32_t timeout_ms, double *latency_ms) {
    if (s == nullptr) {
        set_error("serve_wait: null server");
        return 0;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto done = [&] {
        auto it = s->tickets.find(ticket);
        return it == s->tickets.end() || it->second.state == CS_SERVE_DONE || !s->sched_error.empty();
    };
    if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms ? timeout_ms : 60000u), done)) {
        set_error("serve_wait: ticket %llu not done after %u ms", (unsigned long long) ticket, timeout_ms);
        return 0;
    }
    if (!s->sched_error.empty()) {
        set_error("serve: %s", s->sched_error.c_str());
        return 0;
    }
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) {
        set_error("serve_wait: unknown ticket %llu", (unsigned long long) ticket);
        return 0;
    }
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(it->second.t_done - it->second.t_submit).count();
    return 1;
}

extern "C" int cs_b200_serve_release(cs_server *s, uint64_t ticket) {
    if (s == nullptr) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it != s->tickets.end() && it->second.state == CS_SERVE_DONE) s->tickets.erase(it);
    return 1;
}

extern "C" int cs_b200_serve_stats(cs_server *s, cs_serve_stats *out) {
    if (s == nullptr || out == nullptr) {
        set_error("serve_stats: null argument");
        return 0;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->admitted = s->admitted;
    out->completed = s->completed;
    out->pending = s->pending.size();
    out->kernel_launches = s->kernel_launches;
    out->scratch_in_use = s->pool_used;
    out->scratch_budget = s->pool_bytes;
    uint32_t err = 0u;
    unsigned long long prof[16] = {0};
    cudaMemcpy(&err, s->d_error, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(prof, s->d_prof, sizeof(prof), cudaMemcpyDeviceToHost);
    out->device_error = err;
    for (int k = 0; k < 8; ++k) {
        out->items[k] = prof[k];
        out->item_ns[k] = prof[8 + k];
    }
    return 1;
}

extern "C" int cs_b200_serve_run_trace(cs_server *s, const cs_serve_request *reqs, const uint32_t *req_index,
                                       const double *arrival_s, uint32_t n, double *latency_ms, double *makespan_s,
                                       double *phase_ms) {
    if (s == nullptr || reqs == nullptr || req_index == nullptr || arrival_s == nullptr) {
        set_error("serve_run_trace: null argument");
        return 0;
    }
    std::vector<uint64_t> tk(n, 0);
    const auto t0 = clk::now();
    for (uint32_t i = 0; i < n; ++i) {
        const auto at = t0 + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(arrival_s[i]));
        while (clk::now() < at) {
            const auto left = at - clk::now();
            if (left > std::chrono::microseconds(200))
                std::this_thread::sleep_for(left - std::chrono::microseconds(100));
        }
        if (!cs_b200_serve_submit(s, &reqs[req_index[i]], &tk[i])) return 0;
    }
    for (uint32_t i = 0; i < n; ++i) {
        double ms = 0.0;
        if (!cs_b200_serve_wait(s, tk[i], 120000u, &ms)) return 0;
        if (latency_ms) latency_ms[i] = ms;
    }
    const auto t1 = clk::now();
    if (makespan_s) *makespan_s = std::chrono::duration<double>(t1 - t0).count();
    if (phase_ms) {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t i = 0; i < n; ++i) {
            const ticket_rec &t = s->tickets[tk[i]];
            auto ms = [&](clk::time_point x) { return std::chrono::duration<double, std::milli>(x - t.t_submit).count(); };
            phase_ms[4 * i + 0] = ms(t.t_admit);
            phase_ms[4 * i + 1] = ms(t.t_start);
            phase_ms[4 * i + 2] = ms(t.t_device_done);
            phase_ms[4 * i + 3] = ms(t.t_done);
        }
    }
    for (uint32_t i = 0; i < n; ++i) cs_b200_serve_release(s, tk[i]);
    return 1;
}

extern "C" void cs_b200_serve_close(cs_server *s) {
    if (s == nullptr) return;
    if (s->sched.joinable()) {
        // let admitted work finish (bounded), then stop the scheduler and the kernel
        for (int i = 0; i < 20000; ++i) {
            {
                std::lock_guard<std::mutex> lk(s->mu);
                bool idle = s->pending.empty();
                for (auto &sr : s->slots) idle = idle && sr.state == SLOT_FREE;
                if (idle) break;
            }
            std::this_thread::sleep_for(std::chrono::milliseconds(1));
        }
        s->quit.store(true);
        s->sched.join();
    }
    if (s->d_htail && s->h_zero && s->pstream) {
        s->h_zero[8] = 1u;
        cudaMemcpyAsync(s->d_htail + 1, s->h_zero + 8, 4, cudaMemcpyHostToDevice, s->pstream);
        cudaStreamSynchronize(s->pstream);
    }
    if (s->kstream) cudaStreamSynchronize(s->kstream);
    if (s->cstream) cudaStreamSynchronize(s->cstream);
    for (auto &sr : s->slots)
        if (sr.ev) cudaEventDestroy(sr.ev);
    for (auto *p : s->d_index) cudaFree(p);
    if (s->d_parts) cudaFree(s->d_parts);
    if (s->d_reqs) cudaFree(s->d_reqs);
    if (s->h_reqs) cudaFreeHost(s->h_reqs);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_zero) cudaFreeHost(s->h_zero);
    if (s->d_heads) cudaFree(s->d_heads);
    if (s->d_dslots) cudaFree(s->d_dslots);
    if (s->d_dseq) cudaFree(s->d_dseq);
    if (s->d_hslots) cudaFree(s->d_hslots);
    if (s->d_hseq) cudaFree(s->d_hseq);
    if (s->d_htail) cudaFree(s->d_htail);
    if (s->h_push) cudaFreeHost(s->h_push);
    if (s->d_prof) cudaFree(s->d_prof);
    if (s->d_orph) cudaFree(s->d_orph);
    if (s->pstream) cudaStreamDestroy(s->pstream);
    if (s->d_error) cudaFree(s->d_error);
    if (s->pool) cudaFree(s->pool);
    if (s->kdone) cudaEventDestroy(s->kdone);
    if (s->kstream) cudaStreamDestroy(s->kstream);
    if (s->cstream) cudaStreamDestroy(s->cstream);
    delete s;
}
