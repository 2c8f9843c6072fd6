// Shared device/host helpers for libcellshard_b200.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>

#include "../../include/cellshard_b200.h"

namespace csb {

// ---------------------------------------------------------------------------
// Error reporting: one message per host thread, read by cs_b200_last_error().
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
void clear_error();

inline int cuda_ok(cudaError_t err, const char *what) {
    if (err == cudaSuccess) return 1;
    set_error("CUDA error at %s: %s", what, cudaGetErrorString(err));
    return 0;
}

inline int launch_ok(const char *kernel) {
    return cuda_ok(cudaGetLastError(), kernel);
}

inline cudaStream_t as_stream(cs_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs on the current device (cached per device ordinal).
int sm_count();

// Blocks of `kernel` resident on the whole device at once (SMs x blocks per
// SM for this block size and dynamic shared memory), at most `needed` and
// at least 1: a grid-stride kernel launched with it runs in a single wave.
unsigned resident_grid(const void *kernel, unsigned threads, std::size_t smem, std::size_t needed);

inline std::size_t align_up(std::size_t v, std::size_t a) { return (v + a - 1u) / a * a; }

// Bump allocator over caller scratch; every sub-buffer is 256-byte aligned.
struct scratch_carver {
    char *base;
    std::size_t cap;
    std::size_t used;
    __host__ scratch_carver(void *b, std::size_t c) : base((char *) b), cap(c), used(0) {}
    template <typename T>
    __host__ T *take(std::size_t count) {
        used = align_up(used, 256);
        T *p = (T *) (base ? base + used : nullptr);
        used += count * sizeof(T);
        return p;
    }
    __host__ bool fits() const { return used <= cap; }
};

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float h2f(uint16_t bits) {
    return __half2float(__ushort_as_half(bits));
}

// A fp16 value compares unequal to 0.0f unless it is +0 or -0 (NaN counts as
// nonzero, as `__half2float(v) != 0.0f` does in the reference).
__device__ __forceinline__ bool half_nonzero(uint16_t bits) { return (bits & 0x7fffu) != 0u; }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void status_or(uint32_t *status, uint32_t bits) {
    if (status != nullptr && bits != 0u) atomicOr(status, bits);
}

// Streaming 16-byte load that does not allocate the line in L1 (value
// streams are touched once).
__device__ __forceinline__ uint4 ld_stream_v4(const void *p) {
    uint4 r;
    asm("ld.global.nc.L1::no_allocate.L2::256B.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p));
    return r;
}

__device__ __forceinline__ uint2 ld_stream_v2(const void *p) {
    uint2 r;
    asm("ld.global.nc.L1::no_allocate.L2::256B.v2.u32 {%0,%1}, [%2];" : "=r"(r.x), "=r"(r.y) : "l"(p));
    return r;
}

__device__ __forceinline__ void st_stream_v4(void *p, uint4 v) {
    asm volatile("st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z),
                 "r"(v.w)
                 : "memory");
}

// Warp inclusive scan (all 32 lanes participate).
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (unsigned) o) v += t;
    }
    return v;
}

// Block-wide exclusive scan; blockDim.x must be a multiple of 32 (<= 1024)
// and every thread must call it.  smem holds 33 words.  Safe to call back to
// back (ends with a barrier after the shared reads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *smem, uint32_t &total) {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t incl = warp_inclusive_scan(v);
    if (lane == 31u) smem[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < nw ? smem[lane] : 0u;
        const uint32_t wi = warp_inclusive_scan(w);
        if (lane < nw) smem[lane] = wi - w;
        if (lane == 31u) smem[32] = wi;
    }
    __syncthreads();
    const uint32_t r = smem[warp] + incl - v;
    total = smem[32];
    __syncthreads();
    return r;
}

// Lanes holding the same BITS-bit digit as this lane (this lane included),
// among lanes whose `valid` is set; 0 for an invalid lane.  Built from one
// ballot per digit bit (the multisplit construction), cheaper than a general
// match for small digits.
template <int BITS>
__device__ __forceinline__ uint32_t warp_match_digit(uint32_t d, bool valid) {
    uint32_t m = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < BITS; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bb = __ballot_sync(0xffffffffu, bit);
        m &= bit ? bb : ~bb;
    }
    return valid ? m : 0u;
}

// ---------------------------------------------------------------------------
// 16-byte asynchronous copies global -> shared (per thread; completion is
// tracked per thread in commit groups).  Both addresses 16-byte aligned.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_16(void *sdst, const void *gsrc) {
    const uint32_t s = (uint32_t) __cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Waits until at most N of this thread's committed groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Bulk (TMA) copies shared -> global.  Sizes and both addresses must be
// multiples of 16 bytes.  Generic-proxy shared-memory writes must be fenced
// with fence_proxy_async_smem() (by the writing threads, then a barrier)
// before the bulk copy reads them.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_store_s2g(void *gdst, const void *ssrc, uint32_t bytes) {
    const uint32_t s = (uint32_t) __cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(s), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Waits until at most N of this thread's committed bulk groups are still
// reading shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Waits until all of this thread's committed bulk groups have completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of uint32 (three launches: tile sums, scan of
// tile sums, tile-local scan + add).  out may alias in.  out[n] receives the
// total when write_total is set (so out must hold n + 1 entries).
// ---------------------------------------------------------------------------
std::size_t scan_u32_scratch_bytes(std::size_t n);
int scan_exclusive_u32(const uint32_t *in, uint32_t *out, std::size_t n, bool write_total, void *scratch,
                       std::size_t scratch_bytes, cudaStream_t stream);

// Stable ascending sort of n uint32 keys carrying uint32 values (vals nullptr:
// the indices 0..n-1), LSD radix in 8-bit digit passes (bucket.cu).  Word 0
// of the scratch is a status word (1 = a bounded look-back wait ran out).
std::size_t sort_pairs_u32_scratch_bytes(uint32_t n);
int sort_pairs_u32(const uint32_t *keys, const uint32_t *vals, uint32_t n, uint32_t *out_keys, uint32_t *out_vals,
                   void *tmp, std::size_t tmp_bytes, cudaStream_t stream);

// Owned device memory and stream for the synchronous host entry points.
struct dmem {
    void *p = nullptr;
    dmem() = default;
    dmem(const dmem &) = delete;
    dmem &operator=(const dmem &) = delete;
    ~dmem() {
        if (p) cudaFree(p);
    }
    bool alloc(std::size_t n, const char *what) { return cuda_ok(cudaMalloc(&p, n == 0 ? 16 : n), what) != 0; }
};

struct own_stream {
    cudaStream_t s = nullptr;
    own_stream() = default;
    own_stream(const own_stream &) = delete;
    own_stream &operator=(const own_stream &) = delete;
    ~own_stream() {
        if (s) cudaStreamDestroy(s);
    }
};

// Host Blocked-ELL staged on the device (the reference's upload_async), and
// the shape check of a device Blocked-ELL view (sliced_from_blocked.cu).
struct staged_bell {
    dmem bci, val;
    cs_blocked_ell_view view{};
};
int stage_bell(const cs_host_blocked_ell *src, staged_bell *st, cudaStream_t stream);
int check_bell(const cs_blocked_ell_view *src, const char *who);
// Host-owned Blocked-ELL packed as sparse::allocate lays it out (blocked_ell.cu).
int host_blocked_ell_allocate(cs_host_blocked_ell *m);

// Sliced-ELL pieces shared by the CSR and Blocked-ELL sources (sliced_ell.cu).
int sliced_layout_launch(const cs_compressed_view *src, uint32_t slice_rows, uint32_t *d_offsets, uint32_t *d_widths,
                         uint32_t *d_slot_offsets, uint64_t *d_total, void *scratch, std::size_t scratch_bytes,
                         cudaStream_t stream);
int choose_sliced_rows_core(const cs_compressed_view *v, uint32_t nnz, const unsigned int *candidates,
                            unsigned int candidate_count, cs_sliced_ell_tune_result *out, cudaStream_t stream);
int host_sliced_alloc(cs_host_sliced_ell *dst, uint32_t rows, uint32_t cols, uint32_t nnz, uint32_t S,
                      uint64_t total_slots);

} // namespace csb
