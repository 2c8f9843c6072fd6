// Seeded synthetic cell x gene CSR (tests and benchmark inputs).
//
// One warp per row.  Draw j of row r is the 53-bit uniform u = hash(seed, r, j)
// mapped to a popularity rank by binary search in an integer CDF and to a
// column through a rank -> column permutation.  Draws are resolved 32 at a
// time in draw order (a column is accepted when it is neither already chosen
// nor drawn by an earlier lane of the same round), which reproduces serial
// successive sampling exactly, so the result does not depend on scheduling.
// The chosen set lives in a per-warp shared-memory bitmap and is emitted in
// ascending column order.  Value k of the row is an integer count drawn from
// a second CDF (bucket i -> count i + 1), optionally scaled, rounded to fp16.
#include "common.cuh"

namespace csb {
namespace {

constexpr unsigned kSynthWarps = 4;

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t draw_u53(uint64_t seed_key, uint32_t row, uint32_t j) {
    return splitmix64(seed_key ^ (((uint64_t) row << 32) | (uint64_t) j)) >> 11;
}

// first i in [0, n) with u < cdf[i]; cdf[n-1] == 2^53 so it always exists
__device__ __forceinline__ uint32_t cdf_search(const uint64_t *__restrict__ cdf, uint32_t n, uint64_t u) {
    uint32_t lo = 0, hi = n - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (u < __ldg(cdf + mid))
            hi = mid;
        else
            lo = mid + 1u;
    }
    return lo;
}

__global__ void __launch_bounds__(kSynthWarps * 32) synth_csr_kernel(
    uint32_t rows, uint32_t cols, const uint32_t *__restrict__ row_ptr, const uint64_t *__restrict__ col_cdf,
    const uint32_t *__restrict__ col_of_rank, const uint64_t *__restrict__ val_cdf, uint32_t val_len,
    const float *__restrict__ row_scale, uint64_t seed, uint32_t *__restrict__ out_idx, uint16_t *__restrict__ out_val) {
    extern __shared__ uint32_t synth_smem[];
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t words = (cols + 31u) / 32u;
    uint32_t *bits = synth_smem + (std::size_t) warp * words;
    const uint64_t col_key = splitmix64(seed ^ 0x636f6c756d6e73ull);
    const uint64_t val_key = splitmix64(seed ^ 0x76616c7565737321ull);
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t r = blockIdx.x * kSynthWarps + warp; r < rows; r += gridDim.x * kSynthWarps) {
        for (uint32_t w = lane; w < words; w += 32u) bits[w] = 0u;
        __syncwarp();
        const uint32_t base = row_ptr[r];
        uint32_t need = row_ptr[r + 1u] - base;
        if (need > cols) need = cols;
        uint32_t chosen = 0u;
        const uint32_t max_rounds = (64u * cols + 1024u) / 32u;
        for (uint32_t round = 0; chosen < need && round < max_rounds; ++round) {
            const uint64_t u = draw_u53(col_key, r, round * 32u + lane);
            const uint32_t c = __ldg(col_of_rank + cdf_search(col_cdf, cols, u));
            const uint32_t peers = __match_any_sync(0xffffffffu, c);
            const bool first = lane == (unsigned) (__ffs(peers) - 1);
            const bool fresh = ((bits[c >> 5] >> (c & 31u)) & 1u) == 0u;
            uint32_t acc = __ballot_sync(0xffffffffu, first && fresh);
            const uint32_t room = need - chosen;
            while ((uint32_t) __popc(acc) > room) acc &= ~(1u << (31 - __clz(acc))); // keep the lowest lanes
            __syncwarp();
            if ((acc >> lane) & 1u) atomicOr(bits + (c >> 5), 1u << (c & 31u));
            chosen += __popc(acc);
            __syncwarp();
        }
        // cap reached (never for need <= cols / 2 in practice): lowest free columns
        for (uint32_t w0 = 0; chosen < need && w0 < words; w0 += 32u) {
            const uint32_t w = w0 + lane;
            uint32_t free_bits = 0u;
            if (w < words) {
                free_bits = ~bits[w];
                if (w == words - 1u && (cols & 31u) != 0u) free_bits &= (1u << (cols & 31u)) - 1u;
            }
            const uint32_t cnt = __popc(free_bits);
            const uint32_t incl = warp_inclusive_scan(cnt);
            const uint32_t before = incl - cnt;
            const uint32_t room = need - chosen;
            uint32_t take = 0u;
            if (before < room) take = min(cnt, room - before);
            uint32_t fb = free_bits, t = 0u;
            while (t < take) {
                const uint32_t bit = __ffs(fb) - 1u;
                bits[w] |= 1u << bit;
                fb &= fb - 1u;
                ++t;
            }
            chosen += min(__shfl_sync(0xffffffffu, incl, 31), room);
            __syncwarp();
        }
        __syncwarp();
        // emit ascending columns and their values
        const float scale = row_scale != nullptr ? row_scale[r] : 1.0f;
        uint32_t carry = 0u;
        for (uint32_t w0 = 0; w0 < words; w0 += 32u) {
            const uint32_t w = w0 + lane;
            uint32_t word = w < words ? bits[w] : 0u;
            const uint32_t cnt = __popc(word);
            const uint32_t incl = warp_inclusive_scan(cnt);
            uint32_t pos = carry + incl - cnt;
            while (word != 0u) {
                const uint32_t bit = __ffs(word) - 1u;
                if (pos < need) {
                    out_idx[base + pos] = w * 32u + bit;
                    const uint32_t k = cdf_search(val_cdf, val_len, draw_u53(val_key, r, pos)) + 1u;
                    out_val[base + pos] = __half_as_ushort(__float2half_rn((float) k * scale));
                }
                ++pos;
                word &= word - 1u;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        (void) lt;
        __syncwarp();
    }
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_synth_csr(uint32_t rows, uint32_t cols, const uint32_t *d_row_ptr, const uint64_t *d_col_cdf,
                                 const uint32_t *d_col_of_rank, const uint64_t *d_val_cdf, uint32_t val_cdf_len,
                                 const float *d_row_scale, uint64_t seed, uint32_t *d_minor_idx, uint16_t *d_val,
                                 cs_stream_t s) {
    if (rows == 0u) return 1;
    if (cols == 0u || d_row_ptr == nullptr || d_col_cdf == nullptr || d_col_of_rank == nullptr ||
        d_val_cdf == nullptr || val_cdf_len == 0u) {
        set_error("synth_csr: missing tables or zero columns");
        return 0;
    }
    const std::size_t smem = (std::size_t) kSynthWarps * ((cols + 31u) / 32u) * sizeof(uint32_t);
    if (smem > 200u * 1024u) {
        set_error("synth_csr: %u columns exceed the shared-memory bitmap", cols);
        return 0;
    }
    if (smem > 48u * 1024u &&
        !cuda_ok(cudaFuncSetAttribute(synth_csr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "synth smem attribute"))
        return 0;
    uint32_t grid = (rows + kSynthWarps - 1u) / kSynthWarps;
    const uint32_t cap = (uint32_t) sm_count() * 64u;
    if (grid > cap) grid = cap;
    synth_csr_kernel<<<grid, kSynthWarps * 32, smem, as_stream(s)>>>(rows, cols, d_row_ptr, d_col_cdf, d_col_of_rank,
                                                                     d_val_cdf, val_cdf_len, d_row_scale, seed,
                                                                     d_minor_idx, d_val);
    return launch_ok("synth_csr_kernel");
}
