// 16-byte value-vector helpers for warp-per-row walks over Blocked-ELL rows
// (a lane holds 8 consecutive fp16 values of one slot; block sizes that are
// multiples of 8 keep a vector inside one slot).
#pragma once

#include "common.cuh"

namespace csb {

// 1.0 in each half of w that is nonzero as a float or NaN (either sign of
// zero gives 0.0): one packed-half compare.
__device__ __forceinline__ uint32_t nonzero_halves(uint32_t w) {
    uint32_t d;
    asm("set.neu.f16x2.f16x2 %0, %1, %2;" : "=r"(d) : "r"(w), "r"(0u));
    return d;
}

// Bit q set when fp16 value q of the 8 in v is nonzero as a float (NaN
// counts).  Each half becomes 1.0 (0x3c00) or 0 by a packed compare; a byte
// permute keeps the high byte of every half (bit 5 set for a nonzero value),
// the flags of values 0-3 land at bit 8k + 1 and those of values 4-7 at bit
// 8k + 5, and after a shift one multiply gathers bit 8k into bit 24 + k and
// bit 8k + 4 into bit 28 + k (no two partial products meet).
__device__ __forceinline__ uint32_t live_bits8(const uint4 &v) {
    const uint32_t f01 = __byte_perm(nonzero_halves(v.x), nonzero_halves(v.y), 0x7531u);
    const uint32_t f23 = __byte_perm(nonzero_halves(v.z), nonzero_halves(v.w), 0x7531u);
    const uint32_t g = (f23 & 0x20202020u) | ((f01 >> 4) & 0x02020202u);
    return ((g >> 1) * 0x01020408u) >> 24;
}

// Columns gene0 .. gene0 + 7 of a vector inside slot bc: the mask of those
// that exist (valid block column, column < cols).  gene0 = bc * B + offset:
// for a padding slot (bc = CS_INVALID_COL) it wraps to 2^32 - B + offset,
// past any column count, so one clamp covers both tests.
__device__ __forceinline__ uint32_t in_range8(uint32_t bc, uint32_t gene0, uint32_t cols) {
    (void) bc;
    const uint32_t d = min(max(cols, gene0) - gene0, 8u);
    return (1u << d) - 1u;
}

// e / B and e % B for a block size B: a shift and a mask when B is a power
// of two (every block size the choosers produce), a division otherwise.
struct block_div {
    uint32_t B;
    int shift;
    __device__ __forceinline__ explicit block_div(uint32_t b) : B(b), shift(-1) {
#ifdef __CUDA_ARCH__
        if (b != 0u && (b & (b - 1u)) == 0u) shift = __ffs((int) b) - 1;
#endif
    }
    __device__ __forceinline__ uint32_t div(uint32_t e) const { return shift >= 0 ? e >> shift : e / B; }
    __device__ __forceinline__ uint32_t mod(uint32_t e) const { return shift >= 0 ? e & (B - 1u) : e % B; }
};

__device__ __forceinline__ uint16_t half_of(const uint4 &v, uint32_t q) {
    const uint32_t w = q < 4u ? (q < 2u ? v.x : v.y) : (q < 6u ? v.z : v.w);
    return (uint16_t) (w >> ((q & 1u) * 16u));
}

// N 16-byte value vectors of one lane (256 values apart) and their block
// columns; positions past the row give zeros and CS_INVALID_COL.
template <unsigned N>
__device__ __forceinline__ void load_steps(const uint16_t *vrow, const uint32_t *bci, const block_div &bd,
                                           uint32_t ell_cols, uint32_t first, uint4 (&v)[N], uint32_t (&bc)[N]) {
#pragma unroll
    for (unsigned u = 0; u < N; ++u) {
        const uint32_t e0 = first + u * 256u;
        const bool in = e0 < ell_cols;
        v[u] = in ? ld_stream_v4(vrow + e0) : make_uint4(0u, 0u, 0u, 0u);
        bc[u] = in ? __ldg(bci + bd.div(e0)) : CS_INVALID_COL;
    }
}

} // namespace csb
