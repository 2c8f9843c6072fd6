// Sliced-ELL row emission shared by the single-partition and batched
// converters: row r owns the w slots [base, base + w) of its slice; its n
// real (column, value) pairs go into the first n slots in CSR order, the rest
// is padding (CS_INVALID_COL, 0) -- sliced_ell_from_compressed.cuh:49-80.
//
// A group of GL lanes (GL in {32, 16, 8, 4}) writes one row.  The output is
// written 4 slots per lane with 16-byte column and 8-byte value stores once
// base + k is a multiple of 4; the unaligned head (< 4 slots) and the tail are
// written one slot at a time.  Requires col_idx 16-byte and val 8-byte
// aligned.
#pragma once

#include "common.cuh"

namespace csb {

template <unsigned GL>
__device__ __forceinline__ void sell_emit_row_vec(const uint32_t *__restrict__ idx, const uint16_t *__restrict__ val,
                                                  uint32_t a, uint32_t n, uint32_t w, std::size_t base,
                                                  uint32_t *__restrict__ col_idx, uint16_t *__restrict__ out_val,
                                                  unsigned gl) {
    if (n > w) n = w;
    const uint32_t head = min((uint32_t) ((4u - (uint32_t) (base & 3u)) & 3u), w);
    if (gl < head) {
        const bool real = gl < n;
        col_idx[base + gl] = real ? __ldg(idx + a + gl) : CS_INVALID_COL;
        out_val[base + gl] = real ? __ldg(reinterpret_cast<const unsigned short *>(val) + a + gl) : (uint16_t) 0u;
    }
    const uint32_t body_end = head + ((w - head) & ~3u);
    for (uint32_t k = head + 4u * gl; k < body_end; k += 4u * GL) {
        uint4 ci;
        uint2 vv;
        if (k + 4u <= n) {
            const uint32_t *ip = idx + a + k;
            const unsigned short *vp = reinterpret_cast<const unsigned short *>(val) + a + k;
            ci = make_uint4(__ldg(ip), __ldg(ip + 1), __ldg(ip + 2), __ldg(ip + 3));
            vv.x = (uint32_t) __ldg(vp) | ((uint32_t) __ldg(vp + 1) << 16);
            vv.y = (uint32_t) __ldg(vp + 2) | ((uint32_t) __ldg(vp + 3) << 16);
        } else if (k >= n) {
            ci = make_uint4(CS_INVALID_COL, CS_INVALID_COL, CS_INVALID_COL, CS_INVALID_COL);
            vv = make_uint2(0u, 0u);
        } else {
            uint32_t c[4];
            uint32_t v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool real = k + j < n;
                c[j] = real ? __ldg(idx + a + k + j) : CS_INVALID_COL;
                v[j] = real ? (uint32_t) __ldg(reinterpret_cast<const unsigned short *>(val) + a + k + j) : 0u;
            }
            ci = make_uint4(c[0], c[1], c[2], c[3]);
            vv = make_uint2(v[0] | (v[1] << 16), v[2] | (v[3] << 16));
        }
        *reinterpret_cast<uint4 *>(col_idx + base + k) = ci;
        *reinterpret_cast<uint2 *>(out_val + base + k) = vv;
    }
    for (uint32_t k = body_end + gl; k < w; k += GL) {
        const bool real = k < n;
        col_idx[base + k] = real ? __ldg(idx + a + k) : CS_INVALID_COL;
        out_val[base + k] = real ? __ldg(reinterpret_cast<const unsigned short *>(val) + a + k) : (uint16_t) 0u;
    }
}

} // namespace csb
