// fp16 row-segment loads and compensated fp32 accumulation shared by the
// grouped-moments kernels (single partition and served requests).
#pragma once

#include "common.cuh"

namespace csb {

// Raw loads of L consecutive fp16 values (kept as packed words so a batch of
// rows can be in flight before any conversion).
template <int L>
struct raw_vec {
    static constexpr int W = (L + 1) / 2; // 32-bit words
    uint32_t w[W];
};

template <int L>
__device__ __forceinline__ void load_raw(const uint16_t *p, raw_vec<L> &r) {
    if constexpr (L == 8) {
        const uint4 v = ld_stream_v4(p);
        r.w[0] = v.x;
        r.w[1] = v.y;
        r.w[2] = v.z;
        r.w[3] = v.w;
    } else if constexpr (L == 4) {
        const uint2 v = __ldg(reinterpret_cast<const uint2 *>(p));
        r.w[0] = v.x;
        r.w[1] = v.y;
    } else if constexpr (L == 2) {
        r.w[0] = __ldg(reinterpret_cast<const unsigned int *>(p));
    } else {
        r.w[0] = __ldg(reinterpret_cast<const unsigned short *>(p));
    }
}

template <int L>
__device__ __forceinline__ void zero_raw(raw_vec<L> &r) {
#pragma unroll
    for (int i = 0; i < raw_vec<L>::W; ++i) r.w[i] = 0u;
}

template <int L>
__device__ __forceinline__ void unpack(const raw_vec<L> &r, float *x) {
    if constexpr (L == 1) {
        x[0] = h2f((uint16_t) r.w[0]);
    } else {
#pragma unroll
        for (int i = 0; i < L / 2; ++i) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&r.w[i]));
            x[2 * i] = f.x;
            x[2 * i + 1] = f.y;
        }
    }
}

// Knuth two-sum folded into a running (hi, lo) pair.
__device__ __forceinline__ void two_sum_acc(float &hi, float &lo, float b) {
    const float s = __fadd_rn(hi, b);
    const float bb = __fsub_rn(s, hi);
    const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    hi = s;
    lo = __fadd_rn(lo, err);
}

} // namespace csb
