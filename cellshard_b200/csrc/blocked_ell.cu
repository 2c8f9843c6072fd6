// CSR -> Blocked-ELL on the GPU.
//
// The reference builds Blocked-ELL with two serial host passes per row block
// (src/convert/blocked_ell_from_compressed.cuh:33-91 counts distinct column
// blocks with epoch marks; :294-342 sorts them with qsort, maps block -> slot
// and scatters values into a memset output).  Here:
//
//   shape   one warp per row block sets a shared-memory bitmap over column
//           blocks from the row block's contiguous CSR index range; popc gives
//           the distinct count, atomicMax the global ell_width.  The bitmaps
//           are kept in scratch for the emit pass.
//   emit    one CTA per output row assembles the row's padded ELL segment in
//           shared memory (zero, scatter, then 16-byte streaming stores), the
//           slot of column block b being prefix(word) + popc(word & below(b)),
//           which is exactly the rank of b in the ascending qsort order.  The
//           first row of each row block also writes the row block's
//           blockColIdx (set bits in ascending order, CS_INVALID_COL padding).
//
// Values of duplicate columns inside one row resolve to the last occurrence
// (the reference's overwrite order): such rows are detected with a block-wide
// vote and scattered by one thread in CSR order.
#include "common.cuh"

#include <cstdlib>
#include <cstring>

namespace csb {
namespace {

constexpr unsigned kShapeWarps = 4;
constexpr unsigned kEmitThreads = 256;
constexpr unsigned kSegHalves = 32768; // 64 KB row segment in shared memory

__device__ __forceinline__ uint32_t div_b(uint32_t c, uint32_t B, int shift) {
    return shift >= 0 ? (c >> shift) : (c / B);
}

__global__ void __launch_bounds__(kShapeWarps * 32) bell_shape_kernel(
    const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx, uint32_t rows, uint32_t cols, uint32_t nnz,
    uint32_t B, int shift, uint32_t row_blocks, uint32_t words, uint32_t *__restrict__ bitmaps,
    unsigned long long *__restrict__ shape, uint32_t *status) {
    extern __shared__ uint32_t shape_smem[];
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t *bits = shape_smem + (std::size_t) warp * words;
    uint32_t local_max = 0u;
    unsigned long long local_total = 0ull;
    uint32_t bad = 0u;
    for (uint32_t rb = blockIdx.x * kShapeWarps + warp; rb < row_blocks; rb += gridDim.x * kShapeWarps) {
        for (uint32_t w = lane; w < words; w += 32u) bits[w] = 0u;
        __syncwarp();
        const uint32_t r0 = rb * B;
        const uint32_t r1 = min(rows, r0 + B);
        uint32_t ptr_bad = 0u;
        for (uint32_t r = r0 + lane; r < r1; r += 32u) {
            const uint32_t a = ptr[r], b = ptr[r + 1u];
            if (b < a || b > nnz) ptr_bad = 1u;
        }
        ptr_bad = __any_sync(0xffffffffu, ptr_bad);
        if (ptr_bad) {
            bad |= CS_STATUS_BAD_POINTERS;
        } else {
            const uint32_t b = ptr[r0], e = ptr[r1];
            auto mark = [&](uint32_t c) {
                if (c >= cols) {
                    bad |= CS_STATUS_INDEX_RANGE;
                    return;
                }
                const uint32_t bc = div_b(c, B, shift);
                atomicOr(bits + (bc >> 5), 1u << (bc & 31u));
            };
            // scalar head to a 16-byte boundary, 16-byte body, scalar tail
            const bool vec = (reinterpret_cast<uintptr_t>(idx) & 15u) == 0u;
            const uint32_t head_end = vec ? min(e, (b + 3u) & ~3u) : e;
            for (uint32_t i = b + lane; i < head_end; i += 32u) mark(idx[i]);
            if (vec) {
                const uint32_t nvec = (e - head_end) >> 2;
                const uint4 *v4 = reinterpret_cast<const uint4 *>(idx + head_end);
                // the four columns of a vector usually share a bitmap word (rows are
                // mostly sorted): their bits are OR-ed locally, one atomic per word run
                auto mark4 = [&](const uint4 &q) {
                    const uint32_t c[4] = {q.x, q.y, q.z, q.w};
                    uint32_t word = 0xffffffffu, m = 0u;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if (c[k] >= cols) {
                            bad |= CS_STATUS_INDEX_RANGE;
                            continue;
                        }
                        const uint32_t bc = div_b(c[k], B, shift);
                        if ((bc >> 5) != word) {
                            if (m != 0u) atomicOr(bits + word, m);
                            word = bc >> 5;
                            m = 0u;
                        }
                        m |= 1u << (bc & 31u);
                    }
                    if (m != 0u) atomicOr(bits + word, m);
                };
                // eight vectors per lane loaded before any is marked
                constexpr unsigned kV = 8;
                for (uint32_t k0 = lane; k0 < nvec; k0 += 32u * kV) {
                    uint4 q[kV];
#pragma unroll
                    for (unsigned u = 0; u < kV; ++u) {
                        const uint32_t k = k0 + 32u * u;
                        q[u] = k < nvec ? __ldg(v4 + k) : make_uint4(0u, 0u, 0u, 0u);
                    }
#pragma unroll
                    for (unsigned u = 0; u < kV; ++u)
                        if (k0 + 32u * u < nvec) mark4(q[u]);
                }
                for (uint32_t i = head_end + (nvec << 2) + lane; i < e; i += 32u) mark(idx[i]);
            }
        }
        __syncwarp();
        uint32_t cnt = 0u;
        for (uint32_t w = lane; w < words; w += 32u) {
            const uint32_t word = bits[w];
            cnt += __popc(word);
            if (bitmaps != nullptr) bitmaps[(std::size_t) rb * words + w] = word;
        }
        cnt = __reduce_add_sync(0xffffffffu, cnt);
        local_max = max(local_max, cnt);
        local_total += cnt;
        __syncwarp();
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0u) {
        if (local_max != 0u) atomicMax(shape, (unsigned long long) local_max);
        if (local_total != 0ull) atomicAdd(shape + 1, local_total);
        status_or(status, bad);
    }
}

__global__ void __launch_bounds__(kEmitThreads) bell_emit_kernel(
    const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx, const uint16_t *__restrict__ val, uint32_t rows,
    uint32_t cols, uint32_t nnz, uint32_t B, int shift, uint32_t words, uint32_t width, uint32_t ell_cols,
    const uint32_t *__restrict__ bitmaps, uint32_t *__restrict__ out_bci, uint16_t *__restrict__ out_val,
    uint32_t *__restrict__ d_nnz, uint32_t *status) {
    extern __shared__ __align__(16) unsigned char emit_smem[];
    uint16_t *buf = reinterpret_cast<uint16_t *>(emit_smem);                  // [kSegHalves]
    uint2 *ix = reinterpret_cast<uint2 *>(emit_smem + kSegHalves * sizeof(uint16_t)); // [words]
    __shared__ uint32_t count_smem;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const bool vec_ok = ((ell_cols & 7u) == 0u) && ((reinterpret_cast<uintptr_t>(out_val) & 15u) == 0u);
    uint32_t my_nnz = 0u;
    uint32_t bad = 0u;
    uint32_t prev_rb = 0xffffffffu;
    for (uint32_t r = blockIdx.x; r < rows; r += gridDim.x) {
        const uint32_t rb = div_b(r, B, shift);
        if (rb != prev_rb) {
            __syncthreads();
            if (warp == 0) {
                uint32_t carry = 0u;
                for (uint32_t w0 = 0; w0 < words; w0 += 32u) {
                    const uint32_t w = w0 + lane;
                    const uint32_t word = w < words ? bitmaps[(std::size_t) rb * words + w] : 0u;
                    const uint32_t c = __popc(word);
                    const uint32_t incl = warp_inclusive_scan(c);
                    if (w < words) ix[w] = make_uint2(word, carry + incl - c);
                    carry += __shfl_sync(0xffffffffu, incl, 31);
                }
                if (lane == 0u) count_smem = carry;
            }
            __syncthreads();
            prev_rb = rb;
        }
        const uint32_t count = count_smem;
        if (count > width) bad |= CS_STATUS_INDEX_RANGE;
        if (r == rb * B && out_bci != nullptr) {
            uint32_t *row_bci = out_bci + (std::size_t) rb * width;
            for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
                uint32_t word = ix[w].x;
                uint32_t pos = ix[w].y;
                while (word != 0u) {
                    const uint32_t bit = __ffs(word) - 1u;
                    if (pos < width) row_bci[pos] = w * 32u + bit;
                    ++pos;
                    word &= word - 1u;
                }
            }
            for (uint32_t s = count + threadIdx.x; s < width; s += blockDim.x) row_bci[s] = CS_INVALID_COL;
        }
        const uint32_t a = ptr[r], e = ptr[r + 1u];
        const bool ptr_bad = e < a || e > nnz;
        // rows whose columns are not strictly increasing take the ordered path
        int unordered = 0;
        if (!ptr_bad) {
            for (uint32_t i = a + threadIdx.x; i + 1u < e; i += blockDim.x)
                if (idx[i] >= idx[i + 1u]) unordered = 1;
        }
        unordered = __syncthreads_or(unordered);
        std::size_t row_base = (std::size_t) r * ell_cols;
        for (uint32_t seg0 = 0; seg0 < ell_cols; seg0 += kSegHalves) {
            const uint32_t seg_len = min(kSegHalves, ell_cols - seg0);
            // zero the segment
            for (uint32_t k = threadIdx.x * 8u; k < seg_len; k += blockDim.x * 8u) {
                if (k + 8u <= seg_len)
                    *reinterpret_cast<uint4 *>(buf + k) = make_uint4(0u, 0u, 0u, 0u);
                else
                    for (uint32_t j = k; j < seg_len; ++j) buf[j] = 0u;
            }
            __syncthreads();
            if (!ptr_bad) {
                if (!unordered) {
                    for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
                        const uint32_t c = idx[i];
                        if (c >= cols) continue;
                        const uint32_t bc = div_b(c, B, shift);
                        const uint2 x = ix[bc >> 5];
                        const uint32_t slot = x.y + __popc(x.x & ((1u << (bc & 31u)) - 1u));
                        const uint32_t pos = slot * B + (c - bc * B) - seg0;
                        if (slot < width && pos < seg_len) buf[pos] = val[i];
                    }
                } else if (threadIdx.x == 0) {
                    for (uint32_t i = a; i < e; ++i) {
                        const uint32_t c = idx[i];
                        if (c >= cols) continue;
                        const uint32_t bc = div_b(c, B, shift);
                        const uint2 x = ix[bc >> 5];
                        const uint32_t slot = x.y + __popc(x.x & ((1u << (bc & 31u)) - 1u));
                        const uint32_t pos = slot * B + (c - bc * B) - seg0;
                        if (slot < width && pos < seg_len) buf[pos] = val[i];
                    }
                }
            } else {
                bad |= CS_STATUS_BAD_POINTERS;
            }
            __syncthreads();
            uint16_t *dst = out_val + row_base + seg0;
            if (vec_ok) {
                for (uint32_t k = threadIdx.x * 8u; k < seg_len; k += blockDim.x * 8u) {
                    const uint4 v = *reinterpret_cast<const uint4 *>(buf + k);
                    const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        my_nnz += ((w4[q] & 0x7fffu) != 0u) + ((w4[q] & 0x7fff0000u) != 0u);
                    st_stream_v4(dst + k, v);
                }
            } else {
                for (uint32_t k = threadIdx.x; k < seg_len; k += blockDim.x) {
                    const uint16_t v = buf[k];
                    my_nnz += half_nonzero(v);
                    dst[k] = v;
                }
            }
            __syncthreads();
        }
    }
    my_nnz = __reduce_add_sync(0xffffffffu, my_nnz);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0u) {
        if (my_nnz != 0u) atomicAdd(d_nnz, my_nnz);
        status_or(status, bad);
    }
}


// Emit with shared-memory row staging and bulk (TMA) stores.  A CTA takes
// whole row blocks (the block's column index is loaded once for its B rows)
// and owns NBUF row buffers (~64 KB in total, three CTAs per SM): a row is
// scattered into a zeroed buffer by the threads, then one thread hands the
// whole padded row to the copy engine and the CTA moves on while it streams
// out.  A buffer is re-zeroed only after the bulk store that read it has
// finished reading.  Rows whose columns are not strictly increasing are
// redone in CSR order by one thread (the reference's overwrite order).
template <int NBUF>
__global__ void __launch_bounds__(kEmitThreads, 3) bell_emit_tma_kernel(
    const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx, const uint16_t *__restrict__ val, uint32_t rows,
    uint32_t cols, uint32_t nnz, uint32_t B, int shift, uint32_t words, uint32_t width, uint32_t ell_cols,
    const uint32_t *__restrict__ bitmaps, uint32_t *__restrict__ out_bci, uint16_t *__restrict__ out_val,
    uint32_t *__restrict__ d_nnz, uint32_t *status) {
    extern __shared__ __align__(128) unsigned char tma_smem[];
    constexpr int PF = 8; // entries per thread prefetched for the next row
    const uint32_t row_bytes = ell_cols * 2u;
    const uint32_t stride = (row_bytes + 127u) & ~127u;
    uint2 *ix = reinterpret_cast<uint2 *>(tma_smem + (std::size_t) NBUF * stride);
    uint32_t *rp = reinterpret_cast<uint32_t *>(ix + words); // [B + 1] row pointers of the block
    __shared__ uint32_t count_smem;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t row_blocks = (rows + B - 1u) / B;
    for (uint32_t k = threadIdx.x * 16u; k < NBUF * stride; k += blockDim.x * 16u)
        *reinterpret_cast<uint4 *>(tma_smem + k) = make_uint4(0u, 0u, 0u, 0u);
    uint32_t my_nnz = 0u, bad = 0u, iter = 0u;
    uint32_t nc[PF];
    uint16_t nv[PF];
    auto prefetch = [&](uint32_t a, uint32_t e) {
#pragma unroll
        for (int k = 0; k < PF; ++k) {
            const uint32_t i = a + threadIdx.x + (uint32_t) k * kEmitThreads;
            nc[k] = i < e ? __ldg(idx + i) : 0xffffffffu;
            nv[k] = i < e ? __ldg(reinterpret_cast<const unsigned short *>(val) + i) : (uint16_t) 0u;
        }
    };
    for (uint32_t rb = blockIdx.x; rb < row_blocks; rb += gridDim.x) {
        const uint32_t r_beg = rb * B, r_end = min(rows, rb * B + B);
        __syncthreads();
        if (warp == 0) {
            uint32_t carry = 0u;
            for (uint32_t w0 = 0; w0 < words; w0 += 32u) {
                const uint32_t w = w0 + lane;
                const uint32_t word = w < words ? bitmaps[(std::size_t) rb * words + w] : 0u;
                const uint32_t c = __popc(word);
                const uint32_t incl = warp_inclusive_scan(c);
                if (w < words) ix[w] = make_uint2(word, carry + incl - c);
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0u) count_smem = carry;
        }
        for (uint32_t r = threadIdx.x; r <= r_end - r_beg; r += blockDim.x) rp[r] = ptr[r_beg + r];
        __syncthreads();
        const uint32_t count = count_smem;
        if (count > width) bad |= CS_STATUS_INDEX_RANGE;
        if (out_bci != nullptr) {
            uint32_t *row_bci = out_bci + (std::size_t) rb * width;
            for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
                uint32_t word = ix[w].x;
                uint32_t pos = ix[w].y;
                while (word != 0u) {
                    const uint32_t bit = __ffs(word) - 1u;
                    if (pos < width) row_bci[pos] = w * 32u + bit;
                    ++pos;
                    word &= word - 1u;
                }
            }
            for (uint32_t s2 = count + threadIdx.x; s2 < width; s2 += blockDim.x) row_bci[s2] = CS_INVALID_COL;
        }
        {
            const uint32_t a0 = rp[0], e0 = rp[1];
            prefetch(a0, (e0 < a0 || e0 > nnz) ? a0 : e0);
        }
        for (uint32_t r = r_beg; r < r_end; ++r, ++iter) {
            uint32_t cc[PF];
            uint16_t cv[PF];
#pragma unroll
            for (int k = 0; k < PF; ++k) {
                cc[k] = nc[k];
                cv[k] = nv[k];
            }
            const uint32_t a = rp[r - r_beg], e = rp[r - r_beg + 1u];
            const bool ptr_bad = e < a || e > nnz;
            if (ptr_bad) bad |= CS_STATUS_BAD_POINTERS;
            if (r + 1u < r_end) {
                const uint32_t a1 = rp[r - r_beg + 1u], e1 = rp[r - r_beg + 2u];
                prefetch(a1, (e1 < a1 || e1 > nnz) ? a1 : e1);
            }
            uint16_t *buf = reinterpret_cast<uint16_t *>(tma_smem + (std::size_t) (iter % NBUF) * stride);
            if (iter >= (uint32_t) NBUF) {
                if (threadIdx.x == 0) bulk_wait_read<NBUF - 1>();
                __syncthreads();
                for (uint32_t k = threadIdx.x * 8u; k < ell_cols; k += blockDim.x * 8u)
                    *reinterpret_cast<uint4 *>(buf + k) = make_uint4(0u, 0u, 0u, 0u);
                __syncthreads();
            }
            int unordered = 0;
            uint32_t row_nnz = 0u;
            auto place = [&](uint32_t i, uint32_t c, uint16_t v) {
                if (c >= cols) return;
                const uint32_t bc = div_b(c, B, shift);
                const uint2 x = ix[bc >> 5];
                const uint32_t slot = x.y + __popc(x.x & ((1u << (bc & 31u)) - 1u));
                if (slot >= width) return;
                buf[slot * B + (c - bc * B)] = v;
                row_nnz += half_nonzero(v);
            };
            if (!ptr_bad) {
#pragma unroll
                for (int k = 0; k < PF; ++k) {
                    const uint32_t i = a + threadIdx.x + (uint32_t) k * kEmitThreads;
                    // the next entry belongs to the next lane (or, for lane 31, the next warp)
                    uint32_t nxt = __shfl_down_sync(0xffffffffu, cc[k], 1);
                    if (lane == 31u && i + 1u < e) nxt = __ldg(idx + i + 1u);
                    if (i < e) {
                        if (i + 1u < e && cc[k] >= nxt) unordered = 1;
                        place(i, cc[k], cv[k]);
                    }
                }
                for (uint32_t i = a + PF * kEmitThreads + threadIdx.x; i < e; i += blockDim.x) {
                    const uint32_t c = __ldg(idx + i);
                    if (i + 1u < e && c >= __ldg(idx + i + 1u)) unordered = 1;
                    place(i, c, val[i]);
                }
            }
            if (__syncthreads_or(unordered)) {
                for (uint32_t k = threadIdx.x * 8u; k < ell_cols; k += blockDim.x * 8u)
                    *reinterpret_cast<uint4 *>(buf + k) = make_uint4(0u, 0u, 0u, 0u);
                __syncthreads();
                if (threadIdx.x == 0) {
                    for (uint32_t i = a; i < e; ++i) {
                        const uint32_t c = idx[i];
                        if (c >= cols) continue;
                        const uint32_t bc = div_b(c, B, shift);
                        const uint2 x = ix[bc >> 5];
                        const uint32_t slot = x.y + __popc(x.x & ((1u << (bc & 31u)) - 1u));
                        if (slot < width) buf[slot * B + (c - bc * B)] = val[i];
                    }
                }
                __syncthreads();
                row_nnz = 0u;
                for (uint32_t k = threadIdx.x; k < ell_cols; k += blockDim.x) row_nnz += half_nonzero(buf[k]);
            }
            my_nnz += row_nnz;
            fence_proxy_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                bulk_store_s2g(out_val + (std::size_t) r * ell_cols, buf, row_bytes);
                bulk_commit();
            }
        }
    }
    if (threadIdx.x == 0) bulk_wait_all();
    my_nnz = __reduce_add_sync(0xffffffffu, my_nnz);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0u) {
        if (my_nnz != 0u) atomicAdd(d_nnz, my_nnz);
        status_or(status, bad);
    }
}

int pow2_shift(uint32_t B) {
    if (B == 0u || (B & (B - 1u)) != 0u) return -1;
    int s = 0;
    while ((1u << s) != B) ++s;
    return s;
}

uint32_t col_words(uint32_t cols, uint32_t B) {
    const uint32_t col_blocks = (cols + B - 1u) / B;
    return (col_blocks + 31u) / 32u;
}

constexpr uint32_t kMaxShapeWords = 4096; // 131072 column blocks

int check_src(const cs_compressed_view *src, uint32_t B, const char *who) {
    if (src == nullptr) {
        set_error("%s: null source view", who);
        return 0;
    }
    if (B == 0u) {
        set_error("%s: block_size must be nonzero", who);
        return 0;
    }
    if (src->axis != CS_COMPRESSED_BY_ROW) {
        set_error("%s: source must be compressed by row", who);
        return 0;
    }
    if (col_words(src->cols, B) > kMaxShapeWords) {
        set_error("%s: %u columns at block %u exceed the column-block limit", who, src->cols, B);
        return 0;
    }
    if (src->rows != 0u && src->majorPtr == nullptr) {
        set_error("%s: null majorPtr", who);
        return 0;
    }
    return 1;
}

} // namespace

int blocked_ell_shape_launch(const cs_compressed_view *src, uint32_t B, uint64_t *d_shape, uint32_t *bitmaps,
                             uint32_t *d_status, cudaStream_t stream) {
    const uint32_t row_blocks = (src->rows + B - 1u) / B;
    const uint32_t words = col_words(src->cols, B);
    if (row_blocks == 0u || words == 0u) return 1;
    const std::size_t smem = (std::size_t) kShapeWarps * words * sizeof(uint32_t);
    if (smem > 48u * 1024u &&
        !cuda_ok(cudaFuncSetAttribute(bell_shape_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "bell_shape smem attribute"))
        return 0;
    uint32_t grid = (row_blocks + kShapeWarps - 1u) / kShapeWarps;
    const uint32_t cap = (uint32_t) sm_count() * 32u;
    if (grid > cap) grid = cap;
    bell_shape_kernel<<<grid, kShapeWarps * 32, smem, stream>>>(
        src->majorPtr, src->minorIdx, src->rows, src->cols, src->nnz, B, pow2_shift(B), row_blocks, words, bitmaps,
        reinterpret_cast<unsigned long long *>(d_shape), d_status);
    return launch_ok("bell_shape_kernel");
}

int blocked_ell_emit_launch(const cs_compressed_view *src, const cs_blocked_ell_view *dst, uint32_t *d_nnz,
                            const uint32_t *bitmaps, uint32_t *d_status, cudaStream_t stream) {
    const uint32_t B = dst->block_size;
    const uint32_t words = col_words(src->cols, B);
    const uint32_t width = dst->ell_cols / B;
    if (src->rows == 0u || dst->ell_cols == 0u) return 1;
    // bulk-store path: whole padded rows in shared memory, 16-byte aligned rows
    const std::size_t row_bytes = (std::size_t) dst->ell_cols * 2u;
    const std::size_t stride = (row_bytes + 127u) & ~(std::size_t) 127u;
    const bool tma_ok = (dst->ell_cols % 8u) == 0u && (reinterpret_cast<uintptr_t>(dst->val) & 15u) == 0u &&
                        dst->ell_cols <= kSegHalves;
    if (tma_ok) {
        const int nbuf = stride <= 8192u ? 8 : (stride <= 16384u ? 4 : (stride <= 32768u ? 2 : 1));
        const std::size_t tsmem =
            (std::size_t) nbuf * stride + (std::size_t) words * sizeof(uint2) + ((std::size_t) B + 1u) * 4u;
        if (tsmem <= 72u * 1024u) {
            const uint32_t row_blocks = (src->rows + B - 1u) / B;
            uint32_t tgrid = (uint32_t) sm_count() * 3u;
            if (tgrid > row_blocks) tgrid = row_blocks;
            auto launch = [&](auto kern) {
                if (!cuda_ok(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) tsmem),
                             "bell_emit_tma smem attribute"))
                    return 0;
                kern<<<tgrid, kEmitThreads, tsmem, stream>>>(src->majorPtr, src->minorIdx, src->val, src->rows,
                                                              src->cols, src->nnz, B, pow2_shift(B), words, width,
                                                              dst->ell_cols, bitmaps, dst->blockColIdx, dst->val,
                                                              d_nnz, d_status);
                return launch_ok("bell_emit_tma_kernel");
            };
            if (nbuf == 8) return launch(bell_emit_tma_kernel<8>);
            if (nbuf == 4) return launch(bell_emit_tma_kernel<4>);
            if (nbuf == 2) return launch(bell_emit_tma_kernel<2>);
            return launch(bell_emit_tma_kernel<1>);
        }
    }
    const std::size_t smem = (std::size_t) kSegHalves * sizeof(uint16_t) + (std::size_t) words * sizeof(uint2);
    if (!cuda_ok(cudaFuncSetAttribute(bell_emit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "bell_emit smem attribute"))
        return 0;
    uint32_t grid = src->rows;
    const uint32_t cap = (uint32_t) sm_count() * 64u;
    if (grid > cap) grid = cap;
    bell_emit_kernel<<<grid, kEmitThreads, smem, stream>>>(src->majorPtr, src->minorIdx, src->val, src->rows,
                                                           src->cols, src->nnz, B, pow2_shift(B), words, width,
                                                           dst->ell_cols, bitmaps, dst->blockColIdx, dst->val, d_nnz,
                                                           d_status);
    return launch_ok("bell_emit_kernel");
}

// ---------------------------------------------------------------------------
// Host-owned results (packed exactly like sparse::allocate).
// ---------------------------------------------------------------------------
int host_blocked_ell_allocate(cs_host_blocked_ell *m) {
    const uint32_t B = m->block_size;
    const std::size_t rb = B == 0u ? 0u : (m->rows + B - 1u) / B;
    const std::size_t width = (B == 0u || m->ell_cols == 0u) ? 0u : m->ell_cols / B;
    const std::size_t idx_bytes = rb * width * sizeof(uint32_t);
    const std::size_t val_offset = align_up(idx_bytes, alignof(uint16_t));
    const std::size_t total = val_offset + (std::size_t) m->rows * m->ell_cols * sizeof(uint16_t);
    m->flags = 0u;
    m->storage = nullptr;
    m->blockColIdx = nullptr;
    m->val = nullptr;
    if (total == 0u) return 1;
    void *storage = std::malloc(total);
    if (storage == nullptr) return 0;
    m->storage = storage;
    m->blockColIdx = idx_bytes != 0u ? (uint32_t *) storage : nullptr;
    m->val = (m->rows != 0u && m->ell_cols != 0u) ? (uint16_t *) ((char *) storage + val_offset) : nullptr;
    return 1;
}

// RAII device buffers for the synchronous host wrappers.
struct dev_buf {
    void *p = nullptr;
    ~dev_buf() {
        if (p) cudaFree(p);
    }
    bool alloc(std::size_t bytes, const char *what) {
        if (bytes == 0) bytes = 16;
        return cuda_ok(cudaMalloc(&p, bytes), what) != 0;
    }
};

struct staged_csr {
    dev_buf ptr, idx, val;
    cs_compressed_view view{};
    bool upload(const cs_host_compressed *src, cudaStream_t stream) {
        view.rows = src->rows;
        view.cols = src->cols;
        view.nnz = src->nnz;
        view.axis = src->axis;
        const std::size_t major = (std::size_t) (src->axis == CS_COMPRESSED_BY_COL ? src->cols : src->rows) + 1u;
        if (!ptr.alloc(major * 4u, "cudaMalloc csr ptr") || !idx.alloc((std::size_t) src->nnz * 4u, "cudaMalloc csr idx") ||
            !val.alloc((std::size_t) src->nnz * 2u, "cudaMalloc csr val"))
            return false;
        view.majorPtr = (uint32_t *) ptr.p;
        view.minorIdx = (uint32_t *) idx.p;
        view.val = (uint16_t *) val.p;
        if (src->majorPtr == nullptr) {
            if (!cuda_ok(cudaMemsetAsync(ptr.p, 0, major * 4u, stream), "memset csr ptr")) return false;
        } else if (!cuda_ok(cudaMemcpyAsync(ptr.p, src->majorPtr, major * 4u, cudaMemcpyHostToDevice, stream),
                            "H2D csr ptr")) {
            return false;
        }
        if (src->nnz != 0u) {
            if (!cuda_ok(cudaMemcpyAsync(idx.p, src->minorIdx, (std::size_t) src->nnz * 4u, cudaMemcpyHostToDevice,
                                         stream),
                         "H2D csr idx") ||
                !cuda_ok(cudaMemcpyAsync(val.p, src->val, (std::size_t) src->nnz * 2u, cudaMemcpyHostToDevice, stream),
                         "H2D csr val"))
                return false;
        }
        return true;
    }
};

int shape_on_device(const cs_compressed_view *v, uint32_t B, uint64_t shape[2], dev_buf *bitmaps, uint32_t *status_out,
                    cudaStream_t stream) {
    dev_buf d_shape, d_status;
    if (!d_shape.alloc(32, "cudaMalloc shape") || !d_status.alloc(4, "cudaMalloc status")) return 0;
    if (!cuda_ok(cudaMemsetAsync(d_shape.p, 0, 32, stream), "memset shape") ||
        !cuda_ok(cudaMemsetAsync(d_status.p, 0, 4, stream), "memset status"))
        return 0;
    uint32_t *bm = nullptr;
    if (bitmaps != nullptr) {
        const std::size_t rb = (v->rows + B - 1u) / B;
        if (!bitmaps->alloc(rb * col_words(v->cols, B) * 4u, "cudaMalloc bitmaps")) return 0;
        bm = (uint32_t *) bitmaps->p;
    }
    if (!blocked_ell_shape_launch(v, B, (uint64_t *) d_shape.p, bm, (uint32_t *) d_status.p, stream)) return 0;
    if (!cuda_ok(cudaMemcpyAsync(shape, d_shape.p, 16, cudaMemcpyDeviceToHost, stream), "D2H shape") ||
        !cuda_ok(cudaMemcpyAsync(status_out, d_status.p, 4, cudaMemcpyDeviceToHost, stream), "D2H status") ||
        !cuda_ok(cudaStreamSynchronize(stream), "sync shape"))
        return 0;
    return 1;
}

} // namespace csb

using namespace csb;

extern "C" void cs_b200_host_blocked_ell_clear(cs_host_blocked_ell *m) {
    if (m == nullptr) return;
    if (m->storage != nullptr)
        std::free(m->storage);
    else {
        std::free(m->blockColIdx);
        std::free(m->val);
    }
    std::memset(m, 0, sizeof(*m));
}

extern "C" int cs_b200_blocked_ell_scratch_bytes(uint32_t rows, uint32_t cols, uint32_t block_size,
                                                 size_t *out_bytes) {
    if (out_bytes == nullptr || block_size == 0u) {
        set_error("blocked_ell_scratch_bytes: null output or zero block size");
        return 0;
    }
    const std::size_t rb = (rows + block_size - 1u) / block_size;
    *out_bytes = align_up(rb * col_words(cols, block_size) * sizeof(uint32_t) + 16u, 256);
    return 1;
}

extern "C" int cs_b200_blocked_ell_shape(const cs_compressed_view *src, uint32_t block_size, uint64_t *d_shape,
                                         void *d_scratch, size_t scratch_bytes, uint32_t *d_status, cs_stream_t s) {
    if (!check_src(src, block_size, "blocked_ell_shape")) return 0;
    if (d_shape == nullptr) {
        set_error("blocked_ell_shape: null d_shape");
        return 0;
    }
    if (d_scratch != nullptr) {
        size_t need = 0;
        cs_b200_blocked_ell_scratch_bytes(src->rows, src->cols, block_size, &need);
        if (scratch_bytes < need) {
            set_error("blocked_ell_shape: scratch %zu < %zu", scratch_bytes, need);
            return 0;
        }
    }
    return blocked_ell_shape_launch(src, block_size, d_shape, (uint32_t *) d_scratch, d_status, as_stream(s));
}

extern "C" int cs_b200_blocked_ell_emit(const cs_compressed_view *src, const cs_blocked_ell_view *dst,
                                        uint32_t *d_nnz, const void *d_scratch, size_t scratch_bytes,
                                        uint32_t *d_status, cs_stream_t s) {
    if (dst == nullptr || !check_src(src, dst->block_size, "blocked_ell_emit")) {
        if (dst == nullptr) set_error("blocked_ell_emit: null destination view");
        return 0;
    }
    if (dst->rows != src->rows || dst->cols != src->cols || dst->ell_cols % dst->block_size != 0u) {
        set_error("blocked_ell_emit: destination geometry does not match the source");
        return 0;
    }
    size_t need = 0;
    cs_b200_blocked_ell_scratch_bytes(src->rows, src->cols, dst->block_size, &need);
    if (d_scratch == nullptr || scratch_bytes < need || d_nnz == nullptr) {
        set_error("blocked_ell_emit: scratch (%zu < %zu) or d_nnz missing", scratch_bytes, need);
        return 0;
    }
    return blocked_ell_emit_launch(src, dst, d_nnz, (const uint32_t *) d_scratch, d_status, as_stream(s));
}

extern "C" int cs_b200_blocked_ell_from_compressed(const cs_host_compressed *src, unsigned int block_size,
                                                   cs_host_blocked_ell *dst) {
    if (src == nullptr || dst == nullptr || block_size == 0u) {
        set_error("blocked_ell_from_compressed: null argument or zero block size");
        return 0;
    }
    if (src->axis != CS_COMPRESSED_BY_ROW) {
        set_error("blocked_ell_from_compressed: source must be compressed by row");
        return 0;
    }
    cudaStream_t stream = nullptr;
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream create")) return 0;
    struct stream_guard {
        cudaStream_t s;
        ~stream_guard() { cudaStreamDestroy(s); }
    } guard{stream};
    staged_csr csr;
    if (!csr.upload(src, stream)) return 0;
    if (!check_src(&csr.view, block_size, "blocked_ell_from_compressed")) return 0;
    uint64_t shape[2] = {0, 0};
    uint32_t status = 0;
    dev_buf bitmaps;
    if (src->rows != 0u && src->cols != 0u) {
        if (!shape_on_device(&csr.view, block_size, shape, &bitmaps, &status, stream)) return 0;
        if (status != 0u) {
            set_error("blocked_ell_from_compressed: invalid CSR (status 0x%x)", status);
            return 0;
        }
    }
    const uint32_t ell_width = (uint32_t) shape[0];
    cs_b200_host_blocked_ell_clear(dst);
    dst->rows = src->rows;
    dst->cols = src->cols;
    dst->nnz = src->nnz;
    dst->block_size = block_size;
    dst->ell_cols = ell_width * block_size;
    if (!host_blocked_ell_allocate(dst)) {
        set_error("blocked_ell_from_compressed: host allocation failed");
        return 0;
    }
    const std::size_t rb = (src->rows + block_size - 1u) / block_size;
    const std::size_t idx_bytes = rb * ell_width * sizeof(uint32_t);
    const std::size_t val_bytes = (std::size_t) src->rows * dst->ell_cols * sizeof(uint16_t);
    uint32_t nnz = 0u;
    if (idx_bytes != 0u && val_bytes != 0u) {
        dev_buf d_bci, d_val, d_nnz, d_status;
        if (!d_bci.alloc(idx_bytes, "cudaMalloc bci") || !d_val.alloc(val_bytes, "cudaMalloc ell val") ||
            !d_nnz.alloc(4, "cudaMalloc nnz") || !d_status.alloc(4, "cudaMalloc status")) {
            cs_b200_host_blocked_ell_clear(dst);
            return 0;
        }
        cs_blocked_ell_view dv{};
        dv.rows = dst->rows;
        dv.cols = dst->cols;
        dv.nnz = 0u;
        dv.block_size = block_size;
        dv.ell_cols = dst->ell_cols;
        dv.blockColIdx = (uint32_t *) d_bci.p;
        dv.val = (uint16_t *) d_val.p;
        bool ok = cuda_ok(cudaMemsetAsync(d_nnz.p, 0, 4, stream), "memset nnz") &&
                  cuda_ok(cudaMemsetAsync(d_status.p, 0, 4, stream), "memset status") &&
                  blocked_ell_emit_launch(&csr.view, &dv, (uint32_t *) d_nnz.p, (const uint32_t *) bitmaps.p,
                                          (uint32_t *) d_status.p, stream) &&
                  cuda_ok(cudaMemcpyAsync(dst->blockColIdx, d_bci.p, idx_bytes, cudaMemcpyDeviceToHost, stream),
                          "D2H bci") &&
                  cuda_ok(cudaMemcpyAsync(dst->val, d_val.p, val_bytes, cudaMemcpyDeviceToHost, stream), "D2H val") &&
                  cuda_ok(cudaMemcpyAsync(&nnz, d_nnz.p, 4, cudaMemcpyDeviceToHost, stream), "D2H nnz") &&
                  cuda_ok(cudaMemcpyAsync(&status, d_status.p, 4, cudaMemcpyDeviceToHost, stream), "D2H status") &&
                  cuda_ok(cudaStreamSynchronize(stream), "sync emit");
        if (!ok || status != 0u) {
            if (ok) set_error("blocked_ell_from_compressed: emit status 0x%x", status);
            cs_b200_host_blocked_ell_clear(dst);
            return 0;
        }
    } else if (idx_bytes != 0u) {
        for (std::size_t i = 0; i < rb * ell_width; ++i) dst->blockColIdx[i] = CS_INVALID_COL;
    }
    dst->nnz = nnz;
    return 1;
}

extern "C" int cs_b200_choose_blocked_ell_block_size(const cs_host_compressed *src, const unsigned int *candidates,
                                                     unsigned int candidate_count, cs_blocked_ell_tune_result *out) {
    if (src == nullptr || out == nullptr || candidates == nullptr || candidate_count == 0u) {
        set_error("choose_blocked_ell_block_size: null argument or no candidates");
        return 0;
    }
    if (src->axis != CS_COMPRESSED_BY_ROW) {
        set_error("choose_blocked_ell_block_size: source must be compressed by row");
        return 0;
    }
    cudaStream_t stream = nullptr;
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream create")) return 0;
    struct stream_guard {
        cudaStream_t s;
        ~stream_guard() { cudaStreamDestroy(s); }
    } guard{stream};
    staged_csr csr;
    if (!csr.upload(src, stream)) return 0;
    cs_blocked_ell_tune_result best{0u, 0.0, 0u};
    for (unsigned int i = 0; i < candidate_count; ++i) {
        const unsigned int B = candidates[i];
        if (B == 0u) continue;
        uint32_t ell_width = 0u;
        double fill = 0.0;
        if (src->rows != 0u && src->cols != 0u) {
            if (!check_src(&csr.view, B, "choose_blocked_ell_block_size")) return 0;
            uint64_t shape[2] = {0, 0};
            uint32_t status = 0;
            if (!shape_on_device(&csr.view, B, shape, nullptr, &status, stream)) return 0;
            if (status != 0u) {
                set_error("choose_blocked_ell_block_size: invalid CSR (status 0x%x)", status);
                return 0;
            }
            ell_width = (uint32_t) shape[0];
            const unsigned long row_blocks = (src->rows + B - 1u) / B;
            fill = (row_blocks == 0u || ell_width == 0u)
                       ? 1.0
                       : (double) shape[1] / (double) ((unsigned long) row_blocks * (unsigned long) ell_width);
        }
        const std::size_t padded = (std::size_t) src->rows * (std::size_t) ell_width * (std::size_t) B * 2u;
        if (best.block_size == 0u || padded + 1u < best.padded_bytes ||
            (padded == best.padded_bytes && fill > best.fill_ratio + 1.0e-9) ||
            (padded == best.padded_bytes && fill + 1.0e-9 >= best.fill_ratio && B > best.block_size)) {
            best.block_size = B;
            best.fill_ratio = fill;
            best.padded_bytes = padded;
        }
    }
    if (best.block_size == 0u) {
        set_error("choose_blocked_ell_block_size: no usable candidate");
        return 0;
    }
    *out = best;
    return 1;
}

extern "C" void cs_b200_host_compressed_clear(cs_host_compressed *m) {
    if (m == nullptr) return;
    if (m->storage != nullptr)
        std::free(m->storage);
    else {
        std::free(m->majorPtr);
        std::free(m->minorIdx);
        std::free(m->val);
    }
    std::memset(m, 0, sizeof(*m));
}

extern "C" void cs_b200_host_sliced_ell_clear(cs_host_sliced_ell *m) {
    if (m == nullptr) return;
    if (m->storage != nullptr)
        std::free(m->storage);
    else {
        std::free(m->slice_row_offsets);
        std::free(m->slice_widths);
        std::free(m->col_idx);
        std::free(m->val);
    }
    std::memset(m, 0, sizeof(*m));
}
