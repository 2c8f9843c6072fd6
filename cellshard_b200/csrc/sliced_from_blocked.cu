// Blocked-ELL -> Sliced-ELL on the GPU.
//
// The reference counts each row's live entries on the host
// (count_blocked_ell_row_nnz_, src/convert/sliced_ell_from_blocked_ell.cuh:36-62),
// builds the uniform slice layout on the host (:111-142), uploads both
// matrices and emits with one thread per row (:146-190) before copying the
// result back.  Here:
//
//   row pointers  one warp per row counts the live entries (valid slot,
//                 column < cols, value != 0 as a float) with 16-byte value
//                 loads, four in flight per lane; one device scan turns the
//                 counts into row pointers.  Those pointers are all the CSR
//                 layout, candidate and chooser code reads, so the Sliced-ELL
//                 layout and slice-height choice are the CSR ones unchanged.
//   emit          one warp per row walks its values again in 256-value steps
//                 (a 16-byte vector per lane); per step the lanes' live bits
//                 are ranked by a warp scan, each lane stores its entries at
//                 run + rank, slot order preserved; padding (CS_INVALID_COL,
//                 0) fills the rest of the row's width.
#include "common.cuh"
#include "bell_vec.cuh"

#include <cstdlib>
#include <cstring>

namespace csb {
namespace {

constexpr unsigned kWarps = 8;
constexpr unsigned kThreads = kWarps * 32;
constexpr unsigned kSteps = 4; // 256-value steps per lane in flight

unsigned grid_rows(uint32_t rows) {
    uint32_t g = (rows + kWarps - 1u) / kWarps;
    const uint32_t cap = (uint32_t) sm_count() * 16u;
    if (g > cap) g = cap;
    return g == 0u ? 1u : g;
}

// VEC: block size a multiple of 8 and values 16-byte aligned.
template <bool VEC>
__global__ void __launch_bounds__(kThreads) bell_row_live_kernel(cs_blocked_ell_view src, uint32_t *__restrict__ counts) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t B = src.block_size;
    const uint32_t W = B != 0u ? src.ell_cols / B : 0u;
    const block_div bd(B);
    for (uint32_t row = blockIdx.x * kWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kWarps) {
        const uint32_t *bci = src.blockColIdx + (std::size_t) (row / B) * W;
        const uint16_t *vrow = src.val + (std::size_t) row * src.ell_cols;
        uint32_t n = 0u;
        if (VEC) {
            // the next group of steps is loaded before the current one is counted
            uint4 v[kSteps], vn[kSteps];
            uint32_t bc[kSteps], bcn[kSteps];
            load_steps(vrow, bci, bd, src.ell_cols, lane * 8u, v, bc);
            for (uint32_t base = lane * 8u; base - lane * 8u < src.ell_cols; base += 256u * kSteps) {
                load_steps(vrow, bci, bd, src.ell_cols, base + 256u * kSteps, vn, bcn);
#pragma unroll
                for (unsigned u = 0; u < kSteps; ++u) {
                    const uint32_t e0 = base + u * 256u;
                    n += __popc(live_bits8(v[u]) & in_range8(bc[u], bc[u] * B + bd.mod(e0), src.cols));
                    v[u] = vn[u];
                    bc[u] = bcn[u];
                }
            }
        } else {
            for (uint32_t e = lane; e < src.ell_cols; e += 32u) {
                const uint32_t bc = bci[e / B];
                const uint32_t c = bc * B + e % B;
                n += (bc != CS_INVALID_COL && c < src.cols && half_nonzero(vrow[e])) ? 1u : 0u;
            }
        }
        n = __reduce_add_sync(0xffffffffu, n);
        if (lane == 0u) counts[row] = n;
    }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads) sell_from_bell_emit_kernel(cs_blocked_ell_view src, uint32_t h,
                                                                       const uint32_t *__restrict__ widths,
                                                                       const uint32_t *__restrict__ slot_offsets,
                                                                       uint32_t *__restrict__ col_idx,
                                                                       uint16_t *__restrict__ out_val) {
    static_assert(kSteps % 2 == 0, "steps are ranked in pairs");
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t B = src.block_size;
    const uint32_t W = B != 0u ? src.ell_cols / B : 0u;
    const block_div bd(B);
    for (uint32_t row = blockIdx.x * kWarps + (threadIdx.x >> 5); row < src.rows; row += gridDim.x * kWarps) {
        const uint32_t slice = row / h;
        const uint32_t width = widths[slice];
        const std::size_t base = (std::size_t) slot_offsets[slice] + (std::size_t) (row - slice * h) * width;
        const uint32_t *bci = src.blockColIdx + (std::size_t) (row / B) * W;
        const uint16_t *vrow = src.val + (std::size_t) row * src.ell_cols;
        uint32_t run = 0u; // live entries of the row written so far (warp-uniform)
        if (VEC) {
            for (uint32_t b0 = lane * 8u; b0 - lane * 8u < src.ell_cols; b0 += 256u * kSteps) {
                uint4 v[kSteps];
                uint32_t bc[kSteps];
                load_steps(vrow, bci, bd, src.ell_cols, b0, v, bc);
#pragma unroll
                for (unsigned u = 0; u < kSteps; u += 2u) {
                    // two 256-value steps in slot order (lanes in order, values in
                    // order), ranked by one warp scan of 16-bit count pairs
                    uint32_t bits[2], gene0[2];
#pragma unroll
                    for (unsigned k = 0; k < 2u; ++k) {
                        gene0[k] = bc[u + k] * B + bd.mod(b0 + (u + k) * 256u);
                        bits[k] = live_bits8(v[u + k]) & in_range8(bc[u + k], gene0[k], src.cols);
                    }
                    const uint32_t cnt = __popc(bits[0]) | (__popc(bits[1]) << 16);
                    const uint32_t incl = warp_inclusive_scan(cnt);
                    const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
                    const uint32_t excl = incl - cnt;
#pragma unroll
                    for (unsigned k = 0; k < 2u; ++k) {
                        uint32_t slot = run + (k == 0u ? (excl & 0xffffu) : (tot & 0xffffu) + (excl >> 16));
                        uint32_t b = bits[k];
                        while (b != 0u) {
                            const uint32_t q = __ffs(b) - 1u;
                            b &= b - 1u;
                            if (slot < width) {
                                col_idx[base + slot] = gene0[k] + q;
                                out_val[base + slot] = half_of(v[u + k], q);
                            }
                            ++slot;
                        }
                    }
                    run += (tot & 0xffffu) + (tot >> 16);
                }
            }
        } else {
            for (uint32_t e0 = 0; e0 < src.ell_cols; e0 += 32u) {
                const uint32_t e = e0 + lane;
                bool live = false;
                uint32_t c = 0u;
                uint16_t x = 0u;
                if (e < src.ell_cols) {
                    const uint32_t bc = bci[e / B];
                    c = bc * B + e % B;
                    x = vrow[e];
                    live = bc != CS_INVALID_COL && c < src.cols && half_nonzero(x);
                }
                const uint32_t ballot = __ballot_sync(0xffffffffu, live);
                const uint32_t slot = run + __popc(ballot & lt);
                if (live && slot < width) {
                    col_idx[base + slot] = c;
                    out_val[base + slot] = x;
                }
                run += __popc(ballot);
            }
        }
        for (uint32_t s = (run < width ? run : width) + lane; s < width; s += 32u) {
            col_idx[base + s] = CS_INVALID_COL;
            out_val[base + s] = 0u;
        }
    }
}

bool bell_vec(const cs_blocked_ell_view *src) {
    return src->block_size % 8u == 0u && (reinterpret_cast<uintptr_t>(src->val) & 15u) == 0u;
}

} // namespace

int check_bell(const cs_blocked_ell_view *src, const char *who) {
    if (src == nullptr) {
        set_error("%s: null view", who);
        return 0;
    }
    if (src->rows != 0u && src->ell_cols != 0u &&
        (src->block_size == 0u || src->ell_cols % src->block_size != 0u || src->blockColIdx == nullptr ||
         src->val == nullptr)) {
        set_error("%s: block size must divide ell_cols and the arrays be set", who);
        return 0;
    }
    return 1;
}

int stage_bell(const cs_host_blocked_ell *src, staged_bell *st, cudaStream_t stream) {
    const uint32_t B = src->block_size;
    const std::size_t rb = B != 0u ? ((std::size_t) src->rows + B - 1u) / B : 0u;
    const std::size_t idx_bytes = rb * (B != 0u ? src->ell_cols / B : 0u) * 4u;
    const std::size_t val_bytes = (std::size_t) src->rows * src->ell_cols * 2u;
    if (!st->bci.alloc(idx_bytes, "cudaMalloc blocked_ell idx") || !st->val.alloc(val_bytes, "cudaMalloc blocked_ell val"))
        return 0;
    if ((idx_bytes != 0u &&
         !cuda_ok(cudaMemcpyAsync(st->bci.p, src->blockColIdx, idx_bytes, cudaMemcpyHostToDevice, stream), "H2D idx")) ||
        (val_bytes != 0u &&
         !cuda_ok(cudaMemcpyAsync(st->val.p, src->val, val_bytes, cudaMemcpyHostToDevice, stream), "H2D val")))
        return 0;
    st->view = cs_blocked_ell_view{src->rows, src->cols, src->nnz, src->block_size, src->ell_cols,
                                   (uint32_t *) st->bci.p, (uint16_t *) st->val.p};
    return 1;
}

std::size_t bell_row_ptr_scratch(uint32_t rows) { return scan_u32_scratch_bytes(rows); }

int bell_row_ptr_launch(const cs_blocked_ell_view *src, uint32_t *d_row_ptr, void *scratch, std::size_t scratch_bytes,
                        cudaStream_t stream) {
    if (src->rows == 0u) return cuda_ok(cudaMemsetAsync(d_row_ptr, 0, 4, stream), "row_ptr memset");
    if (src->ell_cols == 0u) {
        return cuda_ok(cudaMemsetAsync(d_row_ptr, 0, ((std::size_t) src->rows + 1u) * 4u, stream), "row_ptr memset");
    }
    if (bell_vec(src))
        bell_row_live_kernel<true><<<grid_rows(src->rows), kThreads, 0, stream>>>(*src, d_row_ptr);
    else
        bell_row_live_kernel<false><<<grid_rows(src->rows), kThreads, 0, stream>>>(*src, d_row_ptr);
    if (!launch_ok("bell_row_live_kernel")) return 0;
    return scan_exclusive_u32(d_row_ptr, d_row_ptr, src->rows, true, scratch, scratch_bytes, stream);
}

int sell_from_bell_emit_launch(const cs_blocked_ell_view *src, const cs_sliced_ell_view *dst, cudaStream_t stream) {
    if (src->rows == 0u) return 1;
    const uint32_t h = dst->slice_rows < src->rows ? (dst->slice_rows == 0u ? 1u : dst->slice_rows) : src->rows;
    if (bell_vec(src) && src->ell_cols != 0u)
        sell_from_bell_emit_kernel<true><<<grid_rows(src->rows), kThreads, 0, stream>>>(
            *src, h, dst->slice_widths, dst->slice_slot_offsets, dst->col_idx, dst->val);
    else
        sell_from_bell_emit_kernel<false><<<grid_rows(src->rows), kThreads, 0, stream>>>(
            *src, h, dst->slice_widths, dst->slice_slot_offsets, dst->col_idx, dst->val);
    return launch_ok("sell_from_bell_emit_kernel");
}

} // namespace csb

using namespace csb;

extern "C" int cs_b200_blocked_ell_row_ptr_scratch_bytes(uint32_t rows, size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("blocked_ell_row_ptr_scratch_bytes: null output");
        return 0;
    }
    *out_bytes = bell_row_ptr_scratch(rows);
    return 1;
}

extern "C" int cs_b200_blocked_ell_row_ptr(const cs_blocked_ell_view *src, uint32_t *d_row_ptr, void *d_scratch,
                                           size_t scratch_bytes, cs_stream_t s) {
    if (!check_bell(src, "blocked_ell_row_ptr")) return 0;
    if (d_row_ptr == nullptr) {
        set_error("blocked_ell_row_ptr: null output");
        return 0;
    }
    return bell_row_ptr_launch(src, d_row_ptr, d_scratch, scratch_bytes, as_stream(s));
}

extern "C" int cs_b200_sliced_ell_emit_from_blocked_ell(const cs_blocked_ell_view *src, const cs_sliced_ell_view *dst,
                                                        cs_stream_t s) {
    if (!check_bell(src, "sliced_ell_emit_from_blocked_ell")) return 0;
    if (dst == nullptr || dst->rows != src->rows) {
        set_error("sliced_ell_emit_from_blocked_ell: destination rows differ");
        return 0;
    }
    if (src->rows != 0u && (dst->slice_rows == 0u || dst->slice_widths == nullptr ||
                            dst->slice_slot_offsets == nullptr)) {
        set_error("sliced_ell_emit_from_blocked_ell: destination needs uniform slice_rows, widths, slot offsets");
        return 0;
    }
    return sell_from_bell_emit_launch(src, dst, as_stream(s));
}

extern "C" int cs_b200_sliced_ell_from_blocked_ell(const cs_host_blocked_ell *src, unsigned int slice_rows,
                                                   cs_host_sliced_ell *dst) {
    if (src == nullptr || dst == nullptr || slice_rows == 0u || src->block_size == 0u) {
        set_error("sliced_ell_from_blocked_ell: null argument, zero slice_rows or zero block size");
        return 0;
    }
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    staged_bell sb;
    if (!stage_bell(src, &sb, g.s)) return 0;
    if (!check_bell(&sb.view, "sliced_ell_from_blocked_ell")) return 0;
    const uint32_t rows = src->rows;
    const uint32_t h = rows == 0u ? 0u : (slice_rows < rows ? slice_rows : rows);
    const uint32_t S = rows == 0u ? 0u : (rows + h - 1u) / h;
    dmem row_ptr, offs, widths, slots, total, scratch;
    size_t lsb = 0;
    cs_b200_sliced_ell_scratch_bytes(rows, slice_rows, &lsb);
    const std::size_t psb = bell_row_ptr_scratch(rows);
    if (!row_ptr.alloc(((std::size_t) rows + 1u) * 4u, "row_ptr") ||
        !offs.alloc(((std::size_t) S + 1u) * 4u, "offsets") || !widths.alloc((std::size_t) S * 4u, "widths") ||
        !slots.alloc((std::size_t) S * 4u, "slots") || !total.alloc(16, "total") ||
        !scratch.alloc(lsb > psb ? lsb : psb, "scratch"))
        return 0;
    if (!bell_row_ptr_launch(&sb.view, (uint32_t *) row_ptr.p, scratch.p, psb, g.s)) return 0;
    const cs_compressed_view rv{rows, src->cols, src->nnz, CS_COMPRESSED_BY_ROW, (uint32_t *) row_ptr.p, nullptr,
                                nullptr};
    if (!sliced_layout_launch(&rv, slice_rows, (uint32_t *) offs.p, (uint32_t *) widths.p, (uint32_t *) slots.p,
                              (uint64_t *) total.p, scratch.p, lsb, g.s))
        return 0;
    uint64_t total_slots = 0;
    if (!cuda_ok(cudaMemcpyAsync(&total_slots, total.p, 8, cudaMemcpyDeviceToHost, g.s), "D2H total") ||
        !cuda_ok(cudaStreamSynchronize(g.s), "sync layout"))
        return 0;
    if (total_slots > 0xffffffffull) {
        set_error("sliced_ell_from_blocked_ell: %llu slots overflow the u32 slot index",
                  (unsigned long long) total_slots);
        return 0;
    }
    // the reference carries the source's nnz field over (sliced_ell_from_blocked_ell.cuh:246)
    if (!host_sliced_alloc(dst, rows, src->cols, src->nnz, S, total_slots)) return 0;
    if (S == 0u) {
        dst->slice_row_offsets[0] = 0u;
        return 1;
    }
    dmem d_col, d_val;
    const std::size_t col_bytes = (std::size_t) total_slots * 4u;
    bool ok = d_col.alloc(col_bytes, "col") && d_val.alloc((std::size_t) total_slots * 2u, "val");
    const cs_sliced_ell_view dv{rows, src->cols, src->nnz, S, h, (uint32_t *) offs.p, (uint32_t *) widths.p,
                                (uint32_t *) slots.p, (uint32_t *) d_col.p, (uint16_t *) d_val.p};
    ok = ok && sell_from_bell_emit_launch(&sb.view, &dv, g.s) &&
         cuda_ok(cudaMemcpyAsync(dst->slice_row_offsets, offs.p, ((std::size_t) S + 1u) * 4u, cudaMemcpyDeviceToHost,
                                 g.s),
                 "D2H offsets") &&
         cuda_ok(cudaMemcpyAsync(dst->slice_widths, widths.p, (std::size_t) S * 4u, cudaMemcpyDeviceToHost, g.s),
                 "D2H widths") &&
         (total_slots == 0u ||
          (cuda_ok(cudaMemcpyAsync(dst->col_idx, d_col.p, col_bytes, cudaMemcpyDeviceToHost, g.s), "D2H col") &&
           cuda_ok(cudaMemcpyAsync(dst->val, d_val.p, (std::size_t) total_slots * 2u, cudaMemcpyDeviceToHost, g.s),
                   "D2H val"))) &&
         cuda_ok(cudaStreamSynchronize(g.s), "sync emit");
    if (!ok) {
        cs_b200_host_sliced_ell_clear(dst);
        return 0;
    }
    return 1;
}

extern "C" int cs_b200_choose_sliced_ell_slice_rows_from_blocked_ell(const cs_host_blocked_ell *src,
                                                                     const unsigned int *candidates,
                                                                     unsigned int candidate_count,
                                                                     cs_sliced_ell_tune_result *out) {
    if (src == nullptr || out == nullptr || candidates == nullptr || candidate_count == 0u || src->block_size == 0u) {
        set_error("choose_sliced_ell_slice_rows_from_blocked_ell: null argument, no candidates or zero block size");
        return 0;
    }
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    staged_bell sb;
    if (!stage_bell(src, &sb, g.s)) return 0;
    if (!check_bell(&sb.view, "choose_sliced_ell_slice_rows_from_blocked_ell")) return 0;
    dmem row_ptr, scratch;
    const std::size_t psb = bell_row_ptr_scratch(src->rows);
    if (!row_ptr.alloc(((std::size_t) src->rows + 1u) * 4u, "row_ptr") || !scratch.alloc(psb, "scratch")) return 0;
    if (!bell_row_ptr_launch(&sb.view, (uint32_t *) row_ptr.p, scratch.p, psb, g.s)) return 0;
    const cs_compressed_view rv{src->rows, src->cols, src->nnz, CS_COMPRESSED_BY_ROW, (uint32_t *) row_ptr.p, nullptr,
                                nullptr};
    return choose_sliced_rows_core(&rv, src->nnz, candidates, candidate_count, out, g.s);
}
