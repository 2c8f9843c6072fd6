// CSR -> Sliced-ELL on the GPU.
//
// The reference computes the layout on the host (count_compressed_row_nnz_ and
// build_uniform_sliced_layout_, src/convert/sliced_ell_from_compressed.cuh:20-45
// and sliced_ell_from_blocked_ell.cuh:111-142), uploads the source and the
// padded destination, scatters with one thread per row (:49-80) and copies the
// result back.  Here the layout is computed on the device:
//
//   layout  one warp per slice: row nnz from the row pointers, warp max ->
//           slice width, slot count = rows_in_slice * width; one device scan
//           -> slot offsets (u32 running sum, as the reference's upload does,
//           sharded_device.cuh:716-723) and the total.
//   emit    one warp per row copies the row's (column, value) pairs into its
//           first slots and writes padding (CS_INVALID_COL, 0) into the rest,
//           both as coalesced contiguous runs.
//   chooser evaluate_sliced_candidate_ (sliced_ell_from_blocked_ell.cuh:64-109)
//           needs sum over slices of rows_in_slice * max nnz per candidate
//           height: one launch accumulates it for every candidate; the score
//           arithmetic stays in host doubles, in the reference's order.
#include "common.cuh"
#include "emit_rows.cuh"

#include <cstdlib>
#include <cstring>

namespace csb {

int transpose_csc_to_csr_staged(const cs_compressed_view *src, uint32_t **d_ptr, uint32_t **d_idx, uint16_t **d_val,
                                cudaStream_t stream);

namespace {

constexpr unsigned kWarps = 8;
constexpr unsigned kMaxCandidates = 16;

uint32_t clamp_rows(uint32_t rows, uint32_t h) {
    if (rows == 0u) return 0u;
    if (h < 1u) h = 1u;
    return h < rows ? h : rows;
}

__global__ void __launch_bounds__(kWarps * 32) sell_layout_kernel(const uint32_t *__restrict__ ptr, uint32_t rows,
                                                                  uint32_t h, uint32_t slices,
                                                                  uint32_t *__restrict__ offsets,
                                                                  uint32_t *__restrict__ widths,
                                                                  uint32_t *__restrict__ slot_counts,
                                                                  unsigned long long *__restrict__ total64) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long local = 0ull;
    for (uint32_t s = blockIdx.x * kWarps + (threadIdx.x >> 5); s < slices; s += gridDim.x * kWarps) {
        const uint32_t r0 = s * h;
        const uint32_t r1 = min(rows, r0 + h);
        uint32_t w = 0u;
        for (uint32_t r = r0 + lane; r < r1; r += 32u) w = max(w, ptr[r + 1u] - ptr[r]);
        w = __reduce_max_sync(0xffffffffu, w);
        if (lane == 0u) {
            widths[s] = w;
            offsets[s + 1u] = r1;
            slot_counts[s] = (r1 - r0) * w;
            local += (unsigned long long) (r1 - r0) * w;
            if (s == 0u) offsets[0] = 0u;
        }
    }
    if (lane == 0u && local != 0ull && total64 != nullptr) atomicAdd(total64, local);
}

// Padded slots for every candidate height in one pass (one warp per row chunk
// of the largest candidate's lcm is not needed: each warp handles one slice
// of each candidate in turn).
struct heights_t {
    uint32_t h[kMaxCandidates];
};

__global__ void __launch_bounds__(kWarps * 32) sell_candidates_kernel(const uint32_t *__restrict__ ptr, uint32_t rows,
                                                                      heights_t heights, uint32_t n_cand,
                                                                      unsigned long long *__restrict__ padded) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t gw = blockIdx.x * kWarps + (threadIdx.x >> 5);
    const uint32_t nw = gridDim.x * kWarps;
    for (uint32_t k = 0; k < n_cand; ++k) {
        const uint32_t h = heights.h[k];
        const uint32_t slices = (rows + h - 1u) / h;
        unsigned long long local = 0ull;
        for (uint32_t s = gw; s < slices; s += nw) {
            const uint32_t r0 = s * h, r1 = min(rows, r0 + h);
            uint32_t w = 0u;
            for (uint32_t r = r0 + lane; r < r1; r += 32u) w = max(w, ptr[r + 1u] - ptr[r]);
            w = __reduce_max_sync(0xffffffffu, w);
            local += (unsigned long long) (r1 - r0) * w;
        }
        if (lane == 0u && local != 0ull) atomicAdd(padded + k, local);
    }
}

__global__ void __launch_bounds__(kWarps * 32) sell_emit_kernel(const uint32_t *__restrict__ ptr,
                                                                const uint32_t *__restrict__ idx,
                                                                const uint16_t *__restrict__ val, uint32_t rows,
                                                                uint32_t h, const uint32_t *__restrict__ widths,
                                                                const uint32_t *__restrict__ slot_offsets,
                                                                uint32_t *__restrict__ col_idx,
                                                                uint16_t *__restrict__ out_val) {
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t r = blockIdx.x * kWarps + (threadIdx.x >> 5); r < rows; r += gridDim.x * kWarps) {
        const uint32_t s = r / h;
        const uint32_t w = widths[s];
        const std::size_t base = (std::size_t) slot_offsets[s] + (std::size_t) (r - s * h) * w;
        const uint32_t a = ptr[r];
        const uint32_t n = min(ptr[r + 1u] - a, w);
        for (uint32_t k = lane; k < w; k += 32u) {
            const bool real = k < n;
            col_idx[base + k] = real ? idx[a + k] : CS_INVALID_COL;
            out_val[base + k] = real ? val[a + k] : (uint16_t) 0u;
        }
    }
}

// Vectorised emit: one group of GL lanes per row (rows_per_warp = 32 / GL).
template <unsigned GL>
__global__ void __launch_bounds__(kWarps * 32) sell_emit_vec_kernel(const uint32_t *__restrict__ ptr,
                                                                    const uint32_t *__restrict__ idx,
                                                                    const uint16_t *__restrict__ val, uint32_t rows,
                                                                    uint32_t h, const uint32_t *__restrict__ widths,
                                                                    const uint32_t *__restrict__ slot_offsets,
                                                                    uint32_t *__restrict__ col_idx,
                                                                    uint16_t *__restrict__ out_val) {
    constexpr unsigned RPW = 32u / GL;
    const unsigned lane = threadIdx.x & 31u, gl = lane % GL;
    const uint32_t warp0 = blockIdx.x * kWarps + (threadIdx.x >> 5);
    for (uint32_t r = warp0 * RPW + lane / GL; r < rows; r += gridDim.x * kWarps * RPW) {
        const uint32_t s = r / h;
        const uint32_t w = widths[s];
        const std::size_t base = (std::size_t) slot_offsets[s] + (std::size_t) (r - s * h) * w;
        const uint32_t a = ptr[r];
        sell_emit_row_vec<GL>(idx, val, a, ptr[r + 1u] - a, w, base, col_idx, out_val, gl);
    }
}

unsigned grid_for(uint32_t items) {
    uint32_t g = (items + kWarps - 1u) / kWarps;
    const uint32_t cap = (uint32_t) sm_count() * 32u;
    if (g > cap) g = cap;
    return g == 0u ? 1u : g;
}

struct dbuf {
    void *p = nullptr;
    ~dbuf() {
        if (p) cudaFree(p);
    }
    bool alloc(std::size_t n, const char *what) {
        return cuda_ok(cudaMalloc(&p, n == 0 ? 16 : n), what) != 0;
    }
};

struct stream_guard {
    cudaStream_t s = nullptr;
    ~stream_guard() {
        if (s) cudaStreamDestroy(s);
    }
};

} // namespace

int sliced_layout_launch(const cs_compressed_view *src, uint32_t slice_rows, uint32_t *d_offsets, uint32_t *d_widths,
                         uint32_t *d_slot_offsets, uint64_t *d_total, void *scratch, std::size_t scratch_bytes,
                         cudaStream_t stream) {
    const uint32_t h = clamp_rows(src->rows, slice_rows);
    const uint32_t S = src->rows == 0u ? 0u : (src->rows + h - 1u) / h;
    if (d_total != nullptr && !cuda_ok(cudaMemsetAsync(d_total, 0, 8, stream), "sliced total memset")) return 0;
    if (S == 0u) {
        if (d_offsets != nullptr && !cuda_ok(cudaMemsetAsync(d_offsets, 0, 4, stream), "sliced offsets memset"))
            return 0;
        return 1;
    }
    scratch_carver c(scratch, scratch_bytes);
    uint32_t *counts = c.take<uint32_t>((std::size_t) S + 1u);
    void *scan_tmp = c.take<char>(scan_u32_scratch_bytes(S));
    if (!c.fits()) {
        set_error("sliced_ell_layout: scratch too small");
        return 0;
    }
    sell_layout_kernel<<<grid_for(S), kWarps * 32, 0, stream>>>(src->majorPtr, src->rows, h, S, d_offsets, d_widths,
                                                                counts,
                                                                reinterpret_cast<unsigned long long *>(d_total));
    if (!launch_ok("sell_layout_kernel")) return 0;
    if (!scan_exclusive_u32(counts, counts, S, true, scan_tmp, scan_u32_scratch_bytes(S), stream)) return 0;
    if (!cuda_ok(cudaMemcpyAsync(d_slot_offsets, counts, (std::size_t) S * 4u, cudaMemcpyDeviceToDevice, stream),
                 "slot offsets copy"))
        return 0;
    return 1;
}

int sliced_emit_launch(const cs_compressed_view *src, const cs_sliced_ell_view *dst, cudaStream_t stream) {
    if (src->rows == 0u) return 1;
    const uint32_t h = clamp_rows(src->rows, dst->slice_rows);
    const bool aligned = ((uintptr_t) dst->col_idx & 15u) == 0u && ((uintptr_t) dst->val & 7u) == 0u;
    if (!aligned) {
        sell_emit_kernel<<<grid_for(src->rows), kWarps * 32, 0, stream>>>(src->majorPtr, src->minorIdx, src->val,
                                                                          src->rows, h, dst->slice_widths,
                                                                          dst->slice_slot_offsets, dst->col_idx,
                                                                          dst->val);
        return launch_ok("sell_emit_kernel");
    }
    // rows narrower than a warp's 128 slots share the warp
    const double mean_nnz = (double) src->nnz / (double) src->rows;
    if (mean_nnz >= 96.0)
        sell_emit_vec_kernel<32><<<grid_for(src->rows), kWarps * 32, 0, stream>>>(
            src->majorPtr, src->minorIdx, src->val, src->rows, h, dst->slice_widths, dst->slice_slot_offsets,
            dst->col_idx, dst->val);
    else
        sell_emit_vec_kernel<8><<<grid_for((src->rows + 3u) / 4u), kWarps * 32, 0, stream>>>(
            src->majorPtr, src->minorIdx, src->val, src->rows, h, dst->slice_widths, dst->slice_slot_offsets,
            dst->col_idx, dst->val);
    return launch_ok("sell_emit_vec_kernel");
}

} // namespace csb

using namespace csb;

extern "C" int cs_b200_sliced_ell_scratch_bytes(uint32_t rows, uint32_t slice_rows, size_t *out_bytes) {
    if (out_bytes == nullptr) {
        set_error("sliced_ell_scratch_bytes: null output");
        return 0;
    }
    const uint32_t h = clamp_rows(rows, slice_rows);
    const std::size_t S = rows == 0u ? 0u : (rows + h - 1u) / h;
    *out_bytes = align_up((S + 1u) * 4u, 256) + scan_u32_scratch_bytes(S) + 256u;
    return 1;
}

extern "C" int cs_b200_sliced_ell_layout(const cs_compressed_view *src, uint32_t slice_rows,
                                         uint32_t *d_slice_row_offsets, uint32_t *d_slice_widths,
                                         uint32_t *d_slice_slot_offsets, uint64_t *d_total_slots, void *d_scratch,
                                         size_t scratch_bytes, cs_stream_t s) {
    if (src == nullptr || slice_rows == 0u || src->axis != CS_COMPRESSED_BY_ROW) {
        set_error("sliced_ell_layout: need a row-compressed source and slice_rows > 0");
        return 0;
    }
    if (src->rows != 0u && (d_slice_row_offsets == nullptr || d_slice_widths == nullptr ||
                            d_slice_slot_offsets == nullptr || src->majorPtr == nullptr)) {
        set_error("sliced_ell_layout: null arrays");
        return 0;
    }
    return sliced_layout_launch(src, slice_rows, d_slice_row_offsets, d_slice_widths, d_slice_slot_offsets,
                                d_total_slots, d_scratch, scratch_bytes, as_stream(s));
}

extern "C" int cs_b200_sliced_ell_emit(const cs_compressed_view *src, const cs_sliced_ell_view *dst, cs_stream_t s) {
    if (src == nullptr || dst == nullptr || src->axis != CS_COMPRESSED_BY_ROW || dst->rows != src->rows) {
        set_error("sliced_ell_emit: need a row-compressed source matching the destination");
        return 0;
    }
    if (src->rows != 0u && (dst->slice_rows == 0u || dst->slice_widths == nullptr ||
                            dst->slice_slot_offsets == nullptr)) {
        set_error("sliced_ell_emit: destination needs uniform slice_rows, widths and slot offsets");
        return 0;
    }
    return sliced_emit_launch(src, dst, as_stream(s));
}

extern "C" int cs_b200_sliced_ell_candidates(const cs_compressed_view *src, const uint32_t *candidates,
                                             uint32_t count, uint64_t *d_padded_slots, cs_stream_t s) {
    if (src == nullptr || candidates == nullptr || d_padded_slots == nullptr || count == 0u ||
        count > kMaxCandidates || src->axis != CS_COMPRESSED_BY_ROW) {
        set_error("sliced_ell_candidates: bad arguments (at most %u candidates)", kMaxCandidates);
        return 0;
    }
    cudaStream_t stream = as_stream(s);
    if (!cuda_ok(cudaMemsetAsync(d_padded_slots, 0, (std::size_t) count * 8u, stream), "candidates memset")) return 0;
    if (src->rows == 0u) return 1;
    heights_t heights{};
    for (uint32_t k = 0; k < count; ++k) heights.h[k] = clamp_rows(src->rows, candidates[k] == 0u ? 1u : candidates[k]);
    sell_candidates_kernel<<<grid_for(src->rows), kWarps * 32, 0, stream>>>(
        src->majorPtr, src->rows, heights, count, reinterpret_cast<unsigned long long *>(d_padded_slots));
    return launch_ok("sell_candidates_kernel");
}

namespace {

// Host result packed as sparse::allocate(sliced_ell) (sliced_ell.cuh:165-224):
// offsets, widths, column indices, values in one malloc'd block.
} // namespace

int csb::host_sliced_alloc(cs_host_sliced_ell *dst, uint32_t rows, uint32_t cols, uint32_t nnz, uint32_t S,
                           uint64_t total_slots) {
    cs_b200_host_sliced_ell_clear(dst);
    dst->rows = rows;
    dst->cols = cols;
    dst->nnz = nnz;
    const std::size_t offsets_bytes = ((std::size_t) S + 1u) * 4u;
    const std::size_t widths_offset = align_up(offsets_bytes, 4);
    const std::size_t widths_bytes = (std::size_t) S * 4u;
    const std::size_t col_offset = align_up(widths_offset + widths_bytes, 4);
    const std::size_t col_bytes = (std::size_t) total_slots * 4u;
    const std::size_t val_offset = align_up(col_offset + col_bytes, 2);
    const std::size_t total_bytes = val_offset + (std::size_t) total_slots * 2u;
    char *storage = (char *) std::malloc(total_bytes);
    if (storage == nullptr) {
        set_error("sliced_ell host allocation failed");
        return 0;
    }
    dst->slice_count = S;
    dst->storage = storage;
    dst->slice_row_offsets = (uint32_t *) storage;
    dst->slice_widths = (uint32_t *) (storage + widths_offset);
    dst->col_idx = (uint32_t *) (storage + col_offset);
    dst->val = (uint16_t *) (storage + val_offset);
    return 1;
}

namespace {

// CSC input: the reference's CPU path (sliced_ell_from_compressed.cuh:144-163)
// appends each column's entries to its rows in column order, i.e. the stable
// transpose; it is staged through the GPU transpose here.
struct row_source {
    cs_compressed_view view{};
    dbuf ptr, idx, val, t_ptr, t_idx, t_val;
};

bool stage_rows(const cs_host_compressed *src, row_source *rs, cudaStream_t stream) {
    const std::size_t major = (std::size_t) (src->axis == CS_COMPRESSED_BY_COL ? src->cols : src->rows) + 1u;
    if (!rs->ptr.alloc(major * 4u, "cudaMalloc ptr") || !rs->idx.alloc((std::size_t) src->nnz * 4u, "cudaMalloc idx") ||
        !rs->val.alloc((std::size_t) src->nnz * 2u, "cudaMalloc val"))
        return false;
    if (src->majorPtr != nullptr) {
        if (!cuda_ok(cudaMemcpyAsync(rs->ptr.p, src->majorPtr, major * 4u, cudaMemcpyHostToDevice, stream), "H2D ptr"))
            return false;
    } else if (!cuda_ok(cudaMemsetAsync(rs->ptr.p, 0, major * 4u, stream), "ptr memset")) {
        return false;
    }
    if (src->nnz != 0u &&
        (!cuda_ok(cudaMemcpyAsync(rs->idx.p, src->minorIdx, (std::size_t) src->nnz * 4u, cudaMemcpyHostToDevice,
                                  stream),
                  "H2D idx") ||
         !cuda_ok(cudaMemcpyAsync(rs->val.p, src->val, (std::size_t) src->nnz * 2u, cudaMemcpyHostToDevice, stream),
                  "H2D val")))
        return false;
    cs_compressed_view v{src->rows, src->cols, src->nnz, src->axis, (uint32_t *) rs->ptr.p, (uint32_t *) rs->idx.p,
                         (uint16_t *) rs->val.p};
    if (src->axis == CS_COMPRESSED_BY_ROW) {
        rs->view = v;
        return true;
    }
    uint32_t *p = nullptr, *i = nullptr;
    uint16_t *x = nullptr;
    if (!transpose_csc_to_csr_staged(&v, &p, &i, &x, stream)) return false;
    rs->t_ptr.p = p;
    rs->t_idx.p = i;
    rs->t_val.p = x;
    rs->view = cs_compressed_view{src->rows, src->cols, src->nnz, CS_COMPRESSED_BY_ROW, p, i, x};
    return true;
}

int padded_slots_host(const cs_compressed_view *v, const unsigned int *candidates, unsigned int count,
                      uint64_t *out, cudaStream_t stream) {
    dbuf d;
    if (!d.alloc(kMaxCandidates * 8u, "cudaMalloc padded")) return 0;
    uint32_t cands[kMaxCandidates];
    for (unsigned k = 0; k < count; ++k) cands[k] = candidates[k];
    if (!cs_b200_sliced_ell_candidates(v, cands, count, (uint64_t *) d.p, (cs_stream_t) stream)) return 0;
    if (!cuda_ok(cudaMemcpyAsync(out, d.p, count * 8u, cudaMemcpyDeviceToHost, stream), "D2H padded") ||
        !cuda_ok(cudaStreamSynchronize(stream), "sync padded"))
        return 0;
    return 1;
}

} // namespace

extern "C" int cs_b200_choose_sliced_ell_slice_rows_from_compressed(const cs_host_compressed *src,
                                                                    const unsigned int *candidates,
                                                                    unsigned int candidate_count,
                                                                    cs_sliced_ell_tune_result *out) {
    if (src == nullptr || out == nullptr || candidates == nullptr || candidate_count == 0u) {
        set_error("choose_sliced_ell_slice_rows: null argument or no candidates");
        return 0;
    }
    stream_guard g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    row_source rs;
    if (!stage_rows(src, &rs, g.s)) return 0;
    return choose_sliced_rows_core(&rs.view, src->nnz, candidates, candidate_count, out, g.s);
}

// evaluate_sliced_candidate_ + choose_sliced_ell_slice_rows
// (sliced_ell_from_blocked_ell.cuh:64-109,196-221) over the row pointers of a
// device view; nnz is the source's nnz field (the storage ratio's divisor).
int csb::choose_sliced_rows_core(const cs_compressed_view *v, uint32_t nnz, const unsigned int *candidates,
                                 unsigned int candidate_count, cs_sliced_ell_tune_result *out, cudaStream_t stream) {
    const uint32_t rows = v->rows;
    cs_sliced_ell_tune_result best{};
    best.slice_rows = 0u;
    best.score = __builtin_inf();
    // non-zero candidates in order, in batches the candidates kernel accepts
    unsigned int live[kMaxCandidates];
    for (unsigned int i0 = 0; i0 < candidate_count;) {
        unsigned int n = 0;
        for (; i0 < candidate_count && n < kMaxCandidates; ++i0) {
            if (candidates[i0] == 0u) continue;
            live[n] = candidates[i0];
            ++n;
        }
        if (n == 0u) break;
        uint64_t padded[kMaxCandidates] = {0};
        if (rows != 0u && !padded_slots_host(v, live, n, padded, stream)) return 0;
        for (unsigned int k = 0; k < n; ++k) {
            cs_sliced_ell_tune_result c{};
            if (rows == 0u) {
                c.slice_rows = 0u;
                c.slice_count = 0u;
                c.padded_slots = 0u;
                c.padded_bytes = 0u;
                c.storage_ratio = 1.0;
                c.slice_penalty = 0.0;
                c.score = 1.0;
            } else {
                const uint32_t h = clamp_rows(rows, live[k]);
                const uint32_t S = (rows + h - 1u) / h;
                c.slice_rows = h;
                c.slice_count = S;
                c.padded_slots = (std::size_t) padded[k];
                c.padded_bytes = c.padded_slots * 6u + ((std::size_t) S * 2u + 1u) * 4u;
                c.storage_ratio = nnz == 0u ? 1.0 : (double) c.padded_slots / (double) nnz;
                c.slice_penalty = 0.25 * ((double) S / (double) rows);
                c.score = c.storage_ratio + c.slice_penalty;
            }
            if (best.slice_rows == 0u || c.score + 1.0e-12 < best.score ||
                (c.score <= best.score + 1.0e-12 && c.padded_bytes < best.padded_bytes) ||
                (c.score <= best.score + 1.0e-12 && c.padded_bytes == best.padded_bytes &&
                 c.slice_rows > best.slice_rows)) {
                best = c;
            }
        }
    }
    if (best.slice_rows == 0u && rows != 0u) {
        set_error("choose_sliced_ell_slice_rows: no usable candidate");
        return 0;
    }
    *out = best;
    return 1;
}

extern "C" int cs_b200_sliced_ell_from_compressed(const cs_host_compressed *src, unsigned int slice_rows,
                                                  cs_host_sliced_ell *dst) {
    if (src == nullptr || dst == nullptr || slice_rows == 0u) {
        set_error("sliced_ell_from_compressed: null argument or zero slice_rows");
        return 0;
    }
    stream_guard g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    row_source rs;
    if (!stage_rows(src, &rs, g.s)) return 0;
    const uint32_t rows = src->rows;
    const uint32_t h = clamp_rows(rows, slice_rows);
    const uint32_t S = rows == 0u ? 0u : (rows + h - 1u) / h;
    dbuf offs, widths, slots, total, scratch;
    size_t sb = 0;
    cs_b200_sliced_ell_scratch_bytes(rows, slice_rows, &sb);
    if (!offs.alloc(((std::size_t) S + 1u) * 4u, "offsets") || !widths.alloc((std::size_t) S * 4u, "widths") ||
        !slots.alloc((std::size_t) S * 4u, "slots") || !total.alloc(16, "total") || !scratch.alloc(sb, "scratch"))
        return 0;
    if (!sliced_layout_launch(&rs.view, slice_rows, (uint32_t *) offs.p, (uint32_t *) widths.p, (uint32_t *) slots.p,
                              (uint64_t *) total.p, scratch.p, sb, g.s))
        return 0;
    uint64_t total_slots = 0;
    if (!cuda_ok(cudaMemcpyAsync(&total_slots, total.p, 8, cudaMemcpyDeviceToHost, g.s), "D2H total") ||
        !cuda_ok(cudaStreamSynchronize(g.s), "sync layout"))
        return 0;
    if (total_slots > 0xffffffffull) {
        set_error("sliced_ell_from_compressed: %llu slots overflow the u32 slot index", (unsigned long long) total_slots);
        return 0;
    }
    if (!host_sliced_alloc(dst, src->rows, src->cols, src->nnz, S, total_slots)) return 0;
    const std::size_t offsets_bytes = ((std::size_t) S + 1u) * 4u;
    const std::size_t widths_bytes = (std::size_t) S * 4u;
    const std::size_t col_bytes = (std::size_t) total_slots * 4u;
    bool ok = true;
    if (S == 0u) {
        dst->slice_row_offsets[0] = 0u;
    } else {
        dbuf d_col, d_val;
        ok = d_col.alloc(col_bytes, "col") && d_val.alloc((std::size_t) total_slots * 2u, "val");
        cs_sliced_ell_view dv{rows, src->cols, src->nnz, S, h, (uint32_t *) offs.p, (uint32_t *) widths.p,
                              (uint32_t *) slots.p, (uint32_t *) d_col.p, (uint16_t *) d_val.p};
        ok = ok && sliced_emit_launch(&rs.view, &dv, g.s) &&
             cuda_ok(cudaMemcpyAsync(dst->slice_row_offsets, offs.p, offsets_bytes, cudaMemcpyDeviceToHost, g.s),
                     "D2H offsets") &&
             cuda_ok(cudaMemcpyAsync(dst->slice_widths, widths.p, widths_bytes, cudaMemcpyDeviceToHost, g.s),
                     "D2H widths") &&
             (total_slots == 0u ||
              (cuda_ok(cudaMemcpyAsync(dst->col_idx, d_col.p, col_bytes, cudaMemcpyDeviceToHost, g.s), "D2H col") &&
               cuda_ok(cudaMemcpyAsync(dst->val, d_val.p, (std::size_t) total_slots * 2u, cudaMemcpyDeviceToHost, g.s),
                       "D2H val"))) &&
             cuda_ok(cudaStreamSynchronize(g.s), "sync emit");
    }
    if (!ok) {
        cs_b200_host_sliced_ell_clear(dst);
        return 0;
    }
    return 1;
}
