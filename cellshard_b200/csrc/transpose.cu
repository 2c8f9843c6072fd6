// Stable compressed transpose: CSR (cDim x uDim) -> CSC, row indices ascending
// inside every column -- the result of cusparseCsr2cscEx2 (ALG1), which the
// reference's build_compressed_transpose_raw uses as its primary path
// (src/convert/compressed_transpose_raw.cuh:43-81).  Its atomic fallback
// (:84-121) is order-nondeterministic and is not reproduced.
//
//   hist     rows are cut into T tiles; each CTA counts its tile's entries
//            per column in shared memory -> H[t][c].
//   colscan  per column, exclusive scan of H over tiles (in place) and the
//            column total; one device scan of the totals gives out_ptr.
//   scatter  each CTA replays its tile 16 rows at a time.  Round A sets, per
//            column, a 16-bit mask of which batch rows hold it (atomicOr in a
//            packed shared word: mask << 16 | running count); round B places
//            entry (r, c) at out_ptr[c] + H[t][c] + count + popc(mask below r);
//            round C advances the count.  Placement is therefore fixed by
//            (tile, row) order alone -- deterministic and stable.
// A row that repeats a column sets CS_STATUS_DUPLICATE_COL in the status word
// at the start of the caller's scratch.
#include "common.cuh"

namespace csb {
namespace {

constexpr unsigned kThreads = 512;
constexpr unsigned kBatchRows = 16;
constexpr uint32_t kColRange = 32768; // columns per shared-memory pass (128 KB)
constexpr uint32_t kMaxTileRows = 65535;

struct tr_layout {
    uint32_t *status;
    uint32_t *hist; // [tiles * uDim]
    void *scan_tmp;
    std::size_t scan_bytes;
    std::size_t bytes;
    uint32_t tiles, tile_rows, passes;
};

void make_layout(uint32_t cDim, uint32_t uDim, void *base, std::size_t cap, tr_layout *l) {
    const uint32_t sms = (uint32_t) sm_count();
    uint32_t tiles = cDim == 0u ? 1u : (cDim + 15u) / 16u;
    if (tiles > 2u * sms) tiles = 2u * sms;
    const uint32_t min_tiles = cDim == 0u ? 1u : (cDim + kMaxTileRows - 1u) / kMaxTileRows;
    if (tiles < min_tiles) tiles = min_tiles;
    if (tiles == 0u) tiles = 1u;
    l->tiles = tiles;
    l->tile_rows = cDim == 0u ? 0u : (cDim + tiles - 1u) / tiles;
    l->passes = uDim == 0u ? 0u : (uDim + kColRange - 1u) / kColRange;
    scratch_carver c(base, cap);
    l->status = c.take<uint32_t>(4);
    l->hist = c.take<uint32_t>((std::size_t) tiles * uDim + 1u);
    l->scan_bytes = scan_u32_scratch_bytes(uDim);
    l->scan_tmp = c.take<char>(l->scan_bytes);
    l->bytes = c.used;
}

__global__ void __launch_bounds__(kThreads) tr_hist_kernel(const uint32_t *__restrict__ ptr,
                                                          const uint32_t *__restrict__ idx, uint32_t cDim,
                                                          uint32_t uDim, uint32_t tile_rows,
                                                          uint32_t *__restrict__ hist, uint32_t *status) {
    extern __shared__ uint32_t tr_counts[];
    const uint32_t t = blockIdx.x;
    const uint32_t c0 = blockIdx.y * kColRange;
    const uint32_t cr = min(kColRange, uDim - c0);
    for (uint32_t k = threadIdx.x; k < cr; k += blockDim.x) tr_counts[k] = 0u;
    __syncthreads();
    const uint32_t r0 = t * tile_rows;
    const uint32_t r1 = min(cDim, r0 + tile_rows);
    uint32_t bad = 0u;
    if (r0 < r1) {
        const uint32_t a = ptr[r0], e = ptr[r1];
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c >= uDim) {
                bad |= CS_STATUS_INDEX_RANGE;
                continue;
            }
            if (c - c0 < cr) atomicAdd(tr_counts + (c - c0), 1u);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cr; k += blockDim.x) hist[(std::size_t) t * uDim + c0 + k] = tr_counts[k];
    if (bad) status_or(status, bad);
}

__global__ void __launch_bounds__(256) tr_colscan_kernel(uint32_t uDim, uint32_t tiles, uint32_t *__restrict__ hist,
                                                         uint32_t *__restrict__ totals) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= uDim) return;
    uint32_t run = 0u;
    for (uint32_t t = 0; t < tiles; ++t) {
        const std::size_t k = (std::size_t) t * uDim + c;
        const uint32_t v = hist[k];
        hist[k] = run;
        run += v;
    }
    totals[c] = run;
}

__global__ void __launch_bounds__(kThreads) tr_scatter_kernel(const uint32_t *__restrict__ ptr,
                                                             const uint32_t *__restrict__ idx,
                                                             const uint16_t *__restrict__ val, uint32_t cDim,
                                                             uint32_t uDim, uint32_t tile_rows,
                                                             const uint32_t *__restrict__ hist,
                                                             const uint32_t *__restrict__ out_ptr,
                                                             uint32_t *__restrict__ out_idx,
                                                             uint16_t *__restrict__ out_val, uint32_t *status) {
    extern __shared__ uint32_t tr_packed[]; // (mask << 16) | count per column of the pass
    __shared__ uint32_t rp[kBatchRows + 1];
    const uint32_t t = blockIdx.x;
    const uint32_t c0 = blockIdx.y * kColRange;
    const uint32_t cr = min(kColRange, uDim - c0);
    for (uint32_t k = threadIdx.x; k < cr; k += blockDim.x) tr_packed[k] = 0u;
    const uint32_t r0 = t * tile_rows;
    const uint32_t r1 = min(cDim, r0 + tile_rows);
    const uint32_t *hrow = hist + (std::size_t) t * uDim;
    uint32_t bad = 0u;
    for (uint32_t b0 = r0; b0 < r1; b0 += kBatchRows) {
        const uint32_t nb = min(kBatchRows, r1 - b0);
        __syncthreads();
        if (threadIdx.x <= nb) rp[threadIdx.x] = ptr[b0 + threadIdx.x];
        __syncthreads();
        const uint32_t a = rp[0], e = rp[nb];
        // round A: which batch rows hold each column
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c - c0 >= cr || c >= uDim) continue;
            uint32_t rl = 0u;
            while (rl + 1u < nb && rp[rl + 1u] <= i) ++rl;
            const uint32_t bit = 1u << (16u + rl);
            if (atomicOr(tr_packed + (c - c0), bit) & bit) bad |= CS_STATUS_DUPLICATE_COL;
        }
        __syncthreads();
        // round B: place
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c - c0 >= cr || c >= uDim) continue;
            uint32_t rl = 0u;
            while (rl + 1u < nb && rp[rl + 1u] <= i) ++rl;
            const uint32_t w = tr_packed[c - c0];
            const uint32_t mask = w >> 16;
            const uint32_t rank = (w & 0xffffu) + __popc(mask & ((1u << rl) - 1u));
            const uint32_t pos = out_ptr[c] + hrow[c] + rank;
            out_idx[pos] = b0 + rl;
            out_val[pos] = val[i];
        }
        __syncthreads();
        // round C: advance the per-column count, clear the mask
        for (uint32_t i = a + threadIdx.x; i < e; i += blockDim.x) {
            const uint32_t c = idx[i];
            if (c - c0 >= cr || c >= uDim) continue;
            uint32_t rl = 0u;
            while (rl + 1u < nb && rp[rl + 1u] <= i) ++rl;
            const uint32_t w = tr_packed[c - c0];
            const uint32_t mask = w >> 16;
            if (rl == (uint32_t) (__ffs(mask) - 1)) tr_packed[c - c0] = ((w & 0xffffu) + __popc(mask)) & 0xffffu;
        }
    }
    if (bad) status_or(status, bad);
}

} // namespace

int transpose_launch(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *ptr, const uint32_t *idx,
                     const uint16_t *val, uint32_t *out_ptr, uint32_t *out_idx, uint16_t *out_val, void *scratch,
                     std::size_t scratch_bytes, cudaStream_t stream) {
    tr_layout l;
    make_layout(cDim, uDim, scratch, scratch_bytes, &l);
    if (scratch == nullptr || l.bytes > scratch_bytes) {
        set_error("compressed_transpose: scratch %zu < %zu bytes", scratch_bytes, l.bytes);
        return 0;
    }
    if (!cuda_ok(cudaMemsetAsync(l.status, 0, 16, stream), "transpose status memset") ||
        !cuda_ok(cudaMemsetAsync(out_ptr, 0, ((std::size_t) uDim + 1u) * 4u, stream), "transpose out_ptr memset"))
        return 0;
    if (nnz == 0u || cDim == 0u || uDim == 0u) return 1;
    const std::size_t smem = (std::size_t) min(uDim, kColRange) * sizeof(uint32_t);
    if (!cuda_ok(cudaFuncSetAttribute(tr_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "hist smem attribute") ||
        !cuda_ok(cudaFuncSetAttribute(tr_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                 "scatter smem attribute"))
        return 0;
    dim3 grid(l.tiles, l.passes);
    tr_hist_kernel<<<grid, kThreads, smem, stream>>>(ptr, idx, cDim, uDim, l.tile_rows, l.hist, l.status);
    if (!launch_ok("tr_hist_kernel")) return 0;
    tr_colscan_kernel<<<(uDim + 255u) / 256u, 256, 0, stream>>>(uDim, l.tiles, l.hist, out_ptr);
    if (!launch_ok("tr_colscan_kernel")) return 0;
    if (!scan_exclusive_u32(out_ptr, out_ptr, uDim, true, l.scan_tmp, l.scan_bytes, stream)) return 0;
    tr_scatter_kernel<<<grid, kThreads, smem, stream>>>(ptr, idx, val, cDim, uDim, l.tile_rows, l.hist, out_ptr,
                                                        out_idx, out_val, l.status);
    return launch_ok("tr_scatter_kernel");
}

std::size_t transpose_scratch(uint32_t cDim, uint32_t uDim) {
    tr_layout l;
    make_layout(cDim, uDim, nullptr, 0, &l);
    return l.bytes;
}

// CSC (cols-major) -> CSR (rows-major) into fresh device buffers (used by the
// host conversion wrappers for column-compressed input).
int transpose_csc_to_csr_staged(const cs_compressed_view *src, uint32_t **d_ptr, uint32_t **d_idx, uint16_t **d_val,
                                cudaStream_t stream) {
    const uint32_t cDim = src->cols, uDim = src->rows;
    void *scratch = nullptr;
    const std::size_t sb = transpose_scratch(cDim, uDim);
    if (!cuda_ok(cudaMalloc((void **) d_ptr, ((std::size_t) uDim + 1u) * 4u), "transpose ptr") ||
        !cuda_ok(cudaMalloc((void **) d_idx, (std::size_t) src->nnz * 4u + 16u), "transpose idx") ||
        !cuda_ok(cudaMalloc((void **) d_val, (std::size_t) src->nnz * 2u + 16u), "transpose val") ||
        !cuda_ok(cudaMalloc(&scratch, sb), "transpose scratch"))
        return 0;
    int ok = transpose_launch(cDim, uDim, src->nnz, src->majorPtr, src->minorIdx, src->val, *d_ptr, *d_idx, *d_val,
                              scratch, sb, stream);
    uint32_t status = 0u;
    if (ok)
        ok = cuda_ok(cudaMemcpyAsync(&status, scratch, 4, cudaMemcpyDeviceToHost, stream), "transpose status") &&
             cuda_ok(cudaStreamSynchronize(stream), "transpose sync");
    cudaFree(scratch);
    if (ok && status != 0u) {
        set_error("column-compressed input rejected (status 0x%x)", status);
        ok = 0;
    }
    return ok;
}

} // namespace csb

using namespace csb;

extern "C" int cs_b200_compressed_transpose_scratch_bytes(uint32_t cDim, uint32_t uDim, uint32_t nnz,
                                                          size_t *out_bytes) {
    (void) nnz;
    if (out_bytes == nullptr) {
        set_error("compressed_transpose_scratch_bytes: null output");
        return 0;
    }
    *out_bytes = transpose_scratch(cDim, uDim);
    return 1;
}

extern "C" int cs_b200_build_compressed_transpose(uint32_t cDim, uint32_t uDim, uint32_t nnz, const uint32_t *d_cAxPtr,
                                                  const uint32_t *d_uAxIdx, const uint16_t *d_val,
                                                  uint32_t *d_out_uAxPtr, uint32_t *d_heads, uint32_t *d_out_cAxIdx,
                                                  uint16_t *d_out_val, void *d_scan_tmp, size_t scan_bytes,
                                                  cs_stream_t s) {
    (void) d_heads;
    if (d_out_uAxPtr == nullptr || (nnz != 0u && (d_cAxPtr == nullptr || d_uAxIdx == nullptr || d_val == nullptr ||
                                                  d_out_cAxIdx == nullptr || d_out_val == nullptr))) {
        set_error("compressed_transpose: null device array");
        return 0;
    }
    return transpose_launch(cDim, uDim, nnz, d_cAxPtr, d_uAxIdx, d_val, d_out_uAxPtr, d_out_cAxIdx, d_out_val,
                            d_scan_tmp, scan_bytes, as_stream(s));
}
