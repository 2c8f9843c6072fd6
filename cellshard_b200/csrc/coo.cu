// COO -> Blocked-ELL.
//
// Reference: convert::blocked_ell_from_coo / choose_blocked_ell_block_size_from_coo
// (src/convert/blocked_ell_from_compressed.cuh:105-257,349-478, serial host
// loops) and blocked_ell_from_coo_cuda / choose_..._from_coo_cuda
// (src/convert/blocked_ell_from_coo_cuda.cuh:17-966: 64-bit (row block, block
// column) keys, CUB sort, head flags, scans, a thread per entry scattering).
//
// Here, when every mapped column is below `cols` (and the column-block
// bitmaps of the CSR kernels stay small), the CSR route: entries whose rows
// never decrease -- COO written row by row -- get row pointers from their row
// runs; other entries are first stably sorted by column and then by row (rows
// in order, columns ascending, a repeated (row, column) keeping its entries'
// COO order) and their columns and values gathered; then the
// library's CSR -> Blocked-ELL shape and emit, which place a row's values in
// that order (a repeated column keeps its last value) and count nnz the same
// way.  Otherwise:
//   scan    one pass over the entries: rows in range and columns inside
//           the column map (others dropped and flagged), the largest mapped
//           column (one small read-back sizes the key)
//   keys    (row block << b | block column) in 32 bits when both fit, sorted
//           by the library's stable radix sort with the entry index as value;
//           otherwise two stable 32-bit sorts (block column, then row block)
//   groups  a head flag where the (row block, block column) pair changes, a
//           count of distinct pairs per row block, scans of both, the width =
//           the largest count; group g's entries start at gs[g]
//   emit    one thread per group: its slot is g - (groups before its row
//           block), it writes the block column and then the group's values
//           in entry order, so a repeated (row, column) keeps its last value
//           as the host routine's loop does, and counts the stored nonzero
//           values by their zero/nonzero transitions (both reference counts)
#include "common.cuh"

#include <cstdlib>
#include <cstring>

namespace csb {
namespace {

constexpr uint32_t kInvalid = 0xffffffffu;

// words: [0] largest mapped column, [1] dropped entries, [2] width, [3] route
// (0 two sorts, 1 one sort, 2 CSR), [4] key shift, [5] kept entries, [6] rows
// decrease somewhere, [7] the CSR route's nnz
constexpr uint32_t kRouteTwoSorts = 0u, kRouteOneSort = 1u, kRouteCsr = 2u, kRouteCsrSorted = 3u;

// The CSR route's column-block bitmaps (one bit per column block per row
// block) must stay small next to the entries themselves.
bool csr_route_fits(uint32_t n, uint32_t rows, uint32_t cols, uint32_t B) {
    std::size_t bytes = 0u;
    cs_b200_blocked_ell_scratch_bytes(rows, cols, B, &bytes);
    return bytes <= ((std::size_t) 64u << 20) || bytes <= (std::size_t) n * 16u;
}

struct coo_scratch {
    uint32_t *words;
    unsigned long long *shape;   // CSR route: width, pairs
    uint32_t *csr_ptr, *mcol;    // CSR route: row pointers, mapped (and row-sorted) columns
    uint16_t *sval;              // CSR route after the row sort: values in row order
    void *csr_tmp;
    uint32_t *keys, *rkeys, *skeys, *spos, *pos1, *flags, *gid, *gs, *rb_count, *rb_off;
    void *sort_tmp, *scan_tmp;
    std::size_t csr_bytes, sort_bytes, scan_bytes, bytes;
};

void carve(void *base, uint32_t n, uint32_t rows, uint32_t cols, uint32_t B, coo_scratch *x) {
    const uint32_t RB = (uint32_t) (((uint64_t) rows + B - 1u) / B);
    scratch_carver c(base, ~std::size_t(0));
    const std::size_t n1 = (std::size_t) n + 1u;
    x->words = c.take<uint32_t>(8);
    x->shape = c.take<unsigned long long>(2);
    x->csr_ptr = c.take<uint32_t>((std::size_t) rows + 1u);
    x->mcol = c.take<uint32_t>(n1);
    x->sval = c.take<uint16_t>(n1);
    x->csr_bytes = 0u;
    if (B != 0u && csr_route_fits(n, rows, cols, B)) cs_b200_blocked_ell_scratch_bytes(rows, cols, B, &x->csr_bytes);
    x->csr_tmp = c.take<char>(x->csr_bytes);
    x->keys = c.take<uint32_t>(n1);
    x->rkeys = c.take<uint32_t>(n1);
    x->skeys = c.take<uint32_t>(n1);
    x->spos = c.take<uint32_t>(n1);
    x->pos1 = c.take<uint32_t>(n1);
    x->flags = c.take<uint32_t>(n1);
    x->gid = c.take<uint32_t>(n1);
    x->gs = c.take<uint32_t>(n1);
    x->rb_count = c.take<uint32_t>((std::size_t) RB + 1u);
    x->rb_off = c.take<uint32_t>((std::size_t) RB + 1u);
    x->sort_bytes = sort_pairs_u32_scratch_bytes(n);
    x->sort_tmp = c.take<char>(x->sort_bytes);
    x->scan_bytes = scan_u32_scratch_bytes(n > RB ? n : RB);
    x->scan_tmp = c.take<char>(x->scan_bytes);
    x->bytes = c.used;
}

__device__ __forceinline__ uint32_t mapped(const uint32_t *col, const uint32_t *map, uint32_t i) {
    const uint32_t c = col[i];
    return map != nullptr ? map[c] : c;
}

// An entry is kept when its row is in range and, with a column map, its
// column indexes the map (the map has one entry per source column).
__device__ __forceinline__ bool entry_ok(const cs_coo_view &src, const uint32_t *map, uint32_t i) {
    return src.rowIdx[i] < src.rows && (map == nullptr || src.colIdx[i] < src.cols);
}

__global__ void __launch_bounds__(256) coo_scan_kernel(const cs_coo_view src, const uint32_t *__restrict__ map,
                                                       uint32_t *__restrict__ words, uint32_t *__restrict__ status) {
    uint32_t mx = 0u, dropped = 0u, down = 0u;
    // four entries per thread, their row and column loads issued together
    constexpr unsigned U = 4;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < src.nnz; i0 += stride * U) {
        uint32_t r[U], rp[U], c[U];
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * stride;
            const bool in = i < src.nnz && i >= i0; // i >= i0: no wrap past 2^32
            r[u] = in ? __ldg(src.rowIdx + i) : 0u;
            rp[u] = in && i != 0u ? __ldg(src.rowIdx + i - 1u) : 0u;
            c[u] = in ? __ldg(src.colIdx + i) : 0u;
        }
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * stride;
            if (i >= src.nnz || i < i0) continue;
            if (i != 0u && r[u] < rp[u]) down = 1u;
            if (!(r[u] < src.rows && (map == nullptr || c[u] < src.cols))) {
                ++dropped;
                continue;
            }
            mx = max(mx, map != nullptr ? __ldg(map + c[u]) : c[u]);
        }
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    dropped = __reduce_add_sync(0xffffffffu, dropped);
    down = __reduce_or_sync(0xffffffffu, down);
    if ((threadIdx.x & 31u) == 0u) {
        if (mx != 0u) atomicMax(words, mx);
        if (down != 0u) atomicOr(words + 6, 1u);
        if (dropped != 0u) {
            atomicAdd(words + 1, dropped);
            if (status != nullptr) atomicOr(status, (uint32_t) CS_STATUS_INDEX_RANGE);
        }
    }
}

// single: key = rb << shift | bc; otherwise keys = bc and rkeys = rb.  Dropped
// entries get the largest key so they sort last.
__global__ void __launch_bounds__(256) coo_key_kernel(const cs_coo_view src, const uint32_t *__restrict__ map,
                                                      uint32_t B, uint32_t shift, bool single,
                                                      uint32_t *__restrict__ keys, uint32_t *__restrict__ rkeys) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < src.nnz; i += gridDim.x * blockDim.x) {
        const uint32_t r = src.rowIdx[i];
        const bool ok = entry_ok(src, map, i);
        const uint32_t bc = ok ? mapped(src.colIdx, map, i) / B : kInvalid;
        if (single) {
            keys[i] = ok ? ((r / B) << shift) | bc : kInvalid;
        } else {
            keys[i] = bc;
            rkeys[i] = ok ? r / B : kInvalid;
        }
    }
}

__global__ void gather_kernel(uint32_t n, const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx,
                              uint32_t *__restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

struct coo_decode {
    const uint32_t *skeys, *spos, *col, *map;
    uint32_t B, shift, mask;
    bool single;
    __device__ __forceinline__ void at(uint32_t i, uint32_t *rb, uint32_t *bc) const {
        const uint32_t k = skeys[i];
        if (single) {
            *rb = shift == 32u ? 0u : k >> shift;
            *bc = k & mask;
        } else {
            *rb = k;
            *bc = mapped(col, map, spos[i]) / B;
        }
    }
};

__global__ void __launch_bounds__(256) coo_head_kernel(coo_decode d, uint32_t n_valid, uint32_t *__restrict__ flags,
                                                       uint32_t *__restrict__ rb_count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_valid; i += gridDim.x * blockDim.x) {
        uint32_t rb, bc;
        d.at(i, &rb, &bc);
        bool head = i == 0u;
        if (!head) {
            uint32_t rp, bp;
            d.at(i - 1u, &rp, &bp);
            head = rp != rb || bp != bc;
        }
        flags[i] = head ? 1u : 0u;
        if (head) atomicAdd(rb_count + rb, 1u);
    }
}

__global__ void __launch_bounds__(256) coo_width_kernel(uint32_t RB, const uint32_t *__restrict__ rb_count,
                                                        uint32_t *__restrict__ words) {
    uint32_t mx = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < RB; i += gridDim.x * blockDim.x)
        mx = max(mx, rb_count[i]);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31u) == 0u && mx != 0u) atomicMax(words + 2, mx);
}

__global__ void __launch_bounds__(256) coo_group_start_kernel(uint32_t n_valid, const uint32_t *__restrict__ flags,
                                                              const uint32_t *__restrict__ gid,
                                                              uint32_t *__restrict__ gs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_valid; i += gridDim.x * blockDim.x) {
        if (i == n_valid)
            gs[gid[n_valid]] = n_valid;
        else if (flags[i] != 0u)
            gs[gid[i]] = i;
    }
}

// One thread per (row block, block column) group, its entries in entry order.
__global__ void __launch_bounds__(256) coo_group_kernel(coo_decode d, const uint32_t *__restrict__ row_idx,
                                                        const uint16_t *__restrict__ val,
                                                        const uint32_t *__restrict__ gs,
                                                        const uint32_t *__restrict__ gid,
                                                        const uint32_t *__restrict__ rb_off, uint32_t n_valid,
                                                        uint32_t cols, uint32_t W, uint32_t *__restrict__ bci,
                                                        uint16_t *__restrict__ out, unsigned long long *__restrict__ nnz) {
    const uint32_t G = gid[n_valid];
    const std::size_t ell = (std::size_t) W * d.B;
    long long all = 0, in = 0;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
        const uint32_t p0 = gs[g], p1 = gs[g + 1u];
        uint32_t rb, bc;
        d.at(p0, &rb, &bc);
        const uint32_t slot = g - rb_off[rb];
        bci[(std::size_t) rb * W + slot] = bc;
        for (uint32_t p = p0; p < p1; ++p) {
            const uint32_t src = d.spos[p];
            const uint32_t c = mapped(d.col, d.map, src);
            uint16_t *cell = out + (std::size_t) row_idx[src] * ell + (std::size_t) slot * d.B + c % d.B;
            const int prev = half_nonzero(*cell) ? 1 : 0;
            const uint16_t v = val[src];
            const int next = half_nonzero(v) ? 1 : 0;
            all += next - prev;
            if (c < cols) in += next - prev;
            *cell = v;
        }
    }
    // every group's cells are written by one thread, so the transitions add up
    // to the final values' counts; a warp's net change fits 32 bits (signed)
    const int wa = (int) __reduce_add_sync(0xffffffffu, (unsigned) all);
    const int wi = (int) __reduce_add_sync(0xffffffffu, (unsigned) in);
    if ((threadIdx.x & 31u) == 0u && nnz != nullptr) {
        if (wa != 0) atomicAdd(nnz, (unsigned long long) (long long) wa);
        if (wi != 0) atomicAdd(nnz + 1, (unsigned long long) (long long) wi);
    }
}

// CSR route: row pointers of rows that never decrease (empty rows between
// runs get the next run's start) and the mapped columns.
__global__ void __launch_bounds__(256) coo_row_ptr_kernel(uint32_t n, uint32_t rows, const uint32_t *__restrict__ row,
                                                          uint32_t *__restrict__ ptr) {
    // four entries per thread, their loads issued together
    constexpr unsigned U = 4;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * U) {
        uint32_t rr[U], rp[U];
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * stride;
            const bool in = i < n && i >= i0;
            rr[u] = in ? __ldg(row + i) : 0u;
            rp[u] = in && i != 0u ? __ldg(row + i - 1u) : 0u;
        }
#pragma unroll
        for (unsigned u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * stride;
            if (i >= n || i < i0) continue;
            const uint32_t r = rr[u];
            const uint32_t lo = i == 0u ? 0u : rp[u] + 1u;
            for (uint32_t q = lo; q <= r && (i == 0u || r != rp[u]); ++q) ptr[q] = i;
            if (i == n - 1u)
                for (uint32_t q = r + 1u; q <= rows; ++q) ptr[q] = n;
        }
    }
}

__global__ void __launch_bounds__(256) coo_map_cols_kernel(uint32_t n, const uint32_t *__restrict__ col,
                                                           const uint32_t *__restrict__ map, uint32_t *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = map[col[i]];
}

// CSR route after the row sort: columns (mapped) and values in row order.
__global__ void __launch_bounds__(256) coo_gather_rows_kernel(uint32_t n, const uint32_t *__restrict__ pos,
                                                              const uint32_t *__restrict__ col,
                                                              const uint32_t *__restrict__ map,
                                                              const uint16_t *__restrict__ val,
                                                              uint32_t *__restrict__ out_col,
                                                              uint16_t *__restrict__ out_val) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = pos[i];
        out_col[i] = mapped(col, map, p);
        out_val[i] = val[p];
    }
}

__global__ void coo_nnz_from_csr_kernel(const uint32_t *__restrict__ count, unsigned long long *__restrict__ nnz) {
    if (threadIdx.x == 0u && blockIdx.x == 0u && nnz != nullptr) {
        nnz[0] += *count;
        nnz[1] += *count;
    }
}

__global__ void fill_u32_kernel(std::size_t n, uint32_t v, uint32_t *__restrict__ dst) {
    for (std::size_t i = blockIdx.x * (std::size_t) blockDim.x + threadIdx.x; i < n;
         i += (std::size_t) gridDim.x * blockDim.x)
        dst[i] = v;
}

uint32_t bits_for(uint32_t v) { return v == 0u ? 0u : 32u - (uint32_t) __builtin_clz(v); }

unsigned grid_for(const void *k, std::size_t n) { return resident_grid(k, 256, 0, (n + 255u) / 256u); }

struct coo_shape {
    uint32_t RB, n_valid, shift, width;
    bool single;
    uint64_t groups;
};

int check_coo(const cs_coo_view *src, uint32_t B, const char *who) {
    if (src == nullptr || B == 0u) {
        set_error("%s: null view or zero block size", who);
        return 0;
    }
    if (src->nnz != 0u && (src->rowIdx == nullptr || src->colIdx == nullptr || src->val == nullptr)) {
        set_error("%s: null COO arrays", who);
        return 0;
    }
    return 1;
}

coo_decode decoder(const cs_coo_view *src, const uint32_t *map, const coo_scratch &x, const coo_shape &s, uint32_t B) {
    coo_decode d;
    d.skeys = x.skeys;
    d.spos = x.spos;
    d.col = src->colIdx;
    d.map = map;
    d.B = B;
    d.shift = s.shift;
    d.mask = s.shift >= 32u ? kInvalid : ((1u << s.shift) - 1u);
    d.single = s.single;
    return d;
}

// The CSR view of the CSR route (row pointers and mapped or row-sorted columns
// in the scratch).
cs_compressed_view csr_of(const cs_coo_view *src, const uint32_t *map, uint32_t cols, const coo_scratch &x,
                          bool sorted) {
    if (sorted) return cs_compressed_view{src->rows, cols, src->nnz, CS_COMPRESSED_BY_ROW, x.csr_ptr, x.mcol, x.sval};
    return cs_compressed_view{src->rows, cols, src->nnz, CS_COMPRESSED_BY_ROW, x.csr_ptr,
                              map != nullptr ? x.mcol : src->colIdx, src->val};
}

// Plan of one block size; leaves the shape words in the scratch for the emit.
int coo_plan(const cs_coo_view *src, const uint32_t *map, uint32_t cols, uint32_t B, void *scratch, std::size_t bytes,
             coo_shape *s, uint32_t *status, cudaStream_t stream) {
    if (!check_coo(src, B, "coo_blocked_ell_plan")) return 0;
    const uint32_t n = src->nnz;
    s->RB = (uint32_t) (((uint64_t) src->rows + B - 1u) / B);
    coo_scratch x;
    carve(nullptr, n, src->rows, cols, B, &x);
    if (scratch == nullptr || bytes < x.bytes) {
        set_error("coo_blocked_ell_plan: scratch %zu < %zu bytes", bytes, x.bytes);
        return 0;
    }
    carve(scratch, n, src->rows, cols, B, &x);
    s->width = 0u;
    s->groups = 0u;
    s->n_valid = 0u;
    s->shift = 0u;
    s->single = true;
    if (!cuda_ok(cudaMemsetAsync(x.words, 0, 32, stream), "coo words")) return 0;
    if (n == 0u) {
        const uint32_t empty[8] = {0, 0, 0, kRouteOneSort, 0, 0, 0, 0};
        return cuda_ok(cudaMemcpyAsync(x.words, empty, 32, cudaMemcpyHostToDevice, stream), "coo words") &&
               cuda_ok(cudaStreamSynchronize(stream), "coo sync");
    }
    coo_scan_kernel<<<grid_for((const void *) coo_scan_kernel, n), 256, 0, stream>>>(*src, map, x.words, status);
    if (!launch_ok("coo_scan_kernel")) return 0;
    uint32_t w[8] = {0};
    if (!cuda_ok(cudaMemcpyAsync(w, x.words, 32, cudaMemcpyDeviceToHost, stream), "D2H coo scan") ||
        !cuda_ok(cudaStreamSynchronize(stream), "coo scan sync"))
        return 0;
    s->n_valid = n - w[1];
    uint32_t route;
    if (w[1] == 0u && w[0] < cols && x.csr_bytes != 0u) {
        // every column fits: the CSR route, after a stable sort by row when rows decrease somewhere
        const bool sorted = w[6] != 0u;
        route = sorted ? kRouteCsrSorted : kRouteCsr;
        const uint32_t *rows_in_order = src->rowIdx;
        if (sorted) {
            // stable by (mapped) column, then stable by row: rows in order, columns ascending
            // inside a row, repeated (row, column) entries next to each other in COO order
            const uint32_t *ckeys = src->colIdx;
            if (map != nullptr) {
                coo_map_cols_kernel<<<grid_for((const void *) coo_map_cols_kernel, n), 256, 0, stream>>>(
                    n, src->colIdx, map, x.keys);
                if (!launch_ok("coo_map_cols_kernel")) return 0;
                ckeys = x.keys;
            }
            if (!sort_pairs_u32(ckeys, nullptr, n, x.flags, x.pos1, x.sort_tmp, x.sort_bytes, stream)) return 0;
            gather_kernel<<<grid_for((const void *) gather_kernel, n), 256, 0, stream>>>(n, src->rowIdx, x.pos1,
                                                                                       x.keys);
            if (!launch_ok("gather_kernel")) return 0;
            if (!sort_pairs_u32(x.keys, x.pos1, n, x.skeys, x.spos, x.sort_tmp, x.sort_bytes, stream)) return 0;
            coo_gather_rows_kernel<<<grid_for((const void *) coo_gather_rows_kernel, n), 256, 0, stream>>>(
                n, x.spos, src->colIdx, map, src->val, x.mcol, x.sval);
            if (!launch_ok("coo_gather_rows_kernel")) return 0;
            rows_in_order = x.skeys;
        } else if (map != nullptr) {
            coo_map_cols_kernel<<<grid_for((const void *) coo_map_cols_kernel, n), 256, 0, stream>>>(n, src->colIdx,
                                                                                                   map, x.mcol);
            if (!launch_ok("coo_map_cols_kernel")) return 0;
        }
        coo_row_ptr_kernel<<<grid_for((const void *) coo_row_ptr_kernel, n), 256, 0, stream>>>(n, src->rows,
                                                                                              rows_in_order, x.csr_ptr);
        if (!launch_ok("coo_row_ptr_kernel")) return 0;
        const cs_compressed_view v = csr_of(src, map, cols, x, sorted);
        unsigned long long shape[2] = {0, 0};
        if (!cuda_ok(cudaMemsetAsync(x.shape, 0, 16, stream), "shape clear") ||
            !cs_b200_blocked_ell_shape(&v, B, (uint64_t *) x.shape, x.csr_tmp, x.csr_bytes, status,
                                       reinterpret_cast<cs_stream_t>(stream)) ||
            !cuda_ok(cudaMemcpyAsync(shape, x.shape, 16, cudaMemcpyDeviceToHost, stream), "D2H shape") ||
            !cuda_ok(cudaStreamSynchronize(stream), "coo csr shape sync"))
            return 0;
        s->width = (uint32_t) shape[0];
        s->groups = shape[1];
        const uint32_t words[4] = {s->width, route, 0u, s->n_valid};
        return cuda_ok(cudaMemcpyAsync(x.words + 2, words, 16, cudaMemcpyHostToDevice, stream), "coo words") &&
               cuda_ok(cudaStreamSynchronize(stream), "coo words sync");
    }
    s->shift = bits_for(w[0] / B);
    s->single = bits_for(s->RB - 1u) + s->shift <= 31u;
    route = s->single ? kRouteOneSort : kRouteTwoSorts;
    coo_key_kernel<<<grid_for((const void *) coo_key_kernel, n), 256, 0, stream>>>(*src, map, B, s->shift, s->single,
                                                                                 x.keys, x.rkeys);
    if (!launch_ok("coo_key_kernel")) return 0;
    if (s->single) {
        if (!sort_pairs_u32(x.keys, nullptr, n, x.skeys, x.spos, x.sort_tmp, x.sort_bytes, stream)) return 0;
    } else {
        // stable by block column, then stable by row block: the (row block, block column) order
        if (!sort_pairs_u32(x.keys, nullptr, n, x.flags, x.pos1, x.sort_tmp, x.sort_bytes, stream)) return 0;
        gather_kernel<<<grid_for((const void *) gather_kernel, n), 256, 0, stream>>>(n, x.rkeys, x.pos1, x.keys);
        if (!launch_ok("gather_kernel")) return 0;
        if (!sort_pairs_u32(x.keys, x.pos1, n, x.skeys, x.spos, x.sort_tmp, x.sort_bytes, stream)) return 0;
    }
    if (!cuda_ok(cudaMemsetAsync(x.rb_count, 0, ((std::size_t) s->RB + 1u) * 4u, stream), "rb counts")) return 0;
    const coo_decode d = decoder(src, map, x, *s, B);
    if (s->n_valid != 0u) {
        coo_head_kernel<<<grid_for((const void *) coo_head_kernel, s->n_valid), 256, 0, stream>>>(d, s->n_valid,
                                                                                                 x.flags, x.rb_count);
        if (!launch_ok("coo_head_kernel")) return 0;
    }
    if (!scan_exclusive_u32(x.flags, x.gid, s->n_valid, true, x.scan_tmp, x.scan_bytes, stream) ||
        !scan_exclusive_u32(x.rb_count, x.rb_off, s->RB, true, x.scan_tmp, x.scan_bytes, stream))
        return 0;
    coo_width_kernel<<<grid_for((const void *) coo_width_kernel, s->RB), 256, 0, stream>>>(s->RB, x.rb_count, x.words);
    coo_group_start_kernel<<<grid_for((const void *) coo_group_start_kernel, (std::size_t) s->n_valid + 1u), 256, 0,
                             stream>>>(s->n_valid, x.flags, x.gid, x.gs);
    if (!launch_ok("coo_group_start_kernel")) return 0;
    uint32_t tail[2] = {0, 0};
    if (!cuda_ok(cudaMemcpyAsync(tail, x.words + 2, 4, cudaMemcpyDeviceToHost, stream), "D2H width") ||
        !cuda_ok(cudaMemcpyAsync(tail + 1, x.rb_off + s->RB, 4, cudaMemcpyDeviceToHost, stream), "D2H groups") ||
        !cuda_ok(cudaStreamSynchronize(stream), "coo plan sync"))
        return 0;
    s->width = tail[0];
    s->groups = tail[1];
    // what the emit needs rides in the words: [3] route, [4] shift, [5] kept entries
    const uint32_t more[3] = {route, s->shift, s->n_valid};
    return cuda_ok(cudaMemcpyAsync(x.words + 3, more, 12, cudaMemcpyHostToDevice, stream), "coo shape") &&
           cuda_ok(cudaStreamSynchronize(stream), "coo shape sync");
}

int coo_emit(const cs_coo_view *src, const uint32_t *map, uint32_t cols, const void *scratch, std::size_t bytes,
             const cs_blocked_ell_view *dst, uint64_t *d_nnz, cudaStream_t stream) {
    if (dst == nullptr || !check_coo(src, dst->block_size, "coo_blocked_ell_emit")) return 0;
    const uint32_t B = dst->block_size, n = src->nnz;
    coo_shape s;
    s.RB = (uint32_t) (((uint64_t) src->rows + B - 1u) / B);
    coo_scratch x;
    carve(nullptr, n, src->rows, cols, B, &x);
    if (scratch == nullptr || bytes < x.bytes) {
        set_error("coo_blocked_ell_emit: scratch %zu < %zu bytes", bytes, x.bytes);
        return 0;
    }
    carve(const_cast<void *>(scratch), n, src->rows, cols, B, &x);
    uint32_t w[8];
    if (!cuda_ok(cudaMemcpyAsync(w, x.words, 32, cudaMemcpyDeviceToHost, stream), "D2H coo words") ||
        !cuda_ok(cudaStreamSynchronize(stream), "coo words sync"))
        return 0;
    s.width = w[2];
    const uint32_t route = w[3];
    s.single = route == kRouteOneSort;
    s.shift = w[4];
    s.n_valid = w[5];
    if (dst->rows != src->rows || dst->ell_cols != s.width * B || dst->cols != cols) {
        set_error("coo_blocked_ell_emit: destination shape differs from the plan (ell_cols %u, width %u x %u)",
                  dst->ell_cols, s.width, B);
        return 0;
    }
    if (s.width == 0u || src->rows == 0u) return 1;
    if (dst->blockColIdx == nullptr || dst->val == nullptr) {
        set_error("coo_blocked_ell_emit: null destination arrays");
        return 0;
    }
    if (route == kRouteCsr || route == kRouteCsrSorted) {
        const cs_compressed_view v = csr_of(src, map, cols, x, route == kRouteCsrSorted);
        if (!cuda_ok(cudaMemsetAsync(x.words + 7, 0, 4, stream), "csr nnz clear") ||
            !cs_b200_blocked_ell_emit(&v, dst, x.words + 7, x.csr_tmp, x.csr_bytes, nullptr,
                                      reinterpret_cast<cs_stream_t>(stream)))
            return 0;
        coo_nnz_from_csr_kernel<<<1, 32, 0, stream>>>(x.words + 7, (unsigned long long *) d_nnz);
        return launch_ok("coo_nnz_from_csr_kernel");
    }
    const std::size_t nb = (std::size_t) s.RB * s.width;
    fill_u32_kernel<<<grid_for((const void *) fill_u32_kernel, nb), 256, 0, stream>>>(nb, kInvalid, dst->blockColIdx);
    if (!launch_ok("fill_u32_kernel") ||
        !cuda_ok(cudaMemsetAsync(dst->val, 0, (std::size_t) dst->rows * dst->ell_cols * 2u, stream), "values memset"))
        return 0;
    if (s.n_valid == 0u) return 1;
    const coo_decode d = decoder(src, map, x, s, B);
    coo_group_kernel<<<grid_for((const void *) coo_group_kernel, s.n_valid), 256, 0, stream>>>(
        d, src->rowIdx, src->val, x.gs, x.gid, x.rb_off, s.n_valid, cols, s.width, dst->blockColIdx, dst->val,
        (unsigned long long *) d_nnz);
    return launch_ok("coo_group_kernel");
}

// Host COO staged on the device (upload_coo, blocked_ell_from_coo_cuda.cuh:
// 462-520): entries and the optional column map.
struct staged_coo {
    dmem row, col, val, map;
    cs_coo_view view{};
    const uint32_t *d_map = nullptr;
};

int stage_coo(const cs_host_coo *src, const uint32_t *feature_to_global, staged_coo *st, cudaStream_t stream) {
    const std::size_t n = src->nnz;
    if (!st->row.alloc(n * 4u, "coo rows") || !st->col.alloc(n * 4u, "coo cols") || !st->val.alloc(n * 2u, "coo val"))
        return 0;
    if (n != 0u && (!cuda_ok(cudaMemcpyAsync(st->row.p, src->rowIdx, n * 4u, cudaMemcpyHostToDevice, stream), "H2D rows") ||
                    !cuda_ok(cudaMemcpyAsync(st->col.p, src->colIdx, n * 4u, cudaMemcpyHostToDevice, stream), "H2D cols") ||
                    !cuda_ok(cudaMemcpyAsync(st->val.p, src->val, n * 2u, cudaMemcpyHostToDevice, stream), "H2D val")))
        return 0;
    if (feature_to_global != nullptr) {
        if (!st->map.alloc((std::size_t) src->cols * 4u, "coo map") ||
            (src->cols != 0u && !cuda_ok(cudaMemcpyAsync(st->map.p, feature_to_global, (std::size_t) src->cols * 4u,
                                                         cudaMemcpyHostToDevice, stream), "H2D map")))
            return 0;
        st->d_map = (const uint32_t *) st->map.p;
    }
    st->view = cs_coo_view{src->rows, src->cols, src->nnz, (uint32_t *) st->row.p, (uint32_t *) st->col.p,
                           (uint16_t *) st->val.p};
    return 1;
}

std::size_t coo_scratch_bytes(uint32_t n, uint32_t rows, uint32_t cols, uint32_t B) {
    coo_scratch x;
    carve(nullptr, n, rows, cols, B, &x);
    return x.bytes;
}

// Host form: stage, plan, allocate, emit, copy back; nnz_index picks the
// host routine's count (0) or the GPU routine's (1).
int host_from_coo(const cs_host_coo *src, uint32_t cols, const uint32_t *map, unsigned int B, cs_host_blocked_ell *dst,
                  int nnz_index, const char *who) {
    if (src == nullptr || dst == nullptr || cols == 0u || B == 0u) {
        set_error("%s: null argument, zero cols or zero block size", who);
        return 0;
    }
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    staged_coo sc;
    if (!stage_coo(src, map, &sc, g.s)) return 0;
    dmem scratch, status, nnz;
    const std::size_t bytes = coo_scratch_bytes(src->nnz, src->rows, cols, B);
    if (!scratch.alloc(bytes, "coo scratch") || !status.alloc(16, "status") || !nnz.alloc(16, "nnz") ||
        !cuda_ok(cudaMemsetAsync(status.p, 0, 16, g.s), "status clear") ||
        !cuda_ok(cudaMemsetAsync(nnz.p, 0, 16, g.s), "nnz clear"))
        return 0;
    coo_shape s;
    if (!coo_plan(&sc.view, sc.d_map, cols, B, scratch.p, bytes, &s, (uint32_t *) status.p, g.s)) return 0;
    if (s.n_valid != src->nnz) {
        set_error("%s: %u entries have a row index >= rows (%u)", who, src->nnz - s.n_valid, src->rows);
        return 0;
    }
    cs_b200_host_blocked_ell_clear(dst);
    dst->rows = src->rows;
    dst->cols = cols;
    dst->nnz = src->nnz;
    dst->block_size = B;
    dst->ell_cols = s.width * B;
    if (!host_blocked_ell_allocate(dst)) {
        set_error("%s: host allocation failed", who);
        return 0;
    }
    const std::size_t nb = (std::size_t) s.RB * s.width, nv = (std::size_t) src->rows * dst->ell_cols;
    dmem d_bci, d_val;
    uint64_t counts[2] = {0, 0};
    const cs_blocked_ell_view dv{src->rows, cols, 0u, B, dst->ell_cols, nullptr, nullptr};
    bool ok = d_bci.alloc(nb * 4u, "bci") && d_val.alloc(nv * 2u, "values");
    cs_blocked_ell_view v = dv;
    v.blockColIdx = (uint32_t *) d_bci.p;
    v.val = (uint16_t *) d_val.p;
    ok = ok && coo_emit(&sc.view, sc.d_map, cols, scratch.p, bytes, &v, (uint64_t *) nnz.p, g.s) &&
         (nb == 0u || cuda_ok(cudaMemcpyAsync(dst->blockColIdx, d_bci.p, nb * 4u, cudaMemcpyDeviceToHost, g.s), "D2H bci")) &&
         (nv == 0u || cuda_ok(cudaMemcpyAsync(dst->val, d_val.p, nv * 2u, cudaMemcpyDeviceToHost, g.s), "D2H values")) &&
         cuda_ok(cudaMemcpyAsync(counts, nnz.p, 16, cudaMemcpyDeviceToHost, g.s), "D2H nnz") &&
         cuda_ok(cudaStreamSynchronize(g.s), "sync coo");
    if (!ok) {
        cs_b200_host_blocked_ell_clear(dst);
        return 0;
    }
    dst->nnz = (uint32_t) counts[nnz_index];
    return 1;
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_coo_blocked_ell_scratch_bytes(uint32_t nnz, uint32_t rows, uint32_t cols,
                                                     uint32_t block_size, size_t *out_bytes) {
    if (out_bytes == nullptr || block_size == 0u) {
        set_error("coo_blocked_ell_scratch_bytes: null output or zero block size");
        return 0;
    }
    *out_bytes = coo_scratch_bytes(nnz, rows, cols, block_size);
    return 1;
}

extern "C" int cs_b200_coo_blocked_ell_plan(const cs_coo_view *src, const uint32_t *d_feature_to_global,
                                            uint32_t cols, uint32_t block_size, void *d_scratch, size_t scratch_bytes,
                                            uint32_t *ell_width_out, uint64_t *total_blocks_out, uint32_t *d_status,
                                            cs_stream_t s) {
    coo_shape sh;
    if (!coo_plan(src, d_feature_to_global, cols, block_size, d_scratch, scratch_bytes, &sh, d_status,
                  as_stream(s)))
        return 0;
    if (ell_width_out != nullptr) *ell_width_out = sh.width;
    if (total_blocks_out != nullptr) *total_blocks_out = sh.groups;
    return 1;
}

extern "C" int cs_b200_coo_blocked_ell_emit(const cs_coo_view *src, const uint32_t *d_feature_to_global,
                                            uint32_t cols, const void *d_scratch, size_t scratch_bytes,
                                            const cs_blocked_ell_view *dst, uint64_t *d_nnz, cs_stream_t s) {
    return coo_emit(src, d_feature_to_global, cols, d_scratch, scratch_bytes, dst, d_nnz, as_stream(s));
}

extern "C" int cs_b200_blocked_ell_from_coo(const cs_host_coo *src, uint32_t cols, const uint32_t *feature_to_global,
                                            unsigned int block_size, cs_host_blocked_ell *dst) {
    return host_from_coo(src, cols, feature_to_global, block_size, dst, 0, "blocked_ell_from_coo");
}

extern "C" int cs_b200_blocked_ell_from_coo_cuda(const cs_host_coo *src, uint32_t cols,
                                                 const uint32_t *feature_to_global, unsigned int block_size,
                                                 cs_host_blocked_ell *dst, int device) {
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return 0;
    return host_from_coo(src, cols, feature_to_global, block_size, dst, 1, "blocked_ell_from_coo_cuda");
}

extern "C" int cs_b200_choose_blocked_ell_block_size_from_coo(const cs_host_coo *src, uint32_t cols,
                                                              const uint32_t *feature_to_global,
                                                              const unsigned int *candidates,
                                                              unsigned int candidate_count,
                                                              cs_blocked_ell_tune_result *out) {
    if (src == nullptr || out == nullptr || candidates == nullptr || candidate_count == 0u || cols == 0u) {
        set_error("choose_blocked_ell_block_size_from_coo: null argument, no candidates or zero cols");
        return 0;
    }
    own_stream g;
    if (!cuda_ok(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking), "stream create")) return 0;
    staged_coo sc;
    if (!stage_coo(src, feature_to_global, &sc, g.s)) return 0;
    std::size_t bytes = 0u;
    for (unsigned int i = 0; i < candidate_count; ++i) {
        if (candidates[i] == 0u) continue;
        const std::size_t b = coo_scratch_bytes(src->nnz, src->rows, cols, candidates[i]);
        if (b > bytes) bytes = b;
    }
    dmem scratch;
    if (!scratch.alloc(bytes, "coo scratch")) return 0;
    cs_blocked_ell_tune_result best{0u, 0.0, 0u};
    for (unsigned int i = 0; i < candidate_count; ++i) {
        const unsigned int B = candidates[i];
        if (B == 0u) continue;
        coo_shape s;
        if (!coo_plan(&sc.view, sc.d_map, cols, B, scratch.p, bytes, &s, nullptr, g.s)) return 0;
        if (s.n_valid != src->nnz) {
            set_error("choose_blocked_ell_block_size_from_coo: entries with a row index >= rows");
            return 0;
        }
        const std::size_t padded = (std::size_t) src->rows * s.width * B * 2u;
        const double fill = (s.RB == 0u || s.width == 0u)
                                ? 1.0
                                : (double) s.groups / (double) ((unsigned long) s.RB * (unsigned long) s.width);
        if (best.block_size == 0u || padded + 1u < best.padded_bytes ||
            (padded == best.padded_bytes && fill > best.fill_ratio + 1.0e-9) ||
            (padded == best.padded_bytes && fill + 1.0e-9 >= best.fill_ratio && B > best.block_size)) {
            best.block_size = B;
            best.fill_ratio = fill;
            best.padded_bytes = padded;
        }
    }
    if (best.block_size == 0u) {
        set_error("choose_blocked_ell_block_size_from_coo: no usable candidate");
        return 0;
    }
    *out = best;
    return 1;
}
