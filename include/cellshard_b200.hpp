/*
 * cellshard_b200.hpp -- C++ drop-in shim over the C ABI of cellshard_b200.h.
 *
 * Host code written against the reference's C++ API (namespaces
 * cellshard::{sparse, device, convert, bucket, runtime}) includes this header
 * instead of the reference's headers for the hot path and keeps its calls:
 * the types below are field for field the reference's (same names, same
 * layouts, __half values), and every function keeps the reference's name,
 * argument order and meaning and its return convention (int 1/0, or
 * cudaError_t for the device:: staging calls).  A translation unit includes
 * either this header or the reference's, not both.
 *
 * Reference declarations mirrored here:
 *   formats/compressed.cuh:24-37, blocked_ell.cuh:15-25, sliced_ell.cuh:16-28
 *   runtime/device/sharded_device.cuh:22-35,67-98,343-991,1050-1083
 *   src/convert/blocked_ell_from_compressed.cuh:157-190,258-347
 *   src/convert/sliced_ell_from_compressed.cuh:96-164,
 *       sliced_ell_from_blocked_ell.cuh:18-26,196-221
 *   src/convert/blocked_ell_from_compressed.cuh:192-257,349-478 (COO),
 *       blocked_ell_from_coo_cuda.cuh:604-966
 *   src/convert/compressed_transpose_raw.cuh:14-123
 *   src/bucket/major_nnz_raw.cuh:12-320, src/bucket/operators/major_nnz.cuh:11-213
 *   include/CellShard/runtime/mask_groups.cuh:14-224
 *   include/CellShard/io/csh5/api.cuh:316-436,726-733 (bucketed partitions),
 *       src/io/csh5/execution_builders_part.hh:1249-1272,1572-1596,
 *       src/bucket/operators/blocked_ell_bucket.cuh:11-210,
 *       include/CellShard/ingest/internal/dataset/internal/convert_layout_support_part.hh:143-181
 * Not mirrored (out of this library's scope): the fleet (multi-GPU) entry
 * points, sharded<T> host containers and their shard-level staging, COO
 * staging and the DIA format.
 */
#ifndef CELLSHARD_B200_HPP_
#define CELLSHARD_B200_HPP_

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cellshard_b200.h"

namespace cellshard {

namespace types {
using dim_t = unsigned int;
using nnz_t = unsigned int;
using idx_t = unsigned int;
using ptr_t = unsigned int;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
} // namespace types

namespace real {
using storage_t = __half;
} // namespace real

// ---------------------------------------------------------------------------
// sparse:: host formats
// ---------------------------------------------------------------------------
namespace sparse {

enum : types::u32 { compressed_by_row = 0u, compressed_by_col = 1u };
enum : types::u32 { blocked_ell_invalid_col = 0xffffffffu, sliced_ell_invalid_col = 0xffffffffu };

struct alignas(16) compressed {
    types::dim_t rows;
    types::dim_t cols;
    types::nnz_t nnz;
    types::u32 axis;
    types::u32 flags;
    void *storage;
    types::ptr_t *majorPtr;
    types::idx_t *minorIdx;
    real::storage_t *val;
};

struct alignas(16) blocked_ell {
    types::dim_t rows;
    types::dim_t cols;
    types::nnz_t nnz;
    types::u32 block_size;
    types::u32 ell_cols;
    types::u32 flags;
    void *storage;
    types::idx_t *blockColIdx;
    real::storage_t *val;
};

struct alignas(16) sliced_ell {
    types::dim_t rows;
    types::dim_t cols;
    types::nnz_t nnz;
    types::u32 slice_count;
    types::u32 flags;
    void *storage;
    types::u32 *slice_row_offsets;
    types::u32 *slice_widths;
    types::idx_t *col_idx;
    real::storage_t *val;
};

// formats/triplet.cuh:14-25
struct alignas(16) coo {
    types::dim_t rows;
    types::dim_t cols;
    types::nnz_t nnz;
    void *storage;
    types::idx_t *rowIdx;
    types::idx_t *colIdx;
    real::storage_t *val;
};

static_assert(sizeof(coo) == sizeof(cs_host_coo) && offsetof(coo, val) == offsetof(cs_host_coo, val),
              "sparse::coo layout");
static_assert(sizeof(compressed) == sizeof(cs_host_compressed) &&
                  offsetof(compressed, val) == offsetof(cs_host_compressed, val),
              "sparse::compressed layout");
static_assert(sizeof(blocked_ell) == sizeof(cs_host_blocked_ell) &&
                  offsetof(blocked_ell, val) == offsetof(cs_host_blocked_ell, val),
              "sparse::blocked_ell layout");
static_assert(sizeof(sliced_ell) == sizeof(cs_host_sliced_ell) &&
                  offsetof(sliced_ell, val) == offsetof(cs_host_sliced_ell, val),
              "sparse::sliced_ell layout");

inline void init(compressed *m) { std::memset(m, 0, sizeof(*m)); }
inline void init(blocked_ell *m) { std::memset(m, 0, sizeof(*m)); }
inline void init(sliced_ell *m) { std::memset(m, 0, sizeof(*m)); }
// Results written by this library own one packed malloc'd block in `storage`.
inline void clear(compressed *m) { cs_b200_host_compressed_clear(reinterpret_cast<cs_host_compressed *>(m)); }
inline void clear(blocked_ell *m) { cs_b200_host_blocked_ell_clear(reinterpret_cast<cs_host_blocked_ell *>(m)); }
inline void clear(sliced_ell *m) { cs_b200_host_sliced_ell_clear(reinterpret_cast<cs_host_sliced_ell *>(m)); }

} // namespace sparse

// ---------------------------------------------------------------------------
// device:: views and single-partition staging
// ---------------------------------------------------------------------------
namespace device {

struct alignas(16) compressed_view {
    unsigned int rows, cols, nnz, axis;
    unsigned int *majorPtr;
    unsigned int *minorIdx;
    __half *val;
};

struct alignas(16) blocked_ell_view {
    unsigned int rows, cols, nnz, block_size, ell_cols;
    unsigned int *blockColIdx;
    __half *val;
};

struct alignas(16) sliced_ell_view {
    unsigned int rows, cols, nnz, slice_count, slice_rows;
    unsigned int *slice_row_offsets;
    unsigned int *slice_widths;
    unsigned int *slice_slot_offsets;
    unsigned int *col_idx;
    __half *val;
};

static_assert(sizeof(compressed_view) == sizeof(cs_compressed_view), "compressed_view layout");
static_assert(sizeof(blocked_ell_view) == sizeof(cs_blocked_ell_view), "blocked_ell_view layout");
static_assert(sizeof(sliced_ell_view) == sizeof(cs_sliced_ell_view), "sliced_ell_view layout");

// device::partition_record<MatrixT> (sharded_device.cuh:22-35): field for
// field the reference's record, the same for every MatrixT.  `view` is the
// device address of the partition's view; a0..a3 its device arrays
// (compressed: majorPtr, minorIdx, val; Blocked-ELL: blockColIdx, val;
// Sliced-ELL: slice_row_offsets, slice_widths, col_idx, val, with the u32
// slot offsets at a1 + round_up(4 * slice_count, 256)).
template <typename MatrixT>
struct alignas(16) partition_record {
    void *allocation;
    std::size_t allocation_bytes;
    void *storage;
    void *view;
    void *a0;
    void *a1;
    void *a2;
    void *a3;
    unsigned long group_begin;
    unsigned long group_end;
    int device_id;
};

// sharded_device.cuh:37-41
struct cached_allocation {
    void *ptr;
    std::size_t bytes;
    int device_id;
};

// sharded_device.cuh:44-51: the residency table of a sharded matrix
template <typename MatrixT>
struct sharded_device {
    unsigned long capacity;
    partition_record<MatrixT> *parts;
    unsigned long cache_count;
    unsigned long cache_capacity;
    cached_allocation *cache;
};

static_assert(sizeof(partition_record<sparse::compressed>) == sizeof(cs_staged_part) &&
                  offsetof(partition_record<sparse::compressed>, device_id) == offsetof(cs_staged_part, device_id) &&
                  offsetof(partition_record<sparse::compressed>, group_begin) ==
                      offsetof(cs_staged_part, group_begin),
              "partition_record layout");
static_assert(sizeof(cached_allocation) == sizeof(cs_cached_allocation), "cached_allocation layout");
static_assert(sizeof(sharded_device<sparse::compressed>) == sizeof(cs_sharded_device) &&
                  offsetof(sharded_device<sparse::compressed>, cache) == offsetof(cs_sharded_device, cache),
              "sharded_device layout");

namespace detail {
inline cudaError_t staged(int ok) {
    if (ok) return cudaSuccess;
    const cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : cudaErrorInvalidValue;
}
template <typename MatrixT>
inline cs_sharded_device *as_state(sharded_device<MatrixT> *s) {
    return reinterpret_cast<cs_sharded_device *>(s);
}
inline const cs_host_compressed *host(const sparse::compressed *m) {
    return reinterpret_cast<const cs_host_compressed *>(m);
}
inline const cs_host_blocked_ell *host(const sparse::blocked_ell *m) {
    return reinterpret_cast<const cs_host_blocked_ell *>(m);
}
inline const cs_host_sliced_ell *host(const sparse::sliced_ell *m) {
    return reinterpret_cast<const cs_host_sliced_ell *>(m);
}
inline int stage_one(cs_sharded_device *st, unsigned long part, const sparse::compressed *m, int dev,
                     cudaStream_t s) {
    return cs_b200_stage_partition_compressed(st, part, host(m), dev, reinterpret_cast<cs_stream_t>(s));
}
inline int stage_one(cs_sharded_device *st, unsigned long part, const sparse::blocked_ell *m, int dev,
                     cudaStream_t s) {
    return cs_b200_stage_partition_blocked_ell(st, part, host(m), dev, reinterpret_cast<cs_stream_t>(s));
}
inline int stage_one(cs_sharded_device *st, unsigned long part, const sparse::sliced_ell *m, int dev,
                     cudaStream_t s) {
    return cs_b200_stage_partition_sliced_ell(st, part, host(m), dev, reinterpret_cast<cs_stream_t>(s));
}
inline int stage_many(cs_sharded_device *st, unsigned long first, unsigned long n, sparse::compressed *const *m,
                      int dev, cudaStream_t s) {
    return cs_b200_stage_shard_compressed(st, first, n, reinterpret_cast<const cs_host_compressed *const *>(m), dev,
                                          reinterpret_cast<cs_stream_t>(s));
}
inline int stage_many(cs_sharded_device *st, unsigned long first, unsigned long n, sparse::blocked_ell *const *m,
                      int dev, cudaStream_t s) {
    return cs_b200_stage_shard_blocked_ell(st, first, n, reinterpret_cast<const cs_host_blocked_ell *const *>(m),
                                           dev, reinterpret_cast<cs_stream_t>(s));
}
inline int stage_many(cs_sharded_device *st, unsigned long first, unsigned long n, sparse::sliced_ell *const *m,
                      int dev, cudaStream_t s) {
    return cs_b200_stage_shard_sliced_ell(st, first, n, reinterpret_cast<const cs_host_sliced_ell *const *>(m), dev,
                                          reinterpret_cast<cs_stream_t>(s));
}
} // namespace detail

inline std::size_t device_partition_bytes(const sparse::compressed *src) {
    size_t n = 0;
    return cs_b200_device_partition_bytes_compressed(reinterpret_cast<const cs_host_compressed *>(src), &n) ? n : 0;
}
inline std::size_t device_partition_bytes(const sparse::blocked_ell *src) {
    size_t n = 0;
    return cs_b200_device_partition_bytes_blocked_ell(reinterpret_cast<const cs_host_blocked_ell *>(src), &n) ? n
                                                                                                               : 0;
}
inline std::size_t device_partition_bytes(const sparse::sliced_ell *src) {
    size_t n = 0;
    return cs_b200_device_partition_bytes_sliced_ell(reinterpret_cast<const cs_host_sliced_ell *>(src), &n) ? n : 0;
}

template <typename MatrixT>
inline void zero_record(partition_record<MatrixT> *record) {
    std::memset(record, 0, sizeof(*record));
    record->device_id = -1;
}

// device::upload_async (sharded_device.cuh:400-756): one packed block on the
// current device holding the view and the arrays; stream-ordered, no sync.
// The record stands alone (empty group range), as the reference's upload
// leaves it; release() frees it.
template <typename MatrixT>
inline cudaError_t upload_async(const MatrixT *src, partition_record<MatrixT> *record, cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    zero_record(record);
    cs_sharded_device one{1ul, reinterpret_cast<cs_staged_part *>(record), 0ul, 0ul, nullptr};
    if (!detail::stage_one(&one, 0ul, src, dev, stream)) return detail::staged(0);
    record->group_begin = record->group_end = 0ul;
    return cudaSuccess;
}
// device::upload: the same, then the stream is synchronised.
template <typename MatrixT>
inline cudaError_t upload(const MatrixT *src, partition_record<MatrixT> *record) {
    cudaError_t e = upload_async(src, record, (cudaStream_t) 0);
    return e != cudaSuccess ? e : cudaStreamSynchronize((cudaStream_t) 0);
}
// device::release (sharded_device.cuh:959-991): frees a standalone record.
template <typename MatrixT>
inline cudaError_t release(partition_record<MatrixT> *record) {
    cs_sharded_device one{1ul, reinterpret_cast<cs_staged_part *>(record), 0ul, 0ul, nullptr};
    record->group_begin = record->group_end = 0ul;
    return detail::staged(cs_b200_release_staged_partition(&one, 0ul));
}

// Host copy of a staged partition's device view, from its host part's
// metadata and the record's arrays (what reference callers assemble by hand
// from a0..a3, e.g. src/convert/sliced_ell_from_compressed.cuh:204-224).
inline compressed_view staged_view(const sparse::compressed *m, const partition_record<sparse::compressed> *r) {
    compressed_view v;
    v.rows = m->rows;
    v.cols = m->cols;
    v.nnz = m->nnz;
    v.axis = m->axis;
    v.majorPtr = static_cast<unsigned int *>(r->a0);
    v.minorIdx = static_cast<unsigned int *>(r->a1);
    v.val = static_cast<__half *>(r->a2);
    return v;
}
inline blocked_ell_view staged_view(const sparse::blocked_ell *m, const partition_record<sparse::blocked_ell> *r) {
    blocked_ell_view v;
    v.rows = m->rows;
    v.cols = m->cols;
    v.nnz = m->nnz;
    v.block_size = m->block_size;
    v.ell_cols = m->ell_cols;
    v.blockColIdx = static_cast<unsigned int *>(r->a0);
    v.val = static_cast<__half *>(r->a1);
    return v;
}
inline sliced_ell_view staged_view(const sparse::sliced_ell *m, const partition_record<sparse::sliced_ell> *r) {
    sliced_ell_view v;
    v.rows = m->rows;
    v.cols = m->cols;
    v.nnz = m->nnz;
    v.slice_count = m->slice_count;
    v.slice_rows = m->slice_count ? m->slice_row_offsets[1] - m->slice_row_offsets[0] : 0u;
    v.slice_row_offsets = static_cast<unsigned int *>(r->a0);
    v.slice_widths = static_cast<unsigned int *>(r->a1);
    v.slice_slot_offsets = reinterpret_cast<unsigned int *>(static_cast<char *>(r->a1) +
                                                           (((std::size_t) m->slice_count * 4u + 255u) / 256u) * 256u);
    v.col_idx = static_cast<unsigned int *>(r->a2);
    v.val = static_cast<__half *>(r->a3);
    return v;
}

} // namespace device

// ---------------------------------------------------------------------------
// sharded<MatrixT>: the metadata-only stitched matrix (runtime/layout/sharded.cuh
// :29-50, 52-362) and its host helpers (runtime/host/sharded_host.cuh:15-395,
// 528-560).  parts[i] may be null (not materialised on the host);
// partition_rows / partition_nnz / partition_aux stay valid as metadata;
// shard_offsets group whole partitions into shards; shard_parts[s] is the
// first partition of shard s.  The cut rules of the re-sharding helpers are
// the reference's, so the same partitions give the same shards.
// ---------------------------------------------------------------------------
template <typename MatrixT>
struct alignas(16) sharded {
    unsigned long rows;
    unsigned long cols;
    unsigned long nnz;
    unsigned long num_partitions;
    unsigned long partition_capacity;
    MatrixT **parts;
    unsigned long *partition_offsets;
    unsigned long *partition_rows;
    unsigned long *partition_nnz;
    unsigned long *partition_aux;
    unsigned long num_shards;
    unsigned long shard_capacity;
    unsigned long *shard_offsets;
    unsigned long *shard_parts;
};

// runtime/storage/shard_storage.cuh:33-41.  The only backend the reference
// fetches partitions from is its `.csh5` (HDF5) dataset, which this library
// does not read: parts must be materialised on the host before they are
// staged, and fetch_partition / fetch_shard report failure with a message.
struct shard_storage;
typedef int (*shard_storage_open_fn)(shard_storage *s);
typedef void (*shard_storage_close_fn)(shard_storage *s);
enum { shard_storage_backend_none = 0, shard_storage_backend_dataset_h5 = 1 };
struct shard_storage {
    unsigned int backend;
    std::uint32_t role;
    std::uint32_t capability_flags;
    char *source_path;
    void *backend_state;
    shard_storage_open_fn open_backend;
    shard_storage_close_fn close_backend;
};
inline void init(shard_storage *s) { std::memset(s, 0, sizeof(*s)); }
inline void clear(shard_storage *s) {
    if (s->close_backend != nullptr) s->close_backend(s);
    std::free(s->source_path);
    std::memset(s, 0, sizeof(*s));
}

namespace sparse {
// formats/blocked_ell.cuh:43-57, sliced_ell.cuh:30-40
inline unsigned long pack_blocked_ell_aux(types::u32 block_size, unsigned long ell_width) {
    return (ell_width << 16u) | (unsigned long) block_size;
}
inline types::u32 unpack_blocked_ell_block_size(unsigned long aux) { return (types::u32) (aux & 0xfffful); }
inline unsigned long unpack_blocked_ell_ell_width(unsigned long aux) { return aux >> 16u; }
inline unsigned long pack_sliced_ell_aux(types::u32 slice_count, types::u32 total_slots) {
    return ((unsigned long) total_slots << 32u) | (unsigned long) slice_count;
}
inline types::u32 unpack_sliced_ell_slice_count(unsigned long aux) { return (types::u32) (aux & 0xfffffffful); }
inline types::u32 unpack_sliced_ell_total_slots(unsigned long aux) { return (types::u32) (aux >> 32u); }
inline types::u32 total_slots(const sliced_ell *m) {
    types::u32 t = 0u;
    for (types::u32 s = 0; s < m->slice_count; ++s)
        t += (m->slice_row_offsets[s + 1u] - m->slice_row_offsets[s]) * m->slice_widths[s];
    return t;
}
} // namespace sparse

template <typename MatrixT>
inline void init(sharded<MatrixT> *m) {
    std::memset(m, 0, sizeof(*m));
}

inline unsigned long partition_nnz(const sparse::compressed *m) { return m->nnz; }
inline unsigned long partition_nnz(const sparse::blocked_ell *m) { return m->nnz; }
inline unsigned long partition_nnz(const sparse::sliced_ell *m) { return m->nnz; }
inline unsigned long partition_aux(const sparse::compressed *m) { return m->axis; }
inline unsigned long partition_aux(const sparse::blocked_ell *m) {
    return sparse::pack_blocked_ell_aux(m->block_size, m->block_size ? m->ell_cols / m->block_size : 0u);
}
inline unsigned long partition_aux(const sparse::sliced_ell *m) {
    return sparse::pack_sliced_ell_aux(m->slice_count, sparse::total_slots(m));
}

// destroy(): the part's packed storage, then the part itself (parts are new'ed)
template <typename MatrixT>
inline void destroy(MatrixT *m) {
    if (m == nullptr) return;
    sparse::clear(m);
    delete m;
}

template <typename MatrixT>
inline void clear(sharded<MatrixT> *m) {
    for (unsigned long i = 0; m->parts != nullptr && i < m->num_partitions; ++i) destroy(m->parts[i]);
    std::free(m->parts);
    std::free(m->partition_offsets);
    std::free(m->partition_rows);
    std::free(m->partition_nnz);
    std::free(m->partition_aux);
    std::free(m->shard_offsets);
    std::free(m->shard_parts);
    init(m);
}

template <typename MatrixT>
inline int reserve_partitions(sharded<MatrixT> *m, unsigned long capacity) {
    if (capacity <= m->partition_capacity) return 1;
    auto *parts = static_cast<MatrixT **>(std::calloc(capacity, sizeof(MatrixT *)));
    auto *offs = static_cast<unsigned long *>(std::calloc(capacity + 1u, sizeof(unsigned long)));
    auto *rows = static_cast<unsigned long *>(std::calloc(capacity, sizeof(unsigned long)));
    auto *nnz = static_cast<unsigned long *>(std::calloc(capacity, sizeof(unsigned long)));
    auto *aux = static_cast<unsigned long *>(std::calloc(capacity, sizeof(unsigned long)));
    if (!parts || !offs || !rows || !nnz || !aux) {
        std::free(parts);
        std::free(offs);
        std::free(rows);
        std::free(nnz);
        std::free(aux);
        return 0;
    }
    const unsigned long n = m->num_partitions;
    if (n != 0u) {
        std::memcpy(parts, m->parts, n * sizeof(MatrixT *));
        std::memcpy(offs, m->partition_offsets, (n + 1u) * sizeof(unsigned long));
        std::memcpy(rows, m->partition_rows, n * sizeof(unsigned long));
        std::memcpy(nnz, m->partition_nnz, n * sizeof(unsigned long));
        std::memcpy(aux, m->partition_aux, n * sizeof(unsigned long));
    }
    std::free(m->parts);
    std::free(m->partition_offsets);
    std::free(m->partition_rows);
    std::free(m->partition_nnz);
    std::free(m->partition_aux);
    m->parts = parts;
    m->partition_offsets = offs;
    m->partition_rows = rows;
    m->partition_nnz = nnz;
    m->partition_aux = aux;
    m->partition_capacity = capacity;
    return 1;
}

template <typename MatrixT>
inline int reserve_shards(sharded<MatrixT> *m, unsigned long capacity) {
    if (capacity <= m->shard_capacity) return 1;
    auto *offs = static_cast<unsigned long *>(std::calloc(capacity + 1u, sizeof(unsigned long)));
    auto *sp = static_cast<unsigned long *>(std::calloc(capacity + 1u, sizeof(unsigned long)));
    if (!offs || !sp) {
        std::free(offs);
        std::free(sp);
        return 0;
    }
    if (m->shard_offsets != nullptr && m->num_shards != 0u) {
        std::memcpy(offs, m->shard_offsets, (m->num_shards + 1u) * sizeof(unsigned long));
        if (m->shard_parts != nullptr) std::memcpy(sp, m->shard_parts, (m->num_shards + 1u) * sizeof(unsigned long));
    }
    std::free(m->shard_offsets);
    std::free(m->shard_parts);
    m->shard_offsets = offs;
    m->shard_parts = sp;
    m->shard_capacity = capacity;
    return 1;
}

// shard s starts at the first partition whose first row is >= its first row
template <typename MatrixT>
inline void rebuild_shard_parts(sharded<MatrixT> *m) {
    if (!m->shard_parts || !m->shard_offsets || !m->partition_offsets) return;
    unsigned long part = 0;
    for (unsigned long s = 0; s < m->num_shards; ++s) {
        while (part < m->num_partitions && m->partition_offsets[part] < m->shard_offsets[s]) ++part;
        m->shard_parts[s] = part;
    }
    m->shard_parts[m->num_shards] = m->num_partitions;
}

template <typename MatrixT>
inline void rebuild_partition_offsets(sharded<MatrixT> *m) {
    m->rows = 0;
    m->nnz = 0;
    if (!m->partition_offsets) return;
    m->partition_offsets[0] = 0;
    for (unsigned long i = 0; i < m->num_partitions; ++i) {
        m->partition_offsets[i + 1u] = m->partition_offsets[i] + m->partition_rows[i];
        m->nnz += m->partition_nnz[i];
    }
    m->rows = m->partition_offsets[m->num_partitions];
}

template <typename MatrixT>
inline int set_shards_to_partitions(sharded<MatrixT> *m) {
    if (!reserve_shards(m, m->num_partitions)) return 0;
    m->num_shards = m->num_partitions;
    for (unsigned long i = 0; i <= m->num_partitions; ++i) {
        m->shard_offsets[i] = m->partition_offsets ? m->partition_offsets[i] : 0u;
        m->shard_parts[i] = i;
    }
    return 1;
}

// metadata-only partitions (parts left null): sharded_host.cuh:145-168
template <typename MatrixT>
inline int define_partitions(sharded<MatrixT> *m, unsigned long cols, unsigned long num_partitions,
                             const unsigned long *partition_rows, const unsigned long *partition_nnz,
                             const unsigned long *partition_aux_in) {
    clear(m);
    if (!reserve_partitions(m, num_partitions)) return 0;
    m->cols = cols;
    m->num_partitions = num_partitions;
    for (unsigned long i = 0; i < num_partitions; ++i) {
        m->parts[i] = nullptr;
        m->partition_rows[i] = partition_rows ? partition_rows[i] : 0u;
        m->partition_nnz[i] = partition_nnz ? partition_nnz[i] : 0u;
        m->partition_aux[i] = partition_aux_in ? partition_aux_in[i] : 0u;
    }
    rebuild_partition_offsets(m);
    return set_shards_to_partitions(m);
}

// takes ownership of `part` (not copied); one shard per partition afterwards
template <typename MatrixT>
inline int append_partition(sharded<MatrixT> *m, MatrixT *part) {
    if (m->num_partitions == m->partition_capacity &&
        !reserve_partitions(m, m->partition_capacity == 0u ? 4u : m->partition_capacity * 2u))
        return 0;
    const unsigned long i = m->num_partitions;
    m->parts[i] = part;
    m->partition_rows[i] = part ? part->rows : 0u;
    m->partition_nnz[i] = part ? partition_nnz(part) : 0u;
    m->partition_aux[i] = part ? partition_aux(part) : 0u;
    ++m->num_partitions;
    if (part && m->cols == 0u) m->cols = part->cols;
    rebuild_partition_offsets(m);
    return set_shards_to_partitions(m);
}

// moves every partition of src to the end of dst (pointers, not payloads)
template <typename MatrixT>
inline int concatenate(sharded<MatrixT> *dst, sharded<MatrixT> *src) {
    if (src->num_partitions == 0u) return 1;
    if (!reserve_partitions(dst, dst->num_partitions + src->num_partitions)) return 0;
    for (unsigned long i = 0; i < src->num_partitions; ++i) {
        const unsigned long d = dst->num_partitions + i;
        dst->parts[d] = src->parts[i];
        dst->partition_rows[d] = src->partition_rows[i];
        dst->partition_nnz[d] = src->partition_nnz[i];
        dst->partition_aux[d] = src->partition_aux[i];
        src->parts[i] = nullptr;
        src->partition_rows[i] = src->partition_nnz[i] = src->partition_aux[i] = 0u;
    }
    dst->num_partitions += src->num_partitions;
    src->num_partitions = 0;
    if (dst->cols == 0u) dst->cols = src->cols;
    rebuild_partition_offsets(dst);
    set_shards_to_partitions(dst);
    rebuild_partition_offsets(src);
    src->rows = src->nnz = src->num_shards = 0u;
    if (src->shard_parts) src->shard_parts[0] = 0u;
    return 1;
}

template <typename MatrixT>
inline unsigned long find_partition(const sharded<MatrixT> *m, unsigned long row) {
    if (!m->partition_offsets || m->num_partitions == 0u) return m->num_partitions;
    unsigned long lo = 0, hi = m->num_partitions;
    while (lo < hi) {
        const unsigned long mid = lo + (hi - lo) / 2u;
        if (row < m->partition_offsets[mid]) hi = mid;
        else if (row >= m->partition_offsets[mid + 1u]) lo = mid + 1u;
        else return mid;
    }
    return m->num_partitions;
}

template <typename MatrixT>
inline unsigned long find_shard(const sharded<MatrixT> *m, unsigned long row) {
    if (!m->shard_offsets || m->num_shards == 0u) return m->num_shards;
    unsigned long lo = 0, hi = m->num_shards;
    while (lo < hi) {
        const unsigned long mid = lo + (hi - lo) / 2u;
        if (row < m->shard_offsets[mid]) hi = mid;
        else if (row >= m->shard_offsets[mid + 1u]) lo = mid + 1u;
        else return mid;
    }
    return m->num_shards;
}

template <typename MatrixT>
inline unsigned long first_row_in_partition(const sharded<MatrixT> *m, unsigned long p) {
    return (p >= m->num_partitions || !m->partition_offsets) ? m->rows : m->partition_offsets[p];
}
template <typename MatrixT>
inline unsigned long last_row_in_partition(const sharded<MatrixT> *m, unsigned long p) {
    return (p >= m->num_partitions || !m->partition_offsets) ? m->rows : m->partition_offsets[p + 1u];
}

template <typename MatrixT>
inline int row_is_partition_boundary(const sharded<MatrixT> *m, unsigned long row) {
    if (row == 0u || row == m->rows) return 1;
    if (!m->partition_offsets || m->num_partitions == 0u) return 0;
    const unsigned long hit = find_partition(m, row);
    return hit < m->num_partitions && m->partition_offsets[hit] == row;
}

template <typename MatrixT>
inline unsigned long first_partition_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    if (m->shard_parts && s < m->num_shards) return m->shard_parts[s];
    if (s >= m->num_shards || m->num_partitions == 0u) return m->num_partitions;
    return find_partition(m, m->shard_offsets[s]);
}
template <typename MatrixT>
inline unsigned long last_partition_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    if (m->shard_parts && s < m->num_shards) return m->shard_parts[s + 1u];
    if (s >= m->num_shards) return m->num_partitions;
    const unsigned long end = m->shard_offsets[s + 1u];
    return end == 0u ? 0u : find_partition(m, end - 1u) + 1u;
}
template <typename MatrixT>
inline unsigned long first_row_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    return (s >= m->num_shards || !m->shard_offsets) ? m->rows : m->shard_offsets[s];
}
template <typename MatrixT>
inline unsigned long last_row_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    return (s >= m->num_shards || !m->shard_offsets) ? m->rows : m->shard_offsets[s + 1u];
}
template <typename MatrixT>
inline unsigned long partition_count_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    const unsigned long b = first_partition_in_shard(m, s), e = last_partition_in_shard(m, s);
    return b >= e ? 0u : e - b;
}
template <typename MatrixT>
inline unsigned long rows_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    const unsigned long b = first_row_in_shard(m, s), e = last_row_in_shard(m, s);
    return b >= e ? 0u : e - b;
}
template <typename MatrixT>
inline int partition_loaded(const sharded<MatrixT> *m, unsigned long p) {
    return p < m->num_partitions && m->parts[p] != nullptr;
}
template <typename MatrixT>
inline int shard_loaded(const sharded<MatrixT> *m, unsigned long s) {
    if (s >= m->num_shards) return 0;
    for (unsigned long i = first_partition_in_shard(m, s); i < last_partition_in_shard(m, s); ++i)
        if (!partition_loaded(m, i)) return 0;
    return 1;
}
template <typename MatrixT>
inline unsigned long nnz_in_shard(const sharded<MatrixT> *m, unsigned long s) {
    if (s >= m->num_shards) return 0;
    unsigned long t = 0;
    for (unsigned long i = first_partition_in_shard(m, s); i < last_partition_in_shard(m, s); ++i)
        t += m->partition_nnz[i];
    return t;
}

// host footprint of one partition (sharded.cuh:236-330): the packed host
// block when materialised, else rebuilt from the metadata
inline std::size_t partition_bytes(const sharded<sparse::compressed> *m, unsigned long p) {
    if (p >= m->num_partitions) return 0;
    const sparse::compressed *h = m->parts[p];
    const unsigned long ptr_dim = m->partition_aux[p] == sparse::compressed_by_col ? m->cols : m->partition_rows[p];
    if (h) {
        const std::size_t major = h->axis == sparse::compressed_by_col ? h->cols : h->rows;
        return sizeof(sparse::compressed) + (major + 1u) * 4u + (std::size_t) h->nnz * 6u;
    }
    return sizeof(sparse::compressed) + (ptr_dim + 1u) * 4u + (std::size_t) m->partition_nnz[p] * 6u;
}
inline std::size_t partition_bytes(const sharded<sparse::blocked_ell> *m, unsigned long p) {
    if (p >= m->num_partitions) return 0;
    const unsigned long aux = m->partition_aux[p];
    const std::size_t B = sparse::unpack_blocked_ell_block_size(aux), W = sparse::unpack_blocked_ell_ell_width(aux);
    const std::size_t rows = m->partition_rows[p];
    return sizeof(sparse::blocked_ell) + (B ? (rows + B - 1u) / B : 0u) * W * 4u + rows * W * B * 2u;
}
inline std::size_t partition_bytes(const sharded<sparse::sliced_ell> *m, unsigned long p) {
    if (p >= m->num_partitions) return 0;
    const unsigned long aux = m->partition_aux[p];
    const std::size_t S = sparse::unpack_sliced_ell_slice_count(aux), T = sparse::unpack_sliced_ell_total_slots(aux);
    return sizeof(sparse::sliced_ell) + (S + 1u) * 4u + S * 4u + T * 6u;
}
template <typename MatrixT>
inline std::size_t bytes(const sharded<MatrixT> *m) {
    std::size_t t = sizeof(*m) + m->partition_capacity * (sizeof(MatrixT *) + 4u * sizeof(unsigned long)) +
                    sizeof(unsigned long) + 2u * (m->shard_capacity + 1u) * sizeof(unsigned long);
    for (unsigned long i = 0; i < m->num_partitions; ++i) t += partition_bytes(m, i);
    return t;
}
template <typename MatrixT>
inline std::size_t shard_bytes(const sharded<MatrixT> *m, unsigned long s) {
    if (s >= m->num_shards) return 0;
    std::size_t t = 0;
    for (unsigned long i = first_partition_in_shard(m, s); i < last_partition_in_shard(m, s); ++i)
        t += partition_bytes(m, i);
    return t;
}

// sharded_host.cuh:232-268: about rows / count rows per shard, cutting only
// where enough partitions remain for the shards still to come
template <typename MatrixT>
inline int set_equal_shards(sharded<MatrixT> *m, unsigned long count) {
    if (count == 0u || m->num_partitions == 0u) {
        m->num_shards = 0;
        return 1;
    }
    if (count >= m->num_partitions) return set_shards_to_partitions(m);
    if (!reserve_shards(m, count)) return 0;
    const unsigned long target = (m->rows + count - 1u) / count;
    unsigned long n = 0, rows = 0;
    m->shard_offsets[0] = 0;
    for (unsigned long i = 0; i < m->num_partitions; ++i) {
        const unsigned long parts_left = m->num_partitions - (i + 1u), shards_left = count - (n + 1u);
        rows += m->partition_rows[i];
        if (shards_left == 0u) continue;
        if (rows >= target && parts_left >= shards_left) {
            m->shard_offsets[++n] = m->partition_offsets[i + 1u];
            rows = 0;
        }
    }
    m->shard_offsets[++n] = m->rows;
    m->num_shards = n;
    rebuild_shard_parts(m);
    return 1;
}

namespace detail {
// greedy cut: a new shard starts at partition i when the running total is
// non-zero and adding i's weight would pass `limit`; zero-weight partitions
// are skipped when `skip_zero` (sharded_host.cuh:335-395,
// sharded_device.cuh:1113-1142)
template <typename MatrixT, typename Weight>
inline int cut_shards(sharded<MatrixT> *m, std::size_t limit, bool skip_zero, Weight w) {
    if (limit == 0u) return set_shards_to_partitions(m);
    if (!reserve_shards(m, m->num_partitions)) return 0;
    std::size_t used = 0;
    unsigned long n = 0;
    m->shard_offsets[0] = 0;
    for (unsigned long i = 0; i < m->num_partitions; ++i) {
        const std::size_t b = w(i);
        if (skip_zero && b == 0u) continue;
        if (used != 0u && used + b > limit) {
            m->shard_offsets[++n] = m->partition_offsets[i];
            used = 0;
        }
        used += b;
    }
    if (m->num_partitions != 0u) m->shard_offsets[++n] = m->rows;
    m->num_shards = n;
    rebuild_shard_parts(m);
    return 1;
}
} // namespace detail

template <typename MatrixT>
inline int set_shards_by_nnz(sharded<MatrixT> *m, unsigned long max_nnz) {
    return detail::cut_shards(m, max_nnz, true, [m](unsigned long i) { return (std::size_t) m->partition_nnz[i]; });
}
template <typename MatrixT>
inline int set_shards_by_part_bytes(sharded<MatrixT> *m, std::size_t max_bytes) {
    return detail::cut_shards(m, max_bytes, true, [m](unsigned long i) { return partition_bytes(m, i); });
}

// shard offsets of about target rows each (sharded_host.cuh:270-311); the
// array is calloc'd for the caller
template <typename MatrixT>
inline int build_shard_offsets_by_rows(const sharded<MatrixT> *m, unsigned long target, unsigned long **out_offsets,
                                       unsigned long *out_count) {
    if (!out_offsets || !out_count) return 0;
    *out_offsets = nullptr;
    *out_count = 0;
    if (m->num_partitions == 0u) return 1;
    auto *o = static_cast<unsigned long *>(std::calloc(m->num_partitions + 1u, sizeof(unsigned long)));
    if (!o) return 0;
    unsigned long n = 0, used = 0;
    if (target == 0u) {
        for (unsigned long i = 0; i <= m->num_partitions; ++i) o[i] = m->partition_offsets[i];
        n = m->num_partitions;
    } else {
        for (unsigned long i = 0; i < m->num_partitions; ++i) {
            if (used != 0u && used + m->partition_rows[i] > target) {
                o[++n] = m->partition_offsets[i];
                used = 0;
            }
            used += m->partition_rows[i];
        }
        o[++n] = m->rows;
    }
    *out_offsets = o;
    *out_count = n;
    return 1;
}

// explicit shard offsets, each a partition boundary (sharded_host.cuh:313-332)
template <typename MatrixT>
inline int reshard(sharded<MatrixT> *m, unsigned long count, const unsigned long *offsets) {
    if (count == 0u || !offsets) {
        m->num_shards = 0;
        return 1;
    }
    if (offsets[0] != 0u || offsets[count] != m->rows) return 0;
    for (unsigned long i = 0; i < count; ++i)
        if (offsets[i] > offsets[i + 1u] || !row_is_partition_boundary(m, offsets[i])) return 0;
    if (!row_is_partition_boundary(m, offsets[count]) || !reserve_shards(m, count)) return 0;
    m->num_shards = count;
    for (unsigned long i = 0; i <= count; ++i) m->shard_offsets[i] = offsets[i];
    rebuild_shard_parts(m);
    return 1;
}

// host materialisation: drop frees a part (metadata stays); fetch needs a
// file backend this library does not have
template <typename MatrixT>
inline int drop_partition(sharded<MatrixT> *m, unsigned long p) {
    if (p >= m->num_partitions) return 0;
    destroy(m->parts[p]);
    m->parts[p] = nullptr;
    return 1;
}
template <typename MatrixT>
inline int drop_all_partitions(sharded<MatrixT> *m) {
    for (unsigned long i = 0; i < m->num_partitions; ++i)
        if (!drop_partition(m, i)) return 0;
    return 1;
}
template <typename MatrixT>
inline int drop_shard(sharded<MatrixT> *m, unsigned long s) {
    if (s >= m->num_shards) return 0;
    for (unsigned long i = first_partition_in_shard(m, s); i < last_partition_in_shard(m, s); ++i)
        if (!drop_partition(m, i)) return 0;
    return 1;
}
template <typename MatrixT>
inline int fetch_partition(sharded<MatrixT> *m, const shard_storage *, unsigned long p) {
    if (p < m->num_partitions && m->parts[p] != nullptr) return 1;
    std::fprintf(stderr,
                 "Error: partition %lu is not materialised on the host and file-backed (.csh5) fetch is not part "
                 "of this library\n",
                 p);
    return 0;
}
template <typename MatrixT>
inline int fetch_shard(sharded<MatrixT> *m, const shard_storage *s, unsigned long shard) {
    if (shard >= m->num_shards) return 0;
    for (unsigned long i = first_partition_in_shard(m, shard); i < last_partition_in_shard(m, shard); ++i)
        if (!fetch_partition(m, s, i)) return 0;
    return 1;
}

namespace device {

template <typename MatrixT>
inline void init(sharded_device<MatrixT> *state) {
    std::memset(state, 0, sizeof(*state));
}
// releases every resident partition and frees the cached blocks
template <typename MatrixT>
inline void clear(sharded_device<MatrixT> *state) {
    cs_b200_sharded_device_clear(detail::as_state(state));
}
template <typename MatrixT>
inline int reserve(sharded_device<MatrixT> *state, unsigned long capacity) {
    return cs_b200_sharded_device_reserve(detail::as_state(state), capacity);
}

template <typename MatrixT>
inline cudaError_t release_partition(sharded_device<MatrixT> *state, unsigned long part_id) {
    return detail::staged(cs_b200_release_staged_partition(detail::as_state(state), part_id));
}

// sharded_device.cuh:1144-1166: the host part must be materialised
template <typename MatrixT>
inline cudaError_t upload_partition_async(sharded_device<MatrixT> *state, const sharded<MatrixT> *view,
                                          unsigned long part_id, int device_id, cudaStream_t stream) {
    if (part_id >= view->num_partitions || part_id >= state->capacity || view->parts[part_id] == nullptr)
        return cudaErrorInvalidValue;
    return detail::staged(detail::stage_one(detail::as_state(state), part_id, view->parts[part_id], device_id,
                                            stream));
}
template <typename MatrixT>
inline cudaError_t upload_partition(sharded_device<MatrixT> *state, const sharded<MatrixT> *view,
                                    unsigned long part_id, int device_id) {
    cudaError_t e = upload_partition_async(state, view, part_id, device_id, (cudaStream_t) 0);
    return e != cudaSuccess ? e : cudaStreamSynchronize((cudaStream_t) 0);
}

// sharded_device.cuh:1437-1539: every partition of the shard in one packed
// block (all three formats)
template <typename MatrixT>
inline cudaError_t upload_shard_async(sharded_device<MatrixT> *state, const sharded<MatrixT> *view,
                                      unsigned long shard_id, int device_id, cudaStream_t stream) {
    if (shard_id >= view->num_shards) return cudaErrorInvalidValue;
    const unsigned long b = first_partition_in_shard(view, shard_id), e = last_partition_in_shard(view, shard_id);
    if (b >= e) return cudaSuccess;
    for (unsigned long i = b; i < e; ++i)
        if (i >= state->capacity || view->parts[i] == nullptr) return cudaErrorInvalidValue;
    return detail::staged(detail::stage_many(detail::as_state(state), b, e - b, view->parts + b, device_id, stream));
}
template <typename MatrixT>
inline cudaError_t upload_shard(sharded_device<MatrixT> *state, const sharded<MatrixT> *view, unsigned long shard_id,
                                int device_id) {
    cudaError_t e = upload_shard_async(state, view, shard_id, device_id, (cudaStream_t) 0);
    return e != cudaSuccess ? e : cudaStreamSynchronize((cudaStream_t) 0);
}

// sharded_device.cuh:1541-1559
template <typename MatrixT>
inline cudaError_t release_shard(sharded_device<MatrixT> *state, const sharded<MatrixT> *view,
                                 unsigned long shard_id) {
    if (shard_id >= view->num_shards) return cudaErrorInvalidValue;
    for (unsigned long i = first_partition_in_shard(view, shard_id); i < last_partition_in_shard(view, shard_id);
         ++i) {
        if (i >= state->capacity || state->parts[i].view == nullptr) continue;
        const cudaError_t e = release_partition(state, i);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// sharded_device.cuh:1569-1630: fetch when absent on the host (needs a
// file backend), upload, optionally drop the host part
template <typename MatrixT>
inline cudaError_t stage_partition_async(sharded_device<MatrixT> *state, sharded<MatrixT> *view,
                                         const shard_storage *files, unsigned long part_id, int device_id,
                                         cudaStream_t stream, int drop_host_after_upload) {
    if (part_id >= view->num_partitions || part_id >= state->capacity) return cudaErrorInvalidValue;
    if (state->parts[part_id].view != nullptr && state->parts[part_id].device_id == device_id) {
        if (drop_host_after_upload && view->parts[part_id] != nullptr && !drop_partition(view, part_id))
            return cudaErrorInvalidValue;
        return cudaSuccess;
    }
    if (view->parts[part_id] == nullptr && !fetch_partition(view, files, part_id)) return cudaErrorInvalidValue;
    cudaError_t e = upload_partition_async(state, view, part_id, device_id, stream);
    if (e != cudaSuccess) return e;
    if (drop_host_after_upload) {
        // the copies read the host part: wait for them before it is freed
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        if (!drop_partition(view, part_id)) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}
template <typename MatrixT>
inline cudaError_t stage_partition(sharded_device<MatrixT> *state, sharded<MatrixT> *view, const shard_storage *files,
                                   unsigned long part_id, int device_id, int drop_host_after_upload) {
    cudaError_t e = stage_partition_async(state, view, files, part_id, device_id, (cudaStream_t) 0,
                                          drop_host_after_upload);
    return e != cudaSuccess ? e : cudaStreamSynchronize((cudaStream_t) 0);
}

// sharded_device.cuh:1632-1677
template <typename MatrixT>
inline cudaError_t stage_shard_async(sharded_device<MatrixT> *state, sharded<MatrixT> *view,
                                     const shard_storage *files, unsigned long shard_id, int device_id,
                                     cudaStream_t stream, int drop_host_after_upload) {
    if (shard_id >= view->num_shards) return cudaErrorInvalidValue;
    if (!shard_loaded(view, shard_id) && !fetch_shard(view, files, shard_id)) return cudaErrorInvalidValue;
    cudaError_t e = upload_shard_async(state, view, shard_id, device_id, stream);
    if (e != cudaSuccess) return e;
    if (drop_host_after_upload) {
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        if (!drop_shard(view, shard_id)) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}
template <typename MatrixT>
inline cudaError_t stage_shard(sharded_device<MatrixT> *state, sharded<MatrixT> *view, const shard_storage *files,
                               unsigned long shard_id, int device_id, int drop_host_after_upload) {
    cudaError_t e = stage_shard_async(state, view, files, shard_id, device_id, (cudaStream_t) 0,
                                      drop_host_after_upload);
    return e != cudaSuccess ? e : cudaStreamSynchronize((cudaStream_t) 0);
}

// sharded_device.cuh:1679-1721: the incoming shard is staged before the
// outgoing one is released, so both are resident for a moment
template <typename MatrixT>
inline cudaError_t swap_shard_async(sharded_device<MatrixT> *state, sharded<MatrixT> *view, const shard_storage *files,
                                    unsigned long out_shard, unsigned long in_shard, int device_id, cudaStream_t stream,
                                    int drop_host_after_upload, int drop_host_after_release) {
    cudaError_t e = stage_shard_async(state, view, files, in_shard, device_id, stream, drop_host_after_upload);
    if (e != cudaSuccess) return e;
    e = release_shard(state, view, out_shard);
    if (e != cudaSuccess) return e;
    if (drop_host_after_release && !drop_shard(view, out_shard)) return cudaErrorInvalidValue;
    return cudaSuccess;
}
template <typename MatrixT>
inline cudaError_t swap_shard(sharded_device<MatrixT> *state, sharded<MatrixT> *view, const shard_storage *files,
                              unsigned long out_shard, unsigned long in_shard, int device_id,
                              int drop_host_after_upload, int drop_host_after_release) {
    cudaError_t e = swap_shard_async(state, view, files, out_shard, in_shard, device_id, (cudaStream_t) 0,
                                     drop_host_after_upload, drop_host_after_release);
    return e != cudaSuccess ? e : cudaStreamSynchronize((cudaStream_t) 0);
}

// Resident device bytes of one partition after upload_partition, from the
// metadata alone (sharded_device.cuh:1050-1095): the view's 256 bytes, then
// each array rounded up to 256 bytes (this library's layout).
namespace detail {
inline std::size_t r256(std::size_t x) { return (x + 255u) / 256u * 256u; }
} // namespace detail
inline std::size_t device_partition_bytes(const sharded<sparse::compressed> *view, unsigned long p) {
    const std::size_t ptr_dim =
        view->partition_aux[p] == sparse::compressed_by_col ? view->cols : view->partition_rows[p];
    const std::size_t nnz = view->partition_nnz[p];
    return 256u + detail::r256((ptr_dim + 1u) * 4u) + detail::r256(nnz * 4u) + detail::r256(nnz * 2u);
}
inline std::size_t device_partition_bytes(const sharded<sparse::blocked_ell> *view, unsigned long p) {
    const unsigned long aux = view->partition_aux[p];
    const std::size_t B = sparse::unpack_blocked_ell_block_size(aux), W = sparse::unpack_blocked_ell_ell_width(aux);
    const std::size_t rows = view->partition_rows[p];
    return 256u + detail::r256((B ? (rows + B - 1u) / B : 0u) * W * 4u) + detail::r256(rows * W * B * 2u);
}
inline std::size_t device_partition_bytes(const sharded<sparse::sliced_ell> *view, unsigned long p) {
    const unsigned long aux = view->partition_aux[p];
    const std::size_t S = sparse::unpack_sliced_ell_slice_count(aux), T = sparse::unpack_sliced_ell_total_slots(aux);
    return 256u + detail::r256(S ? (S + 1u) * 4u : 0u) + 2u * detail::r256(S * 4u) + detail::r256(T * 4u) +
           detail::r256(T * 2u);
}
template <typename MatrixT>
inline std::size_t device_shard_bytes(const sharded<MatrixT> *view, unsigned long shard_id) {
    if (shard_id >= view->num_shards) return 0;
    std::size_t t = 0;
    for (unsigned long i = first_partition_in_shard(view, shard_id); i < last_partition_in_shard(view, shard_id); ++i)
        t += device_partition_bytes(view, i);
    return t;
}
// sharded_device.cuh:1113-1142: shards cut so each fits max_bytes of device memory
template <typename MatrixT>
inline int set_shards_by_device_bytes(sharded<MatrixT> *view, std::size_t max_bytes) {
    return ::cellshard::detail::cut_shards(view, max_bytes, true,
                                           [view](unsigned long i) { return device_partition_bytes(view, i); });
}

} // namespace device

// ---------------------------------------------------------------------------
// convert::
// ---------------------------------------------------------------------------
namespace convert {

struct blocked_ell_tune_result {
    unsigned int block_size;
    double fill_ratio;
    std::size_t padded_bytes;
};

struct sliced_ell_tune_result {
    unsigned int slice_rows;
    unsigned int slice_count;
    std::size_t padded_slots;
    std::size_t padded_bytes;
    double storage_ratio;
    double slice_penalty;
    double score;
};

static_assert(sizeof(blocked_ell_tune_result) == sizeof(cs_blocked_ell_tune_result), "tune layout");
static_assert(sizeof(sliced_ell_tune_result) == sizeof(cs_sliced_ell_tune_result), "tune layout");

inline int blocked_ell_from_compressed(const sparse::compressed *src, unsigned int block_size,
                                       sparse::blocked_ell *dst) {
    return cs_b200_blocked_ell_from_compressed(reinterpret_cast<const cs_host_compressed *>(src), block_size,
                                               reinterpret_cast<cs_host_blocked_ell *>(dst));
}

inline int choose_blocked_ell_block_size(const sparse::compressed *src, const unsigned int *candidates,
                                         unsigned int candidate_count, blocked_ell_tune_result *out) {
    return cs_b200_choose_blocked_ell_block_size(reinterpret_cast<const cs_host_compressed *>(src), candidates,
                                                 candidate_count, reinterpret_cast<cs_blocked_ell_tune_result *>(out));
}

// COO -> Blocked-ELL (blocked_ell_from_compressed.cuh:192-257,349-478;
// blocked_ell_from_coo_cuda.cuh:604-966).  The _cuda forms take the device
// ordinal; workspaces and streams of the reference's _cuda signatures are
// replaced by the library's own.
inline int blocked_ell_from_coo(const sparse::coo *src, types::dim_t cols, const types::u32 *feature_to_global,
                                unsigned int block_size, sparse::blocked_ell *dst) {
    return cs_b200_blocked_ell_from_coo(reinterpret_cast<const cs_host_coo *>(src), cols, feature_to_global,
                                        block_size, reinterpret_cast<cs_host_blocked_ell *>(dst));
}

inline int blocked_ell_from_coo_cuda(const sparse::coo *src, types::dim_t cols, const types::u32 *feature_to_global,
                                     unsigned int block_size, sparse::blocked_ell *dst, int device) {
    return cs_b200_blocked_ell_from_coo_cuda(reinterpret_cast<const cs_host_coo *>(src), cols, feature_to_global,
                                             block_size, reinterpret_cast<cs_host_blocked_ell *>(dst), device);
}

inline int choose_blocked_ell_block_size_from_coo(const sparse::coo *src, types::dim_t cols,
                                                  const types::u32 *feature_to_global, const unsigned int *candidates,
                                                  unsigned int candidate_count, blocked_ell_tune_result *out) {
    return cs_b200_choose_blocked_ell_block_size_from_coo(reinterpret_cast<const cs_host_coo *>(src), cols,
                                                          feature_to_global, candidates, candidate_count,
                                                          reinterpret_cast<cs_blocked_ell_tune_result *>(out));
}

inline int choose_blocked_ell_block_size_from_coo_cuda(const sparse::coo *src, types::dim_t cols,
                                                       const types::u32 *feature_to_global,
                                                       const unsigned int *candidates, unsigned int candidate_count,
                                                       int device, blocked_ell_tune_result *out) {
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    return choose_blocked_ell_block_size_from_coo(src, cols, feature_to_global, candidates, candidate_count, out);
}

inline int blocked_ell_from_coo_auto(const sparse::coo *src, types::dim_t cols, const types::u32 *feature_to_global,
                                     const unsigned int *candidates, unsigned int candidate_count,
                                     sparse::blocked_ell *dst, blocked_ell_tune_result *picked = nullptr) {
    blocked_ell_tune_result t{};
    if (!choose_blocked_ell_block_size_from_coo(src, cols, feature_to_global, candidates, candidate_count, &t) ||
        !blocked_ell_from_coo(src, cols, feature_to_global, t.block_size, dst))
        return 0;
    if (picked != nullptr) *picked = t;
    return 1;
}

inline int blocked_ell_from_coo_cuda_auto(const sparse::coo *src, types::dim_t cols,
                                          const types::u32 *feature_to_global, const unsigned int *candidates,
                                          unsigned int candidate_count, sparse::blocked_ell *dst, int device,
                                          blocked_ell_tune_result *picked = nullptr) {
    blocked_ell_tune_result t{};
    if (!choose_blocked_ell_block_size_from_coo_cuda(src, cols, feature_to_global, candidates, candidate_count, device,
                                                     &t) ||
        !blocked_ell_from_coo_cuda(src, cols, feature_to_global, t.block_size, dst, device))
        return 0;
    if (picked != nullptr) *picked = t;
    return 1;
}

inline int sliced_ell_from_compressed(const sparse::compressed *src, unsigned int slice_rows,
                                      sparse::sliced_ell *dst) {
    return cs_b200_sliced_ell_from_compressed(reinterpret_cast<const cs_host_compressed *>(src), slice_rows,
                                              reinterpret_cast<cs_host_sliced_ell *>(dst));
}
// The reference's GPU route has the same contract (host in, host out).
inline int sliced_ell_from_compressed_cuda(const sparse::compressed *src, unsigned int slice_rows,
                                           sparse::sliced_ell *dst) {
    return sliced_ell_from_compressed(src, slice_rows, dst);
}

inline int choose_sliced_ell_slice_rows_from_compressed(const sparse::compressed *src, const unsigned int *candidates,
                                                        unsigned int candidate_count, sliced_ell_tune_result *out) {
    return cs_b200_choose_sliced_ell_slice_rows_from_compressed(
        reinterpret_cast<const cs_host_compressed *>(src), candidates, candidate_count,
        reinterpret_cast<cs_sliced_ell_tune_result *>(out));
}

// src/convert/sliced_ell_from_blocked_ell.cuh:223-395
inline int choose_sliced_ell_slice_rows_from_blocked_ell(const sparse::blocked_ell *src,
                                                         const unsigned int *candidates,
                                                         unsigned int candidate_count, sliced_ell_tune_result *out) {
    return cs_b200_choose_sliced_ell_slice_rows_from_blocked_ell(
        reinterpret_cast<const cs_host_blocked_ell *>(src), candidates, candidate_count,
        reinterpret_cast<cs_sliced_ell_tune_result *>(out));
}

inline int sliced_ell_from_blocked_ell(const sparse::blocked_ell *src, unsigned int slice_rows,
                                       sparse::sliced_ell *dst) {
    return cs_b200_sliced_ell_from_blocked_ell(reinterpret_cast<const cs_host_blocked_ell *>(src), slice_rows,
                                               reinterpret_cast<cs_host_sliced_ell *>(dst));
}
// The reference's GPU route has the same contract (host in, host out); the
// device and stream arguments select nothing here (the current device runs it).
inline int sliced_ell_from_blocked_ell_cuda(const sparse::blocked_ell *src, unsigned int slice_rows,
                                            sparse::sliced_ell *dst, int device = 0, cudaStream_t stream = 0) {
    (void) device;
    (void) stream;
    return sliced_ell_from_blocked_ell(src, slice_rows, dst);
}

inline int sliced_ell_from_blocked_ell_auto(const sparse::blocked_ell *src, const unsigned int *candidates,
                                            unsigned int candidate_count, sparse::sliced_ell *dst,
                                            sliced_ell_tune_result *picked = 0) {
    sliced_ell_tune_result tune{};
    if (!choose_sliced_ell_slice_rows_from_blocked_ell(src, candidates, candidate_count, &tune)) return 0;
    if (!sliced_ell_from_blocked_ell(src, tune.slice_rows == 0u ? 1u : tune.slice_rows, dst)) return 0;
    if (picked != 0) *picked = tune;
    return 1;
}

inline int sliced_ell_from_blocked_ell_cuda_auto(const sparse::blocked_ell *src, const unsigned int *candidates,
                                                 unsigned int candidate_count, sparse::sliced_ell *dst,
                                                 int device = 0, cudaStream_t stream = 0,
                                                 sliced_ell_tune_result *picked = 0) {
    (void) device;
    (void) stream;
    return sliced_ell_from_blocked_ell_auto(src, candidates, candidate_count, dst, picked);
}

inline std::size_t compressed_transpose_scratch_bytes(types::dim_t cDim, types::dim_t uDim, types::nnz_t nnz) {
    size_t n = 0;
    return cs_b200_compressed_transpose_scratch_bytes(cDim, uDim, nnz, &n) ? n : 0;
}

inline int build_compressed_transpose_raw(types::dim_t cDim, types::dim_t uDim, types::nnz_t nnz,
                                          const types::ptr_t *d_cAxPtr, const types::idx_t *d_uAxIdx,
                                          const real::storage_t *d_val, types::ptr_t *d_out_uAxPtr,
                                          types::ptr_t *d_heads, types::idx_t *d_out_cAxIdx,
                                          real::storage_t *d_out_val, void *d_scan_tmp, std::size_t scan_bytes,
                                          cudaStream_t stream) {
    return cs_b200_build_compressed_transpose(cDim, uDim, nnz, d_cAxPtr, d_uAxIdx,
                                              reinterpret_cast<const uint16_t *>(d_val), d_out_uAxPtr, d_heads,
                                              d_out_cAxIdx, reinterpret_cast<uint16_t *>(d_out_val), d_scan_tmp,
                                              scan_bytes, reinterpret_cast<cs_stream_t>(stream));
}
inline int build_transpose_cs_from_cs_raw(types::dim_t cDim, types::dim_t uDim, types::nnz_t nnz,
                                          const types::ptr_t *p, const types::idx_t *i, const real::storage_t *v,
                                          types::ptr_t *op, types::ptr_t *heads, types::idx_t *oi,
                                          real::storage_t *ov, void *tmp, std::size_t bytes, cudaStream_t s) {
    return build_compressed_transpose_raw(cDim, uDim, nnz, p, i, v, op, heads, oi, ov, tmp, bytes, s);
}

} // namespace convert

// ---------------------------------------------------------------------------
// bucket::
// ---------------------------------------------------------------------------
namespace bucket {

struct alignas(16) major_nnz_bucket_plan_view {
    types::dim_t major_dim;
    types::idx_t bucket_count;
    const types::idx_t *major_order;
    const types::idx_t *major_nnz_sorted;
    const types::idx_t *bucket_offsets;
    const types::idx_t *inverse_major_order;
};

inline std::size_t major_nnz_bucket_sort_scratch_bytes(types::dim_t major_dim) {
    size_t n = 0;
    return cs_b200_major_nnz_bucket_sort_scratch_bytes(major_dim, &n) ? n : 0;
}
inline std::size_t major_nnz_bucket_scan_scratch_bytes(types::dim_t major_dim) {
    size_t n = 0;
    return cs_b200_major_nnz_bucket_scan_scratch_bytes(major_dim, &n) ? n : 0;
}

inline int build_major_nnz_bucket_plan_raw(const types::ptr_t *d_major_ptr, types::dim_t major_dim,
                                           types::idx_t *d_major_nnz, types::idx_t *d_major_nnz_sorted,
                                           types::idx_t *d_major_order_in, types::idx_t *d_major_order_out,
                                           types::idx_t *d_bucket_offsets, types::idx_t requested_bucket_count,
                                           void *d_sort_tmp, std::size_t sort_tmp_bytes, cudaStream_t stream) {
    return cs_b200_build_major_nnz_bucket_plan(d_major_ptr, major_dim, d_major_nnz, d_major_nnz_sorted,
                                               d_major_order_in, d_major_order_out, d_bucket_offsets,
                                               requested_bucket_count, d_sort_tmp, sort_tmp_bytes,
                                               reinterpret_cast<cs_stream_t>(stream));
}

inline int rebuild_compressed_major_order_raw(const types::ptr_t *d_src_major_ptr, const types::idx_t *d_src_minor_idx,
                                              const real::storage_t *d_src_val, types::dim_t major_dim,
                                              const types::idx_t *d_major_order, types::ptr_t *d_dst_major_ptr,
                                              types::idx_t *d_dst_minor_idx, real::storage_t *d_dst_val,
                                              types::idx_t *d_inverse_major_order, void *d_scan_tmp,
                                              std::size_t scan_tmp_bytes, cudaStream_t stream) {
    return cs_b200_rebuild_compressed_major_order(d_src_major_ptr, d_src_minor_idx,
                                                  reinterpret_cast<const uint16_t *>(d_src_val), major_dim,
                                                  d_major_order, d_dst_major_ptr, d_dst_minor_idx,
                                                  reinterpret_cast<uint16_t *>(d_dst_val), d_inverse_major_order,
                                                  d_scan_tmp, scan_tmp_bytes, reinterpret_cast<cs_stream_t>(stream));
}

// Caller-held workspace (operators/major_nnz.cuh:11-44): buffers grow
// monotonically; result views alias it until the next call or clear().
struct alignas(16) compressed_major_bucket_workspace {
    int device;
    cudaStream_t stream;
    types::dim_t major_capacity;
    types::nnz_t nnz_capacity;
    types::idx_t bucket_capacity;
    std::size_t sort_capacity;
    std::size_t scan_capacity;
    void *d_major_block;
    void *d_rebuilt_block;
    types::idx_t *d_major_nnz;
    types::idx_t *d_major_nnz_sorted;
    types::idx_t *d_major_order_in;
    types::idx_t *d_major_order_out;
    types::idx_t *d_inverse_major_order;
    types::idx_t *d_bucket_offsets;
    types::ptr_t *d_rebuilt_major_ptr;
    types::idx_t *d_rebuilt_minor_idx;
    real::storage_t *d_rebuilt_val;
    void *d_sort_tmp;
    void *d_scan_tmp;
};

struct alignas(16) compressed_major_bucket_result {
    device::compressed_view rebuilt;
    major_nnz_bucket_plan_view plan;
};

inline void init(compressed_major_bucket_workspace *ws) {
    std::memset(ws, 0, sizeof(*ws));
    ws->device = -1;
}

inline void clear(compressed_major_bucket_workspace *ws) {
    if (ws->d_major_block) cudaFree(ws->d_major_block);
    if (ws->d_rebuilt_block) cudaFree(ws->d_rebuilt_block);
    if (ws->stream) cudaStreamDestroy(ws->stream);
    init(ws);
}

inline int setup(compressed_major_bucket_workspace *ws, int device) {
    init(ws);
    ws->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    return cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) == cudaSuccess;
}

namespace detail {
inline std::size_t up256(std::size_t x) { return (x + 255u) / 256u * 256u; }
} // namespace detail

inline int reserve(compressed_major_bucket_workspace *ws, types::dim_t major_dim, types::nnz_t nnz,
                   types::idx_t bucket_count) {
    const std::size_t sort_bytes = major_nnz_bucket_sort_scratch_bytes(major_dim);
    const std::size_t scan_bytes = major_nnz_bucket_scan_scratch_bytes(major_dim);
    if (major_dim > ws->major_capacity || bucket_count > ws->bucket_capacity || sort_bytes > ws->sort_capacity ||
        scan_bytes > ws->scan_capacity) {
        if (ws->d_major_block) cudaFree(ws->d_major_block);
        ws->d_major_block = nullptr;
        const std::size_t m = detail::up256(((std::size_t) major_dim + 1u) * 4u);
        const std::size_t b = detail::up256(((std::size_t) bucket_count + 2u) * 4u);
        const std::size_t total = 5u * m + b + detail::up256(sort_bytes) + detail::up256(scan_bytes);
        if (cudaMalloc(&ws->d_major_block, total) != cudaSuccess) return 0;
        unsigned char *p = static_cast<unsigned char *>(ws->d_major_block);
        ws->d_major_nnz = reinterpret_cast<types::idx_t *>(p);
        ws->d_major_nnz_sorted = reinterpret_cast<types::idx_t *>(p + m);
        ws->d_major_order_in = reinterpret_cast<types::idx_t *>(p + 2u * m);
        ws->d_major_order_out = reinterpret_cast<types::idx_t *>(p + 3u * m);
        ws->d_inverse_major_order = reinterpret_cast<types::idx_t *>(p + 4u * m);
        ws->d_bucket_offsets = reinterpret_cast<types::idx_t *>(p + 5u * m);
        ws->d_sort_tmp = p + 5u * m + b;
        ws->d_scan_tmp = p + 5u * m + b + detail::up256(sort_bytes);
        ws->major_capacity = major_dim;
        ws->bucket_capacity = bucket_count;
        ws->sort_capacity = sort_bytes;
        ws->scan_capacity = scan_bytes;
    }
    if (nnz > ws->nnz_capacity || major_dim > ws->major_capacity || !ws->d_rebuilt_block) {
        if (ws->d_rebuilt_block) cudaFree(ws->d_rebuilt_block);
        ws->d_rebuilt_block = nullptr;
        const std::size_t m = detail::up256(((std::size_t) major_dim + 1u) * 4u);
        const std::size_t i = detail::up256((std::size_t) nnz * 4u + 4u);
        const std::size_t v = detail::up256((std::size_t) nnz * 2u + 2u);
        if (cudaMalloc(&ws->d_rebuilt_block, m + i + v) != cudaSuccess) return 0;
        unsigned char *p = static_cast<unsigned char *>(ws->d_rebuilt_block);
        ws->d_rebuilt_major_ptr = reinterpret_cast<types::ptr_t *>(p);
        ws->d_rebuilt_minor_idx = reinterpret_cast<types::idx_t *>(p + m);
        ws->d_rebuilt_val = reinterpret_cast<real::storage_t *>(p + m + i);
        ws->nnz_capacity = nnz;
    }
    return 1;
}

inline int build_plan(const device::compressed_view *src, types::idx_t requested_bucket_count,
                      compressed_major_bucket_workspace *ws, major_nnz_bucket_plan_view *out) {
    if (src == nullptr || ws == nullptr || out == nullptr) return 0;
    const types::dim_t major_dim = src->axis == sparse::compressed_by_col ? src->cols : src->rows;
    const types::idx_t B = major_dim == 0u ? 1u
                                           : (requested_bucket_count < 1u ? 1u
                                                                          : (requested_bucket_count > major_dim
                                                                                 ? major_dim
                                                                                 : requested_bucket_count));
    if (!reserve(ws, major_dim, src->nnz, B)) return 0;
    if (!build_major_nnz_bucket_plan_raw(src->majorPtr, major_dim, ws->d_major_nnz, ws->d_major_nnz_sorted,
                                         ws->d_major_order_in, ws->d_major_order_out, ws->d_bucket_offsets,
                                         requested_bucket_count, ws->d_sort_tmp, ws->sort_capacity, ws->stream))
        return 0;
    out->major_dim = major_dim;
    out->bucket_count = B;
    out->major_order = ws->d_major_order_out;
    out->major_nnz_sorted = ws->d_major_nnz_sorted;
    out->bucket_offsets = ws->d_bucket_offsets;
    out->inverse_major_order = nullptr;
    return 1;
}

inline int rebuild(const device::compressed_view *src, const major_nnz_bucket_plan_view *plan,
                   compressed_major_bucket_workspace *ws, compressed_major_bucket_result *out) {
    if (src == nullptr || plan == nullptr || ws == nullptr || out == nullptr) return 0;
    if (!reserve(ws, plan->major_dim, src->nnz, plan->bucket_count)) return 0;
    if (!rebuild_compressed_major_order_raw(src->majorPtr, src->minorIdx, src->val, plan->major_dim,
                                            plan->major_order, ws->d_rebuilt_major_ptr, ws->d_rebuilt_minor_idx,
                                            ws->d_rebuilt_val, ws->d_inverse_major_order, ws->d_scan_tmp,
                                            ws->scan_capacity, ws->stream))
        return 0;
    out->rebuilt = *src;
    out->rebuilt.majorPtr = ws->d_rebuilt_major_ptr;
    out->rebuilt.minorIdx = ws->d_rebuilt_minor_idx;
    out->rebuilt.val = ws->d_rebuilt_val;
    out->plan = *plan;
    out->plan.inverse_major_order = ws->d_inverse_major_order;
    return 1;
}

inline int build_bucketed_major_view(const device::compressed_view *src, types::idx_t requested_bucket_count,
                                     compressed_major_bucket_workspace *ws, compressed_major_bucket_result *out) {
    major_nnz_bucket_plan_view plan;
    if (!build_plan(src, requested_bucket_count, ws, &plan)) return 0;
    return rebuild(src, &plan, ws, out);
}

} // namespace bucket

// ---------------------------------------------------------------------------
// convert:: filtered Blocked-ELL -> CSR (src/convert/filtered_blocked_ell_to_compressed.cuh)
// ---------------------------------------------------------------------------
namespace convert {

struct alignas(16) filtered_blocked_ell_stats {
    types::dim_t kept_rows;
    types::dim_t output_rows;
    types::dim_t output_cols;
    types::nnz_t live_nnz;
    types::u64 kept_row_slots;
    types::u64 dead_slots;
    double live_fill_ratio;
    std::size_t dead_value_bytes;
};

struct alignas(16) filtered_blocked_ell_result {
    device::compressed_view filtered;
    bucket::compressed_major_bucket_result bucketed;
    filtered_blocked_ell_stats stats;
    int has_bucketed;
};

struct alignas(16) filtered_blocked_ell_workspace {
    int device;
    cudaStream_t stream;
    int owns_stream;
    types::dim_t rows_capacity;
    types::dim_t filtered_rows_capacity;
    types::nnz_t nnz_capacity;
    void *d_counts_block;   // row pointers, kept counters, status
    void *d_values_block;   // filtered column indices and values
    void *d_scan_tmp;
    std::size_t d_scan_tmp_bytes;
    types::ptr_t *d_filtered_major_ptr;
    types::idx_t *d_filtered_minor_idx;
    real::storage_t *d_filtered_val;
    unsigned long long *d_kept; // kept rows, kept row slots
    std::uint32_t *d_status;
    bucket::compressed_major_bucket_workspace bucket_ws;
};

inline void init(filtered_blocked_ell_workspace *ws) {
    std::memset(ws, 0, sizeof(*ws));
    ws->device = -1;
    bucket::init(&ws->bucket_ws);
}

inline void clear(filtered_blocked_ell_workspace *ws) {
    if (ws->device >= 0) cudaSetDevice(ws->device);
    bucket::clear(&ws->bucket_ws);
    if (ws->d_scan_tmp) cudaFree(ws->d_scan_tmp);
    if (ws->d_values_block) cudaFree(ws->d_values_block);
    if (ws->d_counts_block) cudaFree(ws->d_counts_block);
    if (ws->owns_stream && ws->stream) cudaStreamDestroy(ws->stream);
    init(ws);
}

inline int setup(filtered_blocked_ell_workspace *ws, int device, cudaStream_t stream = 0) {
    clear(ws);
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    ws->device = device;
    if (stream == 0) {
        if (cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess) return 0;
        ws->owns_stream = 1;
    } else {
        ws->stream = stream;
    }
    return bucket::setup(&ws->bucket_ws, device);
}

inline int reserve(filtered_blocked_ell_workspace *ws, types::dim_t src_rows, types::dim_t filtered_rows,
                   types::dim_t /*filtered_cols*/, types::nnz_t max_nnz, types::u64 /*total_values*/) {
    if (cudaSetDevice(ws->device >= 0 ? ws->device : 0) != cudaSuccess) return 0;
    size_t scan = 0;
    if (!cs_b200_filter_blocked_ell_scratch_bytes(src_rows, filtered_rows, &scan)) return 0;
    if (filtered_rows + 1u > ws->filtered_rows_capacity + 1u || !ws->d_counts_block) {
        if (ws->d_counts_block) cudaFree(ws->d_counts_block);
        ws->d_counts_block = nullptr;
        const std::size_t ptr_bytes = bucket::detail::up256(((std::size_t) filtered_rows + 1u) * 4u);
        if (cudaMalloc(&ws->d_counts_block, ptr_bytes + 256u) != cudaSuccess) return 0;
        unsigned char *p = static_cast<unsigned char *>(ws->d_counts_block);
        ws->d_filtered_major_ptr = reinterpret_cast<types::ptr_t *>(p);
        ws->d_kept = reinterpret_cast<unsigned long long *>(p + ptr_bytes);
        ws->d_status = reinterpret_cast<std::uint32_t *>(p + ptr_bytes + 64u);
        ws->filtered_rows_capacity = filtered_rows;
    }
    if (max_nnz > ws->nnz_capacity || !ws->d_values_block) {
        if (ws->d_values_block) cudaFree(ws->d_values_block);
        ws->d_values_block = nullptr;
        const std::size_t idx_bytes = bucket::detail::up256((std::size_t) max_nnz * 4u + 4u);
        if (cudaMalloc(&ws->d_values_block, idx_bytes + (std::size_t) max_nnz * 2u + 16u) != cudaSuccess) return 0;
        ws->d_filtered_minor_idx = static_cast<types::idx_t *>(ws->d_values_block);
        ws->d_filtered_val = reinterpret_cast<real::storage_t *>(static_cast<unsigned char *>(ws->d_values_block) +
                                                                 idx_bytes);
        ws->nnz_capacity = max_nnz;
    }
    if (scan > ws->d_scan_tmp_bytes || !ws->d_scan_tmp) {
        if (ws->d_scan_tmp) cudaFree(ws->d_scan_tmp);
        ws->d_scan_tmp = nullptr;
        if (cudaMalloc(&ws->d_scan_tmp, scan) != cudaSuccess) return 0;
        ws->d_scan_tmp_bytes = scan;
    }
    ws->rows_capacity = src_rows;
    return 1;
}

namespace detail {
// Count + emit over a shard's partitions (host array of views); live nnz and
// kept counters come back to the host, as the reference reads them.
inline int filter_parts(const cs_blocked_ell_view *views, std::uint32_t part_count, types::dim_t output_rows,
                        types::dim_t output_cols, const unsigned char *d_keep_rows, const unsigned char *d_keep_cols,
                        const types::idx_t *d_row_remap, const types::idx_t *d_col_remap, types::nnz_t max_nnz,
                        filtered_blocked_ell_workspace *ws, unsigned int *live_nnz, unsigned long long kept[2]) {
    types::dim_t rows = 0;
    for (std::uint32_t k = 0; k < part_count; ++k) rows += views[k].rows;
    if (!reserve(ws, rows, output_rows, output_cols, max_nnz, 0u)) return 0;
    cs_row_feature_mask_view m{d_keep_rows, d_keep_cols, d_row_remap, d_col_remap};
    const cs_stream_t s = reinterpret_cast<cs_stream_t>(ws->stream);
    if (cudaMemsetAsync(ws->d_status, 0, 4, ws->stream) != cudaSuccess) return 0;
    // without remaps, block sizes multiples of 8 and 16-byte aligned values: the
    // marked route (one full read of the kept values, a re-read of the 8-value
    // groups holding kept entries); count + emit otherwise, or when max_nnz is short
    bool vec = d_row_remap == nullptr && d_col_remap == nullptr && output_rows >= rows;
    for (std::uint32_t k = 0; vec && k < part_count; ++k)
        vec = views[k].rows == 0u ||
              (views[k].block_size % 8u == 0u && (reinterpret_cast<std::uintptr_t>(views[k].val) & 15u) == 0u);
    std::size_t need = 0;
    if (vec && cs_b200_filter_blocked_ell_marked_scratch_bytes(views, part_count, &need) && need > 0u) {
        if (need > ws->d_scan_tmp_bytes) {
            cudaFree(ws->d_scan_tmp);
            ws->d_scan_tmp = nullptr;
            ws->d_scan_tmp_bytes = 0u;
            if (cudaMalloc(&ws->d_scan_tmp, need) != cudaSuccess) return 0;
            ws->d_scan_tmp_bytes = need;
        }
        std::uint32_t status = 0u;
        if (!cs_b200_filter_blocked_ell_marked(views, part_count, &m, output_rows, output_cols,
                                               ws->d_filtered_major_ptr, ws->d_filtered_minor_idx,
                                               reinterpret_cast<std::uint16_t *>(ws->d_filtered_val), max_nnz,
                                               reinterpret_cast<std::uint64_t *>(ws->d_kept), ws->d_scan_tmp,
                                               ws->d_scan_tmp_bytes, ws->d_status, s) ||
            cudaMemcpyAsync(live_nnz, ws->d_filtered_major_ptr + output_rows, 4, cudaMemcpyDeviceToHost,
                            ws->stream) != cudaSuccess ||
            cudaMemcpyAsync(kept, ws->d_kept, 16, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
            cudaMemcpyAsync(&status, ws->d_status, 4, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
            cudaStreamSynchronize(ws->stream) != cudaSuccess)
            return 0;
        if (status == 0u) return 1;
        if (status != CS_STATUS_CAPACITY || cudaMemsetAsync(ws->d_status, 0, 4, ws->stream) != cudaSuccess) return 0;
    }
    if (!cs_b200_filter_blocked_ell_count(views, part_count, &m, output_rows, output_cols, ws->d_filtered_major_ptr,
                                          reinterpret_cast<std::uint64_t *>(ws->d_kept), ws->d_scan_tmp,
                                          ws->d_scan_tmp_bytes, ws->d_status, s))
        return 0;
    std::uint32_t status = 0u;
    if (cudaMemcpyAsync(live_nnz, ws->d_filtered_major_ptr + output_rows, 4, cudaMemcpyDeviceToHost, ws->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(kept, ws->d_kept, 16, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaMemcpyAsync(&status, ws->d_status, 4, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaStreamSynchronize(ws->stream) != cudaSuccess)
        return 0;
    if (status != 0u || *live_nnz > max_nnz) return 0;
    if (*live_nnz == 0u) return 1;
    return cs_b200_filter_blocked_ell_emit(views, part_count, &m, output_rows, output_cols, ws->d_filtered_major_ptr,
                                           ws->d_filtered_minor_idx,
                                           reinterpret_cast<std::uint16_t *>(ws->d_filtered_val), s);
}
} // namespace detail

// filtered_blocked_ell_to_compressed.cuh:264-382; stats as the reference fills
// them there (kept_rows = output_rows, kept_row_slots = kept_rows * ell_cols)
inline int filter_blocked_ell_to_compressed(const device::blocked_ell_view *src, types::dim_t output_rows,
                                            types::dim_t output_cols, const unsigned char *d_keep_rows,
                                            const unsigned char *d_keep_cols, const types::idx_t *d_row_remap,
                                            const types::idx_t *d_col_remap, filtered_blocked_ell_workspace *ws,
                                            filtered_blocked_ell_result *out) {
    if (src == nullptr || ws == nullptr) return 0;
    filtered_blocked_ell_result local{};
    unsigned int live = 0u;
    unsigned long long kept[2] = {0ull, 0ull};
    if (output_rows != 0u && output_cols != 0u) {
        const cs_blocked_ell_view v = *reinterpret_cast<const cs_blocked_ell_view *>(src);
        if (!detail::filter_parts(&v, 1u, output_rows, output_cols, d_keep_rows, d_keep_cols, d_row_remap,
                                  d_col_remap, src->nnz, ws, &live, kept))
            return 0;
    } else if (!reserve(ws, src->rows, output_rows, output_cols, src->nnz, 0u)) {
        return 0;
    }
    local.filtered.rows = output_rows;
    local.filtered.cols = output_cols;
    local.filtered.nnz = live;
    local.filtered.axis = sparse::compressed_by_row;
    local.filtered.majorPtr = ws->d_filtered_major_ptr;
    local.filtered.minorIdx = ws->d_filtered_minor_idx;
    local.filtered.val = ws->d_filtered_val;
    const types::u64 slots = (output_rows != 0u && output_cols != 0u) ? (types::u64) output_rows * src->ell_cols : 0u;
    local.stats.kept_rows = output_rows;
    local.stats.output_rows = output_rows;
    local.stats.output_cols = output_cols;
    local.stats.live_nnz = live;
    local.stats.kept_row_slots = slots;
    local.stats.dead_slots = slots > live ? slots - live : 0u;
    local.stats.live_fill_ratio = slots == 0u ? 1.0 : (double) live / (double) slots;
    local.stats.dead_value_bytes = (std::size_t) local.stats.dead_slots * sizeof(real::storage_t);
    local.has_bucketed = 0;
    if (out != nullptr) *out = local;
    return 1;
}

// :384-412
inline int build_bucketed_filtered_blocked_ell_major_view(const device::blocked_ell_view *src,
                                                          types::dim_t output_rows, types::dim_t output_cols,
                                                          const unsigned char *d_keep_rows,
                                                          const unsigned char *d_keep_cols,
                                                          const types::idx_t *d_row_remap,
                                                          const types::idx_t *d_col_remap,
                                                          types::idx_t requested_bucket_count,
                                                          filtered_blocked_ell_workspace *ws,
                                                          filtered_blocked_ell_result *out) {
    filtered_blocked_ell_result local{};
    if (ws == nullptr) return 0;
    if (!filter_blocked_ell_to_compressed(src, output_rows, output_cols, d_keep_rows, d_keep_cols, d_row_remap,
                                          d_col_remap, ws, &local))
        return 0;
    if (cudaStreamSynchronize(ws->stream) != cudaSuccess) return 0;
    if (!bucket::build_bucketed_major_view(&local.filtered, requested_bucket_count, &ws->bucket_ws, &local.bucketed))
        return 0;
    local.has_bucketed = 1;
    if (out != nullptr) *out = local;
    return 1;
}

} // namespace convert

// ---------------------------------------------------------------------------
// repack:: (src/repack/operators/sharded_blocked_ell.cuh).  The reference takes
// a sharded_device<blocked_ell> state and a shard id; sharded<> containers are
// not part of this library, so the shard is passed as its partitions' device
// views in row order (what the reference gathers into part_views).
// ---------------------------------------------------------------------------
namespace repack {

struct alignas(16) sharded_blocked_ell_repack_config {
    types::dim_t output_rows;
    types::dim_t output_cols;
    types::u32 block_size;
    types::idx_t requested_bucket_count;
};

struct alignas(16) sharded_blocked_ell_repack_stats {
    types::dim_t kept_rows;
    types::dim_t output_rows;
    types::dim_t output_cols;
    types::nnz_t live_nnz;
    types::u64 kept_row_slots;
    types::u64 dead_slots;
    double live_fill_ratio;
    std::size_t dead_value_bytes;
    types::u32 ell_width;
};

struct alignas(16) sharded_blocked_ell_repack_result {
    device::compressed_view filtered;
    bucket::compressed_major_bucket_result bucketed;
    device::blocked_ell_view rebuilt;
    bucket::major_nnz_bucket_plan_view bucket_plan;
    sharded_blocked_ell_repack_stats stats;
    unsigned long shard_id;
};

struct alignas(16) sharded_blocked_ell_repack_workspace {
    int device;
    cudaStream_t stream;
    convert::filtered_blocked_ell_workspace filter_ws; // filtered CSR + bucket workspace
    void *d_shape_block;                              // shape words, emitted nnz, status
    void *d_bell_scratch;
    std::size_t bell_scratch_bytes;
    void *d_rebuilt_storage;
    std::size_t rebuilt_storage_capacity_bytes;
    types::idx_t *d_rebuilt_block_cols;
    real::storage_t *d_rebuilt_val;
};

inline void init(sharded_blocked_ell_repack_workspace *ws) {
    std::memset(ws, 0, sizeof(*ws));
    ws->device = -1;
    convert::init(&ws->filter_ws);
}

inline void clear(sharded_blocked_ell_repack_workspace *ws) {
    convert::clear(&ws->filter_ws);
    if (ws->d_rebuilt_storage) cudaFree(ws->d_rebuilt_storage);
    if (ws->d_bell_scratch) cudaFree(ws->d_bell_scratch);
    if (ws->d_shape_block) cudaFree(ws->d_shape_block);
    init(ws);
}

inline int setup(sharded_blocked_ell_repack_workspace *ws, int device, cudaStream_t stream = 0) {
    clear(ws);
    if (!convert::setup(&ws->filter_ws, device, stream)) return 0;
    ws->device = device;
    ws->stream = ws->filter_ws.stream;
    return cudaMalloc(&ws->d_shape_block, 256) == cudaSuccess;
}

// sharded_blocked_ell.cuh:393-726: filter the shard's partitions to CSR, bucket
// its rows by nnz and rebuild them in bucket order, then the rebuilt CSR as
// Blocked-ELL of cfg->block_size in workspace memory.
inline int build_repacked_blocked_ell_parts(const device::blocked_ell_view *const *part_views,
                                            unsigned long part_count, unsigned long shard_id,
                                            const sharded_blocked_ell_repack_config *cfg,
                                            const unsigned char *d_keep_rows, const unsigned char *d_keep_cols,
                                            const types::idx_t *d_row_remap, const types::idx_t *d_col_remap,
                                            sharded_blocked_ell_repack_workspace *ws,
                                            sharded_blocked_ell_repack_result *out) {
    if (part_views == nullptr || cfg == nullptr || ws == nullptr || out == nullptr || cfg->block_size == 0u ||
        part_count == 0u || part_count > CS_MAX_REPACK_PARTS)
        return 0;
    cs_blocked_ell_view views[CS_MAX_REPACK_PARTS];
    types::nnz_t shard_nnz = 0u;
    for (unsigned long k = 0; k < part_count; ++k) {
        if (part_views[k] == nullptr) return 0;
        views[k] = *reinterpret_cast<const cs_blocked_ell_view *>(part_views[k]);
        shard_nnz += part_views[k]->nnz;
    }
    sharded_blocked_ell_repack_result local{};
    local.shard_id = shard_id;
    unsigned int live = 0u;
    unsigned long long kept[2] = {0ull, 0ull};
    if (!convert::detail::filter_parts(views, (std::uint32_t) part_count, cfg->output_rows, cfg->output_cols,
                                       d_keep_rows, d_keep_cols, d_row_remap, d_col_remap, shard_nnz, &ws->filter_ws,
                                       &live, kept))
        return 0;
    convert::filtered_blocked_ell_workspace &fw = ws->filter_ws;
    local.filtered.rows = cfg->output_rows;
    local.filtered.cols = cfg->output_cols;
    local.filtered.nnz = live;
    local.filtered.axis = sparse::compressed_by_row;
    local.filtered.majorPtr = fw.d_filtered_major_ptr;
    local.filtered.minorIdx = fw.d_filtered_minor_idx;
    local.filtered.val = fw.d_filtered_val;
    local.stats.kept_rows = (types::dim_t) kept[0];
    local.stats.output_rows = cfg->output_rows;
    local.stats.output_cols = cfg->output_cols;
    local.stats.live_nnz = live;
    local.stats.kept_row_slots = kept[1];
    local.stats.dead_slots = kept[1] > live ? kept[1] - live : 0u;
    local.stats.live_fill_ratio = kept[1] == 0u ? 1.0 : (double) live / (double) kept[1];
    local.stats.dead_value_bytes = (std::size_t) local.stats.dead_slots * sizeof(real::storage_t);
    local.rebuilt.rows = cfg->output_rows;
    local.rebuilt.cols = cfg->output_cols;
    local.rebuilt.nnz = live;
    local.rebuilt.block_size = cfg->block_size;
    if (cfg->output_rows == 0u || cfg->output_cols == 0u || live == 0u) {
        // as the reference: the filtered CSR doubles as the bucketed view, one bucket
        local.bucketed.rebuilt = local.filtered;
        local.bucketed.plan.major_dim = cfg->output_rows;
        local.bucketed.plan.bucket_count = 1u;
        local.bucket_plan = local.bucketed.plan;
        *out = local;
        return 1;
    }
    if (cudaStreamSynchronize(ws->stream) != cudaSuccess) return 0;
    if (!bucket::build_bucketed_major_view(&local.filtered, cfg->requested_bucket_count, &fw.bucket_ws,
                                           &local.bucketed) ||
        cudaStreamSynchronize(fw.bucket_ws.stream) != cudaSuccess)
        return 0;
    local.bucket_plan = local.bucketed.plan;
    // the rebuilt CSR as Blocked-ELL: shape (ell width), then the emit
    const cs_compressed_view cv = *reinterpret_cast<const cs_compressed_view *>(&local.bucketed.rebuilt);
    size_t sb = 0;
    if (!cs_b200_blocked_ell_scratch_bytes(cv.rows, cv.cols, cfg->block_size, &sb)) return 0;
    if (sb > ws->bell_scratch_bytes || !ws->d_bell_scratch) {
        if (ws->d_bell_scratch) cudaFree(ws->d_bell_scratch);
        ws->d_bell_scratch = nullptr;
        if (cudaMalloc(&ws->d_bell_scratch, sb) != cudaSuccess) return 0;
        ws->bell_scratch_bytes = sb;
    }
    unsigned long long *d_shape = static_cast<unsigned long long *>(ws->d_shape_block);
    std::uint32_t *d_nnz = reinterpret_cast<std::uint32_t *>(d_shape + 2);
    std::uint32_t *d_status = d_nnz + 1;
    const cs_stream_t s = reinterpret_cast<cs_stream_t>(ws->stream);
    unsigned long long shape[2] = {0ull, 0ull};
    std::uint32_t status = 0u;
    if (cudaMemsetAsync(ws->d_shape_block, 0, 32, ws->stream) != cudaSuccess ||
        !cs_b200_blocked_ell_shape(&cv, cfg->block_size, reinterpret_cast<std::uint64_t *>(d_shape),
                                   ws->d_bell_scratch, ws->bell_scratch_bytes, d_status, s) ||
        cudaMemcpyAsync(shape, d_shape, 16, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaMemcpyAsync(&status, d_status, 4, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaStreamSynchronize(ws->stream) != cudaSuccess || status != 0u)
        return 0;
    const types::u32 ell_width = (types::u32) shape[0];
    const types::u32 B = cfg->block_size;
    const std::size_t row_blocks = ((std::size_t) cv.rows + B - 1u) / B;
    const std::size_t idx_bytes = bucket::detail::up256(row_blocks * ell_width * 4u + 4u);
    const std::size_t total = idx_bytes + (std::size_t) cv.rows * ell_width * B * 2u + 16u;
    if (total > ws->rebuilt_storage_capacity_bytes || !ws->d_rebuilt_storage) {
        if (ws->d_rebuilt_storage) cudaFree(ws->d_rebuilt_storage);
        ws->d_rebuilt_storage = nullptr;
        if (cudaMalloc(&ws->d_rebuilt_storage, total) != cudaSuccess) return 0;
        ws->rebuilt_storage_capacity_bytes = total;
    }
    ws->d_rebuilt_block_cols = static_cast<types::idx_t *>(ws->d_rebuilt_storage);
    ws->d_rebuilt_val = reinterpret_cast<real::storage_t *>(static_cast<unsigned char *>(ws->d_rebuilt_storage) +
                                                            idx_bytes);
    local.rebuilt.ell_cols = ell_width * B;
    local.rebuilt.blockColIdx = ell_width ? ws->d_rebuilt_block_cols : nullptr;
    local.rebuilt.val = ell_width ? ws->d_rebuilt_val : nullptr;
    local.stats.ell_width = ell_width;
    if (ell_width != 0u) {
        const cs_blocked_ell_view dv = *reinterpret_cast<const cs_blocked_ell_view *>(&local.rebuilt);
        if (!cs_b200_blocked_ell_emit(&cv, &dv, d_nnz, ws->d_bell_scratch, ws->bell_scratch_bytes, d_status, s) ||
            cudaStreamSynchronize(ws->stream) != cudaSuccess)
            return 0;
    }
    *out = local;
    return 1;
}

} // namespace repack

// ---------------------------------------------------------------------------
// runtime:: mask_groups
// ---------------------------------------------------------------------------
namespace runtime {

static constexpr unsigned int CELLSHARD_MAX_MASK_GROUPS = CS_MAX_MASK_GROUPS;

enum sparse_mask_layout : std::uint32_t {
    sparse_mask_layout_unknown = 0u,
    sparse_mask_layout_blocked_ell = 1u,
    sparse_mask_layout_sliced_ell = 2u,
    sparse_mask_layout_compressed = 3u
};

struct alignas(16) group_mask_config_view {
    unsigned int group_count;
    const char *const *group_names;
    const std::uint32_t *feature_group_masks;
};

struct alignas(16) row_feature_mask_view {
    const unsigned char *row_keep;
    const unsigned char *feature_keep;
    const unsigned int *row_remap;
    const unsigned int *feature_remap;
};

struct alignas(16) sparse_group_filter_params {
    float min_total;
    unsigned int min_detected_features;
    float max_group_fraction;
    unsigned int fraction_group_index;
};

struct alignas(16) sparse_group_reduce_result {
    unsigned int rows;
    unsigned int group_count;
    float *row_totals;
    unsigned int *detected_features;
    float *max_values;
    unsigned char *row_keep;
    float *group_counts;
    float *group_percentages;
};

struct alignas(16) sparse_group_reduce_workspace {
    int device;
    cudaStream_t stream;
    int owns_stream;
    unsigned int rows_capacity;
    unsigned int cols_capacity;
    unsigned int group_capacity;
    unsigned int values_capacity;
    void *row_block;
    void *feature_block;
    void *scratch_block;
    std::size_t scratch_bytes;
    float *row_totals;
    unsigned int *detected_features;
    float *max_values;
    unsigned char *row_keep;
    float *group_counts;
    float *group_percentages;
    std::uint32_t *feature_group_masks;
};

struct alignas(16) masked_sparse_reoptimize_config {
    unsigned int output_rows;
    unsigned int output_cols;
    unsigned int requested_bucket_count;
    unsigned int output_block_size;
    sparse_mask_layout requested_layout;
};

struct alignas(16) masked_sparse_reoptimize_metadata {
    unsigned int kept_rows;
    unsigned int kept_features;
    unsigned int live_nnz;
    unsigned long long bytes_before;
    unsigned long long bytes_after;
    sparse_mask_layout output_layout;
};

struct alignas(16) masked_sparse_reoptimize_result {
    device::compressed_view compressed;
    device::blocked_ell_view blocked_ell;
    masked_sparse_reoptimize_metadata metadata;
};

struct alignas(16) masked_sparse_reoptimize_workspace {
    int device;
    cudaStream_t stream;
    int owns_stream;
    void *private_workspace;
};

struct alignas(16) auto_reoptimize_prediction_input {
    float density_change;
    float row_drop_ratio;
    float feature_drop_ratio;
    float layout_padding_change;
    float estimated_rebuild_cost_ms;
    unsigned int expected_reuse_count;
};

struct alignas(16) auto_reoptimize_prediction {
    unsigned int should_reoptimize;
    float estimated_net_gain_ms;
};

// The reference's predictor is a stub that never asks for a reoptimization
// (mask_groups.cu:526-532); kept with the same answer.
inline int predict_masked_sparse_reoptimization(const auto_reoptimize_prediction_input *input,
                                                auto_reoptimize_prediction *out) {
    if (input == nullptr || out == nullptr) return 0;
    out->should_reoptimize = 0u;
    out->estimated_net_gain_ms = 0.0f;
    return 1;
}

inline void init(sparse_group_reduce_workspace *ws) {
    std::memset(ws, 0, sizeof(*ws));
    ws->device = -1;
}

inline void clear(sparse_group_reduce_workspace *ws) {
    if (ws == nullptr) return;
    if (ws->row_block) cudaFree(ws->row_block);
    if (ws->feature_block) cudaFree(ws->feature_block);
    if (ws->scratch_block) cudaFree(ws->scratch_block);
    if (ws->owns_stream && ws->stream) cudaStreamDestroy(ws->stream);
    init(ws);
}

inline int setup(sparse_group_reduce_workspace *ws, int device, cudaStream_t stream = (cudaStream_t) 0) {
    if (ws == nullptr) return 0;
    ws->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    if (stream != (cudaStream_t) 0) {
        ws->stream = stream;
        ws->owns_stream = 0;
        return 1;
    }
    if (cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess) return 0;
    ws->owns_stream = 1;
    return 1;
}

namespace detail {
inline std::size_t up256(std::size_t x) { return (x + 255u) / 256u * 256u; }
} // namespace detail

// Sizes the per-row outputs for `rows` x `group_count` and the feature masks
// for `cols`; buffers grow monotonically (mask_groups.cu:620-700).
inline int reserve(sparse_group_reduce_workspace *ws, unsigned int rows, unsigned int cols, unsigned int values,
                   unsigned int group_count) {
    if (ws == nullptr || group_count > CELLSHARD_MAX_MASK_GROUPS) return 0;
    if (rows > ws->rows_capacity || group_count > ws->group_capacity || ws->row_block == nullptr) {
        const unsigned int R = rows > ws->rows_capacity ? rows : ws->rows_capacity;
        const unsigned int G = group_count > ws->group_capacity ? group_count : ws->group_capacity;
        const std::size_t r4 = detail::up256((std::size_t) R * 4u + 4u), r1 = detail::up256((std::size_t) R + 1u);
        const std::size_t rg = detail::up256((std::size_t) R * G * 4u + 4u);
        void *p = nullptr;
        if (cudaMalloc(&p, 3u * r4 + r1 + 2u * rg) != cudaSuccess) return 0;
        if (ws->row_block) cudaFree(ws->row_block);
        ws->row_block = p;
        unsigned char *b = static_cast<unsigned char *>(p);
        ws->row_totals = reinterpret_cast<float *>(b);
        ws->detected_features = reinterpret_cast<unsigned int *>(b + r4);
        ws->max_values = reinterpret_cast<float *>(b + 2u * r4);
        ws->row_keep = b + 3u * r4;
        ws->group_counts = reinterpret_cast<float *>(b + 3u * r4 + r1);
        ws->group_percentages = reinterpret_cast<float *>(b + 3u * r4 + r1 + rg);
        ws->rows_capacity = R;
        ws->group_capacity = G;
    }
    if (cols > ws->cols_capacity || ws->feature_block == nullptr) {
        void *p = nullptr;
        if (cudaMalloc(&p, detail::up256((std::size_t) cols * 4u + 4u)) != cudaSuccess) return 0;
        if (ws->feature_block) {
            if (ws->cols_capacity != 0u)
                cudaMemcpy(p, ws->feature_block, (std::size_t) ws->cols_capacity * 4u, cudaMemcpyDeviceToDevice);
            cudaFree(ws->feature_block);
        }
        ws->feature_block = p;
        ws->feature_group_masks = static_cast<std::uint32_t *>(p);
        ws->cols_capacity = cols;
    }
    if (values > ws->values_capacity) ws->values_capacity = values;
    return 1;
}

inline int upload_feature_group_masks(sparse_group_reduce_workspace *ws, unsigned int cols,
                                      const std::uint32_t *host_masks) {
    if (ws == nullptr || host_masks == nullptr) return 0;
    if (!reserve(ws, ws->rows_capacity, cols, ws->values_capacity, ws->group_capacity)) return 0;
    return cudaMemcpy(ws->feature_group_masks, host_masks, (std::size_t) cols * 4u, cudaMemcpyHostToDevice) ==
           cudaSuccess;
}

namespace detail {
inline int bind(sparse_group_reduce_workspace *ws, unsigned int rows, unsigned int G,
                sparse_group_reduce_result *out) {
    out->rows = rows;
    out->group_count = G;
    out->row_totals = ws->row_totals;
    out->detected_features = ws->detected_features;
    out->max_values = ws->max_values;
    out->row_keep = ws->row_keep;
    out->group_counts = G ? ws->group_counts : nullptr;
    out->group_percentages = G ? ws->group_percentages : nullptr;
    return 1;
}

template <typename ViewT, typename CView, typename Fn>
inline int reduce(const ViewT *src, sparse_group_reduce_workspace *ws, const group_mask_config_view *groups,
                  const row_feature_mask_view *masks, const sparse_group_filter_params *filter,
                  sparse_group_reduce_result *out, unsigned int values, Fn fn) {
    if (src == nullptr || ws == nullptr || out == nullptr) return 0;
    const unsigned int G = groups ? groups->group_count : 0u;
    if (G > CELLSHARD_MAX_MASK_GROUPS || !reserve(ws, src->rows, src->cols, values, G)) return 0;
    const std::uint32_t *fm = G == 0u ? nullptr
                                      : (groups->feature_group_masks ? groups->feature_group_masks
                                                                     : ws->feature_group_masks);
    cs_group_reduce_out o{ws->row_totals, ws->detected_features, ws->max_values, ws->row_keep,
                          G ? ws->group_counts : nullptr, G ? ws->group_percentages : nullptr};
    static const row_feature_mask_view no_masks{nullptr, nullptr, nullptr, nullptr};
    if (!fn(reinterpret_cast<const CView *>(src), fm, G,
            reinterpret_cast<const cs_row_feature_mask_view *>(masks ? masks : &no_masks),
            reinterpret_cast<const cs_group_filter_params *>(filter), &o, reinterpret_cast<cs_stream_t>(ws->stream)))
        return 0;
    return bind(ws, src->rows, G, out);
}
} // namespace detail

inline int compute_sparse_group_reduce(const device::blocked_ell_view *src, sparse_group_reduce_workspace *ws,
                                       const group_mask_config_view *groups, const row_feature_mask_view *masks,
                                       const sparse_group_filter_params *filter, sparse_group_reduce_result *out) {
    return detail::reduce<device::blocked_ell_view, cs_blocked_ell_view>(
        src, ws, groups, masks, filter, out, src ? src->rows * src->ell_cols : 0u, cs_b200_group_reduce_blocked_ell);
}

inline int compute_sparse_group_reduce(const device::sliced_ell_view *src, sparse_group_reduce_workspace *ws,
                                       const group_mask_config_view *groups, const row_feature_mask_view *masks,
                                       const sparse_group_filter_params *filter, sparse_group_reduce_result *out) {
    return detail::reduce<device::sliced_ell_view, cs_sliced_ell_view>(src, ws, groups, masks, filter, out, 0u,
                                                                       cs_b200_group_reduce_sliced_ell);
}

inline int compute_sparse_group_reduce_compressed_fallback(const device::compressed_view *src,
                                                           sparse_group_reduce_workspace *ws,
                                                           const group_mask_config_view *groups,
                                                           const row_feature_mask_view *masks,
                                                           const sparse_group_filter_params *filter,
                                                           sparse_group_reduce_result *out) {
    return detail::reduce<device::compressed_view, cs_compressed_view>(src, ws, groups, masks, filter, out,
                                                                       src ? src->nnz : 0u,
                                                                       cs_b200_group_reduce_compressed);
}

inline void init(masked_sparse_reoptimize_workspace *ws) {
    std::memset(ws, 0, sizeof(*ws));
    ws->device = -1;
}

namespace detail {
struct reopt_private {
    void *scratch;
    std::size_t scratch_bytes;
    void *out_block;
    std::size_t out_bytes;
    std::uint32_t *status;
};
} // namespace detail

inline void clear(masked_sparse_reoptimize_workspace *ws) {
    if (ws == nullptr) return;
    auto *pv = static_cast<detail::reopt_private *>(ws->private_workspace);
    if (pv) {
        if (pv->scratch) cudaFree(pv->scratch);
        if (pv->out_block) cudaFree(pv->out_block);
        if (pv->status) cudaFree(pv->status);
        delete pv;
    }
    if (ws->owns_stream && ws->stream) cudaStreamDestroy(ws->stream);
    init(ws);
}

inline int setup(masked_sparse_reoptimize_workspace *ws, int device, cudaStream_t stream = (cudaStream_t) 0) {
    if (ws == nullptr) return 0;
    ws->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    if (stream != (cudaStream_t) 0) {
        ws->stream = stream;
        ws->owns_stream = 0;
    } else {
        if (cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess) return 0;
        ws->owns_stream = 1;
    }
    if (ws->private_workspace == nullptr) {
        auto *pv = new detail::reopt_private{};
        if (cudaMalloc((void **) &pv->status, 4) != cudaSuccess) {
            delete pv;
            return 0;
        }
        ws->private_workspace = pv;
    }
    return 1;
}

// Masked + remapped Blocked-ELL -> CSR.  Synchronises once to size the output
// (as the reference does); the result aliases the workspace.  Entries of an
// output row keep Blocked-ELL slot order; two kept rows remapped to one
// output row are rejected.
inline int manual_reoptimize_masked_sparse(const device::blocked_ell_view *src, const row_feature_mask_view *masks,
                                           const masked_sparse_reoptimize_config *config,
                                           masked_sparse_reoptimize_workspace *ws,
                                           masked_sparse_reoptimize_result *out) {
    if (src == nullptr || ws == nullptr || out == nullptr || ws->private_workspace == nullptr) return 0;
    auto *pv = static_cast<detail::reopt_private *>(ws->private_workspace);
    const unsigned int out_rows = config && config->output_rows ? config->output_rows : src->rows;
    const unsigned int out_cols = config && config->output_cols ? config->output_cols : src->cols;
    static const row_feature_mask_view no_masks{nullptr, nullptr, nullptr, nullptr};
    const auto *m = reinterpret_cast<const cs_row_feature_mask_view *>(masks ? masks : &no_masks);
    const auto *v = reinterpret_cast<const cs_blocked_ell_view *>(src);
    const cs_stream_t s = reinterpret_cast<cs_stream_t>(ws->stream);
    size_t need = 0;
    if (!cs_b200_reoptimize_scratch_bytes(src->rows, out_rows, &need)) return 0;
    const std::size_t ptr_bytes = detail::up256(((std::size_t) out_rows + 1u) * 4u);
    if (need + ptr_bytes > pv->scratch_bytes) {
        if (pv->scratch) cudaFree(pv->scratch);
        pv->scratch = nullptr;
        if (cudaMalloc(&pv->scratch, need + ptr_bytes) != cudaSuccess) return 0;
        pv->scratch_bytes = need + ptr_bytes;
    }
    auto *major = static_cast<std::uint32_t *>(pv->scratch);
    void *scr = static_cast<unsigned char *>(pv->scratch) + ptr_bytes;
    if (cudaMemsetAsync(pv->status, 0, 4, ws->stream) != cudaSuccess) return 0;
    if (!cs_b200_reoptimize_count(v, m, out_rows, out_cols, major, scr, need, pv->status, s)) return 0;
    std::uint32_t nnz = 0, status = 0;
    if (cudaMemcpyAsync(&nnz, major + out_rows, 4, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaMemcpyAsync(&status, pv->status, 4, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaStreamSynchronize(ws->stream) != cudaSuccess || status != 0u)
        return 0;
    const std::size_t need_out = ptr_bytes + detail::up256((std::size_t) nnz * 4u + 4u) +
                                 detail::up256((std::size_t) nnz * 2u + 2u);
    if (need_out > pv->out_bytes) {
        if (pv->out_block) cudaFree(pv->out_block);
        pv->out_block = nullptr;
        if (cudaMalloc(&pv->out_block, need_out) != cudaSuccess) return 0;
        pv->out_bytes = need_out;
    }
    unsigned char *ob = static_cast<unsigned char *>(pv->out_block);
    auto *optr = reinterpret_cast<std::uint32_t *>(ob);
    auto *oidx = reinterpret_cast<std::uint32_t *>(ob + ptr_bytes);
    auto *oval = reinterpret_cast<__half *>(ob + ptr_bytes + detail::up256((std::size_t) nnz * 4u + 4u));
    if (cudaMemcpyAsync(optr, major, ((std::size_t) out_rows + 1u) * 4u, cudaMemcpyDeviceToDevice, ws->stream) !=
            cudaSuccess ||
        !cs_b200_reoptimize_emit(v, m, out_rows, out_cols, optr, oidx, reinterpret_cast<uint16_t *>(oval), s))
        return 0;
    std::memset(out, 0, sizeof(*out));
    out->compressed = device::compressed_view{out_rows, out_cols, nnz, sparse::compressed_by_row, optr, oidx, oval};
    out->metadata.kept_rows = out_rows;
    out->metadata.kept_features = out_cols;
    out->metadata.live_nnz = nnz;
    const unsigned int rb = src->block_size ? (src->rows + src->block_size - 1u) / src->block_size : 0u;
    out->metadata.bytes_before = (unsigned long long) src->rows * src->ell_cols * 2ull +
                                 (unsigned long long) rb * (src->block_size ? src->ell_cols / src->block_size : 0u) *
                                     4ull;
    out->metadata.bytes_after = ((unsigned long long) out_rows + 1ull) * 4ull + (unsigned long long) nnz * 6ull;
    out->metadata.output_layout = sparse_mask_layout_compressed;
    return 1;
}

} // namespace runtime

// ---------------------------------------------------------------------------
// Execution bucketing of one partition (io/csh5/api.cuh:316-436,726-733)
// ---------------------------------------------------------------------------
struct bucketed_blocked_ell_partition {
    types::u32 rows;
    types::u32 cols;
    types::u32 nnz;
    types::u32 segment_count;
    sparse::blocked_ell *segments;
    types::u32 *segment_row_offsets;
    types::u32 *exec_to_canonical_rows;
    types::u32 *canonical_to_exec_rows;
    types::u32 *exec_to_canonical_cols;
    types::u32 *canonical_to_exec_cols;
};

struct bucketed_sliced_ell_partition {
    types::u32 rows;
    types::u32 cols;
    types::u32 nnz;
    types::u32 segment_count;
    sparse::sliced_ell *segments;
    types::u32 *segment_row_offsets;
    types::u32 *exec_to_canonical_rows;
    types::u32 *canonical_to_exec_rows;
    types::u32 canonical_slice_count;
    types::u32 *canonical_slice_row_offsets;
    types::u32 *canonical_slice_widths;
};

static_assert(sizeof(bucketed_blocked_ell_partition) == sizeof(cs_host_bucketed_blocked_ell) &&
                  offsetof(bucketed_blocked_ell_partition, canonical_to_exec_cols) ==
                      offsetof(cs_host_bucketed_blocked_ell, canonical_to_exec_cols),
              "bucketed_blocked_ell_partition layout");
static_assert(sizeof(bucketed_sliced_ell_partition) == sizeof(cs_host_bucketed_sliced_ell) &&
                  offsetof(bucketed_sliced_ell_partition, canonical_slice_widths) ==
                      offsetof(cs_host_bucketed_sliced_ell, canonical_slice_widths),
              "bucketed_sliced_ell_partition layout");

inline void init(bucketed_blocked_ell_partition *p) { std::memset(p, 0, sizeof(*p)); }
inline void init(bucketed_sliced_ell_partition *p) { std::memset(p, 0, sizeof(*p)); }
inline void clear(bucketed_blocked_ell_partition *p) {
    cs_b200_host_bucketed_blocked_ell_clear(reinterpret_cast<cs_host_bucketed_blocked_ell *>(p));
}
inline void clear(bucketed_sliced_ell_partition *p) {
    cs_b200_host_bucketed_sliced_ell_clear(reinterpret_cast<cs_host_bucketed_sliced_ell *>(p));
}

inline int build_bucketed_blocked_ell_partition(bucketed_blocked_ell_partition *out, const sparse::blocked_ell *part,
                                                std::uint32_t requested_bucket_count,
                                                std::uint64_t *bucketed_bytes_out) {
    return cs_b200_build_bucketed_blocked_ell_partition(reinterpret_cast<cs_host_bucketed_blocked_ell *>(out),
                                                        reinterpret_cast<const cs_host_blocked_ell *>(part),
                                                        requested_bucket_count, bucketed_bytes_out);
}

inline int build_bucketed_sliced_ell_partition(bucketed_sliced_ell_partition *out, const sparse::sliced_ell *part,
                                               std::uint32_t requested_bucket_count,
                                               std::uint64_t *bucketed_bytes_out) {
    return cs_b200_build_bucketed_sliced_ell_partition(reinterpret_cast<cs_host_bucketed_sliced_ell *>(out),
                                                       reinterpret_cast<const cs_host_sliced_ell *>(part),
                                                       requested_bucket_count, bucketed_bytes_out);
}

inline int choose_bucket_count_for_part(const sparse::blocked_ell *part, std::uint32_t *bucket_count_out,
                                        std::uint64_t *bucketed_bytes_out) {
    return cs_b200_choose_bucket_count_for_part(reinterpret_cast<const cs_host_blocked_ell *>(part), bucket_count_out,
                                                bucketed_bytes_out);
}

inline int choose_bucket_count_for_sliced_part(const sparse::sliced_ell *part, std::uint32_t *bucket_count_out,
                                               std::uint64_t *bucketed_bytes_out) {
    return cs_b200_choose_bucket_count_for_sliced_part(reinterpret_cast<const cs_host_sliced_ell *>(part),
                                                       bucket_count_out, bucketed_bytes_out);
}

namespace bucket {

// blocked_ell_bucket.cuh:11-29: the plan comes back to the host, the
// workspace owns a stream and grows its device buffers.
struct blocked_ell_bucket_plan {
    std::vector<std::uint32_t> row_block_order;
    std::vector<std::uint32_t> row_block_width_sorted;
};

struct blocked_ell_bucket_workspace {
    int device;
    cudaStream_t stream;
    std::uint32_t row_block_capacity;
    std::uint32_t slot_capacity;
    std::size_t sort_bytes;
    types::idx_t *d_block_col_idx;
    std::uint32_t *d_order;
    std::uint32_t *d_width_sorted;
    void *d_sort_tmp;
};

inline void init(blocked_ell_bucket_workspace *ws) {
    if (ws == nullptr) return;
    std::memset(ws, 0, sizeof(*ws));
    ws->device = -1;
}

inline void clear(blocked_ell_bucket_workspace *ws) {
    if (ws == nullptr) return;
    if (ws->device >= 0) cudaSetDevice(ws->device);
    cudaFree(ws->d_sort_tmp);
    cudaFree(ws->d_width_sorted);
    cudaFree(ws->d_order);
    cudaFree(ws->d_block_col_idx);
    if (ws->stream != nullptr) cudaStreamDestroy(ws->stream);
    init(ws);
}

inline int setup(blocked_ell_bucket_workspace *ws, int device) {
    if (ws == nullptr) return 0;
    init(ws);
    ws->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    return cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) == cudaSuccess;
}

// build_plan (blocked_ell_bucket.cuh:149-210): uploads the block column
// indices, orders the row blocks on the device and copies the plan back.
inline int build_plan(const sparse::blocked_ell *src, blocked_ell_bucket_workspace *ws,
                      blocked_ell_bucket_plan *out) {
    if (src == nullptr || ws == nullptr || out == nullptr || (src->rows != 0u && src->block_size == 0u)) return 0;
    const types::u32 rb = src->rows == 0u ? 0u : (src->rows + src->block_size - 1u) / src->block_size;
    const std::size_t slots = (std::size_t) rb * (src->block_size ? src->ell_cols / src->block_size : 0u);
    out->row_block_order.clear();
    out->row_block_width_sorted.clear();
    if (rb == 0u) return 1;
    if (cudaSetDevice(ws->device >= 0 ? ws->device : 0) != cudaSuccess) return 0;
    std::size_t need = 0u;
    if (!cs_b200_blocked_ell_bucket_plan_scratch_bytes(src->rows, src->block_size, &need)) return 0;
    if (slots > ws->slot_capacity) {
        cudaFree(ws->d_block_col_idx);
        ws->d_block_col_idx = nullptr;
        if (cudaMalloc((void **) &ws->d_block_col_idx, slots * 4u) != cudaSuccess) return 0;
        ws->slot_capacity = (std::uint32_t) slots;
    }
    if (rb > ws->row_block_capacity) {
        cudaFree(ws->d_order);
        cudaFree(ws->d_width_sorted);
        ws->d_order = ws->d_width_sorted = nullptr;
        if (cudaMalloc((void **) &ws->d_order, (std::size_t) rb * 4u) != cudaSuccess ||
            cudaMalloc((void **) &ws->d_width_sorted, (std::size_t) rb * 4u) != cudaSuccess)
            return 0;
        ws->row_block_capacity = rb;
    }
    if (need > ws->sort_bytes) {
        cudaFree(ws->d_sort_tmp);
        ws->d_sort_tmp = nullptr;
        if (cudaMalloc(&ws->d_sort_tmp, need) != cudaSuccess) return 0;
        ws->sort_bytes = need;
    }
    if (slots != 0u && cudaMemcpyAsync(ws->d_block_col_idx, src->blockColIdx, slots * 4u, cudaMemcpyHostToDevice,
                                       ws->stream) != cudaSuccess)
        return 0;
    const cs_blocked_ell_view v{src->rows, src->cols, src->nnz, src->block_size, src->ell_cols, ws->d_block_col_idx,
                                nullptr};
    if (!cs_b200_blocked_ell_bucket_plan(&v, ws->d_order, ws->d_width_sorted, ws->d_sort_tmp, ws->sort_bytes,
                                         ws->stream))
        return 0;
    out->row_block_order.resize(rb);
    out->row_block_width_sorted.resize(rb);
    return cudaMemcpyAsync(out->row_block_order.data(), ws->d_order, (std::size_t) rb * 4u, cudaMemcpyDeviceToHost,
                           ws->stream) == cudaSuccess &&
           cudaMemcpyAsync(out->row_block_width_sorted.data(), ws->d_width_sorted, (std::size_t) rb * 4u,
                           cudaMemcpyDeviceToHost, ws->stream) == cudaSuccess &&
           cudaStreamSynchronize(ws->stream) == cudaSuccess;
}

} // namespace bucket

namespace ingest {
namespace dataset {

// choose_bucket_count_for_part of the ingest path
// (ingest/internal/dataset/internal/convert_layout_support_part.hh:143-181).
inline int choose_bucket_count_for_part(const sparse::blocked_ell *part, int device, std::uint32_t *bucket_count_out) {
    return cs_b200_choose_ingest_bucket_count_for_part(reinterpret_cast<const cs_host_blocked_ell *>(part), device,
                                                       bucket_count_out);
}

} // namespace dataset
} // namespace ingest
} // namespace cellshard

#endif /* CELLSHARD_B200_HPP_ */
