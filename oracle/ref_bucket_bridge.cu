// TEST ORACLE ONLY -- never linked into libcellshard_b200.
//
// extern "C" bridge to the reference's own execution-bucketing builders,
// compiled from the read-only reference tree into oracle/_ref/
// libcs_ref_bucket.so by oracle/Makefile.  Nothing is copied: this file
// includes src/io/csh5/execution_internal.hh (which pulls in
// execution_builders_part.hh:1011-1596) and calls
//   build_bucketed_execution_partition (:1206), choose_bucket_count_for_part (:1249),
//   build_bucketed_sliced_execution_partition (:1529),
//   choose_bucket_count_for_sliced_part (:1572),
// and the .cspack store_*_raw functions of src/io/pack/packfile.cu.
// The header chain also reads and writes HDF5 files; oracle/ref_stub/hdf5.h
// stands in for <hdf5.h> so it compiles without the library (none of those
// paths is called).  The chain opens `namespace cellshard {` and leaves it
// open (the reference's .cc files close it), so the bridge functions sit
// inside it and close it at the end.
#include "src/io/csh5/execution_internal.hh"

#include "cellshard_b200.h"

#include <cstddef>
#include <cstring>

#define SAME_FIELD(A, B, fa, fb) static_assert(offsetof(A, fa) == offsetof(B, fb), #A "." #fa)

static_assert(sizeof(cs_host_bucketed_blocked_ell) == sizeof(bucketed_blocked_ell_partition), "bucketed bell size");
SAME_FIELD(cs_host_bucketed_blocked_ell, bucketed_blocked_ell_partition, segment_count, segment_count);
SAME_FIELD(cs_host_bucketed_blocked_ell, bucketed_blocked_ell_partition, segments, segments);
SAME_FIELD(cs_host_bucketed_blocked_ell, bucketed_blocked_ell_partition, canonical_to_exec_rows, canonical_to_exec_rows);
SAME_FIELD(cs_host_bucketed_blocked_ell, bucketed_blocked_ell_partition, canonical_to_exec_cols, canonical_to_exec_cols);
static_assert(sizeof(cs_host_bucketed_sliced_ell) == sizeof(bucketed_sliced_ell_partition), "bucketed sell size");
SAME_FIELD(cs_host_bucketed_sliced_ell, bucketed_sliced_ell_partition, segments, segments);
SAME_FIELD(cs_host_bucketed_sliced_ell, bucketed_sliced_ell_partition, canonical_to_exec_rows, canonical_to_exec_rows);
SAME_FIELD(cs_host_bucketed_sliced_ell, bucketed_sliced_ell_partition, canonical_slice_count, canonical_slice_count);
SAME_FIELD(cs_host_bucketed_sliced_ell, bucketed_sliced_ell_partition, canonical_slice_widths, canonical_slice_widths);
static_assert(sizeof(cs_host_blocked_ell) == sizeof(sparse::blocked_ell), "blocked_ell size");
static_assert(sizeof(cs_host_sliced_ell) == sizeof(sparse::sliced_ell), "sliced_ell size");

static void csrefb_bell(const cs_host_blocked_ell *s, sparse::blocked_ell *d) {
    sparse::init(d, s->rows, s->cols, s->nnz, s->block_size, s->ell_cols);
    d->blockColIdx = s->blockColIdx;
    d->val = reinterpret_cast<real::storage_t *>(s->val);
}

static void csrefb_sell(const cs_host_sliced_ell *s, sparse::sliced_ell *d) {
    sparse::init(d, s->rows, s->cols, s->nnz);
    d->slice_count = s->slice_count;
    d->slice_row_offsets = s->slice_row_offsets;
    d->slice_widths = s->slice_widths;
    d->col_idx = s->col_idx;
    d->val = reinterpret_cast<real::storage_t *>(s->val);
}

extern "C" int csrefb_build_bucketed_blocked_ell(const cs_host_blocked_ell *part, uint32_t requested,
                                                 cs_host_bucketed_blocked_ell *out, uint64_t *bytes) {
    sparse::blocked_ell p;
    bucketed_blocked_ell_partition o;
    std::uint64_t b = 0u;
    csrefb_bell(part, &p);
    init(&o);
    const int r = build_bucketed_execution_partition(&o, &p, requested, &b);
    std::memcpy(out, &o, sizeof(o));
    if (bytes != nullptr) *bytes = b;
    return r;
}

extern "C" void csrefb_clear_bucketed_blocked_ell(cs_host_bucketed_blocked_ell *out) {
    clear(reinterpret_cast<bucketed_blocked_ell_partition *>(out));
}

extern "C" int csrefb_choose_bucket_count_for_part(const cs_host_blocked_ell *part, uint32_t *count,
                                                   uint64_t *bytes) {
    sparse::blocked_ell p;
    std::uint64_t b = 0u;
    csrefb_bell(part, &p);
    const int r = choose_bucket_count_for_part(&p, count, &b);
    *bytes = b;
    return r;
}

extern "C" int csrefb_build_bucketed_sliced_ell(const cs_host_sliced_ell *part, uint32_t requested,
                                                cs_host_bucketed_sliced_ell *out, uint64_t *bytes) {
    sparse::sliced_ell p;
    bucketed_sliced_ell_partition o;
    std::uint64_t b = 0u;
    csrefb_sell(part, &p);
    init(&o);
    const int r = build_bucketed_sliced_execution_partition(&o, &p, requested, &b);
    std::memcpy(out, &o, sizeof(o));
    if (bytes != nullptr) *bytes = b;
    return r;
}

extern "C" void csrefb_clear_bucketed_sliced_ell(cs_host_bucketed_sliced_ell *out) {
    clear(reinterpret_cast<bucketed_sliced_ell_partition *>(out));
}

extern "C" int csrefb_choose_bucket_count_for_sliced_part(const cs_host_sliced_ell *part, uint32_t *count,
                                                          uint64_t *bytes) {
    sparse::sliced_ell p;
    std::uint64_t b = 0u;
    csrefb_sell(part, &p);
    const int r = choose_bucket_count_for_sliced_part(&p, count, &b);
    *bytes = b;
    return r;
}

// .cspack raw records written by the reference's own codec (src/io/pack/packfile.cu),
// fp16 values.
extern "C" int csrefb_store_blocked_ell_raw(const char *path, uint32_t rows, uint32_t cols, uint32_t nnz,
                                            uint32_t block_size, uint32_t ell_cols, const uint32_t *bci,
                                            const uint16_t *val) {
    return store_blocked_ell_raw(path, rows, cols, nnz, block_size, ell_cols, bci, val, 2u);
}

extern "C" int csrefb_store_sliced_ell_raw(const char *path, uint32_t rows, uint32_t cols, uint32_t nnz,
                                           uint32_t slice_count, const uint32_t *offsets, const uint32_t *widths,
                                           const uint32_t *col_idx, const uint16_t *val) {
    return store_sliced_ell_raw(path, rows, cols, nnz, slice_count, offsets, widths, col_idx, val, 2u);
}

extern "C" int csrefb_store_compressed_raw(const char *path, uint32_t rows, uint32_t cols, uint32_t nnz,
                                           uint32_t axis, const uint32_t *ptr, const uint32_t *idx,
                                           const uint16_t *val) {
    const uint32_t major = axis == sparse::compressed_by_col ? cols : rows;
    return store_compressed_raw(path, rows, cols, nnz, axis, major, ptr, idx, val, 2u);
}

extern "C" int csrefb_store_coo_raw(const char *path, uint32_t rows, uint32_t cols, uint32_t nnz,
                                    const uint32_t *row, const uint32_t *col, const uint16_t *val) {
    return store_coo_raw(path, rows, cols, nnz, row, col, val, 2u);
}

// The public entry point the reference defines in src/io/csh5/runtime/fetch.cc:332-337
// (a one-line forward to build_bucketed_execution_partition); that file needs the
// whole .csh5 runtime, so the ingest bridge links this forward instead.
int build_bucketed_blocked_ell_partition(bucketed_blocked_ell_partition *out, const sparse::blocked_ell *part,
                                         std::uint32_t requested_bucket_count, std::uint64_t *bucketed_bytes_out) {
    return build_bucketed_execution_partition(out, part, requested_bucket_count, bucketed_bytes_out);
}

} // namespace cellshard (opened by the reference's header chain)
