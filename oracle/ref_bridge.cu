// TEST ORACLE ONLY -- never linked into libcellshard_b200.
//
// extern "C" bridge to the reference's own host conversion code, compiled
// from the read-only reference tree (-I <reference>) into oracle/_ref/
// libcs_ref.so by oracle/Makefile.  Nothing is copied: this file only calls
// convert::blocked_ell_from_compressed (src/convert/blocked_ell_from_compressed.cuh:258),
// convert::choose_blocked_ell_block_size (:157),
// convert::sliced_ell_from_compressed (src/convert/sliced_ell_from_compressed.cuh:96),
// convert::choose_sliced_ell_slice_rows_from_compressed (:86),
// convert::sliced_ell_from_blocked_ell (src/convert/sliced_ell_from_blocked_ell.cuh:233) and
// convert::choose_sliced_ell_slice_rows_from_blocked_ell (:223),
// convert::blocked_ell_from_coo (src/convert/blocked_ell_from_compressed.cuh:349) and
// convert::choose_blocked_ell_block_size_from_coo (:192).
// The static_asserts pin the C ABI structs of include/cellshard_b200.h to the
// reference's format structs and device views, field for field.
#include "src/convert/blocked_ell_from_compressed.cuh"
#include "src/convert/sliced_ell_from_compressed.cuh"
#include "src/convert/sliced_ell_from_blocked_ell.cuh"

#include "cellshard_b200.h"

#include <cstddef>
#include <cstdlib>
#include <cstring>

using namespace cellshard;

#define SAME_FIELD(A, B, fa, fb) static_assert(offsetof(A, fa) == offsetof(B, fb), #A "." #fa)

static_assert(sizeof(cs_host_compressed) == sizeof(sparse::compressed), "compressed size");
SAME_FIELD(cs_host_compressed, sparse::compressed, rows, rows);
SAME_FIELD(cs_host_compressed, sparse::compressed, flags, flags);
SAME_FIELD(cs_host_compressed, sparse::compressed, storage, storage);
SAME_FIELD(cs_host_compressed, sparse::compressed, majorPtr, majorPtr);
SAME_FIELD(cs_host_compressed, sparse::compressed, minorIdx, minorIdx);
SAME_FIELD(cs_host_compressed, sparse::compressed, val, val);
static_assert(sizeof(cs_host_blocked_ell) == sizeof(sparse::blocked_ell), "blocked_ell size");
SAME_FIELD(cs_host_blocked_ell, sparse::blocked_ell, ell_cols, ell_cols);
SAME_FIELD(cs_host_blocked_ell, sparse::blocked_ell, storage, storage);
SAME_FIELD(cs_host_blocked_ell, sparse::blocked_ell, blockColIdx, blockColIdx);
SAME_FIELD(cs_host_blocked_ell, sparse::blocked_ell, val, val);
static_assert(sizeof(cs_host_sliced_ell) == sizeof(sparse::sliced_ell), "sliced_ell size");
SAME_FIELD(cs_host_sliced_ell, sparse::sliced_ell, slice_count, slice_count);
SAME_FIELD(cs_host_sliced_ell, sparse::sliced_ell, storage, storage);
SAME_FIELD(cs_host_sliced_ell, sparse::sliced_ell, slice_row_offsets, slice_row_offsets);
SAME_FIELD(cs_host_sliced_ell, sparse::sliced_ell, slice_widths, slice_widths);
SAME_FIELD(cs_host_sliced_ell, sparse::sliced_ell, col_idx, col_idx);
SAME_FIELD(cs_host_sliced_ell, sparse::sliced_ell, val, val);
static_assert(sizeof(cs_compressed_view) == sizeof(device::compressed_view), "compressed_view size");
SAME_FIELD(cs_compressed_view, device::compressed_view, majorPtr, majorPtr);
SAME_FIELD(cs_compressed_view, device::compressed_view, val, val);
static_assert(sizeof(cs_blocked_ell_view) == sizeof(device::blocked_ell_view), "blocked_ell_view size");
SAME_FIELD(cs_blocked_ell_view, device::blocked_ell_view, ell_cols, ell_cols);
SAME_FIELD(cs_blocked_ell_view, device::blocked_ell_view, blockColIdx, blockColIdx);
SAME_FIELD(cs_blocked_ell_view, device::blocked_ell_view, val, val);
static_assert(sizeof(cs_sliced_ell_view) == sizeof(device::sliced_ell_view), "sliced_ell_view size");
SAME_FIELD(cs_sliced_ell_view, device::sliced_ell_view, slice_rows, slice_rows);
SAME_FIELD(cs_sliced_ell_view, device::sliced_ell_view, slice_slot_offsets, slice_slot_offsets);
SAME_FIELD(cs_sliced_ell_view, device::sliced_ell_view, val, val);
static_assert(sizeof(cs_blocked_ell_tune_result) == sizeof(convert::blocked_ell_tune_result), "tune size");
static_assert(sizeof(cs_host_coo) == sizeof(sparse::coo), "coo size");
SAME_FIELD(cs_host_coo, sparse::coo, storage, storage);
SAME_FIELD(cs_host_coo, sparse::coo, rowIdx, rowIdx);
SAME_FIELD(cs_host_coo, sparse::coo, val, val);
static_assert(sizeof(cs_coo_view) == sizeof(device::coo_view), "coo_view size");
SAME_FIELD(cs_coo_view, device::coo_view, rowIdx, rowIdx);
SAME_FIELD(cs_coo_view, device::coo_view, val, val);
static_assert(sizeof(cs_sliced_ell_tune_result) == sizeof(convert::sliced_ell_tune_result), "tune size");
SAME_FIELD(cs_sliced_ell_tune_result, convert::sliced_ell_tune_result, score, score);

namespace {

void to_ref(const cs_host_compressed *s, sparse::compressed *d) {
    sparse::init(d, s->rows, s->cols, s->nnz, s->axis);
    d->majorPtr = s->majorPtr;
    d->minorIdx = s->minorIdx;
    d->val = reinterpret_cast<real::storage_t *>(s->val);
}

void to_ref_bell(const cs_host_blocked_ell *s, sparse::blocked_ell *d) {
    sparse::init(d, s->rows, s->cols, s->nnz, s->block_size, s->ell_cols);
    d->blockColIdx = s->blockColIdx;
    d->val = reinterpret_cast<real::storage_t *>(s->val);
}

void from_ref_sliced(const sparse::sliced_ell &d, cs_host_sliced_ell *dst) {
    dst->rows = d.rows;
    dst->cols = d.cols;
    dst->nnz = d.nnz;
    dst->slice_count = d.slice_count;
    dst->flags = d.flags;
    dst->storage = d.storage;
    dst->slice_row_offsets = d.slice_row_offsets;
    dst->slice_widths = d.slice_widths;
    dst->col_idx = d.col_idx;
    dst->val = reinterpret_cast<uint16_t *>(d.val);
}

void from_ref_tune(const convert::sliced_ell_tune_result &r, cs_sliced_ell_tune_result *out) {
    out->slice_rows = r.slice_rows;
    out->slice_count = r.slice_count;
    out->padded_slots = r.padded_slots;
    out->padded_bytes = r.padded_bytes;
    out->storage_ratio = r.storage_ratio;
    out->slice_penalty = r.slice_penalty;
    out->score = r.score;
}

} // namespace

extern "C" {

int csref_sliced_ell_from_blocked_ell(const cs_host_blocked_ell *src, unsigned int slice_rows,
                                      cs_host_sliced_ell *dst) {
    sparse::blocked_ell s;
    to_ref_bell(src, &s);
    sparse::sliced_ell d;
    sparse::init(&d);
    const int ok = convert::sliced_ell_from_blocked_ell(&s, slice_rows, &d);
    from_ref_sliced(d, dst);
    return ok;
}

int csref_choose_sliced_ell_slice_rows_from_blocked_ell(const cs_host_blocked_ell *src,
                                                        const unsigned int *candidates, unsigned int count,
                                                        cs_sliced_ell_tune_result *out) {
    sparse::blocked_ell s;
    to_ref_bell(src, &s);
    convert::sliced_ell_tune_result r{};
    const int ok = convert::choose_sliced_ell_slice_rows_from_blocked_ell(&s, candidates, count, &r);
    from_ref_tune(r, out);
    return ok;
}

int csref_blocked_ell_from_compressed(const cs_host_compressed *src, unsigned int block_size,
                                      cs_host_blocked_ell *dst) {
    sparse::compressed s;
    to_ref(src, &s);
    sparse::blocked_ell d;
    sparse::init(&d);
    const int ok = convert::blocked_ell_from_compressed(&s, block_size, &d);
    dst->rows = d.rows;
    dst->cols = d.cols;
    dst->nnz = d.nnz;
    dst->block_size = d.block_size;
    dst->ell_cols = d.ell_cols;
    dst->flags = d.flags;
    dst->storage = d.storage;
    dst->blockColIdx = d.blockColIdx;
    dst->val = reinterpret_cast<uint16_t *>(d.val);
    return ok;
}

int csref_choose_blocked_ell_block_size(const cs_host_compressed *src, const unsigned int *candidates,
                                        unsigned int count, cs_blocked_ell_tune_result *out) {
    sparse::compressed s;
    to_ref(src, &s);
    convert::blocked_ell_tune_result r{};
    const int ok = convert::choose_blocked_ell_block_size(&s, candidates, count, &r);
    out->block_size = r.block_size;
    out->fill_ratio = r.fill_ratio;
    out->padded_bytes = r.padded_bytes;
    return ok;
}

int csref_sliced_ell_from_compressed(const cs_host_compressed *src, unsigned int slice_rows,
                                     cs_host_sliced_ell *dst) {
    sparse::compressed s;
    to_ref(src, &s);
    sparse::sliced_ell d;
    sparse::init(&d);
    const int ok = convert::sliced_ell_from_compressed(&s, slice_rows, &d);
    dst->rows = d.rows;
    dst->cols = d.cols;
    dst->nnz = d.nnz;
    dst->slice_count = d.slice_count;
    dst->flags = d.flags;
    dst->storage = d.storage;
    dst->slice_row_offsets = d.slice_row_offsets;
    dst->slice_widths = d.slice_widths;
    dst->col_idx = d.col_idx;
    dst->val = reinterpret_cast<uint16_t *>(d.val);
    return ok;
}

int csref_choose_sliced_ell_slice_rows_from_compressed(const cs_host_compressed *src, const unsigned int *candidates,
                                                       unsigned int count, cs_sliced_ell_tune_result *out) {
    sparse::compressed s;
    to_ref(src, &s);
    convert::sliced_ell_tune_result r{};
    const int ok = convert::choose_sliced_ell_slice_rows_from_compressed(&s, candidates, count, &r);
    out->slice_rows = r.slice_rows;
    out->slice_count = r.slice_count;
    out->padded_slots = r.padded_slots;
    out->padded_bytes = r.padded_bytes;
    out->storage_ratio = r.storage_ratio;
    out->slice_penalty = r.slice_penalty;
    out->score = r.score;
    return ok;
}

unsigned int csref_sliced_total_slots(const cs_host_sliced_ell *m) {
    unsigned int total = 0u;
    for (unsigned int s = 0; s < m->slice_count; ++s)
        total += (m->slice_row_offsets[s + 1u] - m->slice_row_offsets[s]) * m->slice_widths[s];
    return total;
}

void csref_free(void *p) { std::free(p); }

int csref_blocked_ell_from_coo(const cs_host_coo *src, uint32_t cols, const uint32_t *feature_to_global,
                               unsigned int block_size, cs_host_blocked_ell *dst) {
    sparse::coo s;
    std::memcpy(&s, src, sizeof(s));
    s.storage = nullptr;
    sparse::blocked_ell d;
    sparse::init(&d);
    const int ok = convert::blocked_ell_from_coo(&s, cols, feature_to_global, block_size, &d);
    std::memcpy(dst, &d, sizeof(d));
    return ok;
}

int csref_choose_blocked_ell_block_size_from_coo(const cs_host_coo *src, uint32_t cols,
                                                 const uint32_t *feature_to_global, const unsigned int *candidates,
                                                 unsigned int count, cs_blocked_ell_tune_result *out) {
    sparse::coo s;
    std::memcpy(&s, src, sizeof(s));
    s.storage = nullptr;
    convert::blocked_ell_tune_result r{};
    const int ok = convert::choose_blocked_ell_block_size_from_coo(&s, cols, feature_to_global, candidates, count, &r);
    out->block_size = r.block_size;
    out->fill_ratio = r.fill_ratio;
    out->padded_bytes = r.padded_bytes;
    return ok;
}

} // extern "C"
