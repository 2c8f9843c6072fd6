// TEST ORACLE ONLY -- never linked into libcellshard_b200.
//
// extern "C" bridge to the reference's ingest-time bucket-count chooser,
// compiled from the read-only reference tree into oracle/_ref/
// libcs_ref_ingest.so by oracle/Makefile.  Nothing is copied: this file
// includes include/CellShard/ingest/internal/dataset/dataset_ingest.cuh and
// calls
//   bucket::build_plan (src/bucket/operators/blocked_ell_bucket.cuh:149-210,
//     row blocks sorted on the GPU by (valid width << 32 | hash of block columns)),
//   estimate_bucketed_bytes_from_gpu_plan and choose_bucket_count_for_part
//     (include/CellShard/ingest/internal/dataset/internal/convert_layout_support_part.hh:116-181).
// The chain also reads .h5ad files; oracle/ref_stub/hdf5.h stands in for
// <hdf5.h> (none of those paths is called).  build_plan runs on the GPU.
#include "include/CellShard/ingest/internal/dataset/dataset_ingest.cuh"

#include "cellshard_b200.h"

#include <cstring>

namespace {

void csrefi_bell(const cs_host_blocked_ell *s, cellshard::sparse::blocked_ell *d) {
    cellshard::sparse::init(d, s->rows, s->cols, s->nnz, s->block_size, s->ell_cols);
    d->blockColIdx = s->blockColIdx;
    d->val = reinterpret_cast<real::storage_t *>(s->val);
}

} // namespace

extern "C" int csrefi_bucket_plan(const cs_host_blocked_ell *part, uint32_t *order, uint32_t *width_sorted) {
    cellshard::sparse::blocked_ell p;
    cellshard::bucket::blocked_ell_bucket_workspace ws;
    cellshard::bucket::blocked_ell_bucket_plan plan;
    csrefi_bell(part, &p);
    cellshard::bucket::init(&ws);
    int ok = cellshard::bucket::setup(&ws, 0) && cellshard::bucket::build_plan(&p, &ws, &plan);
    if (ok) {
        std::memcpy(order, plan.row_block_order.data(), plan.row_block_order.size() * 4u);
        std::memcpy(width_sorted, plan.row_block_width_sorted.data(), plan.row_block_width_sorted.size() * 4u);
    }
    cellshard::bucket::clear(&ws);
    return ok;
}

extern "C" unsigned long long csrefi_estimate_bucketed_bytes(const cs_host_blocked_ell *part, const uint32_t *order,
                                                             const uint32_t *width_sorted, uint32_t row_blocks,
                                                             uint32_t bucket_count) {
    cellshard::sparse::blocked_ell p;
    cellshard::bucket::blocked_ell_bucket_plan plan;
    csrefi_bell(part, &p);
    plan.row_block_order.assign(order, order + row_blocks);
    plan.row_block_width_sorted.assign(width_sorted, width_sorted + row_blocks);
    return cellshard::ingest::dataset::estimate_bucketed_bytes_from_gpu_plan(&p, plan, bucket_count);
}

extern "C" int csrefi_choose_bucket_count_for_part(const cs_host_blocked_ell *part, uint32_t *count) {
    cellshard::sparse::blocked_ell p;
    csrefi_bell(part, &p);
    return cellshard::ingest::dataset::choose_bucket_count_for_part(&p, 0, count);
}
