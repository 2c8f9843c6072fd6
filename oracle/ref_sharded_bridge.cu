// TEST ORACLE ONLY -- never linked into libcellshard_b200.
//
// extern "C" bridge to the reference's own sharded<T> host helpers
// (include/CellShard/runtime/layout/sharded.cuh, runtime/host/sharded_host.cuh)
// and its device staging state types (runtime/device/sharded_device.cuh),
// compiled from the read-only reference tree into oracle/_ref/
// libcs_ref_sharded.so by oracle/Makefile.  Only host code runs: the shard
// cut rules (set_equal_shards, set_shards_by_nnz, set_shards_by_part_bytes,
// build_shard_offsets_by_rows, reshard) and the row -> partition lookups, on
// metadata-only partitions (define_partitions), so the C++ shim's restated
// helpers can be compared with them on the CPU.  The header chain reaches the
// .csh5 API, whose HDF5 names oracle/ref_stub/hdf5.h stands in for.
#include "include/CellShard/runtime/device/sharded_device.cuh"

#include "cellshard_b200.h"

#include <cstddef>
#include <cstdlib>

using namespace cellshard;

#define SAME_FIELD(A, B, fa, fb) static_assert(offsetof(A, fa) == offsetof(B, fb), #A "." #fa)

// the C ABI staging structs are field for field the reference's
typedef device::partition_record<sparse::blocked_ell> ref_record;
typedef device::sharded_device<sparse::blocked_ell> ref_state;
static_assert(sizeof(cs_staged_part) == sizeof(ref_record), "partition_record size");
SAME_FIELD(cs_staged_part, ref_record, allocation, allocation);
SAME_FIELD(cs_staged_part, ref_record, allocation_bytes, allocation_bytes);
SAME_FIELD(cs_staged_part, ref_record, storage, storage);
SAME_FIELD(cs_staged_part, ref_record, view, view);
SAME_FIELD(cs_staged_part, ref_record, a0, a0);
SAME_FIELD(cs_staged_part, ref_record, a3, a3);
SAME_FIELD(cs_staged_part, ref_record, group_begin, group_begin);
SAME_FIELD(cs_staged_part, ref_record, group_end, group_end);
SAME_FIELD(cs_staged_part, ref_record, device_id, device_id);
static_assert(sizeof(cs_cached_allocation) == sizeof(device::cached_allocation), "cached_allocation size");
SAME_FIELD(cs_cached_allocation, device::cached_allocation, bytes, bytes);
SAME_FIELD(cs_cached_allocation, device::cached_allocation, device_id, device_id);
static_assert(sizeof(cs_sharded_device) == sizeof(ref_state), "sharded_device size");
SAME_FIELD(cs_sharded_device, ref_state, parts, parts);
SAME_FIELD(cs_sharded_device, ref_state, cache_count, cache_count);
SAME_FIELD(cs_sharded_device, ref_state, cache_capacity, cache_capacity);
SAME_FIELD(cs_sharded_device, ref_state, cache, cache);

extern "C" {

// sizeof and field offsets of sharded<blocked_ell>, for the shim's layout check
void csref_sharded_layout(unsigned long *out) {
    typedef sharded<sparse::blocked_ell> S;
    out[0] = sizeof(S);
    out[1] = offsetof(S, parts);
    out[2] = offsetof(S, partition_offsets);
    out[3] = offsetof(S, partition_aux);
    out[4] = offsetof(S, num_shards);
    out[5] = offsetof(S, shard_offsets);
    out[6] = offsetof(S, shard_parts);
}

// mode 0 set_equal_shards(param), 1 set_shards_by_nnz(param),
// 2 set_shards_by_part_bytes(param), 3 build_shard_offsets_by_rows(param),
// 4 reshard(param shards, offsets given in out_offsets).  Partitions are
// Blocked-ELL metadata (rows, nnz, aux).  Writes shard offsets and, for
// modes 0-2 and 4, shard_parts; returns the shard count, or -1 on failure.
long csref_shard_cuts(int mode, unsigned long n, const unsigned long *rows, const unsigned long *nnz,
                      const unsigned long *aux, unsigned long cols, unsigned long param, unsigned long *out_offsets,
                      unsigned long *out_parts) {
    sharded<sparse::blocked_ell> m;
    init(&m);
    if (!define_partitions(&m, cols, n, rows, nnz, aux)) return -1;
    long count = -1;
    if (mode == 0 && set_equal_shards(&m, param)) count = (long) m.num_shards;
    if (mode == 1 && set_shards_by_nnz(&m, param)) count = (long) m.num_shards;
    if (mode == 2 && set_shards_by_part_bytes(&m, param)) count = (long) m.num_shards;
    if (mode == 3) {
        unsigned long *o = nullptr, c = 0;
        if (build_shard_offsets_by_rows(&m, param, &o, &c)) {
            for (unsigned long i = 0; o != nullptr && i <= c; ++i) out_offsets[i] = o[i];
            count = (long) c;
        }
        std::free(o);
        clear(&m);
        return count;
    }
    if (mode == 4) count = reshard(&m, param, out_offsets) ? (long) m.num_shards : -1;
    if (count >= 0) {
        for (unsigned long i = 0; i <= (unsigned long) count; ++i) {
            out_offsets[i] = m.shard_offsets[i];
            out_parts[i] = m.shard_parts[i];
        }
    }
    clear(&m);
    return count;
}

// per row: find_partition; per shard: first/last partition, rows, nnz; per
// partition: partition_bytes (set_shards_to_partitions after the cuts of mode 0)
void csref_shard_queries(unsigned long n, const unsigned long *rows, const unsigned long *nnz, const unsigned long *aux,
                         unsigned long cols, unsigned long equal_shards, unsigned long *part_of_row,
                         unsigned long *shard_info, unsigned long *part_bytes) {
    sharded<sparse::blocked_ell> m;
    init(&m);
    define_partitions(&m, cols, n, rows, nnz, aux);
    set_equal_shards(&m, equal_shards);
    for (unsigned long r = 0; r <= m.rows; ++r) part_of_row[r] = find_partition(&m, r);
    for (unsigned long s = 0; s < m.num_shards; ++s) {
        shard_info[4 * s + 0] = first_partition_in_shard(&m, s);
        shard_info[4 * s + 1] = last_partition_in_shard(&m, s);
        shard_info[4 * s + 2] = rows_in_shard(&m, s);
        shard_info[4 * s + 3] = nnz_in_shard(&m, s);
    }
    for (unsigned long p = 0; p < n; ++p) part_bytes[p] = partition_bytes(&m, p);
    clear(&m);
}

} // extern "C"
