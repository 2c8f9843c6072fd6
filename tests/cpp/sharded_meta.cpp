// The C++ shim's sharded<T> host helpers behind the same extern "C"
// signatures as oracle/ref_sharded_bridge.cu, so tests/test_sharded_meta.py
// can run both on the same partition tables on the CPU (no device work).
#include <cellshard_b200.hpp>

#include <cstddef>
#include <cstdlib>

using namespace cellshard;

extern "C" {

void cs_shim_sharded_layout(unsigned long *out) {
    typedef sharded<sparse::blocked_ell> S;
    out[0] = sizeof(S);
    out[1] = offsetof(S, parts);
    out[2] = offsetof(S, partition_offsets);
    out[3] = offsetof(S, partition_aux);
    out[4] = offsetof(S, num_shards);
    out[5] = offsetof(S, shard_offsets);
    out[6] = offsetof(S, shard_parts);
}

long cs_shim_shard_cuts(int mode, unsigned long n, const unsigned long *rows, const unsigned long *nnz,
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

void cs_shim_shard_queries(unsigned long n, const unsigned long *rows, const unsigned long *nnz,
                           const unsigned long *aux, unsigned long cols, unsigned long equal_shards,
                           unsigned long *part_of_row, unsigned long *shard_info, unsigned long *part_bytes) {
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
