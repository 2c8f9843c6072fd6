// Drives the C++ shim (include/cellshard_b200.hpp) the way reference host
// code drives the reference API: stage host partitions with device::upload
// and whole shards of a sharded<T> through a sharded_device<T> (upload_shard,
// swap_shard, stage_partition, the allocation cache),
// run runtime::compute_sparse_group_reduce over Blocked-ELL, Sliced-ELL and
// compressed views, runtime::manual_reoptimize_masked_sparse, the
// convert:: host conversion and chooser, bucket::build_bucketed_major_view and
// convert::build_compressed_transpose_raw.  Inputs come from a text file of
// lines "name v0 v1 ..."; every result is printed as "name v0 v1 ..." for the
// pytest wrapper (tests/test_gpu_cpp_shim.py) to compare.
#include <cellshard_b200.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace cs = ::cellshard;

namespace {

std::map<std::string, std::vector<double>> read_inputs(const char *path) {
    std::map<std::string, std::vector<double>> m;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string key;
        if (!(is >> key)) continue;
        double v;
        while (is >> v) m[key].push_back(v);
        m[key];
    }
    return m;
}

template <typename T>
std::vector<T> as(const std::vector<double> &v) {
    return std::vector<T>(v.begin(), v.end());
}

std::vector<__half> halves(const std::vector<double> &v) {
    std::vector<__half> h(v.size());
    for (size_t i = 0; i < v.size(); ++i) h[i] = __float2half((float) v[i]);
    return h;
}

template <typename T>
void print_dev(const char *name, const T *d, size_t n) {
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    std::printf("%s", name);
    for (size_t i = 0; i < n; ++i) std::printf(" %.9g", (double) h[i]);
    std::printf("\n");
}

void print_dev_half(const char *name, const __half *d, size_t n) {
    std::vector<__half> h(n);
    if (n) cudaMemcpy(h.data(), d, n * sizeof(__half), cudaMemcpyDeviceToHost);
    std::printf("%s", name);
    for (size_t i = 0; i < n; ++i) std::printf(" %.9g", (double) __half2float(h[i]));
    std::printf("\n");
}

template <typename T>
T *to_device(const std::vector<T> &v) {
    T *d = nullptr;
    cudaMalloc((void **) &d, v.size() * sizeof(T) + 16);
    if (!v.empty()) cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

template <typename T>
void print_host(const std::string &name, const T *v, size_t n) {
    std::printf("%s", name.c_str());
    for (size_t i = 0; i < n; ++i) std::printf(" %.9g", (double) v[i]);
    std::printf("\n");
}

void print_host_half(const std::string &name, const __half *v, size_t n) {
    std::printf("%s", name.c_str());
    for (size_t i = 0; i < n; ++i) std::printf(" %.9g", (double) __half2float(v[i]));
    std::printf("\n");
}

struct lcg {
    std::uint32_t s;
    std::uint32_t next() {
        s = s * 1664525u + 1013904223u;
        return s >> 8;
    }
};

// A Blocked-ELL host partition owning one malloc'd block (as sparse::allocate
// packs it), so cellshard::clear(sharded*) can destroy it: random ascending
// block columns per row block with trailing padding, about a third of the
// valid cells nonzero.
cs::sparse::blocked_ell *make_bell_part(lcg &g, unsigned rows, unsigned cols, unsigned B, unsigned W) {
    auto *m = new cs::sparse::blocked_ell;
    cs::sparse::init(m);
    const unsigned rb = (rows + B - 1u) / B, nb = (cols + B - 1u) / B;
    const std::size_t ib = (std::size_t) rb * W * 4u, vb = (std::size_t) rows * W * B * 2u;
    char *st = static_cast<char *>(std::malloc(ib + vb + 16u));
    m->rows = rows;
    m->cols = cols;
    m->block_size = B;
    m->ell_cols = W * B;
    m->storage = st;
    m->blockColIdx = reinterpret_cast<cs::types::idx_t *>(st);
    m->val = reinterpret_cast<__half *>(st + ib);
    for (unsigned r = 0; r < rb; ++r) {
        const unsigned valid = 1u + g.next() % W;
        unsigned c = g.next() % 3u;
        for (unsigned k = 0; k < W; ++k) {
            unsigned bc = 0xffffffffu;
            if (k < valid && c < nb) {
                bc = c;
                c += 1u + g.next() % 3u;
            }
            m->blockColIdx[(std::size_t) r * W + k] = bc;
        }
    }
    for (unsigned r = 0; r < rows; ++r)
        for (unsigned k = 0; k < W * B; ++k) {
            const unsigned bc = m->blockColIdx[(std::size_t) (r / B) * W + k / B];
            float v = 0.0f;
            if (bc != 0xffffffffu && bc * B + k % B < cols && g.next() % 3u == 0u) v = (float) (1u + g.next() % 7u);
            m->val[(std::size_t) r * W * B + k] = __float2half(v);
            m->nnz += v != 0.0f ? 1u : 0u;
        }
    return m;
}

// The same kind of matrix as a compressed partition (sorted distinct columns).
cs::sparse::compressed *make_csr_part(lcg &g, unsigned rows, unsigned cols) {
    auto *m = new cs::sparse::compressed;
    cs::sparse::init(m);
    std::vector<unsigned> ptr(rows + 1u, 0u), idx;
    std::vector<__half> val;
    for (unsigned r = 0; r < rows; ++r) {
        for (unsigned c = g.next() % 4u; c < cols; c += 1u + g.next() % 6u) {
            idx.push_back(c);
            val.push_back(__float2half((float) (1u + g.next() % 9u)));
        }
        ptr[r + 1u] = (unsigned) idx.size();
    }
    const std::size_t pb = (rows + 1u) * 4u, ib = idx.size() * 4u, vb = val.size() * 2u;
    char *st = static_cast<char *>(std::malloc(pb + ib + vb + 16u));
    m->rows = rows;
    m->cols = cols;
    m->nnz = (unsigned) idx.size();
    m->axis = cs::sparse::compressed_by_row;
    m->storage = st;
    m->majorPtr = reinterpret_cast<cs::types::ptr_t *>(st);
    m->minorIdx = reinterpret_cast<cs::types::idx_t *>(st + pb);
    m->val = reinterpret_cast<__half *>(st + pb + ib);
    std::memcpy(m->majorPtr, ptr.data(), pb);
    std::memcpy(m->minorIdx, idx.data(), ib);
    std::memcpy(m->val, val.data(), vb);
    return m;
}

int fail(int code, const char *what) {
    std::fprintf(stderr, "%s failed: %s\n", what, cs_b200_last_error());
    return code;
}

} // namespace

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    auto in = read_inputs(argv[1]);
    const unsigned rows = (unsigned) in["rows"][0], cols = (unsigned) in["cols"][0];
    auto group_masks = as<std::uint32_t>(in["group_masks"]);
    auto row_keep = as<unsigned char>(in["row_keep"]);
    auto feature_keep = as<unsigned char>(in["feature_keep"]);
    unsigned char *d_rk = to_device(row_keep), *d_fk = to_device(feature_keep);

    cs::runtime::sparse_group_reduce_workspace ws;
    cs::runtime::init(&ws);
    if (!cs::runtime::setup(&ws, 0)) return fail(3, "setup");
    if (!cs::runtime::upload_feature_group_masks(&ws, cols, group_masks.data())) return fail(4, "upload masks");
    const unsigned G = (unsigned) in["group_count"][0];
    cs::runtime::group_mask_config_view groups{G, nullptr, ws.feature_group_masks};
    cs::runtime::row_feature_mask_view masks{d_rk, d_fk, nullptr, nullptr};
    const auto &fp = in["filter"];
    cs::runtime::sparse_group_filter_params filter{(float) fp[0], (unsigned) fp[1], (float) fp[2], (unsigned) fp[3]};
    cs::runtime::sparse_group_reduce_result res;

    auto dump = [&](const char *tag) {
        cudaStreamSynchronize(ws.stream);
        std::string t(tag);
        print_dev((t + ".row_totals").c_str(), res.row_totals, res.rows);
        print_dev((t + ".detected").c_str(), res.detected_features, res.rows);
        print_dev((t + ".keep").c_str(), res.row_keep, res.rows);
        if (res.group_count) {
            print_dev((t + ".group_counts").c_str(), res.group_counts, (size_t) res.rows * res.group_count);
            print_dev((t + ".group_percentages").c_str(), res.group_percentages, (size_t) res.rows * res.group_count);
        }
    };

    // Blocked-ELL staged through device::upload
    const unsigned B = (unsigned) in["blocked.block_size"][0], ell_cols = (unsigned) in["blocked.ell_cols"][0];
    auto bci = as<std::uint32_t>(in["blocked.block_cols"]);
    auto bval = halves(in["blocked.values"]);
    cs::sparse::blocked_ell hb;
    cs::sparse::init(&hb);
    hb.rows = rows;
    hb.cols = cols;
    hb.block_size = B;
    hb.ell_cols = ell_cols;
    hb.blockColIdx = bci.data();
    hb.val = bval.data();
    for (const auto &x : bval) hb.nnz += __half2float(x) != 0.0f ? 1u : 0u; // the stored nonzeros
    cs::device::partition_record<cs::sparse::blocked_ell> rb;
    if (cs::device::upload(&hb, &rb) != cudaSuccess) return fail(5, "upload blocked_ell");
    std::printf("blocked.partition_bytes %zu %zu\n", cs::device::device_partition_bytes(&hb), rb.allocation_bytes);
    auto bview = cs::device::staged_view(&hb, &rb);
    if (!cs::runtime::compute_sparse_group_reduce(&bview, &ws, &groups, &masks, &filter, &res))
        return fail(6, "reduce blocked_ell");
    dump("blocked");
    cs::runtime::group_mask_config_view no_groups{0u, nullptr, nullptr};
    if (!cs::runtime::compute_sparse_group_reduce(&bview, &ws, &no_groups, nullptr, &filter, &res))
        return fail(7, "reduce blocked_ell without groups");
    dump("no_groups");
    // a missing filter is refused, as the reference refuses it
    std::printf("null_filter %d\n", cs::runtime::compute_sparse_group_reduce(&bview, &ws, &no_groups, nullptr,
                                                                             nullptr, &res));

    // compressed fallback
    auto cptr = as<std::uint32_t>(in["compressed.ptr"]);
    auto cidx = as<std::uint32_t>(in["compressed.idx"]);
    auto cval = halves(in["compressed.values"]);
    cs::sparse::compressed hc;
    cs::sparse::init(&hc);
    hc.rows = rows;
    hc.cols = cols;
    hc.nnz = (unsigned) cidx.size();
    hc.axis = cs::sparse::compressed_by_row;
    hc.majorPtr = cptr.data();
    hc.minorIdx = cidx.data();
    hc.val = cval.data();
    cs::device::partition_record<cs::sparse::compressed> rc;
    if (cs::device::upload(&hc, &rc) != cudaSuccess) return fail(8, "upload compressed");
    auto cview = cs::device::staged_view(&hc, &rc);
    if (!cs::runtime::compute_sparse_group_reduce_compressed_fallback(&cview, &ws, &groups, &masks, &filter, &res))
        return fail(9, "reduce compressed");
    dump("compressed");

    // Sliced-ELL (host format has no slot offsets or slice height: derived on upload)
    auto soff = as<std::uint32_t>(in["sliced.offsets"]);
    auto sw = as<std::uint32_t>(in["sliced.widths"]);
    auto sci = as<std::uint32_t>(in["sliced.col_idx"]);
    auto sval = halves(in["sliced.values"]);
    cs::sparse::sliced_ell hs;
    cs::sparse::init(&hs);
    hs.rows = rows;
    hs.cols = cols;
    hs.nnz = (unsigned) in["sliced.nnz"][0];
    hs.slice_count = (unsigned) sw.size();
    hs.slice_row_offsets = soff.data();
    hs.slice_widths = sw.data();
    hs.col_idx = sci.data();
    hs.val = sval.data();
    cs::device::partition_record<cs::sparse::sliced_ell> rs;
    if (cs::device::upload(&hs, &rs) != cudaSuccess) return fail(10, "upload sliced_ell");
    auto sview = cs::device::staged_view(&hs, &rs);
    std::printf("sliced.view %u %u\n", sview.slice_rows, sview.slice_count);
    print_dev("sliced.slot_offsets", sview.slice_slot_offsets, sview.slice_count);
    if (!cs::runtime::compute_sparse_group_reduce(&sview, &ws, &groups, &masks, &filter, &res))
        return fail(11, "reduce sliced_ell");
    dump("sliced");

    // reoptimize with remaps
    auto rr = as<std::uint32_t>(in["reoptimize.row_remap"]);
    auto fr = as<std::uint32_t>(in["reoptimize.feature_remap"]);
    std::uint32_t *d_rr = to_device(rr), *d_fr = to_device(fr);
    cs::runtime::row_feature_mask_view rmasks{d_rk, d_fk, d_rr, d_fr};
    cs::runtime::masked_sparse_reoptimize_config cfg{(unsigned) in["reoptimize.output_rows"][0],
                                                     (unsigned) in["reoptimize.output_cols"][0], 0u, 0u,
                                                     cs::runtime::sparse_mask_layout_compressed};
    cs::runtime::masked_sparse_reoptimize_workspace rws;
    cs::runtime::init(&rws);
    if (!cs::runtime::setup(&rws, 0)) return fail(12, "reoptimize setup");
    cs::runtime::masked_sparse_reoptimize_result rres;
    if (!cs::runtime::manual_reoptimize_masked_sparse(&bview, &rmasks, &cfg, &rws, &rres))
        return fail(13, "reoptimize");
    cudaStreamSynchronize(rws.stream);
    std::printf("reoptimize.meta %u %u %u\n", rres.metadata.kept_rows, rres.metadata.kept_features,
                rres.metadata.live_nnz);
    print_dev("reoptimize.ptr", rres.compressed.majorPtr, rres.compressed.rows + 1u);
    print_dev("reoptimize.idx", rres.compressed.minorIdx, rres.compressed.nnz);
    print_dev_half("reoptimize.val", rres.compressed.val, rres.compressed.nnz);

    // filtered Blocked-ELL -> CSR and the repack (one partition, block size 2, 2 buckets)
    {
        const unsigned orows = (unsigned) in["reoptimize.output_rows"][0];
        const unsigned ocols = (unsigned) in["reoptimize.output_cols"][0];
        cs::convert::filtered_blocked_ell_workspace fws;
        cs::convert::init(&fws);
        if (!cs::convert::setup(&fws, 0)) return fail(21, "filter setup");
        cs::convert::filtered_blocked_ell_result fres;
        if (!cs::convert::build_bucketed_filtered_blocked_ell_major_view(&bview, orows, ocols, d_rk, d_fk, d_rr, d_fr,
                                                                         2u, &fws, &fres))
            return fail(22, "filter + bucket");
        cudaStreamSynchronize(fws.bucket_ws.stream);
        std::printf("filter.meta %u %u %d\n", fres.filtered.nnz, fres.stats.kept_rows, fres.has_bucketed);
        print_dev("filter.ptr", fres.filtered.majorPtr, orows + 1u);
        print_dev("filter.idx", fres.filtered.minorIdx, fres.filtered.nnz);
        print_dev("filter.bucket_order", fres.bucketed.plan.major_order, orows);
        cs::convert::clear(&fws);

        cs::repack::sharded_blocked_ell_repack_workspace pws;
        cs::repack::init(&pws);
        if (!cs::repack::setup(&pws, 0)) return fail(23, "repack setup");
        const cs::device::blocked_ell_view *pv[1] = {&bview};
        const cs::repack::sharded_blocked_ell_repack_config pcfg{orows, ocols, 2u, 2u};
        cs::repack::sharded_blocked_ell_repack_result pres;
        if (!cs::repack::build_repacked_blocked_ell_parts(pv, 1ul, 0ul, &pcfg, d_rk, d_fk, d_rr, d_fr, &pws, &pres))
            return fail(24, "repack");
        std::printf("repack.meta %u %u %u %u\n", pres.stats.kept_rows, pres.stats.live_nnz, pres.stats.ell_width,
                    pres.rebuilt.ell_cols);
        print_dev("repack.block_cols", pres.rebuilt.blockColIdx,
                  ((orows + 1u) / 2u) * pres.stats.ell_width);
        print_dev_half("repack.values", pres.rebuilt.val, orows * pres.rebuilt.ell_cols);
        cs::repack::clear(&pws);
    }

    // host conversion + chooser through convert::
    cs::sparse::blocked_ell conv;
    cs::sparse::init(&conv);
    if (!cs::convert::blocked_ell_from_compressed(&hc, 2u, &conv)) return fail(14, "blocked_ell_from_compressed");
    std::printf("convert.blocked %u %u %u\n", conv.block_size, conv.ell_cols, conv.nnz);
    {
        const unsigned rbk = (conv.rows + conv.block_size - 1u) / conv.block_size;
        std::printf("convert.block_cols");
        for (unsigned i = 0; i < rbk * (conv.ell_cols / conv.block_size); ++i) std::printf(" %u", conv.blockColIdx[i]);
        std::printf("\nconvert.values");
        for (unsigned i = 0; i < conv.rows * conv.ell_cols; ++i) std::printf(" %g", __half2float(conv.val[i]));
        std::printf("\n");
    }
    {
        // Blocked-ELL -> Sliced-ELL with the slice height chosen from 2 / 4 / 8
        const unsigned bcands[3] = {2u, 4u, 8u};
        cs::sparse::sliced_ell sconv;
        cs::sparse::init(&sconv);
        cs::convert::sliced_ell_tune_result picked;
        if (!cs::convert::sliced_ell_from_blocked_ell_auto(&conv, bcands, 3u, &sconv, &picked))
            return fail(20, "sliced_ell_from_blocked_ell_auto");
        unsigned total = 0u;
        for (unsigned s = 0; s < sconv.slice_count; ++s)
            total += (sconv.slice_row_offsets[s + 1u] - sconv.slice_row_offsets[s]) * sconv.slice_widths[s];
        std::printf("convert.sell_from_bell %u %u %u\n", picked.slice_rows, sconv.slice_count, sconv.nnz);
        std::printf("convert.sell_from_bell.col");
        for (unsigned i = 0; i < total; ++i) std::printf(" %u", sconv.col_idx[i]);
        std::printf("\nconvert.sell_from_bell.val");
        for (unsigned i = 0; i < total; ++i) std::printf(" %g", __half2float(sconv.val[i]));
        std::printf("\n");
        // execution bucketing of the Sliced-ELL (2 buckets) and its chooser
        cs::bucketed_sliced_ell_partition sb;
        cs::init(&sb);
        std::uint64_t sbytes = 0u;
        if (!cs::build_bucketed_sliced_ell_partition(&sb, &sconv, 2u, &sbytes)) return fail(25, "bucketed sliced");
        std::printf("exec.sell %u %llu", sb.segment_count, (unsigned long long) sbytes);
        for (unsigned s = 0; s < sb.segment_count; ++s)
            std::printf(" %u %u %u", sb.segments[s].rows, sb.segments[s].slice_count ? sb.segments[s].slice_widths[0] : 0u,
                        sb.segments[s].nnz);
        std::printf("\nexec.sell.e2c");
        for (unsigned r = 0; r < sb.rows; ++r) std::printf(" %u", sb.exec_to_canonical_rows[r]);
        std::printf("\n");
        cs::clear(&sb);
        std::uint32_t sc = 0u;
        if (!cs::choose_bucket_count_for_sliced_part(&sconv, &sc, &sbytes)) return fail(26, "choose sliced");
        std::printf("exec.sell.choose %u %llu\n", sc, (unsigned long long) sbytes);
        cs::sparse::clear(&sconv);
    }
    {
        // execution bucketing of the Blocked-ELL (2 buckets), both choosers, bucket::build_plan
        cs::bucketed_blocked_ell_partition bb;
        cs::init(&bb);
        std::uint64_t bbytes = 0u;
        if (!cs::build_bucketed_blocked_ell_partition(&bb, &conv, 2u, &bbytes)) return fail(27, "bucketed blocked");
        std::printf("exec.bell %u %llu", bb.segment_count, (unsigned long long) bbytes);
        for (unsigned s = 0; s < bb.segment_count; ++s)
            std::printf(" %u %u %u", bb.segments[s].rows, bb.segments[s].ell_cols, bb.segments[s].nnz);
        std::printf("\nexec.bell.block_cols");
        for (unsigned s = 0; s < bb.segment_count; ++s) {
            const cs::sparse::blocked_ell &g = bb.segments[s];
            const unsigned n = ((g.rows + g.block_size - 1u) / g.block_size) * (g.ell_cols / g.block_size);
            for (unsigned i = 0; i < n; ++i) std::printf(" %u", g.blockColIdx[i]);
        }
        std::printf("\nexec.bell.e2c");
        for (unsigned r = 0; r < bb.rows; ++r) std::printf(" %u", bb.exec_to_canonical_rows[r]);
        std::printf("\n");
        cs::clear(&bb);
        std::uint32_t bc = 0u, ic = 0u;
        if (!cs::choose_bucket_count_for_part(&conv, &bc, &bbytes)) return fail(28, "choose blocked");
        if (!cs::ingest::dataset::choose_bucket_count_for_part(&conv, 0, &ic)) return fail(29, "choose ingest");
        std::printf("exec.bell.choose %u %llu %u\n", bc, (unsigned long long) bbytes, ic);
        cs::bucket::blocked_ell_bucket_workspace pws;
        cs::bucket::init(&pws);
        cs::bucket::blocked_ell_bucket_plan plan;
        if (!cs::bucket::setup(&pws, 0) || !cs::bucket::build_plan(&conv, &pws, &plan)) return fail(30, "build_plan");
        std::printf("exec.plan.order");
        for (auto x : plan.row_block_order) std::printf(" %u", x);
        std::printf("\nexec.plan.width");
        for (auto x : plan.row_block_width_sorted) std::printf(" %u", x);
        std::printf("\n");
        cs::bucket::clear(&pws);
    }
    cs::sparse::clear(&conv);
    {
        // the same matrix as COO (entries in reverse order), through the COO chooser and builder
        std::vector<cs::types::idx_t> cr, cc;
        std::vector<__half> cv;
        for (unsigned r = 0; r < hc.rows; ++r)
            for (unsigned k = hc.majorPtr[r]; k < hc.majorPtr[r + 1u]; ++k) {
                cr.insert(cr.begin(), r);
                cc.insert(cc.begin(), hc.minorIdx[k]);
                cv.insert(cv.begin(), hc.val[k]);
            }
        cs::sparse::coo coo{hc.rows, hc.cols, (cs::types::nnz_t) cr.size(), nullptr, cr.data(), cc.data(), cv.data()};
        const unsigned coo_cands[2] = {2u, 4u};
        cs::convert::blocked_ell_tune_result ct;
        cs::sparse::blocked_ell cb;
        cs::sparse::init(&cb);
        if (!cs::convert::blocked_ell_from_coo_cuda_auto(&coo, hc.cols, nullptr, coo_cands, 2u, &cb, 0, &ct))
            return fail(31, "blocked_ell_from_coo_cuda_auto");
        std::printf("coo.blocked %u %u %u", ct.block_size, cb.ell_cols, cb.nnz);
        const unsigned cn = ((cb.rows + cb.block_size - 1u) / cb.block_size) * (cb.ell_cols / cb.block_size);
        std::printf("\ncoo.block_cols");
        for (unsigned i = 0; i < cn; ++i) std::printf(" %u", cb.blockColIdx[i]);
        std::printf("\ncoo.values");
        for (unsigned i = 0; i < cb.rows * cb.ell_cols; ++i) std::printf(" %g", __half2float(cb.val[i]));
        std::printf("\n");
        cs::sparse::clear(&cb);
    }
    const unsigned cands[3] = {16u, 32u, 64u};
    cs::convert::sliced_ell_tune_result tune;
    if (!cs::convert::choose_sliced_ell_slice_rows_from_compressed(&hc, cands, 3u, &tune))
        return fail(15, "choose slice rows");
    std::printf("convert.slice_choice %u %u %zu %.17g\n", tune.slice_rows, tune.slice_count, tune.padded_slots,
                tune.score);

    // bucketing through the operator workspace
    cs::bucket::compressed_major_bucket_workspace bws;
    cs::bucket::init(&bws);
    if (!cs::bucket::setup(&bws, 0)) return fail(16, "bucket setup");
    cs::bucket::compressed_major_bucket_result bres;
    if (!cs::bucket::build_bucketed_major_view(&cview, 2u, &bws, &bres)) return fail(17, "bucketed view");
    cudaStreamSynchronize(bws.stream);
    print_dev("bucket.order", bres.plan.major_order, rows);
    print_dev("bucket.offsets", bres.plan.bucket_offsets, bres.plan.bucket_count + 1u);
    print_dev("bucket.rebuilt_ptr", bres.rebuilt.majorPtr, rows + 1u);
    print_dev("bucket.inverse", bres.plan.inverse_major_order, rows);

    // transpose raw
    const size_t tb = cs::convert::compressed_transpose_scratch_bytes(rows, cols, hc.nnz);
    void *tscr = nullptr;
    std::uint32_t *tptr = nullptr, *tidx = nullptr;
    __half *tval = nullptr;
    cudaMalloc(&tscr, tb);
    cudaMalloc((void **) &tptr, (cols + 1u) * 4u);
    cudaMalloc((void **) &tidx, hc.nnz * 4u + 16u);
    cudaMalloc((void **) &tval, hc.nnz * 2u + 16u);
    if (!cs::convert::build_compressed_transpose_raw(rows, cols, hc.nnz, cview.majorPtr, cview.minorIdx, cview.val,
                                                     tptr, nullptr, tidx, tval, tscr, tb, (cudaStream_t) 0))
        return fail(18, "transpose");
    cudaDeviceSynchronize();
    print_dev("transpose.ptr", tptr, cols + 1u);
    print_dev("transpose.idx", tidx, hc.nnz);
    print_dev_half("transpose.val", tval, hc.nnz);


    // ---------------------------------------------------------------------
    // Shard-level staging: a sharded<blocked_ell> of five uneven partitions
    // cut into two shards, staged through a sharded_device (one packed block
    // per shard), swapped, restaged from the allocation cache; every staged
    // partition reduced through runtime::compute_sparse_group_reduce.
    // ---------------------------------------------------------------------
    {
        const unsigned scols = 48u, SB = 4u, SG = 4u;
        lcg g{12345u};
        std::vector<std::uint32_t> smask(scols);
        for (auto &x : smask) x = g.next() & 0xfu;
        print_host("shard.group_masks", smask.data(), smask.size());
        cs::runtime::sparse_group_reduce_workspace ws2;
        cs::runtime::init(&ws2);
        if (!cs::runtime::setup(&ws2, 0) || !cs::runtime::upload_feature_group_masks(&ws2, scols, smask.data()))
            return fail(40, "shard workspace");
        cs::runtime::group_mask_config_view g2{SG, nullptr, ws2.feature_group_masks};
        cs::runtime::sparse_group_filter_params f2{1.0f, 1u, 0.9f, 0u};
        cs::runtime::sparse_group_reduce_result r2;
        auto dump2 = [&](const std::string &t) {
            cudaStreamSynchronize(ws2.stream);
            print_dev((t + ".row_totals").c_str(), r2.row_totals, r2.rows);
            print_dev((t + ".detected").c_str(), r2.detected_features, r2.rows);
            print_dev((t + ".max").c_str(), r2.max_values, r2.rows);
            print_dev((t + ".keep").c_str(), r2.row_keep, r2.rows);
            print_dev((t + ".group_counts").c_str(), r2.group_counts, (size_t) r2.rows * SG);
        };

        const unsigned prow[5] = {37u, 64u, 21u, 50u, 9u}, pw[5] = {3u, 5u, 2u, 4u, 1u};
        cs::sharded<cs::sparse::blocked_ell> m;
        cs::init(&m);
        for (unsigned p = 0; p < 5u; ++p) {
            cs::sparse::blocked_ell *part = make_bell_part(g, prow[p], scols, SB, pw[p]);
            const std::string t = "shard.part" + std::to_string(p);
            std::printf("%s.meta %u %u %u %u\n", t.c_str(), part->rows, part->ell_cols, part->nnz, SB);
            print_host(t + ".bci", part->blockColIdx, (size_t) ((part->rows + SB - 1u) / SB) * pw[p]);
            print_host_half(t + ".val", part->val, (size_t) part->rows * part->ell_cols);
            if (!cs::append_partition(&m, part)) return fail(41, "append_partition");
        }
        if (!cs::set_equal_shards(&m, 2u)) return fail(42, "set_equal_shards");
        print_host("shard.offsets", m.shard_offsets, m.num_shards + 1u);
        print_host("shard.parts", m.shard_parts, m.num_shards + 1u);

        cs::device::sharded_device<cs::sparse::blocked_ell> st;
        cs::device::init(&st);
        if (!cs::device::reserve(&st, m.num_partitions)) return fail(43, "reserve");
        auto reduce_resident = [&](const std::string &tag) -> int {
            for (unsigned long p = 0; p < m.num_partitions; ++p) {
                if (st.parts[p].view == nullptr) continue;
                auto v = cs::device::staged_view(m.parts[p], &st.parts[p]);
                if (!cs::runtime::compute_sparse_group_reduce(&v, &ws2, &g2, nullptr, &f2, &r2)) return 0;
                dump2(tag + ".p" + std::to_string(p));
            }
            return 1;
        };
        auto records = [&](const std::string &tag) {
            std::printf("%s", tag.c_str());
            for (unsigned long p = 0; p < m.num_partitions; ++p) {
                const auto &r = st.parts[p];
                const long vo = r.view ? (long) ((char *) r.view - (char *) st.parts[r.group_begin].view) : -1;
                std::printf(" %lu %lu %d %d %ld", r.group_begin, r.group_end, r.allocation != nullptr ? 1 : 0,
                            r.device_id, vo);
            }
            std::printf("\n%s.cache %lu\n", tag.c_str(), st.cache_count);
        };
        if (cs::device::stage_shard(&st, &m, nullptr, 0ul, 0, 0) != cudaSuccess) return fail(44, "stage_shard 0");
        records("shard.records.s0");
        if (!reduce_resident("shard.s0")) return fail(45, "reduce shard 0");
        void *block0 = st.parts[0].allocation;
        const std::size_t bytes0 = st.parts[0].allocation_bytes;
        if (cs::device::swap_shard(&st, &m, nullptr, 0ul, 1ul, 0, 0, 0) != cudaSuccess) return fail(46, "swap_shard");
        records("shard.records.swapped");
        if (!reduce_resident("shard.s1")) return fail(47, "reduce shard 1");
        // shard 0 again: its block comes back from the cache
        if (cs::device::stage_shard(&st, &m, nullptr, 0ul, 0, 0) != cudaSuccess) return fail(48, "restage shard 0");
        records("shard.records.restaged");
        std::printf("shard.reuse %d %d\n", st.parts[0].allocation == block0 ? 1 : 0,
                    st.parts[0].allocation_bytes == bytes0 ? 1 : 0);
        if (!reduce_resident("shard.both")) return fail(49, "reduce both shards");
        // staging a resident shard again does nothing
        void *b1 = st.parts[m.shard_parts[1]].allocation;
        if (cs::device::upload_shard(&st, &m, 1ul, 0) != cudaSuccess || st.parts[m.shard_parts[1]].allocation != b1)
            return fail(50, "upload resident shard");
        // footprints: per-partition bytes from the metadata equal the C ABI's for the materialised part
        std::printf("shard.bytes");
        for (unsigned long p = 0; p < m.num_partitions; ++p)
            std::printf(" %zu %zu", cs::device::device_partition_bytes(&m, p),
                        cs::device::device_partition_bytes(m.parts[p]));
        std::printf(" %zu %zu %zu\n", cs::device::device_shard_bytes(&m, 0ul), cs::device::device_shard_bytes(&m, 1ul),
                    bytes0);
        // shards by device bytes, by nnz, by host bytes; explicit offsets
        const std::size_t lim = cs::device::device_partition_bytes(&m, 0ul) + cs::device::device_partition_bytes(&m, 1ul);
        cs::device::release_shard(&st, &m, 0ul);
        cs::device::release_shard(&st, &m, 1ul);
        if (!cs::device::set_shards_by_device_bytes(&m, lim)) return fail(51, "set_shards_by_device_bytes");
        print_host("shard.by_device_bytes", m.shard_offsets, m.num_shards + 1u);
        if (!cs::set_shards_by_nnz(&m, 400ul)) return fail(52, "set_shards_by_nnz");
        print_host("shard.by_nnz", m.shard_offsets, m.num_shards + 1u);
        const unsigned long cuts[3] = {0ul, m.partition_offsets[3], m.rows};
        std::printf("shard.reshard %d %d\n", cs::reshard(&m, 2ul, cuts), cs::reshard(&m, 1ul, cuts + 1));
        // stage_partition with the host part dropped after upload; a dropped,
        // non-resident part cannot be fetched (no file backend)
        if (cs::device::stage_partition(&st, &m, nullptr, 4ul, 0, 1) != cudaSuccess) return fail(53, "stage_partition");
        std::printf("shard.dropped %d %lu %lu\n", m.parts[4] == nullptr ? 1 : 0, st.parts[4].group_begin,
                    st.parts[4].group_end);
        const cudaError_t again = cs::device::stage_partition(&st, &m, nullptr, 4ul, 0, 0);
        cs::device::release_partition(&st, 4ul);
        const cudaError_t absent = cs::device::stage_partition(&st, &m, nullptr, 4ul, 0, 0);
        std::printf("shard.stage_codes %d %d\n", (int) again, absent == cudaSuccess ? 0 : 1);
        cs::device::clear(&st);
        cs::clear(&m);
        cs::runtime::clear(&ws2);
    }

    // compressed and Sliced-ELL shards: one packed block each, the Sliced-ELL
    // slot offsets computed on the device per partition
    {
        const unsigned scols = 48u, SG = 4u;
        lcg g{777u};
        std::vector<std::uint32_t> smask(scols);
        for (auto &x : smask) x = g.next() & 0xfu;
        print_host("cshard.group_masks", smask.data(), smask.size());
        cs::runtime::sparse_group_reduce_workspace ws3;
        cs::runtime::init(&ws3);
        if (!cs::runtime::setup(&ws3, 0) || !cs::runtime::upload_feature_group_masks(&ws3, scols, smask.data()))
            return fail(60, "cshard workspace");
        cs::runtime::group_mask_config_view g3{SG, nullptr, ws3.feature_group_masks};
        cs::runtime::sparse_group_filter_params f3{1.0f, 1u, 0.9f, 0u};
        cs::runtime::sparse_group_reduce_result r3;
        auto dump3 = [&](const std::string &t) {
            cudaStreamSynchronize(ws3.stream);
            print_dev((t + ".row_totals").c_str(), r3.row_totals, r3.rows);
            print_dev((t + ".detected").c_str(), r3.detected_features, r3.rows);
            print_dev((t + ".group_counts").c_str(), r3.group_counts, (size_t) r3.rows * SG);
        };
        const unsigned crow[3] = {29u, 70u, 13u};
        cs::sharded<cs::sparse::compressed> mc;
        cs::sharded<cs::sparse::sliced_ell> ms;
        cs::init(&mc);
        cs::init(&ms);
        for (unsigned p = 0; p < 3u; ++p) {
            cs::sparse::compressed *c = make_csr_part(g, crow[p], scols);
            const std::string t = "cshard.part" + std::to_string(p);
            print_host(t + ".ptr", c->majorPtr, c->rows + 1u);
            print_host(t + ".idx", c->minorIdx, c->nnz);
            print_host_half(t + ".val", c->val, c->nnz);
            auto *sl = new cs::sparse::sliced_ell;
            cs::sparse::init(sl);
            if (!cs::convert::sliced_ell_from_compressed(c, 8u, sl)) return fail(61, "sliced_ell_from_compressed");
            if (!cs::append_partition(&mc, c) || !cs::append_partition(&ms, sl)) return fail(62, "append");
        }
        cs::set_equal_shards(&mc, 1u);
        cs::set_equal_shards(&ms, 1u);
        cs::device::sharded_device<cs::sparse::compressed> sc;
        cs::device::sharded_device<cs::sparse::sliced_ell> ss;
        cs::device::init(&sc);
        cs::device::init(&ss);
        if (!cs::device::reserve(&sc, 3ul) || !cs::device::reserve(&ss, 3ul)) return fail(63, "reserve");
        if (cs::device::upload_shard_async(&sc, &mc, 0ul, 0, ws3.stream) != cudaSuccess ||
            cs::device::upload_shard_async(&ss, &ms, 0ul, 0, ws3.stream) != cudaSuccess)
            return fail(64, "upload_shard_async");
        for (unsigned long p = 0; p < 3ul; ++p) {
            auto cv = cs::device::staged_view(mc.parts[p], &sc.parts[p]);
            if (!cs::runtime::compute_sparse_group_reduce_compressed_fallback(&cv, &ws3, &g3, nullptr, &f3, &r3))
                return fail(65, "reduce staged compressed");
            dump3("cshard.c" + std::to_string(p));
            auto sv = cs::device::staged_view(ms.parts[p], &ss.parts[p]);
            cudaStreamSynchronize(ws3.stream);
            print_dev(("cshard.s" + std::to_string(p) + ".slot_offsets").c_str(), sv.slice_slot_offsets,
                      sv.slice_count);
            if (!cs::runtime::compute_sparse_group_reduce(&sv, &ws3, &g3, nullptr, &f3, &r3))
                return fail(66, "reduce staged sliced");
            dump3("cshard.s" + std::to_string(p));
            std::printf("cshard.group %lu %lu %lu %lu\n", sc.parts[p].group_begin, sc.parts[p].group_end,
                        ss.parts[p].group_begin, ss.parts[p].group_end);
        }
        cs::device::clear(&sc);
        cs::device::clear(&ss);
        cs::clear(&mc);
        cs::clear(&ms);
        cs::runtime::clear(&ws3);
    }

    cs::bucket::clear(&bws);
    cs::runtime::clear(&rws);
    cs::runtime::clear(&ws);
    if (cs::device::release(&rb) != cudaSuccess || cs::device::release(&rc) != cudaSuccess ||
        cs::device::release(&rs) != cudaSuccess)
        return fail(19, "release");
    cudaFree(tscr);
    cudaFree(tptr);
    cudaFree(tidx);
    cudaFree(tval);
    cudaFree(d_rk);
    cudaFree(d_fk);
    cudaFree(d_rr);
    cudaFree(d_fr);
    std::printf("done 0\n");
    return 0;
}
