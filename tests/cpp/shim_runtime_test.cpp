// Drives the C++ shim (include/cellshard_b200.hpp) the way reference host
// code drives the reference API: stage host partitions with device::upload,
// run runtime::compute_sparse_group_reduce over Blocked-ELL, Sliced-ELL and
// compressed views, runtime::manual_reoptimize_masked_sparse, the
// convert:: host conversion and chooser, bucket::build_bucketed_major_view and
// convert::build_compressed_transpose_raw.  Inputs come from a text file of
// lines "name v0 v1 ..."; every result is printed as "name v0 v1 ..." for the
// pytest wrapper (tests/test_gpu_cpp_shim.py) to compare.
#include <cellshard_b200.hpp>

#include <cstdio>
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
    std::printf("blocked.partition_bytes %zu %zu\n", cs::device::device_partition_bytes(&hb),
                rb.rec.allocation_bytes);
    auto bview = cs::device::staged_view<cs::device::blocked_ell_view>(&rb);
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
    auto cview = cs::device::staged_view<cs::device::compressed_view>(&rc);
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
    auto sview = cs::device::staged_view<cs::device::sliced_ell_view>(&rs);
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
