// Partition staging: one packed device allocation per partition holding the
// device view descriptor followed by the payload arrays, filled by
// stream-ordered copies -- what device::upload[_async] does for the
// compressed, Blocked-ELL and Sliced-ELL formats
// (include/CellShard/runtime/device/sharded_device.cuh:343-756, 959-991).
// Arrays start on 256-byte boundaries (the kernels here use 16-byte vector
// loads and stores).  The Sliced-ELL device view carries the uniform slice
// height and the u32 slot offsets the host format does not store; they are
// derived on upload as the reference does (sharded_device.cuh:604-620,716-723).
// The reference's 16-entry allocation cache is not reproduced: callers that
// restage often keep their records (release + upload is one cudaFree and one
// cudaMalloc).
#include "common.cuh"

#include <cstring>
#include <vector>

namespace csb {
namespace {

std::size_t align256(std::size_t x) { return (x + 255u) / 256u * 256u; }

struct packer {
    std::size_t used = 256; // the view descriptor lives in the first 256 bytes
    std::size_t take(std::size_t bytes) {
        const std::size_t at = used;
        used = align256(used + bytes);
        return at;
    }
};

int finish_upload(cs_partition_record *rec, const void *view, std::size_t view_bytes,
                  const std::vector<std::pair<std::size_t, std::pair<const void *, std::size_t>>> &copies,
                  cudaStream_t stream) {
    unsigned char *base = static_cast<unsigned char *>(rec->allocation);
    for (const auto &c : copies)
        if (c.second.second != 0u &&
            !cuda_ok(cudaMemcpyAsync(base + c.first, c.second.first, c.second.second, cudaMemcpyHostToDevice, stream),
                     "upload payload copy"))
            return 0;
    // the view descriptor comes from this call's stack, so the call waits for
    // its copies (device::upload is synchronous too)
    if (!cuda_ok(cudaMemcpyAsync(base, view, view_bytes, cudaMemcpyHostToDevice, stream), "upload view copy") ||
        !cuda_ok(cudaStreamSynchronize(stream), "upload view sync"))
        return 0;
    return 1;
}

int alloc_record(cs_partition_record *rec, std::size_t bytes, uint32_t format) {
    std::memset(rec, 0, sizeof(*rec));
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "upload device")) return 0;
    void *p = nullptr;
    if (!cuda_ok(cudaMalloc(&p, bytes), "upload allocation")) return 0;
    rec->allocation = p;
    rec->allocation_bytes = bytes;
    rec->view = p;
    rec->device_id = dev;
    rec->format = format;
    return 1;
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_device_partition_bytes_compressed(const cs_host_compressed *src, size_t *out_bytes) {
    if (src == nullptr || out_bytes == nullptr) {
        set_error("device_partition_bytes: null argument");
        return 0;
    }
    const std::size_t major = src->axis == CS_COMPRESSED_BY_COL ? src->cols : src->rows;
    packer pk;
    pk.take((major + 1u) * 4u);
    pk.take((std::size_t) src->nnz * 4u);
    pk.take((std::size_t) src->nnz * 2u);
    *out_bytes = pk.used;
    return 1;
}

extern "C" int cs_b200_device_partition_bytes_blocked_ell(const cs_host_blocked_ell *src, size_t *out_bytes) {
    if (src == nullptr || out_bytes == nullptr || src->block_size == 0u) {
        set_error("device_partition_bytes: null argument or zero block size");
        return 0;
    }
    const std::size_t rb = ((std::size_t) src->rows + src->block_size - 1u) / src->block_size;
    packer pk;
    pk.take(rb * (src->ell_cols / src->block_size) * 4u);
    pk.take((std::size_t) src->rows * src->ell_cols * 2u);
    *out_bytes = pk.used;
    return 1;
}

namespace {
std::size_t sliced_total_slots(const cs_host_sliced_ell *src) {
    std::size_t total = 0;
    for (uint32_t s = 0; s < src->slice_count; ++s)
        total += (std::size_t) (src->slice_row_offsets[s + 1u] - src->slice_row_offsets[s]) * src->slice_widths[s];
    return total;
}
} // namespace

extern "C" int cs_b200_device_partition_bytes_sliced_ell(const cs_host_sliced_ell *src, size_t *out_bytes) {
    if (src == nullptr || out_bytes == nullptr || (src->slice_count != 0u && src->slice_row_offsets == nullptr)) {
        set_error("device_partition_bytes: null argument");
        return 0;
    }
    const std::size_t S = src->slice_count, total = sliced_total_slots(src);
    packer pk;
    pk.take((S + 1u) * 4u);
    pk.take(S * 4u);
    pk.take(S * 4u);
    pk.take(total * 4u);
    pk.take(total * 2u);
    *out_bytes = pk.used;
    return 1;
}

extern "C" int cs_b200_upload_compressed(const cs_host_compressed *src, cs_partition_record *rec, cs_stream_t s) {
    if (src == nullptr || rec == nullptr || (src->nnz != 0u && (src->minorIdx == nullptr || src->val == nullptr))) {
        set_error("upload_compressed: null argument");
        return 0;
    }
    const std::size_t major = src->axis == CS_COMPRESSED_BY_COL ? src->cols : src->rows;
    packer pk;
    const std::size_t o_ptr = pk.take((major + 1u) * 4u);
    const std::size_t o_idx = pk.take((std::size_t) src->nnz * 4u);
    const std::size_t o_val = pk.take((std::size_t) src->nnz * 2u);
    if (!alloc_record(rec, pk.used, CS_FORMAT_COMPRESSED)) return 0;
    unsigned char *b = static_cast<unsigned char *>(rec->allocation);
    cs_compressed_view v{};
    v.rows = src->rows;
    v.cols = src->cols;
    v.nnz = src->nnz;
    v.axis = src->axis;
    v.majorPtr = reinterpret_cast<uint32_t *>(b + o_ptr);
    v.minorIdx = reinterpret_cast<uint32_t *>(b + o_idx);
    v.val = reinterpret_cast<uint16_t *>(b + o_val);
    rec->a0 = v.majorPtr;
    rec->a1 = v.minorIdx;
    rec->a2 = v.val;
    std::memcpy(rec->host_view, &v, sizeof(v));
    const int ok = finish_upload(rec, &v, sizeof(v),
                                 {{o_ptr, {src->majorPtr, src->majorPtr ? (major + 1u) * 4u : 0u}},
                                  {o_idx, {src->minorIdx, (std::size_t) src->nnz * 4u}},
                                  {o_val, {src->val, (std::size_t) src->nnz * 2u}}},
                                 as_stream(s));
    if (!ok) cs_b200_release_partition(rec);
    return ok;
}

extern "C" int cs_b200_upload_blocked_ell(const cs_host_blocked_ell *src, cs_partition_record *rec, cs_stream_t s) {
    if (src == nullptr || rec == nullptr || src->block_size == 0u || src->ell_cols % src->block_size != 0u) {
        set_error("upload_blocked_ell: null argument or block size not dividing ell_cols");
        return 0;
    }
    const std::size_t rb = ((std::size_t) src->rows + src->block_size - 1u) / src->block_size;
    const std::size_t idx_bytes = rb * (src->ell_cols / src->block_size) * 4u;
    const std::size_t val_bytes = (std::size_t) src->rows * src->ell_cols * 2u;
    packer pk;
    const std::size_t o_idx = pk.take(idx_bytes);
    const std::size_t o_val = pk.take(val_bytes);
    if (!alloc_record(rec, pk.used, CS_FORMAT_BLOCKED_ELL)) return 0;
    unsigned char *b = static_cast<unsigned char *>(rec->allocation);
    cs_blocked_ell_view v{};
    v.rows = src->rows;
    v.cols = src->cols;
    v.nnz = src->nnz;
    v.block_size = src->block_size;
    v.ell_cols = src->ell_cols;
    v.blockColIdx = reinterpret_cast<uint32_t *>(b + o_idx);
    v.val = reinterpret_cast<uint16_t *>(b + o_val);
    rec->a0 = v.blockColIdx;
    rec->a1 = v.val;
    std::memcpy(rec->host_view, &v, sizeof(v));
    const int ok = finish_upload(rec, &v, sizeof(v),
                                 {{o_idx, {src->blockColIdx, idx_bytes}}, {o_val, {src->val, val_bytes}}},
                                 as_stream(s));
    if (!ok) cs_b200_release_partition(rec);
    return ok;
}

extern "C" int cs_b200_upload_sliced_ell(const cs_host_sliced_ell *src, cs_partition_record *rec, cs_stream_t s) {
    if (src == nullptr || rec == nullptr || (src->slice_count != 0u && src->slice_row_offsets == nullptr)) {
        set_error("upload_sliced_ell: null argument");
        return 0;
    }
    const std::size_t S = src->slice_count, total = sliced_total_slots(src);
    if (total > 0xffffffffull) {
        set_error("upload_sliced_ell: %zu slots exceed the u32 slot offsets", total);
        return 0;
    }
    std::vector<uint32_t> slot_off(S ? S : 1u, 0u);
    uint32_t run = 0u, h = 0u;
    for (std::size_t k = 0; k < S; ++k) {
        const uint32_t rin = src->slice_row_offsets[k + 1u] - src->slice_row_offsets[k];
        if (k == 0u) h = rin;
        slot_off[k] = run;
        run += rin * src->slice_widths[k];
    }
    packer pk;
    const std::size_t o_off = pk.take((S + 1u) * 4u);
    const std::size_t o_w = pk.take(S * 4u);
    const std::size_t o_so = pk.take(S * 4u);
    const std::size_t o_ci = pk.take(total * 4u);
    const std::size_t o_v = pk.take(total * 2u);
    if (!alloc_record(rec, pk.used, CS_FORMAT_SLICED_ELL)) return 0;
    unsigned char *b = static_cast<unsigned char *>(rec->allocation);
    cs_sliced_ell_view v{};
    v.rows = src->rows;
    v.cols = src->cols;
    v.nnz = src->nnz;
    v.slice_count = (uint32_t) S;
    v.slice_rows = h;
    v.slice_row_offsets = reinterpret_cast<uint32_t *>(b + o_off);
    v.slice_widths = reinterpret_cast<uint32_t *>(b + o_w);
    v.slice_slot_offsets = reinterpret_cast<uint32_t *>(b + o_so);
    v.col_idx = reinterpret_cast<uint32_t *>(b + o_ci);
    v.val = reinterpret_cast<uint16_t *>(b + o_v);
    rec->a0 = v.slice_row_offsets;
    rec->a1 = v.slice_widths;
    rec->a2 = v.col_idx;
    rec->a3 = v.val;
    std::memcpy(rec->host_view, &v, sizeof(v));
    // slot offsets come from a host vector local to this call
    const bool ok0 = S == 0u || cuda_ok(cudaMemcpy(b + o_so, slot_off.data(), S * 4u, cudaMemcpyHostToDevice),
                                        "upload slot offsets");
    const int ok = ok0 && finish_upload(rec, &v, sizeof(v),
                                        {{o_off, {src->slice_row_offsets, S ? (S + 1u) * 4u : 0u}},
                                         {o_w, {src->slice_widths, S * 4u}},
                                         {o_ci, {src->col_idx, total * 4u}},
                                         {o_v, {src->val, total * 2u}}},
                                        as_stream(s));
    if (!ok) cs_b200_release_partition(rec);
    return ok;
}

extern "C" int cs_b200_release_partition(cs_partition_record *rec) {
    if (rec == nullptr) {
        set_error("release_partition: null record");
        return 0;
    }
    int ok = 1;
    if (rec->allocation != nullptr) {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != rec->device_id) cudaSetDevice(rec->device_id);
        ok = cuda_ok(cudaFree(rec->allocation), "release partition");
        if (cur != rec->device_id) cudaSetDevice(cur);
    }
    std::memset(rec, 0, sizeof(*rec));
    return ok;
}
