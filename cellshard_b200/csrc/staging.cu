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

#include <algorithm>
#include <cstdlib>
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

// ===========================================================================
// Shard-level staging over a device::sharded_device-shaped state
// (sharded_device.cuh:136-243, 992-1212, 1436-1721).  One packed block per
// staged group: the group's device views back to back, then every
// partition's arrays on 256-byte boundaries.  The views and the Sliced-ELL
// slot offsets are written by kernels whose launch arguments carry the data,
// so the calls are stream-ordered end to end and keep no host memory alive
// after they return.
// ===========================================================================
namespace csb {
namespace {

constexpr std::size_t kViewBlob = 3072; // bytes of views one descriptor launch carries

struct view_blob {
    unsigned char b[kViewBlob];
};

// Writes `bytes` bytes of views (passed by value) to dst.
__global__ void write_views_kernel(unsigned char *dst, view_blob blob, unsigned bytes) {
    for (unsigned i = threadIdx.x; i < bytes; i += blockDim.x) dst[i] = blob.b[i];
}

// Slot offsets of one Sliced-ELL partition: exclusive scan of
// (rows in slice k) x width[k], in u32 (the host checked the total fits).
__global__ void __launch_bounds__(1024) sell_slot_offsets_kernel(const uint32_t *__restrict__ row_off,
                                                                 const uint32_t *__restrict__ widths, uint32_t S,
                                                                 uint32_t *__restrict__ out) {
    __shared__ uint32_t sm[33];
    uint32_t carry = 0u;
    for (uint32_t base = 0; base < S; base += blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        const uint32_t v = k < S ? (row_off[k + 1u] - row_off[k]) * widths[k] : 0u;
        uint32_t total = 0u;
        const uint32_t ex = block_exclusive_scan(v, sm, total);
        if (k < S) out[k] = carry + ex;
        carry += total;
    }
}

std::size_t view_bytes_of(uint32_t format) {
    switch (format) {
    case CS_FORMAT_COMPRESSED: return sizeof(cs_compressed_view);
    case CS_FORMAT_BLOCKED_ELL: return sizeof(cs_blocked_ell_view);
    default: return sizeof(cs_sliced_ell_view);
    }
}

// One partition's arrays: host sources, byte counts, and (once placed) the
// device addresses; `view` is filled with the device view.
struct part_arrays {
    const void *src[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    std::size_t bytes[5] = {0, 0, 0, 0, 0};
    unsigned char *dev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int n = 0;
    bool slot_offsets = false; // array 2 of a Sliced-ELL part is computed on the device
    uint32_t slices = 0;
    std::size_t payload() const {
        std::size_t t = 0;
        for (int i = 0; i < n; ++i) t += align256(bytes[i]);
        return t;
    }
};

int plan_compressed(const cs_host_compressed *src, part_arrays *p, bool arrays = true) {
    if (src == nullptr || (arrays && ((src->nnz != 0u && (src->minorIdx == nullptr || src->val == nullptr)) ||
                                      src->majorPtr == nullptr))) {
        set_error("stage compressed: null partition or arrays");
        return 0;
    }
    const std::size_t major = src->axis == CS_COMPRESSED_BY_COL ? src->cols : src->rows;
    p->n = 3;
    p->src[0] = src->majorPtr;
    p->bytes[0] = (major + 1u) * 4u;
    p->src[1] = src->minorIdx;
    p->bytes[1] = (std::size_t) src->nnz * 4u;
    p->src[2] = src->val;
    p->bytes[2] = (std::size_t) src->nnz * 2u;
    return 1;
}

int plan_blocked_ell(const cs_host_blocked_ell *src, part_arrays *p, bool arrays = true) {
    if (src == nullptr || src->block_size == 0u || src->ell_cols % src->block_size != 0u ||
        (arrays && src->rows != 0u && src->ell_cols != 0u && (src->blockColIdx == nullptr || src->val == nullptr))) {
        set_error("stage blocked_ell: null partition, zero block size or block size not dividing ell_cols");
        return 0;
    }
    const std::size_t rb = ((std::size_t) src->rows + src->block_size - 1u) / src->block_size;
    p->n = 2;
    p->src[0] = src->blockColIdx;
    p->bytes[0] = rb * (src->ell_cols / src->block_size) * 4u;
    p->src[1] = src->val;
    p->bytes[1] = (std::size_t) src->rows * src->ell_cols * 2u;
    return 1;
}

int plan_sliced_ell(const cs_host_sliced_ell *src, part_arrays *p, bool arrays = true) {
    if (src == nullptr || (src->slice_count != 0u && (src->slice_row_offsets == nullptr ||
                                                      src->slice_widths == nullptr))) {
        set_error("stage sliced_ell: null partition or slice arrays");
        return 0;
    }
    const std::size_t S = src->slice_count, total = S ? sliced_total_slots(src) : 0u;
    if (total > 0xffffffffull) {
        set_error("stage sliced_ell: %zu slots exceed the u32 slot offsets", total);
        return 0;
    }
    if (arrays && total != 0u && (src->col_idx == nullptr || src->val == nullptr)) {
        set_error("stage sliced_ell: null slot arrays");
        return 0;
    }
    p->n = 5;
    p->src[0] = src->slice_row_offsets;
    p->bytes[0] = S ? (S + 1u) * 4u : 0u;
    p->src[1] = src->slice_widths;
    p->bytes[1] = S * 4u;
    p->src[2] = nullptr; // slot offsets: computed on the device
    p->bytes[2] = S * 4u;
    p->slot_offsets = true;
    p->slices = (uint32_t) S;
    p->src[3] = src->col_idx;
    p->bytes[3] = total * 4u;
    p->src[4] = src->val;
    p->bytes[4] = total * 2u;
    return 1;
}

std::size_t group_bytes(const std::vector<part_arrays> &parts, uint32_t format) {
    std::size_t t = align256(parts.size() * view_bytes_of(format));
    for (const auto &p : parts) t += p.payload();
    return t;
}

// --- the allocation cache (sharded_device.cuh:199-243) ---
void *take_cached(cs_sharded_device *st, int dev, std::size_t min_bytes, std::size_t *out_bytes) {
    *out_bytes = 0;
    if (st->cache == nullptr) return nullptr;
    unsigned long best = (unsigned long) -1;
    for (unsigned long i = 0; i < st->cache_count; ++i) {
        const cs_cached_allocation &c = st->cache[i];
        if (c.ptr == nullptr || c.device_id != dev || c.bytes < min_bytes) continue;
        if (best == (unsigned long) -1 || c.bytes < st->cache[best].bytes) best = i;
    }
    if (best == (unsigned long) -1) return nullptr;
    void *p = st->cache[best].ptr;
    *out_bytes = st->cache[best].bytes;
    st->cache[best] = st->cache[st->cache_count - 1u];
    --st->cache_count;
    return p;
}

int give_to_cache(cs_sharded_device *st, int dev, void *p, std::size_t bytes) {
    if (p == nullptr) return 1;
    if (bytes == 0u || st->cache_count >= CS_STAGE_CACHE_ENTRIES) return cuda_ok(cudaFree(p), "release free");
    if (st->cache_count == st->cache_capacity) {
        const unsigned long cap = CS_STAGE_CACHE_ENTRIES;
        auto *grown = static_cast<cs_cached_allocation *>(std::realloc(st->cache, cap * sizeof(cs_cached_allocation)));
        if (grown == nullptr) return cuda_ok(cudaFree(p), "release free");
        st->cache = grown;
        st->cache_capacity = cap;
    }
    st->cache[st->cache_count++] = cs_cached_allocation{p, bytes, dev};
    return 1;
}

void zero_part(cs_staged_part *r) {
    std::memset(r, 0, sizeof(*r));
    r->device_id = -1;
}

// Places the group's arrays in `base`, fills each view and record, enqueues
// the copies and kernels.  `views` receives the host copies of the views.
template <typename ViewFill>
int place_group(cs_sharded_device *st, unsigned long first, std::vector<part_arrays> &parts, uint32_t format,
                int dev, cudaStream_t stream, ViewFill fill_view) {
    const std::size_t need = group_bytes(parts, format);
    std::size_t got = 0;
    unsigned char *base = static_cast<unsigned char *>(take_cached(st, dev, need, &got));
    if (base == nullptr) {
        void *p = nullptr;
        if (!cuda_ok(cudaMalloc(&p, need), "stage allocation")) return 0;
        base = static_cast<unsigned char *>(p);
        got = need;
    }
    const std::size_t vb = view_bytes_of(format);
    std::vector<unsigned char> views(parts.size() * vb);
    std::size_t at = align256(parts.size() * vb);
    for (std::size_t k = 0; k < parts.size(); ++k) {
        part_arrays &p = parts[k];
        for (int i = 0; i < p.n; ++i) {
            p.dev[i] = base + at;
            at += align256(p.bytes[i]);
        }
        fill_view(k, p, views.data() + k * vb);
    }
    int ok = 1;
    for (std::size_t k = 0; k < parts.size() && ok; ++k) {
        const part_arrays &p = parts[k];
        for (int i = 0; i < p.n && ok; ++i)
            if (p.src[i] != nullptr && p.bytes[i] != 0u)
                ok = cuda_ok(cudaMemcpyAsync(p.dev[i], p.src[i], p.bytes[i], cudaMemcpyHostToDevice, stream),
                             "stage payload copy");
        if (ok && p.slot_offsets && p.slices != 0u) {
            sell_slot_offsets_kernel<<<1, 1024, 0, stream>>>(reinterpret_cast<const uint32_t *>(p.dev[0]),
                                                             reinterpret_cast<const uint32_t *>(p.dev[1]), p.slices,
                                                             reinterpret_cast<uint32_t *>(p.dev[2]));
            ok = launch_ok("sell_slot_offsets_kernel");
        }
    }
    for (std::size_t off = 0; off < views.size() && ok; off += kViewBlob) {
        const std::size_t n = std::min(kViewBlob, views.size() - off);
        view_blob blob;
        std::memcpy(blob.b, views.data() + off, n);
        write_views_kernel<<<1, 256, 0, stream>>>(base + off, blob, (unsigned) n);
        ok = launch_ok("write_views_kernel");
    }
    if (!ok) {
        // the copies may still be in flight: wait before the block is freed
        cudaStreamSynchronize(stream);
        cudaFree(base);
        return 0;
    }
    const unsigned long count = (unsigned long) parts.size();
    for (unsigned long k = 0; k < count; ++k) {
        cs_staged_part &r = st->parts[first + k];
        zero_part(&r);
        r.allocation = k == 0 ? base : nullptr;
        r.allocation_bytes = k == 0 ? got : 0u;
        r.storage = k == 0 ? base : nullptr;
        r.view = base + k * vb;
        void *arr[4] = {nullptr, nullptr, nullptr, nullptr};
        const part_arrays &p = parts[k];
        if (format == CS_FORMAT_SLICED_ELL) {
            arr[0] = p.dev[0];
            arr[1] = p.dev[1];
            arr[2] = p.dev[3];
            arr[3] = p.dev[4];
        } else {
            for (int i = 0; i < p.n && i < 4; ++i) arr[i] = p.dev[i];
        }
        r.a0 = arr[0];
        r.a1 = arr[1];
        r.a2 = arr[2];
        r.a3 = arr[3];
        r.group_begin = first;
        r.group_end = first + count;
        r.device_id = dev;
    }
    return 1;
}

int release_one(cs_sharded_device *st, unsigned long part_id) {
    if (st == nullptr) {
        set_error("release: null state");
        return 0;
    }
    if (part_id >= st->capacity || st->parts == nullptr || st->parts[part_id].view == nullptr) return 1;
    cs_staged_part &r = st->parts[part_id];
    if (!cuda_ok(cudaSetDevice(r.device_id >= 0 ? r.device_id : 0), "release set device")) return 0;
    const unsigned long b = r.group_begin, e = r.group_end;
    if (e <= b || e > st->capacity) {
        // standalone record: free its own block
        void *p = r.allocation != nullptr ? r.allocation : r.storage;
        const int ok = p == nullptr || cuda_ok(cudaFree(p), "release free");
        zero_part(&r);
        return ok;
    }
    cs_staged_part &owner = st->parts[b];
    int ok = 1;
    if (owner.allocation != nullptr)
        ok = give_to_cache(st, owner.device_id, owner.allocation, owner.allocation_bytes);
    else if (owner.storage != nullptr)
        ok = cuda_ok(cudaFree(owner.storage), "release free");
    if (!ok) return 0;
    for (unsigned long i = b; i < e; ++i) zero_part(&st->parts[i]);
    return 1;
}

void fill_compressed_view(const cs_host_compressed *src, const part_arrays &p, unsigned char *out) {
    cs_compressed_view v{};
    v.rows = src->rows;
    v.cols = src->cols;
    v.nnz = src->nnz;
    v.axis = src->axis;
    v.majorPtr = reinterpret_cast<uint32_t *>(p.dev[0]);
    v.minorIdx = reinterpret_cast<uint32_t *>(p.dev[1]);
    v.val = reinterpret_cast<uint16_t *>(p.dev[2]);
    std::memcpy(out, &v, sizeof(v));
}

void fill_blocked_ell_view(const cs_host_blocked_ell *src, const part_arrays &p, unsigned char *out) {
    cs_blocked_ell_view v{};
    v.rows = src->rows;
    v.cols = src->cols;
    v.nnz = src->nnz;
    v.block_size = src->block_size;
    v.ell_cols = src->ell_cols;
    v.blockColIdx = reinterpret_cast<uint32_t *>(p.dev[0]);
    v.val = reinterpret_cast<uint16_t *>(p.dev[1]);
    std::memcpy(out, &v, sizeof(v));
}

void fill_sliced_ell_view(const cs_host_sliced_ell *src, const part_arrays &p, unsigned char *out) {
    cs_sliced_ell_view v{};
    v.rows = src->rows;
    v.cols = src->cols;
    v.nnz = src->nnz;
    v.slice_count = src->slice_count;
    v.slice_rows = src->slice_count ? src->slice_row_offsets[1] - src->slice_row_offsets[0] : 0u;
    v.slice_row_offsets = reinterpret_cast<uint32_t *>(p.dev[0]);
    v.slice_widths = reinterpret_cast<uint32_t *>(p.dev[1]);
    v.slice_slot_offsets = reinterpret_cast<uint32_t *>(p.dev[2]);
    v.col_idx = reinterpret_cast<uint32_t *>(p.dev[3]);
    v.val = reinterpret_cast<uint16_t *>(p.dev[4]);
    std::memcpy(out, &v, sizeof(v));
}

template <typename HostT, typename PlanFn, typename FillFn>
int stage_range(cs_sharded_device *st, unsigned long first, unsigned long count, const HostT *const *srcs, int dev,
                cudaStream_t stream, uint32_t format, PlanFn plan, FillFn fill, const char *what) {
    if (st == nullptr || (count != 0u && srcs == nullptr)) {
        set_error("%s: null state or partition list", what);
        return 0;
    }
    if (count == 0u) return 1;
    if (first >= st->capacity || count > st->capacity - first || st->parts == nullptr) {
        set_error("%s: partitions [%lu, %lu) outside the state's %lu records", what, first, first + count,
                  st->capacity);
        return 0;
    }
    unsigned long i = first;
    for (; i < first + count; ++i)
        if (st->parts[i].view == nullptr || st->parts[i].device_id != dev) break;
    if (i == first + count) return 1; // every partition already resident on this device
    std::vector<part_arrays> parts(count);
    for (unsigned long k = 0; k < count; ++k)
        if (!plan(srcs[k], &parts[k], true)) return 0;
    for (i = first; i < first + count; ++i)
        if (st->parts[i].view != nullptr && !release_one(st, i)) return 0;
    if (!cuda_ok(cudaSetDevice(dev), "stage set device")) return 0;
    return place_group(st, first, parts, format, dev, stream,
                       [&](std::size_t k, const part_arrays &p, unsigned char *out) { fill(srcs[k], p, out); });
}

} // namespace
} // namespace csb

extern "C" int cs_b200_sharded_device_reserve(cs_sharded_device *st, unsigned long capacity) {
    if (st == nullptr) {
        set_error("sharded_device_reserve: null state");
        return 0;
    }
    if (capacity <= st->capacity) return 1;
    auto *rec = static_cast<cs_staged_part *>(std::malloc(capacity * sizeof(cs_staged_part)));
    if (rec == nullptr) {
        set_error("sharded_device_reserve: out of host memory for %lu records", capacity);
        return 0;
    }
    for (unsigned long i = 0; i < capacity; ++i) zero_part(&rec[i]);
    if (st->parts != nullptr && st->capacity != 0u) std::memcpy(rec, st->parts, st->capacity * sizeof(cs_staged_part));
    std::free(st->parts);
    st->parts = rec;
    st->capacity = capacity;
    return 1;
}

extern "C" int cs_b200_sharded_device_clear(cs_sharded_device *st) {
    if (st == nullptr) {
        set_error("sharded_device_clear: null state");
        return 0;
    }
    int ok = 1;
    for (unsigned long i = 0; st->parts != nullptr && i < st->capacity; ++i)
        if (st->parts[i].view != nullptr && !release_one(st, i)) ok = 0;
    for (unsigned long i = 0; st->cache != nullptr && i < st->cache_count; ++i) {
        if (st->cache[i].ptr == nullptr) continue;
        cudaSetDevice(st->cache[i].device_id >= 0 ? st->cache[i].device_id : 0);
        if (!cuda_ok(cudaFree(st->cache[i].ptr), "clear cached block")) ok = 0;
    }
    std::free(st->parts);
    std::free(st->cache);
    std::memset(st, 0, sizeof(*st));
    return ok;
}

extern "C" int cs_b200_stage_partition_compressed(cs_sharded_device *st, unsigned long part_id,
                                                  const cs_host_compressed *src, int dev, cs_stream_t s) {
    return stage_range(st, part_id, 1ul, &src, dev, as_stream(s), CS_FORMAT_COMPRESSED, plan_compressed,
                       fill_compressed_view, "stage_partition_compressed");
}

extern "C" int cs_b200_stage_partition_blocked_ell(cs_sharded_device *st, unsigned long part_id,
                                                   const cs_host_blocked_ell *src, int dev, cs_stream_t s) {
    return stage_range(st, part_id, 1ul, &src, dev, as_stream(s), CS_FORMAT_BLOCKED_ELL, plan_blocked_ell,
                       fill_blocked_ell_view, "stage_partition_blocked_ell");
}

extern "C" int cs_b200_stage_partition_sliced_ell(cs_sharded_device *st, unsigned long part_id,
                                                  const cs_host_sliced_ell *src, int dev, cs_stream_t s) {
    return stage_range(st, part_id, 1ul, &src, dev, as_stream(s), CS_FORMAT_SLICED_ELL, plan_sliced_ell,
                       fill_sliced_ell_view, "stage_partition_sliced_ell");
}

extern "C" int cs_b200_stage_shard_compressed(cs_sharded_device *st, unsigned long first, unsigned long count,
                                              const cs_host_compressed *const *parts, int dev, cs_stream_t s) {
    return stage_range(st, first, count, parts, dev, as_stream(s), CS_FORMAT_COMPRESSED, plan_compressed,
                       fill_compressed_view, "stage_shard_compressed");
}

extern "C" int cs_b200_stage_shard_blocked_ell(cs_sharded_device *st, unsigned long first, unsigned long count,
                                               const cs_host_blocked_ell *const *parts, int dev, cs_stream_t s) {
    return stage_range(st, first, count, parts, dev, as_stream(s), CS_FORMAT_BLOCKED_ELL, plan_blocked_ell,
                       fill_blocked_ell_view, "stage_shard_blocked_ell");
}

extern "C" int cs_b200_stage_shard_sliced_ell(cs_sharded_device *st, unsigned long first, unsigned long count,
                                              const cs_host_sliced_ell *const *parts, int dev, cs_stream_t s) {
    return stage_range(st, first, count, parts, dev, as_stream(s), CS_FORMAT_SLICED_ELL, plan_sliced_ell,
                       fill_sliced_ell_view, "stage_shard_sliced_ell");
}

extern "C" int cs_b200_release_staged_partition(cs_sharded_device *st, unsigned long part_id) {
    return release_one(st, part_id);
}

namespace {
template <typename HostT, typename PlanFn>
int staged_bytes(const HostT *const *parts, unsigned long count, size_t *out, uint32_t format, PlanFn plan) {
    if (out == nullptr || (count != 0u && parts == nullptr)) {
        set_error("staged_bytes: null argument");
        return 0;
    }
    std::vector<part_arrays> p(count);
    for (unsigned long k = 0; k < count; ++k)
        if (!plan(parts[k], &p[k], false)) return 0;
    *out = group_bytes(p, format);
    return 1;
}
} // namespace

extern "C" int cs_b200_staged_bytes_compressed(const cs_host_compressed *const *parts, unsigned long count,
                                               size_t *out) {
    return staged_bytes(parts, count, out, CS_FORMAT_COMPRESSED, plan_compressed);
}

extern "C" int cs_b200_staged_bytes_blocked_ell(const cs_host_blocked_ell *const *parts, unsigned long count,
                                                size_t *out) {
    return staged_bytes(parts, count, out, CS_FORMAT_BLOCKED_ELL, plan_blocked_ell);
}

extern "C" int cs_b200_staged_bytes_sliced_ell(const cs_host_sliced_ell *const *parts, unsigned long count,
                                               size_t *out) {
    return staged_bytes(parts, count, out, CS_FORMAT_SLICED_ELL, plan_sliced_ell);
}
