// .cspack raw partition records straight between a file and device memory.
//
// Record layout (src/io/pack/packfile.cu:13-47,265-272,351-369,597-621,715-721;
// little-endian, no padding): a 13-byte header (u8 format, u32 rows, u32 cols,
// u32 nnz), then per format
//   compressed  (2)  u32 axis, val[nnz], majorPtr[major + 1] (when major > 0), minorIdx[nnz]
//   COO         (3)  val[nnz], rowIdx[nnz], colIdx[nnz]
//   Blocked-ELL (6)  u32 block_size, u32 ell_cols, blockColIdx[row_blocks x width], val[rows x ell_cols]
//   Sliced-ELL  (7)  u32 slice_count, slice_row_offsets[S + 1], slice_widths[S], col_idx[slots], val[slots]
// with fp16 values.  The reference stores and loads through host arrays
// (fwrite / fread); here each array moves through two pinned staging buffers:
// while one chunk is copied between device and pinned memory on the stream,
// the other is written to or read from the file.
#include "common.cuh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace csb {
namespace {

constexpr std::size_t kChunk = (std::size_t) 32 << 20;
constexpr uint8_t kFmtCompressed = 2u, kFmtCoo = 3u, kFmtBlockedEll = 6u, kFmtSlicedEll = 7u;

struct file_guard {
    std::FILE *fp = nullptr;
    ~file_guard() {
        if (fp) std::fclose(fp);
    }
};

// Two pinned buffers and their copy events.
struct staging {
    void *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t s = nullptr;
    ~staging() {
        for (int i = 0; i < 2; ++i) {
            if (ev[i]) cudaEventDestroy(ev[i]);
            if (buf[i]) cudaFreeHost(buf[i]);
        }
        if (s) cudaStreamDestroy(s);
    }
    std::size_t chunk = kChunk;
    // buffers no larger than the record's largest array needs
    bool open(std::size_t largest = kChunk) {
        chunk = largest < kChunk ? (largest < 4096u ? 4096u : largest) : kChunk;
        for (int i = 0; i < 2; ++i)
            if (!cuda_ok(cudaMallocHost(&buf[i], chunk), "pinned staging") ||
                !cuda_ok(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming), "staging event"))
                return false;
        return cuda_ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "staging stream") != 0;
    }
};

bool put(std::FILE *fp, const void *p, std::size_t n) { return n == 0u || std::fwrite(p, 1, n, fp) == n; }
bool get(std::FILE *fp, void *p, std::size_t n) { return n == 0u || std::fread(p, 1, n, fp) == n; }

// device -> file: chunk i is copied while chunk i - 1 is written.
bool store_array(std::FILE *fp, staging &st, const void *dev, std::size_t bytes) {
    const char *src = (const char *) dev;
    std::size_t prev_n = 0u;
    int prev = -1;
    for (std::size_t off = 0, i = 0; off < bytes; off += st.chunk, ++i) {
        const int b = (int) (i & 1u);
        const std::size_t n = bytes - off < st.chunk ? bytes - off : st.chunk;
        if (!cuda_ok(cudaMemcpyAsync(st.buf[b], src + off, n, cudaMemcpyDeviceToHost, st.s), "D2H chunk") ||
            !cuda_ok(cudaEventRecord(st.ev[b], st.s), "chunk event"))
            return false;
        if (prev >= 0) {
            if (!cuda_ok(cudaEventSynchronize(st.ev[prev]), "chunk wait") || !put(fp, st.buf[prev], prev_n)) return false;
        }
        prev = b;
        prev_n = n;
    }
    if (prev >= 0)
        return cuda_ok(cudaEventSynchronize(st.ev[prev]), "chunk wait") && put(fp, st.buf[prev], prev_n);
    return true;
}

// file -> device: chunk i is read while chunk i - 1 is copied.
bool load_array(std::FILE *fp, staging &st, void *dev, std::size_t bytes) {
    char *dst = (char *) dev;
    bool used[2] = {false, false};
    for (std::size_t off = 0, i = 0; off < bytes; off += st.chunk, ++i) {
        const int b = (int) (i & 1u);
        const std::size_t n = bytes - off < st.chunk ? bytes - off : st.chunk;
        if (used[b] && !cuda_ok(cudaEventSynchronize(st.ev[b]), "buffer wait")) return false;
        if (!get(fp, st.buf[b], n)) {
            set_error("cspack: file ends inside an array");
            return false;
        }
        if (!cuda_ok(cudaMemcpyAsync(dst + off, st.buf[b], n, cudaMemcpyHostToDevice, st.s), "H2D chunk") ||
            !cuda_ok(cudaEventRecord(st.ev[b], st.s), "chunk event"))
            return false;
        used[b] = true;
    }
    return cuda_ok(cudaStreamSynchronize(st.s), "load sync") != 0;
}

bool write_header(std::FILE *fp, uint8_t fmt, uint32_t rows, uint32_t cols, uint32_t nnz) {
    return put(fp, &fmt, 1) && put(fp, &rows, 4) && put(fp, &cols, 4) && put(fp, &nnz, 4);
}

bool open_file(file_guard &g, const char *path, const char *mode, const char *who) {
    g.fp = path != nullptr ? std::fopen(path, mode) : nullptr;
    if (g.fp == nullptr) {
        set_error("%s: cannot open %s", who, path != nullptr ? path : "(null)");
        return false;
    }
    std::setvbuf(g.fp, nullptr, _IOFBF, (std::size_t) 8u << 20u);
    return true;
}

bool read_info(std::FILE *fp, cs_cspack_info *info, std::vector<uint32_t> *offsets, std::vector<uint32_t> *widths) {
    std::memset(info, 0, sizeof(*info));
    uint8_t fmt = 0;
    if (!get(fp, &fmt, 1) || !get(fp, &info->rows, 4) || !get(fp, &info->cols, 4) || !get(fp, &info->nnz, 4)) {
        set_error("cspack: short header");
        return false;
    }
    info->format = fmt;
    switch (fmt) {
    case kFmtCompressed:
        return get(fp, &info->axis, 4);
    case kFmtCoo:
        return true;
    case kFmtBlockedEll:
        return get(fp, &info->block_size, 4) && get(fp, &info->ell_cols, 4);
    case kFmtSlicedEll: {
        if (!get(fp, &info->slice_count, 4)) return false;
        offsets->resize((std::size_t) info->slice_count + 1u);
        widths->resize(info->slice_count);
        if (!get(fp, offsets->data(), offsets->size() * 4u) || !get(fp, widths->data(), widths->size() * 4u))
            return false;
        uint32_t total = 0u; // u32 as the reference's total_slots
        for (uint32_t s = 0; s < info->slice_count; ++s) total += ((*offsets)[s + 1u] - (*offsets)[s]) * (*widths)[s];
        info->total_slots = total;
        return true;
    }
    default:
        set_error("cspack: format %u is not one of compressed (2), COO (3), Blocked-ELL (6), Sliced-ELL (7)", fmt);
        return false;
    }
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_cspack_peek(const char *path, cs_cspack_info *info) {
    if (info == nullptr) {
        set_error("cspack_peek: null info");
        return 0;
    }
    file_guard g;
    if (!open_file(g, path, "rb", "cspack_peek")) return 0;
    std::vector<uint32_t> offs, widths;
    if (!read_info(g.fp, info, &offs, &widths)) {
        set_error("cspack_peek: %s is not a readable record", path);
        return 0;
    }
    return 1;
}

extern "C" int cs_b200_cspack_store_blocked_ell(const char *path, const cs_blocked_ell_view *part) {
    if (part == nullptr || (part->rows != 0u && part->block_size == 0u)) {
        set_error("cspack_store_blocked_ell: null view or zero block size");
        return 0;
    }
    const uint32_t B = part->block_size;
    const std::size_t rb = B == 0u ? 0u : ((std::size_t) part->rows + B - 1u) / B;
    const std::size_t w = B == 0u ? 0u : part->ell_cols / B;
    file_guard g;
    staging st;
    if (!open_file(g, path, "wb", "cspack_store_blocked_ell") ||
        !st.open((std::size_t) part->rows * part->ell_cols * 2u > rb * w * 4u ? (std::size_t) part->rows * part->ell_cols * 2u
                                                                              : rb * w * 4u))
        return 0;
    if (!write_header(g.fp, kFmtBlockedEll, part->rows, part->cols, part->nnz) || !put(g.fp, &B, 4) ||
        !put(g.fp, &part->ell_cols, 4) || !store_array(g.fp, st, part->blockColIdx, rb * w * 4u) ||
        !store_array(g.fp, st, part->val, (std::size_t) part->rows * part->ell_cols * 2u)) {
        set_error("cspack_store_blocked_ell: write to %s failed", path);
        return 0;
    }
    return 1;
}

extern "C" int cs_b200_cspack_load_blocked_ell(const char *path, const cs_blocked_ell_view *dst) {
    file_guard g;
    staging st;
    cs_cspack_info info;
    std::vector<uint32_t> o, w;
    if (dst == nullptr || !open_file(g, path, "rb", "cspack_load_blocked_ell") || !read_info(g.fp, &info, &o, &w))
        return 0;
    if (info.format != kFmtBlockedEll || info.rows != dst->rows || info.block_size != dst->block_size ||
        info.ell_cols != dst->ell_cols) {
        set_error("cspack_load_blocked_ell: %s holds format %u, %u rows, block %u, ell_cols %u; the destination "
                  "differs", path, info.format, info.rows, info.block_size, info.ell_cols);
        return 0;
    }
    const uint32_t B = info.block_size;
    const std::size_t rb = B == 0u ? 0u : ((std::size_t) info.rows + B - 1u) / B;
    const std::size_t wd = B == 0u ? 0u : info.ell_cols / B;
    const std::size_t vb = (std::size_t) info.rows * info.ell_cols * 2u, ib = rb * wd * 4u;
    return st.open(vb > ib ? vb : ib) && load_array(g.fp, st, dst->blockColIdx, rb * wd * 4u) &&
           load_array(g.fp, st, dst->val, (std::size_t) info.rows * info.ell_cols * 2u);
}

extern "C" int cs_b200_cspack_store_sliced_ell(const char *path, const cs_sliced_ell_view *part) {
    if (part == nullptr) {
        set_error("cspack_store_sliced_ell: null view");
        return 0;
    }
    const uint32_t S = part->slice_count;
    std::vector<uint32_t> offs((std::size_t) S + 1u, 0u), widths(S);
    if ((S != 0u && (!cuda_ok(cudaMemcpy(offs.data(), part->slice_row_offsets, offs.size() * 4u,
                                         cudaMemcpyDeviceToHost), "D2H offsets") ||
                     !cuda_ok(cudaMemcpy(widths.data(), part->slice_widths, widths.size() * 4u,
                                         cudaMemcpyDeviceToHost), "D2H widths"))))
        return 0;
    uint32_t total = 0u;
    for (uint32_t s = 0; s < S; ++s) total += (offs[s + 1u] - offs[s]) * widths[s];
    file_guard g;
    staging st;
    if (!open_file(g, path, "wb", "cspack_store_sliced_ell") || !st.open((std::size_t) total * 4u)) return 0;
    if (!write_header(g.fp, kFmtSlicedEll, part->rows, part->cols, part->nnz) || !put(g.fp, &S, 4) ||
        !put(g.fp, offs.data(), offs.size() * 4u) || !put(g.fp, widths.data(), widths.size() * 4u) ||
        !store_array(g.fp, st, part->col_idx, (std::size_t) total * 4u) ||
        !store_array(g.fp, st, part->val, (std::size_t) total * 2u)) {
        set_error("cspack_store_sliced_ell: write to %s failed", path);
        return 0;
    }
    return 1;
}

extern "C" int cs_b200_cspack_load_sliced_ell(const char *path, const cs_sliced_ell_view *dst) {
    file_guard g;
    staging st;
    cs_cspack_info info;
    std::vector<uint32_t> offs, widths;
    if (dst == nullptr || !open_file(g, path, "rb", "cspack_load_sliced_ell") || !read_info(g.fp, &info, &offs, &widths))
        return 0;
    if (info.format != kFmtSlicedEll || info.rows != dst->rows || info.slice_count != dst->slice_count) {
        set_error("cspack_load_sliced_ell: %s holds format %u, %u rows, %u slices; the destination differs", path,
                  info.format, info.rows, info.slice_count);
        return 0;
    }
    // slot offsets of the device view: running sum of rows x width per slice
    std::vector<uint32_t> slots(info.slice_count);
    uint32_t run = 0u;
    for (uint32_t s = 0; s < info.slice_count; ++s) {
        slots[s] = run;
        run += (offs[s + 1u] - offs[s]) * widths[s];
    }
    if (!st.open((std::size_t) info.total_slots * 4u)) return 0;
    if (info.slice_count != 0u &&
        (!cuda_ok(cudaMemcpyAsync(dst->slice_row_offsets, offs.data(), offs.size() * 4u, cudaMemcpyHostToDevice, st.s),
                  "H2D offsets") ||
         !cuda_ok(cudaMemcpyAsync(dst->slice_widths, widths.data(), widths.size() * 4u, cudaMemcpyHostToDevice, st.s),
                  "H2D widths") ||
         (dst->slice_slot_offsets != nullptr &&
          !cuda_ok(cudaMemcpyAsync(dst->slice_slot_offsets, slots.data(), slots.size() * 4u, cudaMemcpyHostToDevice,
                                   st.s), "H2D slot offsets")) ||
         !cuda_ok(cudaStreamSynchronize(st.s), "slice tables")))
        return 0;
    return load_array(g.fp, st, dst->col_idx, (std::size_t) info.total_slots * 4u) &&
           load_array(g.fp, st, dst->val, (std::size_t) info.total_slots * 2u);
}

extern "C" int cs_b200_cspack_store_compressed(const char *path, const cs_compressed_view *part) {
    if (part == nullptr) {
        set_error("cspack_store_compressed: null view");
        return 0;
    }
    const uint32_t major = part->axis == CS_COMPRESSED_BY_COL ? part->cols : part->rows;
    file_guard g;
    staging st;
    const std::size_t big = (std::size_t) (part->nnz > major + 1u ? part->nnz : major + 1u) * 4u;
    if (!open_file(g, path, "wb", "cspack_store_compressed") || !st.open(big)) return 0;
    if (!write_header(g.fp, kFmtCompressed, part->rows, part->cols, part->nnz) || !put(g.fp, &part->axis, 4) ||
        !store_array(g.fp, st, part->val, (std::size_t) part->nnz * 2u) ||
        (major != 0u && !store_array(g.fp, st, part->majorPtr, ((std::size_t) major + 1u) * 4u)) ||
        !store_array(g.fp, st, part->minorIdx, (std::size_t) part->nnz * 4u)) {
        set_error("cspack_store_compressed: write to %s failed", path);
        return 0;
    }
    return 1;
}

extern "C" int cs_b200_cspack_load_compressed(const char *path, const cs_compressed_view *dst) {
    file_guard g;
    staging st;
    cs_cspack_info info;
    std::vector<uint32_t> o, w;
    if (dst == nullptr || !open_file(g, path, "rb", "cspack_load_compressed") || !read_info(g.fp, &info, &o, &w))
        return 0;
    if (info.format != kFmtCompressed || info.rows != dst->rows || info.cols != dst->cols || info.nnz != dst->nnz ||
        info.axis != dst->axis) {
        set_error("cspack_load_compressed: %s holds format %u, %u x %u, %u nnz, axis %u; the destination differs",
                  path, info.format, info.rows, info.cols, info.nnz, info.axis);
        return 0;
    }
    const uint32_t major = info.axis == CS_COMPRESSED_BY_COL ? info.cols : info.rows;
    const std::size_t big = (std::size_t) (info.nnz > major + 1u ? info.nnz : major + 1u) * 4u;
    return st.open(big) && load_array(g.fp, st, dst->val, (std::size_t) info.nnz * 2u) &&
           (major == 0u || load_array(g.fp, st, dst->majorPtr, ((std::size_t) major + 1u) * 4u)) &&
           load_array(g.fp, st, dst->minorIdx, (std::size_t) info.nnz * 4u);
}

extern "C" int cs_b200_cspack_store_coo(const char *path, const cs_coo_view *part) {
    if (part == nullptr) {
        set_error("cspack_store_coo: null view");
        return 0;
    }
    file_guard g;
    staging st;
    if (!open_file(g, path, "wb", "cspack_store_coo") || !st.open((std::size_t) part->nnz * 4u)) return 0;
    if (!write_header(g.fp, kFmtCoo, part->rows, part->cols, part->nnz) ||
        !store_array(g.fp, st, part->val, (std::size_t) part->nnz * 2u) ||
        !store_array(g.fp, st, part->rowIdx, (std::size_t) part->nnz * 4u) ||
        !store_array(g.fp, st, part->colIdx, (std::size_t) part->nnz * 4u)) {
        set_error("cspack_store_coo: write to %s failed", path);
        return 0;
    }
    return 1;
}

extern "C" int cs_b200_cspack_load_coo(const char *path, const cs_coo_view *dst) {
    file_guard g;
    staging st;
    cs_cspack_info info;
    std::vector<uint32_t> o, w;
    if (dst == nullptr || !open_file(g, path, "rb", "cspack_load_coo") || !read_info(g.fp, &info, &o, &w)) return 0;
    if (info.format != kFmtCoo || info.nnz != dst->nnz) {
        set_error("cspack_load_coo: %s holds format %u with %u entries; the destination differs", path, info.format,
                  info.nnz);
        return 0;
    }
    return st.open((std::size_t) info.nnz * 4u) && load_array(g.fp, st, dst->val, (std::size_t) info.nnz * 2u) &&
           load_array(g.fp, st, dst->rowIdx, (std::size_t) info.nnz * 4u) &&
           load_array(g.fp, st, dst->colIdx, (std::size_t) info.nnz * 4u);
}
