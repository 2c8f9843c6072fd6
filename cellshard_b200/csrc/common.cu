// Error state, device queries and the device-wide uint32 scan.
#include "common.cuh"

#include <cstdarg>
#include <cstring>

namespace csb {

namespace {
thread_local char g_last_error[512] = {0};
int g_sm_count[64] = {0};
} // namespace

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

void clear_error() { g_last_error[0] = '\0'; }

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (g_sm_count[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        g_sm_count[dev] = n;
    }
    return g_sm_count[dev];
}

unsigned resident_grid(const void *kernel, unsigned threads, std::size_t smem, std::size_t needed) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int) threads, smem) != cudaSuccess ||
        per_sm <= 0)
        per_sm = 1;
    std::size_t g = (std::size_t) sm_count() * (std::size_t) per_sm;
    if (g > needed) g = needed;
    return g == 0u ? 1u : (unsigned) g;
}

// ---------------------------------------------------------------------------
// Scan: 256 threads x 16 items = 4096 items per tile.
// ---------------------------------------------------------------------------
namespace {

constexpr unsigned kScanThreads = 256;
constexpr unsigned kScanItems = 16;
constexpr unsigned kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_kernel(const uint32_t *__restrict__ in, std::size_t n,
                                                                       uint32_t *__restrict__ tile_sums) {
    __shared__ uint32_t smem[33];
    uint32_t total;
    const std::size_t base = (std::size_t) blockIdx.x * kScanTile + (std::size_t) threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (unsigned i = 0; i < kScanItems; ++i) {
        const std::size_t k = base + i;
        if (k < n) s += in[k];
    }
    (void) block_exclusive_scan(s, smem, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) scan_of_tile_sums_kernel(uint32_t *__restrict__ tile_sums, std::size_t tiles,
                                                                 uint32_t *__restrict__ total_out) {
    __shared__ uint32_t smem[33];
    uint32_t total;
    uint32_t carry = 0;
    for (std::size_t base = 0; base < tiles; base += blockDim.x) {
        const std::size_t k = base + threadIdx.x;
        const uint32_t v = k < tiles ? tile_sums[k] : 0u;
        const uint32_t ex = block_exclusive_scan(v, smem, total);
        if (k < tiles) tile_sums[k] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && total_out != nullptr) *total_out = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint32_t *in, uint32_t *out, std::size_t n,
                                                                   const uint32_t *__restrict__ tile_offsets) {
    __shared__ uint32_t smem[33];
    uint32_t total;
    const std::size_t base = (std::size_t) blockIdx.x * kScanTile + (std::size_t) threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (unsigned i = 0; i < kScanItems; ++i) {
        const std::size_t k = base + i;
        v[i] = k < n ? in[k] : 0u;
        s += v[i];
    }
    uint32_t run = block_exclusive_scan(s, smem, total) + tile_offsets[blockIdx.x];
#pragma unroll
    for (unsigned i = 0; i < kScanItems; ++i) {
        const std::size_t k = base + i;
        if (k < n) out[k] = run;
        run += v[i];
    }
}

} // namespace

std::size_t scan_u32_scratch_bytes(std::size_t n) {
    const std::size_t tiles = (n + kScanTile - 1) / kScanTile;
    return align_up((tiles == 0 ? 1 : tiles) * sizeof(uint32_t), 256);
}

int scan_exclusive_u32(const uint32_t *in, uint32_t *out, std::size_t n, bool write_total, void *scratch,
                       std::size_t scratch_bytes, cudaStream_t stream) {
    const std::size_t tiles = (n + kScanTile - 1) / kScanTile;
    if (n == 0) {
        if (write_total) return cuda_ok(cudaMemsetAsync(out, 0, sizeof(uint32_t), stream), "scan empty total");
        return 1;
    }
    if (scratch == nullptr || scratch_bytes < scan_u32_scratch_bytes(n)) {
        set_error("scan scratch too small (%zu < %zu)", scratch_bytes, scan_u32_scratch_bytes(n));
        return 0;
    }
    if (tiles > 0x7fffffffu) {
        set_error("scan too large");
        return 0;
    }
    uint32_t *tile_sums = (uint32_t *) scratch;
    scan_tile_sums_kernel<<<(unsigned) tiles, kScanThreads, 0, stream>>>(in, n, tile_sums);
    if (!launch_ok("scan_tile_sums_kernel")) return 0;
    scan_of_tile_sums_kernel<<<1, 1024, 0, stream>>>(tile_sums, tiles, write_total ? out + n : nullptr);
    if (!launch_ok("scan_of_tile_sums_kernel")) return 0;
    scan_apply_kernel<<<(unsigned) tiles, kScanThreads, 0, stream>>>(in, out, n, tile_sums);
    return launch_ok("scan_apply_kernel");
}

} // namespace csb

extern "C" int cs_b200_abi_version(void) { return CS_B200_ABI_VERSION; }

extern "C" const char *cs_b200_last_error(void) { return csb::g_last_error; }
