// Grouped moments over a fixed, library-owned scratch array: the entry point
// for callers that must not allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a plugin running inside
// a host process whose device memory belongs to another allocator (a
// framework's caching pool, a serving loop that admits requests against a
// fixed HBM budget) may not create allocations of its own, both because
// cudaMalloc synchronises the device in the middle of other work and because
// it would change the process's memory footprint behind the owner's back.
// This entry point takes the caller's inputs and outputs and does everything
// else inside one statically sized device array that the library owns.
//
// The array below is CS_NOALLOC_SCRATCH_BYTES large.  Every GPU on which this
// file's module is loaded holds it until the process exits.  In host code its
// name is only a host-side stand-in, never a device address: the device
// address is obtained once per device with cudaGetSymbolAddress (with that
// device current) and cached.  The first call on each device performs that
// set-up, so that first call should come before any stream capture.  The
// cached address belongs to the device's primary context: after
// cudaDeviceReset the module is loaded again and the array may move, so a
// process that resets a device must not use this entry point on it again.
//
// All calls share the one array and the array keeps the previous call's
// contents.  The reduction writes every scratch byte it reads during the same
// call before reading it, so nothing has to be cleared between calls, but
// calls whose work overlaps on the GPU (concurrent streams, or several host
// threads on one device) race on the array and must be serialised by the
// caller.
#include "common.cuh"

#include <atomic>

namespace csb {

std::size_t group_moments_scratch_needed(const cs_blocked_ell_view *src, const cs_group_moments_params *params);
int group_moments_launch(const cs_blocked_ell_view *src, const uint8_t *d_row_keep, const uint8_t *d_feature_keep,
                         const uint32_t *d_row_labels, const cs_group_moments_params *params,
                         const cs_group_moments_out *out, void *d_scratch, size_t scratch_bytes, cs_stream_t s);

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[CS_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::atomic<void *> g_scratch_ptr[kMaxDevices];

// Device address of g_noalloc_scratch on the current device (set up on first use).
void *scratch_address() {
    int dev = -1;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice (static scratch)")) return nullptr;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("group_moments_noalloc: device ordinal %d outside the supported range", dev);
        return nullptr;
    }
    void *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (p != nullptr) return p;
    if (!cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress (static scratch)")) return nullptr;
    if (p == nullptr) {
        set_error("group_moments_noalloc: cudaGetSymbolAddress returned a null address");
        return nullptr;
    }
    g_scratch_ptr[dev].store(p, std::memory_order_release);
    return p;
}

} // namespace
} // namespace csb

using namespace csb;

extern "C" int cs_b200_group_moments_blocked_ell_noalloc(const cs_blocked_ell_view *src, const uint8_t *d_row_keep,
                                                          const uint8_t *d_feature_keep, const uint32_t *d_row_labels,
                                                          const cs_group_moments_params *params,
                                                          const cs_group_moments_out *out, cs_stream_t stream) {
    const std::size_t need = group_moments_scratch_needed(src, params);
    if (need == 0) return 0;
    if (need > (std::size_t) CS_NOALLOC_SCRATCH_BYTES) {
        set_error("group_moments_noalloc: this partition needs %zu bytes of scratch but the static scratch holds "
                  "%zu; use fewer rows per call, a larger chunk_rows, or cs_b200_group_moments_blocked_ell with "
                  "caller scratch",
                  need, (std::size_t) CS_NOALLOC_SCRATCH_BYTES);
        return 0;
    }
    void *scratch = scratch_address();
    if (scratch == nullptr) return 0;
    return group_moments_launch(src, d_row_keep, d_feature_keep, d_row_labels, params, out, scratch,
                                (std::size_t) CS_NOALLOC_SCRATCH_BYTES, stream);
}
