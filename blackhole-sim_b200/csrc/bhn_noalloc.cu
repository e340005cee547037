// bhn_noalloc.cu -- the fused renderer for callers that cannot allocate device
// memory.
//
// bhn_render_launch needs a scratch buffer (work-queue head, per-view camera
// tables, launch totals) that the caller normally allocates.  Some callers
// cannot: hosts whose device memory is owned by their own allocator or by a
// pool sized at start-up, where a library they load may not allocate beside
// it, and real-time loops that may not take the device-wide synchronisation
// that cudaMalloc / cudaFree can imply.  This entry point keeps that scratch in
// a fixed, file-scope device array, so the caller passes only its inputs and
// outputs.
#include <cuda_runtime.h>

#include <atomic>

#include "bhn_internal.cuh"

namespace {

// The scratch of every bhn_render_noalloc call on a device.  The array is part
// of the library's device image: every GPU that loads the library holds these
// 64 KiB until the process exits.
constexpr int64_t kNoAllocScratchBytes = 64 * 1024;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static_assert(bhn::scratch_layout(BHN_NOALLOC_MAX_VIEWS).total <= kNoAllocScratchBytes,
              "BHN_NOALLOC_MAX_VIEWS views must fit the fixed scratch array");

// Device address of g_noalloc_scratch per device (the host-side name of a
// __device__ array is only a stand-in, never a device address).  It is looked
// up once per device and process; a cudaDeviceReset would invalidate it.
constexpr int kMaxDevices = 64;
std::atomic<void *> g_noalloc_ptr[kMaxDevices];

}  // namespace

using namespace bhn;

extern "C" int bhn_render_noalloc(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np,
                                  const bhn_view *h_views, int32_t n_views, const bhn_render_config *cfg, void *out,
                                  const bhn_ray_outputs *ray_out, bhn_render_stats *stats, void *stream) {
    if (n_views < 1 || n_views > BHN_NOALLOC_MAX_VIEWS)
        return fail(BHN_ERR_VALUE, "bhn_render_noalloc renders 1 to " + std::to_string(BHN_NOALLOC_MAX_VIEWS) +
                                       " views per call; got " + std::to_string(n_views));
    const int64_t need = bhn_render_scratch_bytes(n_views);
    if (need > kNoAllocScratchBytes)
        return fail(BHN_ERR_VALUE, "bhn_render_noalloc: " + std::to_string(n_views) + " views need " +
                                       std::to_string(need) + " scratch bytes, more than the fixed " +
                                       std::to_string(kNoAllocScratchBytes));
    int dev = 0;
    BHN_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(BHN_ERR_UNSUPPORTED, "device ordinal out of range");
    // Set-up on the first call on this device (with the device current): look up
    // the array's device address once and keep it.
    void *scratch = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev].store(scratch, std::memory_order_release);
    }
    // The launch zeroes the work-queue head and the launch totals it uses; the
    // per-view tables are rewritten by the set-up below.
    int rc = bhn_render_prepare(h_views, n_views, scratch, kNoAllocScratchBytes, stream);
    if (rc != BHN_OK) return rc;
    return bhn_render_launch(records, tables, nr, nt, np, n_views, cfg, out, ray_out, scratch, kNoAllocScratchBytes,
                             stats, stream);
}
