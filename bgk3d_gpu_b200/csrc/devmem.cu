// Device memory of library-owned objects (lattices, batches, masks,
// reduction workspaces): one stream-ordered memory pool per device, set-up
// copies and kernels on a private non-blocking stream.
//
// A request server creates and destroys lattices of many sizes while other
// lattices step.  cudaMalloc/cudaFree map and unmap the memory each time
// (milliseconds for GB-sized lattices) and cudaMemcpy on the legacy stream
// waits for every kernel in flight.  Here an allocation comes from the pool
// (memory freed earlier is reused without mapping when the pool retains it),
// is zeroed on the private stream and is ready for any stream on return; a
// free waits for the device like cudaFree does, then returns the block to the
// pool.  With the default retention of 0 bytes the pool gives freed memory
// back to the device at once, which is cudaFree's behaviour.
#include <cstdint>
#include <mutex>

#include "bgk3d_lattice.h"
#include "bgk_internal.h"

namespace bgk {
namespace {

struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    size_t retain = 0;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
DevicePool g_pools[kMaxDevices];

int current_pool(DevicePool** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "device: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(BGK_ERR_UNSUPPORTED, "device %d", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    DevicePool& P = g_pools[dev];
    if (!P.pool) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        e = cudaMemPoolCreate(&P.pool, &props);
        if (e != cudaSuccess) { P.pool = nullptr; return set_error(BGK_ERR_CUDA, "memory pool: %s", cudaGetErrorString(e)); }
        uint64_t thr = P.retain;
        cudaMemPoolSetAttribute(P.pool, cudaMemPoolAttrReleaseThreshold, &thr);
        e = cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(P.pool);
            P.pool = nullptr; P.stream = nullptr;
            return set_error(BGK_ERR_CUDA, "set-up stream: %s", cudaGetErrorString(e));
        }
    }
    *out = &P;
    return BGK_OK;
}

}  // namespace

int dev_alloc(void** p, size_t bytes, bool zero, const char* what) {
    *p = nullptr;
    DevicePool* P = nullptr;
    if (int rc = current_pool(&P)) return rc;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, P->pool, P->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_error(BGK_ERR_NOMEM, "%s (%zu bytes): %s", what, bytes, cudaGetErrorString(e));
    }
    if (zero && bytes) e = cudaMemsetAsync(*p, 0, bytes, P->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(P->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(*p, P->stream);
        *p = nullptr;
        return set_error(BGK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    return BGK_OK;
}

void dev_free(void* p) {
    if (!p) return;
    DevicePool* P = nullptr;
    if (current_pool(&P)) return;
    cudaDeviceSynchronize();            // no kernel of any stream may still use p
    cudaFreeAsync(p, P->stream);
    if (P->retain == 0) {
        cudaStreamSynchronize(P->stream);
        cudaMemPoolTrimTo(P->pool, 0);
    }
}

void dev_free_async(void* p, cudaStream_t st) {
    if (!p) return;
    cudaFreeAsync(p, st);               // after the work queued on st
}

cudaStream_t setup_stream() {
    DevicePool* P = nullptr;
    if (current_pool(&P)) return nullptr;
    return P->stream;
}

}  // namespace bgk

using namespace bgk;

extern "C" int bgk_set_retained_bytes(size_t bytes) {
    DevicePool* P = nullptr;
    if (int rc = current_pool(&P)) return rc;
    P->retain = bytes;
    uint64_t thr = bytes;
    cudaError_t e = cudaMemPoolSetAttribute(P->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "release threshold: %s", cudaGetErrorString(e));
    if (bytes == 0) {
        cudaStreamSynchronize(P->stream);
        cudaMemPoolTrimTo(P->pool, 0);
    }
    return BGK_OK;
}

extern "C" int bgk_trim_memory(void) {
    DevicePool* P = nullptr;
    if (int rc = current_pool(&P)) return rc;
    cudaError_t e = cudaStreamSynchronize(P->stream);
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(P->pool, 0);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "trim: %s", cudaGetErrorString(e));
    return BGK_OK;
}
