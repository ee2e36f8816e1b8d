// bgk_moments_noalloc: the FP64 moments reduction with its scratch in a
// fixed device array of this library instead of a caller-provided workspace.
//
// Some callers cannot allocate device memory where they need the
// diagnostic: a Fortran/OpenACC driver whose device arrays are all owned by
// the directive runtime and that links only a C ABI without a device
// allocator, or a long-running solver or server that reserves its whole
// device-memory budget up front and forbids allocation (and the implicit
// synchronisation cudaMalloc may bring) inside its time loop.  This entry
// point serves them: it calls no cudaMalloc, cudaFree or allocating library
// routine.
//
// The scratch array is a file-scope __device__ array of kNoallocBytes; every
// GPU that loads the library keeps it until the process exits.  Its name in
// host code is only a host-side stand-in, so the device address is obtained
// with cudaGetSymbolAddress, once per device, with that device current, on
// the first call made on that device (make that first call before any stream
// capture).  The address is kept for the life of the process: do not call
// this entry point on a device after cudaDeviceReset of that device (the
// module may then be loaded again elsewhere and the kept address would be
// stale).  The 2 MiB hold the 40-byte partial sums of 52428 blocks of the
// moments pass, ceil(l/tx) x ceil(m/ty) x min(n, 64) blocks with tx x ty =
// 256 threads, tx the smallest power of two >= l in 32..256: 256^3 needs
// 16384 blocks and is served, 512^3 needs 65536 and is rejected.  All calls share the array and it keeps the previous call's
// contents: each launch overwrites every partial-sum slot it later reads, so
// nothing has to start at zero, but calls that overlap on the GPU (different
// streams, or different host threads, on the same device) race on it.
#include <cuda_runtime.h>
#include <mutex>
#include "bgk3d_b200.h"
#include "bgk_internal.h"

namespace {
constexpr size_t kNoallocBytes = size_t(2) << 20;   // 2 MiB of per-block partial sums
constexpr size_t kNoallocSlots = kNoallocBytes / sizeof(double);
constexpr int kMaxDevices = 64;
}  // namespace

static __device__ __align__(256) double g_moments_scratch[kNoallocSlots];

namespace {
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_moments_scratch on the current device (set up once).
int scratch_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return bgk::set_error(BGK_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return bgk::set_error(BGK_ERR_UNSUPPORTED, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_moments_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            return bgk::set_error(BGK_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", dev,
                                  cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(ptr);
    }
    *out = g_scratch_addr[dev];
    return BGK_OK;
}

}  // namespace

extern "C" {

size_t bgk_moments_noalloc_max_bytes(void) { return kNoallocBytes; }

int bgk_moments_noalloc(const bgk_sweep_params* p, void* const* a, double* out_dev, void* stream) {
    if (int e = bgk::validate(p)) return e;
    if (!a || !out_dev) return bgk::set_error(BGK_ERR_ARG, "null pointer");
    const size_t need = bgk_reduce_workspace_bytes(p->l, p->m, p->n);
    if (need > kNoallocBytes)
        return bgk::set_error(BGK_ERR_ARG,
                              "lattice %dx%dx%d needs %zu bytes of reduction scratch; the allocation-free "
                              "bgk_moments_noalloc holds at most %zu bytes (use bgk_moments with a workspace)",
                              p->l, p->m, p->n, need, kNoallocBytes);
    double* scratch = nullptr;
    if (int e = scratch_address(&scratch)) return e;
    return bgk::moments_launch(p, a, out_dev, scratch, (cudaStream_t)stream);
}

}  // extern "C"
