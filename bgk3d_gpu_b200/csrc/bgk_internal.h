// Internal helpers shared by the library's translation units.
#pragma once
#include <cstdarg>
#include <cuda_runtime.h>
#include "bgk3d_b200.h"

namespace bgk {
// TMA-staged sweep switch for library-owned lattices (bgk_set_tma_kernels).
// Off by default: bit-exact, 280 instead of 408 instructions per node for
// FP16, but measured at half the one-node kernel's rate on 256^3 (B200).
inline bool g_tma_kernels = false;
// Two-node sweep for the 16-bit kinds (sweep_ab2_kernel): on by default;
// bgk_set_pair_kernels(0) selects the one-node sweep (tests compare both).
inline bool g_pair_kernels = true;
// Record a formatted message as the calling thread's last error; returns code.
int set_error(int code, const char* fmt, ...);
// cudaGetLastError after a launch, recorded as an error when it failed.
int check_launch(const char* what);
// Block shape for one-thread-per-node sweeps over (i, j) rows: TX x TY = 256.
dim3 row_block(int l);
// Grid of the moments pass: rows of the (i, j) plane x KB blocks striding k.
void moments_grid(int l, int m, int n, dim3& grd, dim3& blk);
// Parameter checks shared by every entry point (returns BGK_OK or an error).
int validate(const struct bgk_sweep_params* p);
// The two launches of the FP64 moments reduction, with the per-block
// partials in ws (bgk_reduce_workspace_bytes(l, m, n) bytes).
int moments_launch(const struct bgk_sweep_params* p, void* const* a, double* out, double* ws,
                   cudaStream_t st);
// The fused sweep launch(es) without argument validation.
int sweep_launch(const struct bgk_sweep_params* p, void* const* a, void* const* b, cudaStream_t st);
// Same, with the per-block FP64 moments of the new state written to mom.
int sweep_launch_mom(const struct bgk_sweep_params* p, void* const* a, void* const* b, double* mom,
                     cudaStream_t st);
// Blocks of a sweep launch that also produces moments: a fixed grid (20
// blocks per SM of the current device, fewer for small lattices) strides over
// the step's warps.  The partial sums, and so the last bits of the moments,
// depend on the device's SM count, never on timing.
long long mom_grid(long long blocks);
// Number of blocks (= partial-moment slots) of the sweep launch with moments
// for p with population 01 at a0 (nullptr: the upper bound for any alignment).
long long sweep_blocks(const struct bgk_sweep_params* p, const void* a0);
// Second pass over nparts partials of 5 doubles into out[0..4].
int finalize_moments(const double* partials, long long nparts, double* out, cudaStream_t st);
// Device memory of library-owned objects from the per-device pool
// (zeroed when asked), ready for any stream on return; dev_free waits for
// the device, as cudaFree does, and returns the block to the pool.
int dev_alloc(void** p, size_t bytes, bool zero, const char* what);
void dev_free(void* p);
// Private non-blocking stream for set-up kernels and copies.
cudaStream_t setup_stream();
// The two launches of the FP64 drag/lift reduction.
int draglift_launch(const struct bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks,
                    int ke, double* out, double* ws, size_t ws_bytes, cudaStream_t st);
}  // namespace bgk
