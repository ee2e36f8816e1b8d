// Internal helpers shared by the library's translation units.
#pragma once
#include <cstdarg>
#include <cuda_runtime.h>
#include "bgk3d_b200.h"

namespace bgk {
// Warps of one step of the warp-segment sweeps (see sweep_ab.cuh).  Rows
// that start on a 32-element boundary (the library's padded layout) take
// ceil(l/32) warps each; other rows one more, unless the plane mapping
// (allowed for the one-node AB sweep only) needs fewer warps: it tiles each
// z plane's rows 1..m as one range, ceil((nx (m - 1) + l + 31) / 32) warps
// for any start alignment.
struct SegPlan {
    bool aligned, flat;
    long long nseg;    // warps per row (row mapping)
    long long wpp;     // warps per plane (plane mapping)
    long long warps;   // warps of one step
};
inline SegPlan seg_plan(int l, int m, int n, long long nx, long long align_base, bool allow_flat) {
    SegPlan s;
    s.aligned = ((align_base + 1) % 32 == 0) && (nx % 32 == 0);
    s.nseg = s.aligned ? (l + 31) / 32 : (l + 62) / 32;
    s.wpp = (nx * (m - 1) + l + 62) / 32;
    s.flat = allow_flat && !s.aligned && nx * m < (1LL << 31) && s.wpp < s.nseg * m;
    s.warps = s.flat ? s.wpp * n : s.nseg * m * n;
    return s;
}

// TMA-staged sweep switch for library-owned lattices (bgk_set_tma_kernels).
// Off by default: bit-exact, 280 instead of 408 instructions per node for
// FP16, but measured at half the one-node kernel's rate on 256^3 (B200).
inline bool g_tma_kernels = false;
// One-node AB sweep with an obstacle as two launches (the obstacle-free
// variant outside the obstacle's grown box, sweep_box_kernel inside it):
// bgk_set_obstacle_split(1).  Off by default: measured 4-7 % slower than one
// launch with the obstacle logic (FP32 sphere case at 256^3, B200).
inline bool g_obstacle_split = false;
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
// Same, with the per-block FP64 moments of the new state written to mom;
// halo (inflow, nullable): in, a's outflow plane is fresh (no pre-pass); out,
// the launch wrote the next state's outflow plane into b.  With mom (the
// records of fused_ws, reduce.cuh), mom_out and mom_ticket (its counters,
// zero before the launch and left zero) are required: the launch sums the
// moments into mom_out[0..4] itself (finalize_by_tickets).
int sweep_launch_mom(const struct bgk_sweep_params* p, void* const* a, void* const* b, double* mom,
                     cudaStream_t st, int* halo = nullptr, double* mom_out = nullptr,
                     unsigned* mom_ticket = nullptr);
// Grid of a time-step launch that also sums moments, over `warps` warp
// segments: block b advances the run of span segments from b * span
// (block_segments, reduce.cuh); span is a multiple of 8.
struct MomPlan {
    long long blocks, span;
};
MomPlan mom_plan(long long warps);
// Number of blocks (= moment records) of the sweep launch with moments
// for p with population 01 at a0 (nullptr: the upper bound for any alignment);
// one_node_ab: the launch is the one-node AB sweep (plane mapping allowed),
// false for the AA steps.
long long sweep_blocks(const struct bgk_sweep_params* p, const void* a0, bool one_node_ab = true);
// Second pass over nparts partials of 5 doubles into out[0..4].
int finalize_moments(const double* partials, long long nparts, double* out, cudaStream_t st);
// Device memory of library-owned objects from the per-device pool
// (zeroed when asked), ready for any stream on return; dev_free waits for
// the device, as cudaFree does, and returns the block to the pool.
int dev_alloc(void** p, size_t bytes, bool zero, const char* what);
void dev_free(void* p);
// Return the block to the pool ordered after the work queued on st (no
// device-wide wait): every use of p must be on st or ordered before it.
void dev_free_async(void* p, cudaStream_t st);
// Private non-blocking stream for set-up kernels and copies.
cudaStream_t setup_stream();
// The launches of the turbulence diagnostics (TKE, dissipation, mean
// squares, enstrophy) into out[0..6], partials in ws.
int dissipation_launch(const struct bgk_sweep_params* p, void* const* a, double nu, double* out, double* ws,
                       cudaStream_t st);
// Bytes of partial sums of dissipation_launch.
size_t dissipation_workspace(int l, int m, int n);
// The two launches of the FP64 drag/lift reduction.
int draglift_launch(const struct bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks,
                    int ke, double* out, double* ws, size_t ws_bytes, cudaStream_t st);
}  // namespace bgk
