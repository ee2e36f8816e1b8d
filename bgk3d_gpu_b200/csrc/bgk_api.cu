// C ABI of libbgk3d_b200.so: validation, kind/case dispatch and launch
// shapes around the kernels of sweep_ab.cuh and reduce.cuh.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include "bgk3d_b200.h"
#include "bgk3d_lattice.h"
#include "bgk_internal.h"
#include "kernels.h"
#include "reduce.cuh"
#include "dissipation.cuh"

namespace bgk {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "%s: launch failed: %s", what, cudaGetErrorString(e));
    return BGK_OK;
}

dim3 row_block(int l) {
    int tx = 32;
    while (tx < l && tx < 256) tx <<= 1;
    return dim3(tx, 256 / tx, 1);
}

void moments_grid(int l, int m, int n, dim3& grd, dim3& blk) {
    blk = row_block(l);
    int kb = n < 64 ? n : 64;
    grd = dim3((l + blk.x - 1) / blk.x, (m + blk.y - 1) / blk.y, kb);
}

long long sweep_blocks(const bgk_sweep_params* p, const void* a0, bool one_node_ab) {
    // the warp-segment launch of sweep_ab_kernel / the AA kernels (seg_plan);
    // without a0 the upper bound over start alignments: the unaligned row
    // mapping, which the plane mapping only replaces where it needs fewer warps
    const size_t es = p->kind == 0 ? 8 : (p->kind == 2 || p->kind == 3) ? 2 : 4;
    const long long align = a0 ? (long long)(((uintptr_t)a0 / es) & 31) : 0;
    const long long warps = a0 ? seg_plan(p->l, p->m, p->n, p->nx, align, one_node_ab).warps
                               : (long long)((p->l + 62) / 32) * p->m * p->n;
    return mom_plan(warps).blocks;
}

MomPlan mom_plan(long long warps) {
    // Runs of 64 segments (eight rounds of a block's 8 warps, 2048 nodes)
    // keep the partials few enough for one finalizing block; blocks that
    // stride over the lattice or live longer run slower (measured on the
    // 256^3 FP32 step, B200: grids of 4 / 20 / 80 blocks per SM striding,
    // 596 / 498 / 473 us; runs of 64 segments 471 us; the step without
    // moments 441 us; shorter runs in the last wave changed nothing).
    MomPlan m;
    m.span = 64;
    m.blocks = (warps + m.span - 1) / m.span;
    return m;
}

int finalize_moments(const double* partials, long long nparts, double* out, cudaStream_t st) {
    finalize_partials_kernel<5><<<1, kFinalizeThreads, 0, st>>>(partials, nparts, out);
    return check_launch("finalize_partials_kernel");
}

int validate(const bgk_sweep_params* p) {
    if (!p) return set_error(BGK_ERR_ARG, "null params");
    if (p->kind < 0 || p->kind > 4) return set_error(BGK_ERR_ARG, "kind %d out of range", p->kind);
    if (p->bcase < -1 || p->bcase > 3) return set_error(BGK_ERR_ARG, "bcase %d out of range", p->bcase);
    if (p->l < 1 || p->m < 1 || p->n < 1) return set_error(BGK_ERR_ARG, "extents must be >= 1");
    if (p->nx < (long long)p->l + 2 || p->ny < (long long)p->m + 2)
        return set_error(BGK_ERR_ARG, "leading dimensions nx=%lld ny=%lld too small for l=%d m=%d", p->nx,
                         p->ny, p->l, p->m);
    if (p->m > 65535 * 256 || p->n > 65535) return set_error(BGK_ERR_ARG, "m or n too large");
    if (p->kind == K_F16 || p->kind == K_BF16) {
        int e;
        float f = frexpf(p->scale, &e);
        if (!(p->scale > 0.f) || f != 0.5f) return set_error(BGK_ERR_ARG, "scale must be a power of two");
    }
    if (p->obs) {
        if (p->imin <= p->imax && p->jmin <= p->jmax && p->kmin <= p->kmax) {
            if (p->imin < 2 || p->imax > p->l - 1 || p->jmin < 2 || p->jmax > p->m - 1 || p->kmin < 2 ||
                p->kmax > p->n - 1)
                return set_error(BGK_ERR_ARG,
                                 "obstacle box [%d,%d]x[%d,%d]x[%d,%d] must stay one node inside the lattice",
                                 p->imin, p->imax, p->jmin, p->jmax, p->kmin, p->kmax);
            if (p->obs_nx < p->l || p->obs_ny < p->m)
                return set_error(BGK_ERR_ARG, "obstacle leading dimensions too small");
        }
    }
    if (p->zhalo & ~3) return set_error(BGK_ERR_ARG, "zhalo %d: only bits 0 and 1", p->zhalo);
    if (p->zhalo) {
        // a slab face reads the neighbour's populations from the halo plane; the
        // outflow plane and the obstacle mask would need the neighbour's too
        if (p->bcase == BC_INFLOW)
            return set_error(BGK_ERR_UNSUPPORTED, "z-slab faces (zhalo) are not supported for the inflow case");
        if (p->obs && p->imin <= p->imax)
            return set_error(BGK_ERR_UNSUPPORTED, "z-slab faces (zhalo) are not supported with an obstacle");
    }
    return BGK_OK;
}

}  // namespace bgk

using namespace bgk;

int bgk::moments_launch(const bgk_sweep_params* p, void* const* a, double* out, double* ws, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_moments<S, C>(p, a, out, ws, st)));
}

int bgk::sweep_launch(const bgk_sweep_params* p, void* const* a, void* const* b, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_sweep<S, C>(p, a, b, nullptr, st)));
}

int bgk::sweep_launch_mom(const bgk_sweep_params* p, void* const* a, void* const* b, double* mom,
                          cudaStream_t st, int* halo, double* mom_out, unsigned* mom_ticket) {
    KIND_DISPATCH(p->kind, (launch_sweep<S, C>(p, a, b, mom, st, halo, mom_out, mom_ticket)));
}

int bgk::dissipation_launch(const bgk_sweep_params* p, void* const* a, double nu, double* out, double* ws,
                            cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_dissipation<S, C>(p, a, nu, out, ws, st)));
}

size_t bgk::dissipation_workspace(int l, int m, int n) {
    dim3 grd, blk;
    moments_grid(l, m, n, grd, blk);
    const dim3 eg = enstrophy_grid(l, m, n);
    return ((size_t)grd.x * grd.y * grd.z * 5 + (size_t)eg.x * eg.y * eg.z * 2) * sizeof(double);
}

int bgk::draglift_launch(const bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks,
                         int ke, double* out, double* ws, size_t ws_bytes, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_draglift<S, C>(p, a, is, ie, js, je, ks, ke, out, ws, ws_bytes, st)));
}

extern "C" {

int bgk_set_obstacle_split(int enable) {
    const int prev = g_obstacle_split ? 1 : 0;
    g_obstacle_split = enable != 0;
    return prev;
}

int bgk_set_pair_kernels(int enable) {
    const int prev = g_pair_kernels ? 1 : 0;
    g_pair_kernels = enable != 0;
    return prev;
}

void bgk_sweep_params_init(bgk_sweep_params* p, int kind, int l, int m, int n, double omega) {
    std::memset(p, 0, sizeof *p);
    p->kind = kind; p->bcase = BGK_BC_NONE;
    p->l = l; p->m = m; p->n = n;
    p->nx = (long long)l + 2; p->ny = (long long)m + 2;
    p->omega = omega;
    p->cte1 = 1.0; p->cte0 = 0.0;
    p->p0 = 1.0 / 3.0; p->p1 = 1.0 / 18.0; p->p2 = 1.0 / (3.0 * 3.0 * (1.0 + 3.0));
    p->rf = 3.0; p->qf = 1.5; p->tre = 3.0;
    p->scale = 1.0f;
    p->obs_nx = l; p->obs_ny = m;
    p->imin = 1; p->imax = 0; p->jmin = 1; p->jmax = 0; p->kmin = 1; p->kmax = 0;
}

int bgk_sweep(const bgk_sweep_params* p, void* const* a, void* const* b, void* stream) {
    if (int e = validate(p)) return e;
    if (!a || !b) return set_error(BGK_ERR_ARG, "null population pointer array");
    for (int d = 0; d < 19; ++d)
        if (!a[d] || (d < 18 && !b[d])) return set_error(BGK_ERR_ARG, "null population %d", d + 1);
    return bgk::sweep_launch(p, a, b, (cudaStream_t)stream);
}

size_t bgk_sweep_moments_workspace_bytes(const bgk_sweep_params* p) {
    if (!p) return 0;
    return bgk::fused_workspace_bytes(bgk::sweep_blocks(p, nullptr), 5);
}

int bgk_sweep_moments(const bgk_sweep_params* p, void* const* a, void* const* b, double* out_dev, void* workspace,
                      size_t workspace_bytes, void* stream) {
    if (int e = validate(p)) return e;
    if (!a || !b || !out_dev || !workspace) return set_error(BGK_ERR_ARG, "null pointer");
    for (int d = 0; d < 19; ++d)
        if (!a[d] || (d < 18 && !b[d])) return set_error(BGK_ERR_ARG, "null population %d", d + 1);
    const long long nb_max = bgk::sweep_blocks(p, nullptr);
    const size_t need = bgk::fused_workspace_bytes(nb_max, 5);
    if (workspace_bytes < need) return set_error(BGK_ERR_ARG, "workspace too small: %zu < %zu", workspace_bytes, need);
    cudaStream_t st = (cudaStream_t)stream;
    const bgk::FusedWs fw = bgk::fused_ws(workspace, nb_max);
    // the caller's workspace holds anything: clear the counters
    cudaError_t e = cudaMemsetAsync(fw.tickets, 0, bgk::fused_ticket_bytes(nb_max), st);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    return bgk::sweep_launch_mom(p, a, b, fw.records, st, nullptr, out_dev, fw.tickets);
}

size_t bgk_reduce_workspace_bytes(int l, int m, int n) {
    dim3 grd, blk;
    moments_grid(l, m, n, grd, blk);
    const size_t nparts = (size_t)grd.x * grd.y * grd.z;
    return nparts * 5 * sizeof(double);
}

int bgk_moments(const bgk_sweep_params* p, void* const* a, double* out_dev, void* workspace,
                size_t workspace_bytes, void* stream) {
    if (int e = validate(p)) return e;
    if (!a || !out_dev || !workspace) return set_error(BGK_ERR_ARG, "null pointer");
    if (workspace_bytes < bgk_reduce_workspace_bytes(p->l, p->m, p->n))
        return set_error(BGK_ERR_ARG, "workspace too small: %zu < %zu", workspace_bytes,
                         bgk_reduce_workspace_bytes(p->l, p->m, p->n));
    return bgk::moments_launch(p, a, out_dev, (double*)workspace, (cudaStream_t)stream);
}

size_t bgk_dissipation_workspace_bytes(int l, int m, int n) {
    if (l < 1 || m < 1 || n < 1) return 0;
    return bgk::dissipation_workspace(l, m, n);
}

int bgk_dissipation(const bgk_sweep_params* p, void* const* a, double nu, double* out_dev, void* workspace,
                    size_t workspace_bytes, void* stream) {
    if (int e = validate(p)) return e;
    if (!a || !out_dev || !workspace) return set_error(BGK_ERR_ARG, "null pointer");
    for (int d = 0; d < 19; ++d)
        if (!a[d]) return set_error(BGK_ERR_ARG, "null population %d", d + 1);
    const size_t need = bgk::dissipation_workspace(p->l, p->m, p->n);
    if (workspace_bytes < need) return set_error(BGK_ERR_ARG, "workspace too small: %zu < %zu", workspace_bytes, need);
    if (!(nu >= 0.0)) return set_error(BGK_ERR_ARG, "viscosity must be >= 0");
    return bgk::dissipation_launch(p, a, nu, out_dev, (double*)workspace, (cudaStream_t)stream);
}

int bgk_draglift(const bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks, int ke,
                 double* out_dev, void* workspace, size_t workspace_bytes, void* stream) {
    if (int e = validate(p)) return e;
    if (!a || !out_dev || !workspace) return set_error(BGK_ERR_ARG, "null pointer");
    if (ie < is || je < js || ke < ks) return set_error(BGK_ERR_ARG, "empty draglift box");
    return bgk::draglift_launch(p, a, is, ie, js, je, ks, ke, out_dev, (double*)workspace, workspace_bytes,
                                (cudaStream_t)stream);
}

int bgk_device_sync(void) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "device sync failed: %s", cudaGetErrorString(e));
    return BGK_OK;
}

size_t bgk_dropin_tracked_workspace_bytes(const bgk_sweep_params* p) {
    if (!p) return 0;
    return bgk::fused_workspace_bytes(bgk::sweep_blocks(p, nullptr), 5);
}

int bgk_dropin_sweep_tracked(const bgk_sweep_params* p, void* const* a, void* const* b, void* workspace,
                             size_t bytes, double* out_dev) {
    if (int e = validate(p)) return e;
    if (!a || !b || !workspace || !out_dev) return set_error(BGK_ERR_ARG, "null pointer");
    const long long nb_max = bgk::sweep_blocks(p, nullptr);
    if (bytes < bgk::fused_workspace_bytes(nb_max, 5))
        return set_error(BGK_ERR_ARG, "workspace too small: %zu < %zu", bytes,
                         bgk::fused_workspace_bytes(nb_max, 5));
    const bgk::FusedWs fw = bgk::fused_ws(workspace, nb_max);
    return bgk::sweep_launch_mom(p, a, b, fw.records, nullptr, nullptr, out_dev, fw.tickets);
}

const char* bgk_last_error(void) { return g_last_error.c_str(); }

const char* bgk_version(void) { return "bgk3d_b200 0.1 (sm_100a)"; }

long long bgk_abi_field_offset(int which, int field) {
#define BGK_OFF(T, f) (long long)offsetof(T, f)
    static const long long sweep[] = {
        BGK_OFF(bgk_sweep_params, kind), BGK_OFF(bgk_sweep_params, bcase), BGK_OFF(bgk_sweep_params, l),
        BGK_OFF(bgk_sweep_params, m), BGK_OFF(bgk_sweep_params, n), BGK_OFF(bgk_sweep_params, nx),
        BGK_OFF(bgk_sweep_params, ny), BGK_OFF(bgk_sweep_params, omega), BGK_OFF(bgk_sweep_params, cte0),
        BGK_OFF(bgk_sweep_params, cte1), BGK_OFF(bgk_sweep_params, p0), BGK_OFF(bgk_sweep_params, p1),
        BGK_OFF(bgk_sweep_params, p2), BGK_OFF(bgk_sweep_params, rf), BGK_OFF(bgk_sweep_params, qf),
        BGK_OFF(bgk_sweep_params, tre), BGK_OFF(bgk_sweep_params, force_mode), BGK_OFF(bgk_sweep_params, fx),
        BGK_OFF(bgk_sweep_params, fy), BGK_OFF(bgk_sweep_params, fz), BGK_OFF(bgk_sweep_params, lid_force),
        BGK_OFF(bgk_sweep_params, u_inflow), BGK_OFF(bgk_sweep_params, inflow_cte1),
        BGK_OFF(bgk_sweep_params, scale), BGK_OFF(bgk_sweep_params, obs), BGK_OFF(bgk_sweep_params, obs_nx),
        BGK_OFF(bgk_sweep_params, obs_ny), BGK_OFF(bgk_sweep_params, imin), BGK_OFF(bgk_sweep_params, imax),
        BGK_OFF(bgk_sweep_params, jmin), BGK_OFF(bgk_sweep_params, jmax), BGK_OFF(bgk_sweep_params, kmin),
        BGK_OFF(bgk_sweep_params, kmax), BGK_OFF(bgk_sweep_params, fast), BGK_OFF(bgk_sweep_params, zhalo)};
    static const long long desc[] = {
        BGK_OFF(bgk_lattice_desc, kind), BGK_OFF(bgk_lattice_desc, bcase), BGK_OFF(bgk_lattice_desc, pattern),
        BGK_OFF(bgk_lattice_desc, l), BGK_OFF(bgk_lattice_desc, m), BGK_OFF(bgk_lattice_desc, n),
        BGK_OFF(bgk_lattice_desc, omega), BGK_OFF(bgk_lattice_desc, force_mode), BGK_OFF(bgk_lattice_desc, fx),
        BGK_OFF(bgk_lattice_desc, fy), BGK_OFF(bgk_lattice_desc, fz), BGK_OFF(bgk_lattice_desc, lid_force),
        BGK_OFF(bgk_lattice_desc, u_inflow), BGK_OFF(bgk_lattice_desc, scale), BGK_OFF(bgk_lattice_desc, fast)};
#undef BGK_OFF
    if (field < 0) return -1;
    if (which == 0) return field < (int)(sizeof sweep / sizeof *sweep) ? sweep[field] : -1;
    if (which == 1) return field < (int)(sizeof desc / sizeof *desc) ? desc[field] : -1;
    return -1;
}

size_t bgk_abi_struct_size(int which) {
    switch (which) {
        case 0: return sizeof(bgk_sweep_params);
        case 1: return sizeof(bgk_lattice_desc);
        default: return 0;
    }
}

}  // extern "C"
