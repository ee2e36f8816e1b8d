// C ABI of libbgk3d_b200.so: validation, kind/case dispatch and launch
// shapes around the kernels of sweep_ab.cuh and reduce.cuh.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <string>
#include "bgk3d_b200.h"
#include "bgk_internal.h"
#include "sweep_ab.cuh"
#include "reduce.cuh"
#include "host_args.cuh"

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
    return BGK_OK;
}

template <class S, class C, int BC>
void launch_sweep_bc(const SweepArgs<S, C>& A, long long nelem, unsigned blocks, bool generic,
                     cudaStream_t st) {
    if (nelem < (1LL << 31)) {
        if (generic) sweep_ab_kernel<S, C, BC, int, true><<<blocks, 256, 0, st>>>(A);
        else sweep_ab_kernel<S, C, BC, int, false><<<blocks, 256, 0, st>>>(A);
    } else {
        if (generic) sweep_ab_kernel<S, C, BC, long long, true><<<blocks, 256, 0, st>>>(A);
        else sweep_ab_kernel<S, C, BC, long long, false><<<blocks, 256, 0, st>>>(A);
    }
}

template <class S, class C>
int launch_sweep(const bgk_sweep_params* p, void* const* a, void* const* b, cudaStream_t st) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, a, b);
    segment_geometry(A, a[0]);
    if (p->bcase == BC_INFLOW) {
        dim3 blk(128), grd((p->m + 127) / 128, p->n);
        outflow_halo_kernel<S, C><<<grd, blk, 0, st>>>(A);
        if (int e = check_launch("outflow_halo_kernel")) return e;
    }
    const long long warps = (long long)A.nseg * p->m * p->n;
    const long long blocks = (warps + 7) / 8;
    if (warps >= (1LL << 32) - 8) return set_error(BGK_ERR_ARG, "lattice too large for one launch");
    const long long nelem = p->nx * p->ny * ((long long)p->n + 2) + 64;
    const bool g = generic_collision(p);
    const unsigned nb = (unsigned)blocks;
    switch (p->bcase) {
        case BC_NONE: launch_sweep_bc<S, C, BC_NONE>(A, nelem, nb, g, st); break;
        case BC_DRIVEN: launch_sweep_bc<S, C, BC_DRIVEN>(A, nelem, nb, g, st); break;
        case BC_PERIODIC: launch_sweep_bc<S, C, BC_PERIODIC>(A, nelem, nb, g, st); break;
        case BC_CHANNEL: launch_sweep_bc<S, C, BC_CHANNEL>(A, nelem, nb, g, st); break;
        case BC_INFLOW: launch_sweep_bc<S, C, BC_INFLOW>(A, nelem, nb, g, st); break;
    }
    return check_launch("sweep_ab_kernel");
}

// Grid of the moments pass: rows of the (i, j) plane x KB blocks striding k.
void moments_grid(int l, int m, int n, dim3& grd, dim3& blk) {
    blk = row_block(l);
    int kb = n < 64 ? n : 64;
    grd = dim3((l + blk.x - 1) / blk.x, (m + blk.y - 1) / blk.y, kb);
}

template <class S, class C>
int launch_moments(const bgk_sweep_params* p, void* const* a, double* out, double* ws, cudaStream_t st) {
    FieldArgs<S, C> F = field_args<S, C>(p, a);
    dim3 grd, blk;
    moments_grid(p->l, p->m, p->n, grd, blk);
    moments_partial_kernel<S, C><<<grd, blk, 0, st>>>(F, ws);
    if (int e = check_launch("moments_partial_kernel")) return e;
    const long long nparts = (long long)grd.x * grd.y * grd.z;
    finalize_partials_kernel<5><<<1, 256, 0, st>>>(ws, nparts, out);
    return check_launch("finalize_partials_kernel");
}

template <class S, class C>
int launch_draglift(const bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks, int ke,
                    double* out, double* ws, size_t ws_bytes, cudaStream_t st) {
    FieldArgs<S, C> F = field_args<S, C>(p, a);
    const int ni = ie - is + 1, nj = je - js + 1, nk = ke - ks + 1;
    const long long tot = (long long)ni * nj * nk;
    const long long nb = (tot + 255) / 256;
    if ((size_t)nb * 3 * sizeof(double) > ws_bytes)
        return set_error(BGK_ERR_ARG, "draglift box needs %lld bytes of workspace", nb * 3 * 8);
    draglift_partial_kernel<S, C><<<(unsigned)nb, 256, 0, st>>>(F, is, js, ks, ni, nj, nk, ws);
    if (int e = check_launch("draglift_partial_kernel")) return e;
    finalize_partials_kernel<3><<<1, 256, 0, st>>>(ws, nb, out);
    return check_launch("finalize_partials_kernel");
}

}  // namespace bgk

using namespace bgk;

#define KIND_DISPATCH(kind, CALL)                                                     \
    switch (kind) {                                                                   \
        case K_F64: { typedef double S; typedef double C; return CALL; }              \
        case K_F32: { typedef float S; typedef float C; return CALL; }                \
        case K_F16: { typedef __half S; typedef float C; return CALL; }               \
        case K_BF16: { typedef __nv_bfloat16 S; typedef float C; return CALL; }       \
        case K_F32_F64: { typedef float S; typedef double C; return CALL; }           \
    }                                                                                 \
    return set_error(BGK_ERR_ARG, "bad kind");

int bgk::moments_launch(const bgk_sweep_params* p, void* const* a, double* out, double* ws, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_moments<S, C>(p, a, out, ws, st)));
}

int bgk::sweep_launch(const bgk_sweep_params* p, void* const* a, void* const* b, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_sweep<S, C>(p, a, b, st)));
}

int bgk::draglift_launch(const bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks,
                         int ke, double* out, double* ws, size_t ws_bytes, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_draglift<S, C>(p, a, is, ie, js, je, ks, ke, out, ws, ws_bytes, st)));
}

extern "C" {

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

const char* bgk_last_error(void) { return g_last_error.c_str(); }

const char* bgk_version(void) { return "bgk3d_b200 0.1 (sm_100a)"; }

}  // extern "C"
