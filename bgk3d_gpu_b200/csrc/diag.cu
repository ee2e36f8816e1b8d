// Device-side profiles, probes and slices: the reference's per-icheck /
// per-ivtim outputs computed where the populations live, so that only the
// line, point or plane crosses to the host instead of the whole state.
//
//   profile  SRC/prof_i.F90, SRC/prof_j.F90, SRC/prof_k.F90:47-77
//   probe    SRC/probe.F90:50-78
//   slice    SRC/vtk_xy.binary.F90:78-97 (vtk_xz, vtk_yz likewise)
//
// Each follows its routine's arithmetic: the profiles sum the storage arrays
// directly (storage arithmetic; the density then adds cte1 in the compute
// type and the velocities divide in the compute type), the probe copies the
// populations into compute-type variables first, and the slices work in
// single precision.  The 16-bit kinds are read as unscaled float values.  The
// library is built without FMA contraction, so every result is the CPU
// restatement's bit for bit.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "bgk_internal.h"
#include "d3q19.cuh"
#include "lattice_internal.h"

using namespace bgk;

namespace {

template <class S> struct Arith;
template <> struct Arith<double> {
    typedef double R;
    static __device__ __forceinline__ double ld(const double* p, long long c, float) { return p[c]; }
};
template <> struct Arith<float> {
    typedef float R;
    static __device__ __forceinline__ float ld(const float* p, long long c, float) { return p[c]; }
};
template <> struct Arith<__half> {
    typedef float R;
    static __device__ __forceinline__ float ld(const __half* p, long long c, float inv) {
        return __fmul_rn(__half2float(p[c]), inv);
    }
};
template <> struct Arith<__nv_bfloat16> {
    typedef float R;
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p, long long c, float inv) {
        return __fmul_rn(__bfloat162float(p[c]), inv);
    }
};

template <class S> struct Pops {
    const S* f[19];
    long long nx, nxy;
    float inv_scale;
};

template <class S, class T>
__device__ __forceinline__ void load19(const Pops<S>& P, long long c, T* x) {
#pragma unroll
    for (int p = 0; p < 19; ++p) x[p] = (T)Arith<S>::ld(P.f[p], c, P.inv_scale);
}

template <class T> __device__ __forceinline__ T sum19(const T* x) {
    return x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] +
           x[14] + x[15] + x[16] + x[17] + x[18];
}
template <class T> __device__ __forceinline__ T mom_x(const T* x) {
    return x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13];
}
template <class T> __device__ __forceinline__ T mom_y(const T* x) {
    return x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17];
}
template <class T> __device__ __forceinline__ T mom_z(const T* x) {
    return x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15];
}

// axis 0: i runs at (j, k) = (c1, c2); 1: j runs at (i, k); 2: k runs at (i, j)
template <class S, class C>
__global__ void profile_kernel(const Pops<S> P, int axis, int c1, int c2, int len, C cte1, double* out) {
    typedef typename Arith<S>::R R;
    const int t = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (t > len) return;
    const int i = axis == 0 ? t : c1, j = axis == 1 ? t : (axis == 0 ? c1 : c2), k = axis == 2 ? t : c2;
    R x[19];
    load19(P, i + P.nx * j + P.nxy * k, x);
    const C den = (C)sum19(x) + cte1;
    double* o = out + 4 * (long long)(t - 1);
    o[0] = (double)((C)mom_x(x) / den);
    o[1] = (double)((C)mom_y(x) / den);
    o[2] = (double)((C)mom_z(x) / den);
    o[3] = (double)den;
}

template <class S, class C>
__global__ void probe_kernel(const Pops<S> P, int i, int j, int k, C cte1, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    C x[19];
    load19(P, i + P.nx * j + P.nxy * k, x);
    const C rho = sum19(x) + cte1;
    out[0] = (double)(mom_x(x) / rho);
    out[1] = (double)(mom_y(x) / rho);
    out[2] = (double)(mom_z(x) / rho);
    out[3] = (double)rho;
}

// plane 0: xy at k = index (out[j][i]); 1: xz at j = index (out[k][i]);
// 2: yz at i = index (out[k][j]); 3 floats per node
template <class S>
__global__ void slice_kernel(const Pops<S> P, int plane, int index, int n1, int n2, float* out) {
    typedef typename Arith<S>::R R;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n1 * n2) return;
    const int a = (int)(t % n1) + 1, b = (int)(t / n1) + 1;
    const int i = plane == 2 ? index : a;
    const int j = plane == 0 ? b : (plane == 1 ? index : a);
    const int k = plane == 0 ? index : b;
    R x[19];
    load19(P, i + P.nx * j + P.nxy * k, x);
    const float u = (float)mom_x(x), w = (float)mom_y(x), v = (float)mom_z(x);
    const float den = (float)(sum19(x) + (R)1.0);
    out[3 * t + 0] = u / den;
    out[3 * t + 1] = w / den;
    out[3 * t + 2] = v / den;
}

template <class S> Pops<S> pops_of(const bgk_sweep_params* p, void* const* a) {
    Pops<S> P;
    for (int d = 0; d < 19; ++d) P.f[d] = (const S*)a[d];
    P.nx = p->nx;
    P.nxy = (long long)p->nx * p->ny;
    P.inv_scale = (p->kind == K_F16 || p->kind == K_BF16) ? 1.0f / p->scale : 1.0f;
    return P;
}

#define DIAG_DISPATCH(kind, ...)                                                              \
    switch (kind) {                                                                           \
        case K_F64: { typedef double S; typedef double C; __VA_ARGS__ } break;               \
        case K_F32: { typedef float S; typedef float C; __VA_ARGS__ } break;                 \
        case K_F16: { typedef __half S; typedef float C; __VA_ARGS__ } break;                \
        case K_BF16: { typedef __nv_bfloat16 S; typedef float C; __VA_ARGS__ } break;        \
        case K_F32_F64: { typedef float S; typedef double C; __VA_ARGS__ } break;            \
        default: return set_error(BGK_ERR_ARG, "unknown kind %d", kind);                      \
    }

int check_layout(const bgk_sweep_params* p, void* const* a, const void* out) {
    if (!p || !a || !out) return set_error(BGK_ERR_ARG, "null argument");
    if (p->l < 1 || p->m < 1 || p->n < 1 || p->nx < p->l + 2 || p->ny < p->m + 2)
        return set_error(BGK_ERR_ARG, "bad extents");
    if ((p->kind == K_F16 || p->kind == K_BF16) && !(p->scale > 0.0f))
        return set_error(BGK_ERR_ARG, "16-bit kinds need a positive scale");
    for (int d = 0; d < 19; ++d)
        if (!a[d]) return set_error(BGK_ERR_ARG, "population %d is null", d + 1);
    return BGK_OK;
}

bool in_box(const bgk_sweep_params* p, int i, int j, int k) {
    return i >= 1 && i <= p->l && j >= 1 && j <= p->m && k >= 1 && k <= p->n;
}

int lattice_params(const bgk_lattice* L, bgk_sweep_params* q, void** a) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    if (L->desc.pattern == BGK_PATTERN_AA && (L->steps % 2) != 0)
        return set_error(BGK_ERR_STATE, "AA lattice after an odd number of steps holds no observable state");
    *q = L->p;
    bgk_lat::observable(L, a);
    return BGK_OK;
}

}  // namespace

extern "C" {

int bgk_profile(const bgk_sweep_params* p, void* const* a, int axis, int c1, int c2, double* out_dev,
                void* stream) {
    if (int e = check_layout(p, a, out_dev)) return e;
    if (axis < 0 || axis > 2) return set_error(BGK_ERR_ARG, "axis must be 0 (i), 1 (j) or 2 (k)");
    const int ci = axis == 0 ? 1 : c1, cj = axis == 1 ? 1 : (axis == 0 ? c1 : c2), ck = axis == 2 ? 1 : c2;
    if (!in_box(p, ci, cj, ck)) return set_error(BGK_ERR_ARG, "profile line (%d, %d) outside the lattice", c1, c2);
    const int len = axis == 0 ? p->l : (axis == 1 ? p->m : p->n);
    cudaStream_t st = (cudaStream_t)stream;
    DIAG_DISPATCH(p->kind, {
        profile_kernel<S, C><<<(len + 127) / 128, 128, 0, st>>>(pops_of<S>(p, a), axis, c1, c2, len, (C)1.0,
                                                               out_dev);
    });
    return check_launch("profile_kernel");
}

int bgk_probe(const bgk_sweep_params* p, void* const* a, int i, int j, int k, double* out_dev, void* stream) {
    if (int e = check_layout(p, a, out_dev)) return e;
    if (!in_box(p, i, j, k)) return set_error(BGK_ERR_ARG, "probe (%d, %d, %d) outside the lattice", i, j, k);
    cudaStream_t st = (cudaStream_t)stream;
    DIAG_DISPATCH(p->kind, { probe_kernel<S, C><<<1, 32, 0, st>>>(pops_of<S>(p, a), i, j, k, (C)1.0, out_dev); });
    return check_launch("probe_kernel");
}

int bgk_slice(const bgk_sweep_params* p, void* const* a, int plane, int index, float* out_dev, void* stream) {
    if (int e = check_layout(p, a, out_dev)) return e;
    if (plane < 0 || plane > 2) return set_error(BGK_ERR_ARG, "plane must be 0 (xy), 1 (xz) or 2 (yz)");
    const int lim = plane == 0 ? p->n : (plane == 1 ? p->m : p->l);
    if (index < 1 || index > lim) return set_error(BGK_ERR_ARG, "slice index %d outside 1..%d", index, lim);
    const int n1 = plane == 2 ? p->m : p->l, n2 = plane == 0 ? p->m : p->n;
    const long long nodes = (long long)n1 * n2;
    cudaStream_t st = (cudaStream_t)stream;
    DIAG_DISPATCH(p->kind, {
        (void)sizeof(C);
        slice_kernel<S><<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(pops_of<S>(p, a), plane, index, n1, n2,
                                                                        out_dev);
    });
    return check_launch("slice_kernel");
}

int bgk_lattice_profile(const bgk_lattice* L, int axis, int c1, int c2, double* out_dev, void* stream) {
    bgk_sweep_params q;
    void* a[19];
    if (int e = lattice_params(L, &q, a)) return e;
    return bgk_profile(&q, a, axis, c1, c2, out_dev, stream);
}

int bgk_lattice_probe(const bgk_lattice* L, int i, int j, int k, double* out_dev, void* stream) {
    bgk_sweep_params q;
    void* a[19];
    if (int e = lattice_params(L, &q, a)) return e;
    return bgk_probe(&q, a, i, j, k, out_dev, stream);
}

int bgk_lattice_slice(const bgk_lattice* L, int plane, int index, float* out_dev, void* stream) {
    bgk_sweep_params q;
    void* a[19];
    if (int e = lattice_params(L, &q, a)) return e;
    return bgk_slice(&q, a, plane, index, out_dev, stream);
}

}  // extern "C"
