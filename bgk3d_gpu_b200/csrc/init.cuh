// On-device initial conditions: equilibrium populations of an analytic flow
// written straight into a lattice (no host round trip), the device form of
// SRC/init.F90:113-201.
//
// Flows (the benchmark forms of the reference's cases: grid points at 2 pi (i-1)/l, ...):
//   INIT_UNIFORM  rho = p[0], u = (p[1], p[2], p[3])   (rest: 1, 0, 0, 0)
//   INIT_TGV      Taylor-Green: x = 2 pi (i-1)/l, ...,
//                 u = u0 sin x cos y cos z, v = -u0 cos x sin y cos z, w = 0,
//                 rho = 1 + 3 (u0^2/16)(cos 2x + cos 2y)(cos 2z + 2),  u0 = p[0]
//   INIT_KIDA     Kida vortex, rho = 1,                  u0 = p[0]
// Populations are f_p^eq - w_p = w_p (rho - 1) + w_p rho (3 c.u + 4.5 (c.u)^2
// - 1.5 u^2) in double, rounded once to the storage kind.  (The reference's
// init.F90 drops the w_p (rho - 1) term for shifted storage, :179-197.)
//
// The reference's own forms, in its arithmetic (init_reference_kernel):
//   INIT_TGV_REF  the TGV3D form of SRC/init.F90:141-148: x = (i - 0.5)/l,
//                 u = u00 sin(2 pi x) cos(2 pi y) cos(2 pi z), v = -u00 cos
//                 sin cos, w = 0, rho = 1 + (u00^2 / (4 4 3)) (cos 4 pi x +
//                 cos 4 pi y)(cos 4 pi z + 2),  u00 = p[0]
//   INIT_TG2D_REF the default periodic 2-D Taylor-Green form (:125-130):
//                 u = 0.1 sin(2 pi x) cos(2 pi z), w = -0.1 cos(2 pi x)
//                 sin(2 pi z), rho = 1
// Both compute in the compute type C with the reference's literals: pi is a
// default-real (single precision) constant (:63), the coordinates are
// formed in double and rounded to C (the 0.5d0 literal), the 2-D form's
// products are double (0.1d0); populations crho p_w (cte1 + cx_p) with cte1
// = 0 (shifted storage, :150-197), so w_p (rho - 1) is dropped as the
// reference drops it.
#pragma once
#include "d3q19.cuh"

namespace bgk {

enum InitFlow : int { INIT_UNIFORM = 0, INIT_TGV = 1, INIT_KIDA = 2, INIT_TGV_REF = 3, INIT_TG2D_REF = 4 };

template <class S> struct InitArgs {
    S* f[19];            // destination arrays of populations 01..19 (AA: slot arrays already permuted)
    long long nx, nxy;
    int l, m, n;
    int flow;
    double p[4];
    float scale;
};

__device__ __forceinline__ double weight_of(int d) {
    const int s = abs(cx_of(d)) + abs(cy_of(d)) + abs(cz_of(d));
    return s == 2 ? 1.0 / 36.0 : (s == 1 ? 1.0 / 18.0 : 1.0 / 3.0);
}

template <class S> __device__ __forceinline__ S store_from_double(double v, float scl);
template <> __device__ __forceinline__ double store_from_double<double>(double v, float) { return v; }
template <> __device__ __forceinline__ float store_from_double<float>(double v, float) { return __double2float_rn(v); }
template <> __device__ __forceinline__ __half store_from_double<__half>(double v, float scl) {
    return __float2half_rn(__fmul_rn(__double2float_rn(v), scl));
}
template <> __device__ __forceinline__ __nv_bfloat16 store_from_double<__nv_bfloat16>(double v, float scl) {
    return __float2bfloat16_rn(__fmul_rn(__double2float_rn(v), scl));
}

// One thread per node (0..l+1, 0..m+1, 0..n+1): the halo gets the flow
// evaluated at its own coordinates (periodic images coincide).
template <class S>
__global__ void init_equilibrium_kernel(const InitArgs<S> A) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ni = A.l + 2, nj = A.m + 2, nk = A.n + 2;
    if (t >= ni * nj * nk) return;
    const int i = (int)(t % ni), j = (int)((t / ni) % nj), k = (int)(t / (ni * nj));
    double rho = 1.0, ux = 0.0, uy = 0.0, uz = 0.0;
    if (A.flow == INIT_UNIFORM) {
        rho = A.p[0]; ux = A.p[1]; uy = A.p[2]; uz = A.p[3];
    } else {
        const double tp = 6.283185307179586476925286766559;
        const double x = tp * (i - 1) / A.l, y = tp * (j - 1) / A.m, z = tp * (k - 1) / A.n;
        const double u0 = A.p[0];
        if (A.flow == INIT_TGV) {
            ux = u0 * sin(x) * cos(y) * cos(z);
            uy = -u0 * cos(x) * sin(y) * cos(z);
            rho = 1.0 + 3.0 * (u0 * u0 / 16.0) * (cos(2.0 * x) + cos(2.0 * y)) * (cos(2.0 * z) + 2.0);
        } else {
            ux = u0 * sin(x) * (cos(3.0 * y) * cos(z) - cos(y) * cos(3.0 * z));
            uy = u0 * sin(y) * (cos(3.0 * z) * cos(x) - cos(z) * cos(3.0 * x));
            uz = u0 * sin(z) * (cos(3.0 * x) * cos(y) - cos(x) * cos(3.0 * y));
        }
    }
    const double usq = ux * ux + uy * uy + uz * uz;
    const long long c = i + A.nx * j + A.nxy * k;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
        const double cu = cx_of(d) * ux + cy_of(d) * uy + cz_of(d) * uz;
        const double w = weight_of(d);
        A.f[d][c] = store_from_double<S>(w * (rho - 1.0) + w * rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * usq), A.scale);
    }
}

// Sine / cosine of the compute type: for float the double function rounded
// once (the correctly rounded value, as libm's sinf gives it), for double the
// double function.
__device__ __forceinline__ float ref_sin(float a) { return __double2float_rn(sin((double)a)); }
__device__ __forceinline__ float ref_cos(float a) { return __double2float_rn(cos((double)a)); }
__device__ __forceinline__ double ref_sin(double a) { return sin(a); }
__device__ __forceinline__ double ref_cos(double a) { return cos(a); }

template <class S, class C> struct InitRefArgs {
    S* f[19];
    long long nx, nxy;
    int l, m, n;
    int flow;
    C u00, rf, qf, tre, p0, p1, p2;
    float scale;
};

// One thread per node of the box (0..l+1, 0..m+1, 0..n+1).
template <class S, class C>
__global__ void init_reference_kernel(const InitRefArgs<S, C> A) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ni = A.l + 2, nj = A.m + 2, nk = A.n + 2;
    if (t >= ni * nj * nk) return;
    const int i = (int)(t % ni), j = (int)((t / ni) % nj), k = (int)(t / (ni * nj));
    const C pi = C(3.14159265358979323846f);
    const C x = (C)(((double)i - 0.5) / (double)A.l);
    const C y = (C)(((double)j - 0.5) / (double)A.m);
    const C z = (C)(((double)k - 0.5) / (double)A.n);
    C xj, yj, zj, crho = C(1);
    const C rf = A.rf, qf = A.qf, tre = A.tre;
    if (A.flow == INIT_TGV_REF) {
        const C u00 = A.u00, due = C(2), qua = C(4);
        xj = u00 * ref_sin(due * pi * x) * ref_cos(due * pi * y) * ref_cos(due * pi * z);
        yj = -(u00 * ref_cos(due * pi * x) * ref_sin(due * pi * y) * ref_cos(due * pi * z));
        zj = C(0);
        crho = C(1) + ((u00 * u00) / (qua * qua * tre)) * (ref_cos(qua * pi * x) + ref_cos(qua * pi * y)) *
                          (ref_cos(qua * pi * z) + due);
    } else {
        const C two = C(2);
        xj = (C)(0.1 * (double)ref_sin(two * pi * x) * (double)ref_cos(two * pi * z));
        yj = C(0);
        zj = (C)(-(0.1 * (double)ref_cos(two * pi * x) * (double)ref_sin(two * pi * z)));
    }
    const C cte1 = C(0);
    const C cvsq = xj * xj + yj * yj + zj * zj;
    C cx[19];
    cx[0] = rf * (xj - yj) + qf * (tre * (xj - yj) * (xj - yj) - cvsq);
    cx[1] = rf * (xj - zj) + qf * (tre * (xj - zj) * (xj - zj) - cvsq);
    cx[2] = rf * (xj + yj) + qf * (tre * (xj + yj) * (xj + yj) - cvsq);
    cx[3] = rf * (xj + zj) + qf * (tre * (xj + zj) * (xj + zj) - cvsq);
    cx[4] = rf * (xj) + qf * (tre * (xj) * (xj) - cvsq);
    cx[5] = rf * (zj) + qf * (tre * (zj) * (zj) - cvsq);
    cx[6] = rf * (yj + zj) + qf * (tre * (yj + zj) * (yj + zj) - cvsq);
    cx[7] = rf * (yj) + qf * (tre * (yj) * (yj) - cvsq);
    cx[8] = rf * (yj - zj) + qf * (tre * (yj - zj) * (yj - zj) - cvsq);
    cx[9] = rf * (-xj - yj) + qf * (tre * (xj + yj) * (xj + yj) - cvsq);
    cx[10] = rf * (-xj - zj) + qf * (tre * (xj + zj) * (xj + zj) - cvsq);
    cx[11] = rf * (-xj + yj) + qf * (tre * (xj - yj) * (xj - yj) - cvsq);
    cx[12] = rf * (-xj + zj) + qf * (tre * (xj - zj) * (xj - zj) - cvsq);
    cx[13] = rf * (-xj) + qf * (tre * (xj) * (xj) - cvsq);
    cx[14] = rf * (-zj) + qf * (tre * (zj) * (zj) - cvsq);
    cx[15] = rf * (-yj - zj) + qf * (tre * (yj + zj) * (yj + zj) - cvsq);
    cx[16] = rf * (-yj) + qf * (tre * (yj) * (yj) - cvsq);
    cx[17] = rf * (-yj + zj) + qf * (tre * (yj - zj) * (yj - zj) - cvsq);
    cx[18] = rf * C(0) + qf * (tre * C(0) * C(0) - cvsq);
    const long long c = i + A.nx * j + A.nxy * k;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
        const int s = abs(cx_of(d)) + abs(cy_of(d)) + abs(cz_of(d));
        const C w = s == 0 ? A.p0 : (s == 1 ? A.p1 : A.p2);
        A.f[d][c] = Conv<S, C>::st(crho * w * (cte1 + cx[d]), A.scale);
    }
}

}  // namespace bgk
