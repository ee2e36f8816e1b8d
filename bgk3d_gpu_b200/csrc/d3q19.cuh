// D3Q19 lattice tables, storage conversions and the BGK collision shared by
// every kernel of the library.
//
// Population numbering, velocities and the pull offsets follow the reference
// exactly (SRC/alloca.F90:29-148 for c_x, c_y, c_z; SRC/col_MC.F90:275-293 for
// the pull x_p = a_p(x - c_p)).  Index 0..18 here is population 01..19.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

namespace bgk {

// velocity components of populations 01..19
__host__ __device__ constexpr int cx_of(int d) {
    return d < 5 ? 1 : (d >= 9 && d < 14 ? -1 : 0);
}
__host__ __device__ constexpr int cy_of(int d) {
    // 01:-1 02:0 03:1 04:0 05:0 06:0 07:1 08:1 09:1 10:-1 11:0 12:1 13:0 14:0 15:0 16:-1 17:-1 18:-1 19:0
    return (d == 0 || d == 9 || d == 15 || d == 16 || d == 17) ? -1
         : (d == 2 || d == 6 || d == 7 || d == 8 || d == 11) ? 1 : 0;
}
__host__ __device__ constexpr int cz_of(int d) {
    // 01:0 02:-1 03:0 04:1 05:0 06:1 07:1 08:0 09:-1 10:0 11:-1 12:0 13:1 14:0 15:-1 16:-1 17:0 18:1 19:0
    return (d == 1 || d == 8 || d == 10 || d == 14 || d == 15) ? -1
         : (d == 3 || d == 5 || d == 6 || d == 12 || d == 17) ? 1 : 0;
}
// opposite population: 01<->12, 02<->13, 03<->10, 04<->11, 05<->14,
// 06<->15, 07<->16, 08<->17, 09<->18, 19<->19
__host__ __device__ constexpr int opp_of(int d) {
    return d == 18 ? 18 : (d < 5 ? (d == 0 ? 11 : d == 1 ? 12 : d == 2 ? 9 : d == 3 ? 10 : 13)
                         : d < 9 ? d + 9
                         : d < 14 ? (d == 9 ? 2 : d == 10 ? 3 : d == 11 ? 0 : d == 12 ? 1 : 4)
                         : d - 9);
}

// Storage kinds (identical numbering in the C-ABI and in the oracle)
enum Kind : int { K_F64 = 0, K_F32 = 1, K_F16 = 2, K_BF16 = 3, K_F32_F64 = 4 };
// Boundary cases (SRC/boundaries.F90:31-43) plus NONE: halos are the caller's.
enum BCase : int { BC_NONE = -1, BC_DRIVEN = 0, BC_PERIODIC = 1, BC_CHANNEL = 2, BC_INFLOW = 3 };

// ------------------------------------------------------------------ storage
// Conv<S,C>: storage element S <-> compute value C.  16-bit kinds hold
// scale*(f - w) rounded to nearest even; scale is a power of two so the
// multiplications are exact.
template <class S, class C> struct Conv;
template <> struct Conv<double, double> {
    __device__ __forceinline__ static double ld(double v, float) { return v; }
    __device__ __forceinline__ static double st(double v, float) { return v; }
};
template <> struct Conv<float, float> {
    __device__ __forceinline__ static float ld(float v, float) { return v; }
    __device__ __forceinline__ static float st(float v, float) { return v; }
};
template <> struct Conv<float, double> {
    __device__ __forceinline__ static double ld(float v, float) { return (double)v; }
    __device__ __forceinline__ static float st(double v, float) { return __double2float_rn(v); }
};
template <> struct Conv<__half, float> {
    __device__ __forceinline__ static float ld(__half v, float inv) { return __fmul_rn(__half2float(v), inv); }
    __device__ __forceinline__ static __half st(float v, float scl) { return __float2half_rn(__fmul_rn(v, scl)); }
};
template <> struct Conv<__nv_bfloat16, float> {
    __device__ __forceinline__ static float ld(__nv_bfloat16 v, float inv) { return __fmul_rn(__bfloat162float(v), inv); }
    __device__ __forceinline__ static __nv_bfloat16 st(float v, float scl) { return __float2bfloat16_rn(__fmul_rn(v, scl)); }
};

// Read-only streamed load for populations that the launch never writes.
template <class S> __device__ __forceinline__ S ldro(const S* p) { return __ldg(p); }
template <> __device__ __forceinline__ __half ldro<__half>(const __half* p) {
    unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
    return __ushort_as_half(u);
}
template <> __device__ __forceinline__ __nv_bfloat16 ldro<__nv_bfloat16>(const __nv_bfloat16* p) {
    unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
    return __ushort_as_bfloat16(u);
}

// Unsigned 32-bit division by a runtime constant with a multiply-high and a
// shift (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, round-up variant).  Exact for every n < 2^32.
struct FastDiv {
    uint32_t d, mul, shift;
    __host__ void init(uint32_t divisor) {
        d = divisor;
        uint32_t l = 0;
        while ((1ull << l) < divisor) ++l;
        // mul = floor(2^32 (2^l - d) / d) + 1
        mul = (uint32_t)((((1ull << l) - divisor) << 32) / divisor + 1);
        shift = l;
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        if (shift == 0) return n;   // d == 1
        const uint32_t t = __umulhi(n, mul);
        return (t + ((n - t) >> 1)) >> (shift - 1);
    }
};

// Collision constants in the compute type.  Weights are computed in double
// and rounded once, as the reference's parameters are (SRC/storage.F90:58-82,
// 147-151).
template <class C> struct ColConst {
    C omega, cte0, cte1, p0, p1, p2, rf, qf, tre;
    int force_mode;  // 0: constant forces; 1: force = f * rho
    C fx, fy, fz;
};

// BGK collision of the 19 pulled values x[] into y[], in the exact operation
// order of SRC/col_MC.F90:295-379 and :501-519.  The library is compiled with
// --fmad=false, so every + and * below rounds separately, as in the reference
// source.  Returns rho, vx, vy, vz (before the rf scaling) through mom[].
//
// GENERIC = false is the specialisation for shifted storage (cte1 = 1,
// cte0 = 0) without forcing: it omits the terms that are then additions of
// +0 or multiplications by 1, which changes no result except possibly the
// sign of an exact zero.
template <class C, bool GENERIC = true>
__device__ __forceinline__ void bgk_collide(const C (&x)[19], C (&y)[19], const ColConst<C>& P,
                                            C* mom = nullptr) {
    const C cte0 = P.cte0, cte1 = P.cte1, tre = P.tre, qf = P.qf, rf = P.rf;
    const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] +
                  x[11] + x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + cte1;
    const C rhoinv = C(1) / rho;
    C vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
    C vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
    C vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
    if (mom) { mom[0] = rho; mom[1] = vx; mom[2] = vy; mom[3] = vz; }
    const C vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    const C vsq = vx2 + vy2 + vz2;
    auto q = [&](C t) -> C { return GENERIC ? cte0 + qf * t : qf * t; };
    C vxpy = vx + vy;
    const C qxpy = q(tre * vxpy * vxpy - vsq);
    C vxmy = vx - vy;
    const C qxmy = q(tre * vxmy * vxmy - vsq);
    C vxpz = vx + vz;
    const C qxpz = q(tre * vxpz * vxpz - vsq);
    C vxmz = vx - vz;
    const C qxmz = q(tre * vxmz * vxmz - vsq);
    C vypz = vy + vz;
    const C qypz = q(tre * vypz * vypz - vsq);
    C vymz = vy - vz;
    const C qymz = q(tre * vymz * vymz - vsq);
    const C qx = q(tre * vx2 - vsq);
    const C qy = q(tre * vy2 - vsq);
    const C qz = q(tre * vz2 - vsq);
    const C q0 = q(-vsq);
    vx = rf * vx; vy = rf * vy; vz = rf * vz;
    vxpy = rf * vxpy; vxmy = rf * vxmy; vxpz = rf * vxpz;
    vxmz = rf * vxmz; vypz = rf * vypz; vymz = rf * vymz;
    const C p0 = P.p0, p1 = P.p1, p2 = P.p2;
    const C rp0 = rho * p0, rp1 = rho * p1, rp2 = rho * p2;
    const C s2 = GENERIC ? cte1 * (rp2 - p2) : rp2 - p2;
    const C s1 = GENERIC ? cte1 * (rp1 - p1) : rp1 - p1;
    const C s0 = GENERIC ? cte1 * (rp0 - p0) : rp0 - p0;
    C e[19];
    e[0] = rp2 * (+vxmy + qxmy) + s2;
    e[1] = rp2 * (+vxmz + qxmz) + s2;
    e[2] = rp2 * (+vxpy + qxpy) + s2;
    e[3] = rp2 * (+vxpz + qxpz) + s2;
    e[4] = rp1 * (+vx + qx) + s1;
    e[5] = rp1 * (+vz + qz) + s1;
    e[6] = rp2 * (+vypz + qypz) + s2;
    e[7] = rp1 * (+vy + qy) + s1;
    e[8] = rp2 * (+vymz + qymz) + s2;
    e[9] = rp2 * (-vxpy + qxpy) + s2;
    e[10] = rp2 * (-vxpz + qxpz) + s2;
    e[11] = rp2 * (-vxmy + qxmy) + s2;
    e[12] = rp2 * (-vxmz + qxmz) + s2;
    e[13] = rp1 * (-vx + qx) + s1;
    e[14] = rp1 * (-vz + qz) + s1;
    e[15] = rp2 * (-vypz + qypz) + s2;
    e[16] = rp1 * (-vy + qy) + s1;
    e[17] = rp2 * (-vymz + qymz) + s2;
    e[18] = rp0 * (+q0) + s0;
    const C om = P.omega;
    if (!GENERIC) {
#pragma unroll
        for (int d = 0; d < 18; ++d) y[d] = x[d] - om * (x[d] - e[d]);
    } else {
    C fx = P.fx, fy = P.fy, fz = P.fz;
    if (P.force_mode == 1) { fx = P.fx * rho; fy = P.fy * rho; fz = P.fz * rho; }
    y[0] = x[0] - om * (x[0] - e[0]) + fx - fy;
    y[1] = x[1] - om * (x[1] - e[1]) + fx - fz;
    y[2] = x[2] - om * (x[2] - e[2]) + fx + fy;
    y[3] = x[3] - om * (x[3] - e[3]) + fx + fz;
    y[4] = x[4] - om * (x[4] - e[4]) + fx;
    y[5] = x[5] - om * (x[5] - e[5]) + fz;
    y[6] = x[6] - om * (x[6] - e[6]) + fy + fz;
    y[7] = x[7] - om * (x[7] - e[7]) + fy;
    y[8] = x[8] - om * (x[8] - e[8]) + fy - fz;
    y[9] = x[9] - om * (x[9] - e[9]) - fx - fy;
    y[10] = x[10] - om * (x[10] - e[10]) - fx - fz;
    y[11] = x[11] - om * (x[11] - e[11]) - fx + fy;
    y[12] = x[12] - om * (x[12] - e[12]) - fx + fz;
    y[13] = x[13] - om * (x[13] - e[13]) - fx;
    y[14] = x[14] - om * (x[14] - e[14]) - fz;
    y[15] = x[15] - om * (x[15] - e[15]) - fy - fz;
    y[16] = x[16] - om * (x[16] - e[16]) - fy;
    y[17] = x[17] - om * (x[17] - e[17]) - fy + fz;
    }
    y[18] = x[18] - om * (x[18] - e[18]);
}

}  // namespace bgk
