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
// multiplications are exact.  ld/st convert physical values; raw/pack
// convert storage units (the scaled value itself), which is what the
// time-step kernels compute in: with power-of-two scales every intermediate
// rounding of the collision is the physical one times the scale, so the
// results are bit-identical and 38 multiplications per node are saved.
template <class S, class C> struct Conv;
template <> struct Conv<double, double> {
    __device__ __forceinline__ static double ld(double v, float) { return v; }
    __device__ __forceinline__ static double st(double v, float) { return v; }
    __device__ __forceinline__ static double raw(double v) { return v; }
    __device__ __forceinline__ static double pack(double v) { return v; }
};
template <> struct Conv<float, float> {
    __device__ __forceinline__ static float ld(float v, float) { return v; }
    __device__ __forceinline__ static float st(float v, float) { return v; }
    __device__ __forceinline__ static float raw(float v) { return v; }
    __device__ __forceinline__ static float pack(float v) { return v; }
};
template <> struct Conv<float, double> {
    __device__ __forceinline__ static double ld(float v, float) { return (double)v; }
    __device__ __forceinline__ static float st(double v, float) { return __double2float_rn(v); }
    __device__ __forceinline__ static double raw(float v) { return (double)v; }
    __device__ __forceinline__ static float pack(double v) { return __double2float_rn(v); }
};
template <> struct Conv<__half, float> {
    __device__ __forceinline__ static float ld(__half v, float inv) { return __fmul_rn(__half2float(v), inv); }
    __device__ __forceinline__ static __half st(float v, float scl) { return __float2half_rn(__fmul_rn(v, scl)); }
    __device__ __forceinline__ static float raw(__half v) { return __half2float(v); }
    __device__ __forceinline__ static __half pack(float v) { return __float2half_rn(v); }
};
template <> struct Conv<__nv_bfloat16, float> {
    __device__ __forceinline__ static float ld(__nv_bfloat16 v, float inv) { return __fmul_rn(__bfloat162float(v), inv); }
    __device__ __forceinline__ static __nv_bfloat16 st(float v, float scl) { return __float2bfloat16_rn(__fmul_rn(v, scl)); }
    __device__ __forceinline__ static float raw(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ __forceinline__ static __nv_bfloat16 pack(float v) { return __float2bfloat16_rn(v); }
};

// True for the kinds stored scaled (the 16-bit ones).
template <class S> struct Scaled { static constexpr bool value = sizeof(S) == 2; };

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
// Resident 256-thread blocks per SM that the two-lattice one-node sweep is
// compiled for (the register cap follows: 64K / (256 x blocks)).  FP64
// compute needs the most registers; the 16-bit kinds move half the bytes of
// FP32 per node, so they need more warps in flight to cover memory latency
// (5 blocks = 48 registers; measured on 256^3 against 4 blocks: FP16 +5 %
// periodic, +6 % driven).  The in-place and batched sweeps keep 4: they
// spill at 48.
template <class S, class C> struct SweepBlocks {
    static constexpr int value = sizeof(C) == 8 ? 3 : (sizeof(S) == 2 ? 5 : 4);
};

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
// 147-151).  In the time-step kernels p0, p1, p2 and the forces are in
// storage units (multiplied by the 16-bit scale).
template <class C> struct ColConst {
    C omega, cte0, cte1, p0, p1, p2, rf, qf, tre;
    int force_mode;  // 0: constant forces; 1: force = f * rho
    C fx, fy, fz;
};

// Round-to-nearest reciprocal, the correctly rounded 1 / a: the same value as
// the IEEE division 1 / a (so the reference-order collision stays
// bit-identical), in fewer instructions than a general division.  An
// approximate reciprocal would bias the velocity in one direction every step
// and the momentum would drift (measured: 5e-5 relative kinetic-energy error
// after 400 TGV steps, against 1.5e-5 for the reference order).
__device__ __forceinline__ float rcp_c(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double rcp_c(double a) { return 1.0 / a; }
// 1 / a correctly rounded, as the reference-order collision forms it: the IEEE
// division for one value (measured faster there than the reciprocal
// instruction sequence, 40 vs 36 GLUPS on the FP32 channel case), the
// reciprocal for a packed pair (f2.cuh: two reciprocals are cheaper than two
// divisions; FP16 reference order +5 %).  The same bits either way.
__device__ __forceinline__ float inv_rn(float a) { return 1.0f / a; }
__device__ __forceinline__ double inv_rn(double a) { return 1.0 / a; }

// Collision modes of the time-step kernels.
enum CollMode : int {
    CM_STRICT = 0,          // reference operation order, shifted storage, no force
    CM_STRICT_GENERIC = 1,  // reference operation order, any cte0/cte1, forces
    CM_FAST = 2,            // fused multiply-adds, shifted storage, no force
    CM_FAST_GENERIC = 3,    // fused multiply-adds, any cte0/cte1, forces
};
__host__ __device__ constexpr bool cm_generic(int cm) { return (cm & 1) != 0; }
__host__ __device__ constexpr bool cm_fast(int cm) { return cm >= 2; }

// BGK collision of the 19 pulled values x[] into y[], in the exact operation
// order of SRC/col_MC.F90:295-379 and :501-519.  The library is compiled with
// --fmad=false, so every + and * below rounds separately, as in the reference
// source.  x and y are in storage units; with SCALED (16-bit kinds) the four
// sums that give rho and the velocity are unscaled by inv (exact).
//
// GENERIC = false is the specialisation for shifted storage (cte1 = 1,
// cte0 = 0) without forcing: it omits the terms that are then additions of
// +0 or multiplications by 1, which changes no result except possibly the
// sign of an exact zero.
//
// bgk_collide_f reads population d through xs(d) for the moment sums and
// through xp(d) for the relaxation, and hands y_d to ys(d, y_d); the
// equilibria are formed pair by pair (+-c share their velocity term), so
// that a caller short of registers never holds all 19 of them.  Every value
// is computed by the same operations in the same order as in the reference.
template <class V, class C, bool GENERIC, bool SCALED, class XS, class XP, class YS>
__device__ __forceinline__ void bgk_collide_f(XS xs, XP xp, YS ys, const ColConst<C>& P, float inv) {
    const V cte0 = V(P.cte0), cte1 = V(P.cte1), tre = V(P.tre), qf = V(P.qf), rf = V(P.rf);
    V sum = xs(0) + xs(1) + xs(2) + xs(3) + xs(4) + xs(5) + xs(6) + xs(7) + xs(8) + xs(9) + xs(10) +
            xs(11) + xs(12) + xs(13) + xs(14) + xs(15) + xs(16) + xs(17) + xs(18);
    if (SCALED) sum = sum * V((C)inv);
    const V rho = sum + cte1;
    const V rhoinv = inv_rn(rho);   // the correctly rounded 1 / rho
    V mx = xs(0) + xs(1) + xs(2) + xs(3) + xs(4) - xs(9) - xs(10) - xs(11) - xs(12) - xs(13);
    V my = xs(2) + xs(6) + xs(7) + xs(8) + xs(11) - xs(0) - xs(9) - xs(15) - xs(16) - xs(17);
    V mz = xs(3) + xs(5) + xs(6) + xs(12) + xs(17) - xs(1) - xs(8) - xs(10) - xs(14) - xs(15);
    if (SCALED) { mx = mx * V((C)inv); my = my * V((C)inv); mz = mz * V((C)inv); }
    const V vx = mx * rhoinv, vy = my * rhoinv, vz = mz * rhoinv;
    const V vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    const V vsq = vx2 + vy2 + vz2;
    auto q = [&](V t) -> V { return GENERIC ? cte0 + qf * t : qf * t; };
    const V p0 = V(P.p0), p1 = V(P.p1), p2 = V(P.p2);
    const V rp0 = rho * p0, rp1 = rho * p1, rp2 = rho * p2;
    const V s2 = GENERIC ? cte1 * (rp2 - p2) : rp2 - p2;
    const V s1 = GENERIC ? cte1 * (rp1 - p1) : rp1 - p1;
    const V s0 = GENERIC ? cte1 * (rp0 - p0) : rp0 - p0;
    const V om = V(P.omega);
    V fx = V(C(0)), fy = V(C(0)), fz = V(C(0));
    if (GENERIC) {
        fx = V(P.fx); fy = V(P.fy); fz = V(P.fz);
        if (P.force_mode == 1) { fx = V(P.fx) * rho; fy = V(P.fy) * rho; fz = V(P.fz) * rho; }
    }
    // relaxation of population d towards its equilibrium e (x read once: a
    // caller's xp may convert a packed word, and that conversion is opaque
    // to the compiler)
    auto relax = [&](int d, V e) -> V {
        const V x = xp(d);
        return x - om * (x - e);
    };
    // axis pair dp / dm along v_a: q from tre (v_a v_a); force +-f
    auto axis = [&](int dp, int dm, V v, V v2, V f) {
        const V qa = q(tre * v2 - vsq);
        const V lin = rf * v;
        const V yp = relax(dp, rp1 * (+lin + qa) + s1), ym = relax(dm, rp1 * (-lin + qa) + s1);
        ys(dp, GENERIC ? yp + f : yp);
        ys(dm, GENERIC ? ym - f : ym);
    };
    // diagonal pair dp / dm along v = v_a +- v_b: q from (tre v) v; forces
    // added one at a time as the reference writes them, dp: + fa +- fb,
    // dm: - fa -+ fb (bminus: the sign of fb in dp is minus)
    auto diag = [&](int dp, int dm, V v, V fa, V fb, bool bminus) {
        const V qd = q(tre * v * v - vsq);
        const V lin = rf * v;
        const V yp = relax(dp, rp2 * (+lin + qd) + s2), ym = relax(dm, rp2 * (-lin + qd) + s2);
        if (GENERIC) {
            const V yp1 = yp + fa, ym1 = ym - fa;
            ys(dp, bminus ? yp1 - fb : yp1 + fb);
            ys(dm, bminus ? ym1 + fb : ym1 - fb);
        } else {
            ys(dp, yp);
            ys(dm, ym);
        }
    };
    diag(0, 11, vx - vy, fx, fy, true);
    diag(1, 12, vx - vz, fx, fz, true);
    diag(2, 9, vx + vy, fx, fy, false);
    diag(3, 10, vx + vz, fx, fz, false);
    axis(4, 13, vx, vx2, fx);
    axis(5, 14, vz, vz2, fz);
    diag(6, 15, vy + vz, fy, fz, false);
    axis(7, 16, vy, vy2, fy);
    diag(8, 17, vy - vz, fy, fz, true);
    ys(18, relax(18, rp0 * (+q(-vsq)) + s0));
}

template <class V, class C, bool GENERIC, bool SCALED>
__device__ __forceinline__ void bgk_collide_v(const V (&x)[19], V (&y)[19], const ColConst<C>& P, float inv) {
    auto xr = [&](int d) { return x[d]; };
    bgk_collide_f<V, C, GENERIC, SCALED>(xr, xr, [&](int d, V v) { y[d] = v; }, P, inv);
}

// The collision on one node's compute values.
template <class C, bool GENERIC = true, bool SCALED = false>
__device__ __forceinline__ void bgk_collide(const C (&x)[19], C (&y)[19], const ColConst<C>& P,
                                            float inv = 1.0f) {
    bgk_collide_v<C, C, GENERIC, SCALED>(x, y, P, inv);
}

// Constants of the fused-multiply-add collision, in storage units, computed
// on the host in double and rounded once: with u = rho (cte0 - qf |v|^2) +
// cte1 (rho - 1), omega times the equilibrium of the pair +-c is
//   omega e_+- = b_w u + rho a_w (c.v)^2 +- rho r_w (c.v),
// a_w = omega qf tre p_w, r_w = omega rf p_w, b_w = omega p_w -- the same
// polynomial as SRC/col_MC.F90:361-379, regrouped.
template <class C> struct FastConst {
    C omc;                 // 1 - omega
    C a1, a2, r1, r2;      // axis (p1) and diagonal (p2) classes
    C b0, b1, b2;          // rest, axis, diagonal
    C qf, cte0, cte1;
    int force_mode;
    C fx, fy, fz;          // storage units
};

__device__ __forceinline__ float fma_c(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_c(double a, double b, double c) { return __fma_rn(a, b, c); }

// The BGK collision as pairs of opposite populations with fused
// multiply-adds: y_+- = (1 - omega) x_+- + omega e_+- (+- the body force,
// which is odd in c).  About 140 operations per node instead of 240; not
// bit-identical to the reference order (the results differ by a few units in
// the last place of the compute type per step).
//
// bgk_collide_fast_f reads population d through xs(d) for the moment sums and
// through xp(d) for the relaxation, and hands y_d to ys(d, y_d): a caller
// short of registers can keep the inputs packed and convert them twice, and
// store each result as soon as it is known.
template <class V, class C, bool GENERIC, bool SCALED, class XS, class XP, class YS>
__device__ __forceinline__ void bgk_collide_fast_f(XS xs, XP xp, YS ys, const FastConst<C>& K, float inv) {
    const V sum = xs(0) + xs(1) + xs(2) + xs(3) + xs(4) + xs(5) + xs(6) + xs(7) + xs(8) + xs(9) + xs(10) +
                  xs(11) + xs(12) + xs(13) + xs(14) + xs(15) + xs(16) + xs(17) + xs(18);
    const V rho = SCALED ? fma_c(sum, V((C)inv), V(K.cte1)) : sum + V(K.cte1);
    const V ri = rcp_c(rho);
    const V mx = xs(0) + xs(1) + xs(2) + xs(3) + xs(4) - xs(9) - xs(10) - xs(11) - xs(12) - xs(13);
    const V my = xs(2) + xs(6) + xs(7) + xs(8) + xs(11) - xs(0) - xs(9) - xs(15) - xs(16) - xs(17);
    const V mz = xs(3) + xs(5) + xs(6) + xs(12) + xs(17) - xs(1) - xs(8) - xs(10) - xs(14) - xs(15);
    const V g = SCALED ? V((C)inv) * ri : ri;
    const V vx = mx * g, vy = my * g, vz = mz * g;
    const V vsq = fma_c(vz, vz, fma_c(vy, vy, vx * vx));
    const V t = GENERIC ? fma_c(V(-K.qf), vsq, V(K.cte0)) : V(-K.qf) * vsq;
    const V u = GENERIC ? fma_c(rho, t, V(K.cte1) * (rho - V(C(1)))) : fma_c(rho, t, rho - V(C(1)));
    const V B0 = V(K.b0) * u, B1 = V(K.b1) * u, B2 = V(K.b2) * u;
    const V A1 = rho * V(K.a1), A2 = rho * V(K.a2), R1 = rho * V(K.r1), R2 = rho * V(K.r2);
    V fx = V(C(0)), fy = V(C(0)), fz = V(C(0));
    if (GENERIC) {
        fx = V(K.fx); fy = V(K.fy); fz = V(K.fz);
        if (K.force_mode == 1) { fx = fx * rho; fy = fy * rho; fz = fz * rho; }
    }
    const V om = V(K.omc);
    auto pair = [&](int dp, int dm, V v, V A, V B, V R, V f) {
        const V sym = fma_c(A, v * v, B);
        const V an = GENERIC ? fma_c(R, v, f) : R * v;
        ys(dp, fma_c(xp(dp), om, sym) + an);
        ys(dm, fma_c(xp(dm), om, sym) - an);
    };
    pair(0, 11, vx - vy, A2, B2, R2, fx - fy);
    pair(1, 12, vx - vz, A2, B2, R2, fx - fz);
    pair(2, 9, vx + vy, A2, B2, R2, fx + fy);
    pair(3, 10, vx + vz, A2, B2, R2, fx + fz);
    pair(4, 13, vx, A1, B1, R1, fx);
    pair(5, 14, vz, A1, B1, R1, fz);
    pair(6, 15, vy + vz, A2, B2, R2, fy + fz);
    pair(7, 16, vy, A1, B1, R1, fy);
    pair(8, 17, vy - vz, A2, B2, R2, fy - fz);
    ys(18, fma_c(xp(18), om, B0));
}

template <class V, class C, bool GENERIC, bool SCALED>
__device__ __forceinline__ void bgk_collide_fast_v(const V (&x)[19], V (&y)[19], const FastConst<C>& K,
                                                   float inv) {
    auto xr = [&](int d) { return x[d]; };
    bgk_collide_fast_f<V, C, GENERIC, SCALED>(xr, xr, [&](int d, V v) { y[d] = v; }, K, inv);
}

template <class C, bool GENERIC, bool SCALED>
__device__ __forceinline__ void bgk_collide_fast(const C (&x)[19], C (&y)[19], const FastConst<C>& K,
                                                 float inv = 1.0f) {
    bgk_collide_fast_v<C, C, GENERIC, SCALED>(x, y, K, inv);
}

// Collision of one node in storage units under collision mode CM.
template <class S, class C, int CM>
__device__ __forceinline__ void collide_cm(const C (&x)[19], C (&y)[19], const ColConst<C>& K,
                                           const FastConst<C>& F, float inv) {
    constexpr bool SC = Scaled<S>::value;
    if constexpr (cm_fast(CM)) bgk_collide_fast<C, cm_generic(CM), SC>(x, y, F, inv);
    else bgk_collide<C, cm_generic(CM), SC>(x, y, K, inv);
}

}  // namespace bgk
