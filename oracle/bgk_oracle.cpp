// ============================================================================
//  bgk_oracle.cpp -- CPU ORACLE (test infrastructure only).
//
//  A plain, loop-by-loop restatement of the reference's fused D3Q19 BGK time
//  step, used ONLY by tests/, __graft_entry__.smoke() and bench.py's
//  cpu_baseline / reference arm to check (never to produce) the CUDA results.
//  Nothing in the product path links or calls this file.
//
//  What it restates (paths relative to the reference project):
//    * SRC/col_MC.F90:255-536       fused pull-stream + BGK collision, written
//                                   to b01..b18 and in place to a19, in the
//                                   exact source order of the arithmetic
//                                   (the same order SRC/col_MC_gpu.hpp:163-255
//                                   uses), optional forcing :472-488 / :501-519
//    * SRC/bcond.driven.F90:107-247  x -> y -> z halo bounce-back, lid force
//    * SRC/bcond.periodic.F90:107-252 x -> y -> z periodic halo copies
//    * SRC/bcond.channel.F90:124-267 x,y periodic, z no-slip (GPU-branch ranges
//                                   1..l, 1..m of :245-251; the do-concurrent
//                                   branch :253 indexes out of bounds)
//    * SRC/bcond.inflow.F90:131-313  outflow/inflow equilibria + y,z periodic
//    * SRC/bcond.obs.F90:103-122     obstacle bounce-back into solid nodes,
//                                   executed serially in Fortran loop order
//    * SRC/diagno.F90:87-138         per-node moments, FP64 accumulation
//    * SRC/draglift.F90:77-176       momentum-exchange drag/lift (accumulated
//                                   in FP64 here; the reference uses mykind)
//    * SRC/dissipation.F90:136-338   tke, 2 nu Pi:Pi dissipation and the mean
//                                   squared velocity components (per-node in
//                                   the compute type, sums in FP64; the
//                                   reference sums in mykind), the pull read
//                                   from the halo as stored
//    * SRC/vtk_om.xy.binary.F90:49-87 node velocities and their central
//                                   differences (the vorticity), summed here
//                                   as the enstrophy 0.5 |w|^2 (FP64)
//    * SRC/init.F90:113-201          initial populations: the TGV3D form and
//                                   the default periodic 2-D Taylor-Green form,
//                                   in mykind arithmetic with the reference's
//                                   literals (pi is a default-real constant,
//                                   0.1d0 promotes its products to double),
//                                   shifted storage dropping w (rho - 1)
//                                   (cte1 = 0); next to them the benchmark
//                                   forms (uniform, Taylor-Green and Kida at
//                                   2 pi (i-1)/l, in double, keeping w (rho - 1))
//
//  Storage kinds (kind argument):
//    0  f64 storage, f64 compute      (DOUBLE)
//    1  f32 storage, f32 compute      (SINGLE)
//    2  f16 storage, f32 compute      (MIXED1 analogue: f - w stored as half,
//                                      optionally multiplied by a power-of-two
//                                      scale before rounding)
//    3  bf16 storage, f32 compute     (same, bfloat16)
//    4  f32 storage, f64 compute      (MIXED2)
//  Conversions to 16-bit formats round to nearest even (IEEE default), the
//  same rounding the Fortran assignment and the CUDA __float2half_rn /
//  __float2bfloat16_rn intrinsics use.
//
//  Build: strict IEEE, no contraction (-O2 -ffp-contract=off -fno-fast-math),
//  OpenMP only over independent (k) planes, which does not change any per-node
//  arithmetic.  The obstacle loop always runs serially.
// ============================================================================
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cstdlib>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- 16-bit RNE
inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// binary32 -> binary16, round to nearest even (IEEE 754).
uint16_t float_to_half(float f) {
    uint32_t x = f2u(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) {                       // inf or nan
        if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u | ((ax >> 13) & 0x3ffu));
        return (uint16_t)(sign | 0x7c00u);
    }
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);   // rounds to >= 65520 -> inf
    if (ax < 0x38800000u) {                        // result is subnormal or zero
        if (ax < 0x33000000u) return (uint16_t)sign; // < 2^-25: rounds to zero
        uint32_t e = ax >> 23;                     // biased exponent (102..112)
        uint32_t mant = (ax & 0x7fffffu) | 0x800000u;
        uint32_t shift = 126u - e;                 // 14..24 ; value = mant * 2^(e-150)
        // half subnormal unit = 2^-24 -> q = mant * 2^(e-150+24) = mant >> (126-e)
        uint32_t q = mant >> shift;
        uint32_t rem = mant & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (q & 1u))) q += 1u;
        return (uint16_t)(sign | q);
    }
    // normal range
    uint32_t e = (ax >> 23) - 127u + 15u;
    uint32_t mant = ax & 0x7fffffu;
    uint32_t q = (e << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q += 1u;  // may carry into exponent: fine
    return (uint16_t)(sign | q);
}

float half_to_float(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1fu;
    uint32_t mant = h & 0x3ffu;
    if (e == 0) {
        if (mant == 0) return u2f(sign);
        // subnormal: mant * 2^-24
        float v = (float)mant * 5.9604644775390625e-08f;   // exact
        return sign ? -v : v;
    }
    if (e == 31) return u2f(sign | 0x7f800000u | (mant << 13));
    return u2f(sign | ((e - 15u + 127u) << 23) | (mant << 13));
}

// binary32 -> bfloat16, round to nearest even.
uint16_t float_to_bf16(float f) {
    uint32_t x = f2u(f);
    if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);  // quiet nan
    uint32_t lsb = (x >> 16) & 1u;
    x += 0x7fffu + lsb;
    return (uint16_t)(x >> 16);
}
float bf16_to_float(uint16_t b) { return u2f((uint32_t)b << 16); }

// ------------------------------------------------------------ storage traits
// Store<S,C>: how a storage element S is read into / written from compute C.
template <class S, class C> struct Store;
template <> struct Store<double, double> {
    static double ld(double v, const double&) { return v; }
    static double st(double v, const double&) { return v; }
};
template <> struct Store<float, float> {
    static float ld(float v, const float&) { return v; }
    static float st(float v, const float&) { return v; }
};
template <> struct Store<float, double> {
    static double ld(float v, const double&) { return (double)v; }
    static float st(double v, const double&) { return (float)v; }   // RNE
};
struct Half { uint16_t b; };
struct BF16 { uint16_t b; };
// scale[0] = scale, scale[1] = 1/scale (both powers of two)
template <> struct Store<Half, float> {
    static float ld(Half v, const float* s) { return half_to_float(v.b) * s[1]; }
    static Half st(float v, const float* s) { return Half{float_to_half(v * s[0])}; }
};
template <> struct Store<BF16, float> {
    static float ld(BF16 v, const float* s) { return bf16_to_float(v.b) * s[1]; }
    static BF16 st(float v, const float* s) { return BF16{float_to_bf16(v * s[0])}; }
};

// Uniform accessor: ScaleArg is `const C&` (unused) for native types and
// `const float*` for 16-bit types.
template <class S, class C> struct ScaleArgOf { typedef C type; };
template <> struct ScaleArgOf<Half, float> { typedef const float* type; };
template <> struct ScaleArgOf<BF16, float> { typedef const float* type; };

template <class S, class C> struct Ctx {
    S* a[19];
    long nx, nxy;
    typename ScaleArgOf<S, C>::type sc;
    float scl[2];
    inline long idx(long i, long j, long k) const { return i + nx * j + nxy * k; }
    inline S& at(int p, long i, long j, long k) { return a[p - 1][idx(i, j, k)]; }
    inline C ld(int p, long i, long j, long k) { return Store<S, C>::ld(at(p, i, j, k), sc); }
    inline void st(int p, long i, long j, long k, C v) { at(p, i, j, k) = Store<S, C>::st(v, sc); }
};

template <class S, class C>
void make_ctx(Ctx<S, C>& c, void** a, int nx, int ny, const float* scale);
template <class S, class C>
void make_ctx_common(Ctx<S, C>& c, void** a, int nx, int ny, const float* scale) {
    for (int p = 0; p < 19; ++p) c.a[p] = (S*)a[p];
    c.nx = nx; c.nxy = (long)nx * (long)ny;
    c.scl[0] = scale ? scale[0] : 1.0f;
    c.scl[1] = scale ? scale[1] : 1.0f;
}
template <class S, class C> struct SetSc {
    static void set(Ctx<S, C>& c) { c.sc = C(0); }
};
template <> struct SetSc<Half, float> { static void set(Ctx<Half, float>& c) { c.sc = c.scl; } };
template <> struct SetSc<BF16, float> { static void set(Ctx<BF16, float>& c) { c.sc = c.scl; } };

// Velocity components of populations 01..19 (index 0..18), SRC/alloca.F90:29-148.
inline int cx_tab(int p) {
    static const int t[19] = {1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0};
    return t[p];
}
inline int cy_tab(int p) {
    static const int t[19] = {-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0};
    return t[p];
}
inline int cz_tab(int p) {
    static const int t[19] = {0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0};
    return t[p];
}

// A double rounded to storage kind S the way the library's initial-state
// kernel rounds it: to float first for the 4- and 2-byte kinds, then (16-bit
// kinds) times the power-of-two scale and to nearest even.
template <class S> struct StoreD;
template <> struct StoreD<double> { static double st(double v, const float*) { return v; } };
template <> struct StoreD<float> { static float st(double v, const float*) { return (float)v; } };
template <> struct StoreD<Half> {
    static Half st(double v, const float* s) { return Half{float_to_half((float)v * s[0])}; }
};
template <> struct StoreD<BF16> {
    static BF16 st(double v, const float* s) { return BF16{float_to_bf16((float)v * s[0])}; }
};

// ------------------------------------------------------ boundary conditions
// SRC/bcond.periodic.F90:107-252 (x, then y, then z; full halo ranges)
template <class S, class C>
void bc_periodic(Ctx<S, C>& A, int l, int m, int n) {
    const int l1 = l + 1, m1 = m + 1, n1 = n + 1;
    for (int k = 0; k <= n + 1; ++k)
        for (int j = 0; j <= m + 1; ++j) {
            A.at(1, 0, j, k) = A.at(1, l, j, k);
            A.at(2, 0, j, k) = A.at(2, l, j, k);
            A.at(3, 0, j, k) = A.at(3, l, j, k);
            A.at(4, 0, j, k) = A.at(4, l, j, k);
            A.at(5, 0, j, k) = A.at(5, l, j, k);
            A.at(10, l1, j, k) = A.at(10, 1, j, k);
            A.at(11, l1, j, k) = A.at(11, 1, j, k);
            A.at(12, l1, j, k) = A.at(12, 1, j, k);
            A.at(13, l1, j, k) = A.at(13, 1, j, k);
            A.at(14, l1, j, k) = A.at(14, 1, j, k);
        }
    for (int k = 0; k <= n + 1; ++k)
        for (int i = 0; i <= l + 1; ++i) {
            A.at(3, i, 0, k) = A.at(3, i, m, k);
            A.at(7, i, 0, k) = A.at(7, i, m, k);
            A.at(8, i, 0, k) = A.at(8, i, m, k);
            A.at(9, i, 0, k) = A.at(9, i, m, k);
            A.at(12, i, 0, k) = A.at(12, i, m, k);
            A.at(1, i, m1, k) = A.at(1, i, 1, k);
            A.at(10, i, m1, k) = A.at(10, i, 1, k);
            A.at(16, i, m1, k) = A.at(16, i, 1, k);
            A.at(17, i, m1, k) = A.at(17, i, 1, k);
            A.at(18, i, m1, k) = A.at(18, i, 1, k);
        }
    for (int j = 0; j <= m + 1; ++j)
        for (int i = 0; i <= l + 1; ++i) {
            A.at(4, i, j, 0) = A.at(4, i, j, n);
            A.at(6, i, j, 0) = A.at(6, i, j, n);
            A.at(7, i, j, 0) = A.at(7, i, j, n);
            A.at(13, i, j, 0) = A.at(13, i, j, n);
            A.at(18, i, j, 0) = A.at(18, i, j, n);
            A.at(2, i, j, n1) = A.at(2, i, j, 1);
            A.at(9, i, j, n1) = A.at(9, i, j, 1);
            A.at(11, i, j, n1) = A.at(11, i, j, 1);
            A.at(15, i, j, n1) = A.at(15, i, j, 1);
            A.at(16, i, j, n1) = A.at(16, i, j, 1);
        }
}

// x periodic (SRC/bcond.channel.F90:124-135) + y periodic (:190-201)
template <class S, class C>
void bc_xy_periodic(Ctx<S, C>& A, int l, int m, int n) {
    const int l1 = l + 1, m1 = m + 1;
    for (int k = 0; k <= n + 1; ++k)
        for (int j = 0; j <= m + 1; ++j) {
            A.at(10, l1, j, k) = A.at(10, 1, j, k);
            A.at(11, l1, j, k) = A.at(11, 1, j, k);
            A.at(12, l1, j, k) = A.at(12, 1, j, k);
            A.at(13, l1, j, k) = A.at(13, 1, j, k);
            A.at(14, l1, j, k) = A.at(14, 1, j, k);
            A.at(1, 0, j, k) = A.at(1, l, j, k);
            A.at(2, 0, j, k) = A.at(2, l, j, k);
            A.at(3, 0, j, k) = A.at(3, l, j, k);
            A.at(4, 0, j, k) = A.at(4, l, j, k);
            A.at(5, 0, j, k) = A.at(5, l, j, k);
        }
    for (int k = 0; k <= n + 1; ++k)
        for (int i = 0; i <= l + 1; ++i) {
            A.at(3, i, 0, k) = A.at(3, i, m, k);
            A.at(7, i, 0, k) = A.at(7, i, m, k);
            A.at(8, i, 0, k) = A.at(8, i, m, k);
            A.at(9, i, 0, k) = A.at(9, i, m, k);
            A.at(12, i, 0, k) = A.at(12, i, m, k);
            A.at(1, i, m1, k) = A.at(1, i, 1, k);
            A.at(10, i, m1, k) = A.at(10, i, 1, k);
            A.at(16, i, m1, k) = A.at(16, i, 1, k);
            A.at(17, i, m1, k) = A.at(17, i, 1, k);
            A.at(18, i, m1, k) = A.at(18, i, 1, k);
        }
}

// z no-slip walls, loop over the interior 1..l, 1..m (SRC/bcond.channel.F90:245-267;
// with the lid force: SRC/bcond.driven.F90:236-247)
template <class S, class C>
void bc_z_walls(Ctx<S, C>& A, int l, int m, int n, bool lid, C force) {
    const int n1 = n + 1;
    for (int j = 1; j <= m; ++j)
        for (int i = 1; i <= l; ++i) {
            A.at(6, i, j, 0) = A.at(15, i, j, 1);
            A.at(4, i - 1, j, 0) = A.at(11, i, j, 1);
            A.at(7, i, j - 1, 0) = A.at(16, i, j, 1);
            A.at(13, i + 1, j, 0) = A.at(2, i, j, 1);
            A.at(18, i, j + 1, 0) = A.at(9, i, j, 1);
            A.at(15, i, j, n1) = A.at(6, i, j, n);
            if (lid) A.st(2, i - 1, j, n1, A.ld(13, i, j, n) + force);
            else A.at(2, i - 1, j, n1) = A.at(13, i, j, n);
            A.at(9, i, j - 1, n1) = A.at(18, i, j, n);
            if (lid) A.st(11, i + 1, j, n1, A.ld(4, i, j, n) - force);
            else A.at(11, i + 1, j, n1) = A.at(4, i, j, n);
            A.at(16, i, j + 1, n1) = A.at(7, i, j, n);
        }
}

// SRC/bcond.driven.F90:107-247
template <class S, class C>
void bc_driven(Ctx<S, C>& A, int l, int m, int n, C force) {
    const int l1 = l + 1, m1 = m + 1;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j) {
            A.at(12, l1, j - 1, k) = A.at(1, l, j, k);
            A.at(13, l1, j, k - 1) = A.at(2, l, j, k);
            A.at(10, l1, j + 1, k) = A.at(3, l, j, k);
            A.at(11, l1, j, k + 1) = A.at(4, l, j, k);
            A.at(14, l1, j, k) = A.at(5, l, j, k);
            A.at(3, 0, j - 1, k) = A.at(10, 1, j, k);
            A.at(4, 0, j, k - 1) = A.at(11, 1, j, k);
            A.at(1, 0, j + 1, k) = A.at(12, 1, j, k);
            A.at(2, 0, j, k + 1) = A.at(13, 1, j, k);
            A.at(5, 0, j, k) = A.at(14, 1, j, k);
        }
    for (int k = 1; k <= n; ++k)
        for (int i = 1; i <= l; ++i) {
            A.at(8, i, 0, k) = A.at(17, i, 1, k);
            A.at(12, i + 1, 0, k) = A.at(1, i, 1, k);
            A.at(3, i - 1, 0, k) = A.at(10, i, 1, k);
            A.at(7, i, 0, k - 1) = A.at(16, i, 1, k);
            A.at(9, i, 0, k + 1) = A.at(18, i, 1, k);
            A.at(10, i + 1, m1, k) = A.at(3, i, m, k);
            A.at(16, i, m1, k + 1) = A.at(7, i, m, k);
            A.at(17, i, m1, k) = A.at(8, i, m, k);
            A.at(18, i, m1, k - 1) = A.at(9, i, m, k);
            A.at(1, i - 1, m1, k) = A.at(12, i, m, k);
        }
    bc_z_walls(A, l, m, n, true, force);
}

// SRC/bcond.inflow.F90:131-181 then periodic y (:236-247) and z (:302-313).
// cte1 is the inflow routine's own constant: 0 for shifted storage.
template <class S, class C>
void bc_inflow(Ctx<S, C>& A, int l, int m, int n, C u_inflow, C cte1) {
    const int l1 = l + 1, m1 = m + 1, n1 = n + 1;
    const C rf = C(3), qf = C(1.5), three = C(3);
    const C p1 = (C)(1.0 / 18.0);
    const C p2 = (C)(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
    const C crho = C(1), rhoinv = C(1), zero = C(0);
    for (int k = 0; k <= n + 1; ++k)
        for (int j = 0; j <= m + 1; ++j) {
            C xj = (A.ld(1, l, j, k) + A.ld(2, l, j, k) + A.ld(3, l, j, k) + A.ld(4, l, j, k) +
                    A.ld(5, l, j, k) - A.ld(10, l, j, k) - A.ld(11, l, j, k) - A.ld(12, l, j, k) -
                    A.ld(13, l, j, k) - A.ld(14, l, j, k)) * rhoinv;
            C yj = (A.ld(3, l, j, k) + A.ld(7, l, j, k) + A.ld(8, l, j, k) + A.ld(9, l, j, k) +
                    A.ld(12, l, j, k) - A.ld(1, l, j, k) - A.ld(10, l, j, k) - A.ld(16, l, j, k) -
                    A.ld(17, l, j, k) - A.ld(18, l, j, k)) * rhoinv;
            C zj = (A.ld(4, l, j, k) + A.ld(6, l, j, k) + A.ld(7, l, j, k) + A.ld(13, l, j, k) +
                    A.ld(18, l, j, k) - A.ld(2, l, j, k) - A.ld(9, l, j, k) - A.ld(11, l, j, k) -
                    A.ld(15, l, j, k) - A.ld(16, l, j, k)) * rhoinv;
            C cvsq = xj * xj + yj * yj + zj * zj;
            C cx10 = rf * (-xj - yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
            C cx11 = rf * (-xj - zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
            C cx12 = rf * (-xj + yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
            C cx13 = rf * (-xj + zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
            C cx14 = rf * (-xj) + qf * (three * (xj) * (xj) - cvsq);
            A.st(10, l1, j, k, crho * p2 * (cte1 + cx10));
            A.st(11, l1, j, k, crho * p2 * (cte1 + cx11));
            A.st(12, l1, j, k, crho * p2 * (cte1 + cx12));
            A.st(13, l1, j, k, crho * p2 * (cte1 + cx13));
            A.st(14, l1, j, k, crho * p1 * (cte1 + cx14));
            xj = u_inflow; yj = zero; zj = zero;
            cvsq = xj * xj + yj * yj + zj * zj;
            C cx01 = rf * (xj - yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
            C cx02 = rf * (xj - zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
            C cx03 = rf * (xj + yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
            C cx04 = rf * (xj + zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
            C cx05 = rf * (xj) + qf * (three * (xj) * (xj) - cvsq);
            A.st(1, 0, j, k, crho * p2 * (cte1 + cx01));
            A.st(2, 0, j, k, crho * p2 * (cte1 + cx02));
            A.st(3, 0, j, k, crho * p2 * (cte1 + cx03));
            A.st(4, 0, j, k, crho * p2 * (cte1 + cx04));
            A.st(5, 0, j, k, crho * p1 * (cte1 + cx05));
        }
    for (int k = 0; k <= n + 1; ++k)
        for (int i = 0; i <= l + 1; ++i) {
            A.at(3, i, 0, k) = A.at(3, i, m, k);
            A.at(7, i, 0, k) = A.at(7, i, m, k);
            A.at(8, i, 0, k) = A.at(8, i, m, k);
            A.at(9, i, 0, k) = A.at(9, i, m, k);
            A.at(12, i, 0, k) = A.at(12, i, m, k);
            A.at(1, i, m1, k) = A.at(1, i, 1, k);
            A.at(10, i, m1, k) = A.at(10, i, 1, k);
            A.at(16, i, m1, k) = A.at(16, i, 1, k);
            A.at(17, i, m1, k) = A.at(17, i, 1, k);
            A.at(18, i, m1, k) = A.at(18, i, 1, k);
        }
    for (int j = 0; j <= m + 1; ++j)
        for (int i = 0; i <= l + 1; ++i) {
            A.at(4, i, j, 0) = A.at(4, i, j, n);
            A.at(6, i, j, 0) = A.at(6, i, j, n);
            A.at(7, i, j, 0) = A.at(7, i, j, n);
            A.at(13, i, j, 0) = A.at(13, i, j, n);
            A.at(18, i, j, 0) = A.at(18, i, j, n);
            A.at(2, i, j, n1) = A.at(2, i, j, 1);
            A.at(9, i, j, n1) = A.at(9, i, j, 1);
            A.at(11, i, j, n1) = A.at(11, i, j, 1);
            A.at(15, i, j, n1) = A.at(15, i, j, 1);
            A.at(16, i, j, n1) = A.at(16, i, j, 1);
        }
}

// SRC/bcond.obs.F90:103-122, serial Fortran order (k, j, i).
template <class S, class C>
void bc_obs(Ctx<S, C>& A, const int32_t* obs, int l, int m, int imin, int imax, int jmin,
            int jmax, int kmin, int kmax) {
    for (int k = kmin; k <= kmax; ++k)
        for (int j = jmin; j <= jmax; ++j)
            for (int i = imin; i <= imax; ++i) {
                long o = (long)(i - 1) + (long)l * (j - 1) + (long)l * m * (k - 1);
                if (obs[o] != 1) continue;
                A.at(1, i, j, k) = A.at(12, i + 1, j - 1, k);
                A.at(2, i, j, k) = A.at(13, i + 1, j, k - 1);
                A.at(3, i, j, k) = A.at(10, i + 1, j + 1, k);
                A.at(4, i, j, k) = A.at(11, i + 1, j, k + 1);
                A.at(5, i, j, k) = A.at(14, i + 1, j, k);
                A.at(6, i, j, k) = A.at(15, i, j, k + 1);
                A.at(7, i, j, k) = A.at(16, i, j + 1, k + 1);
                A.at(8, i, j, k) = A.at(17, i, j + 1, k);
                A.at(9, i, j, k) = A.at(18, i, j + 1, k - 1);
                A.at(10, i, j, k) = A.at(3, i - 1, j - 1, k);
                A.at(11, i, j, k) = A.at(4, i - 1, j, k - 1);
                A.at(12, i, j, k) = A.at(1, i - 1, j + 1, k);
                A.at(13, i, j, k) = A.at(2, i - 1, j, k + 1);
                A.at(14, i, j, k) = A.at(5, i - 1, j, k);
                A.at(15, i, j, k) = A.at(6, i, j, k - 1);
                A.at(16, i, j, k) = A.at(7, i, j - 1, k - 1);
                A.at(17, i, j, k) = A.at(8, i, j - 1, k);
                A.at(18, i, j, k) = A.at(9, i, j - 1, k + 1);
            }
}

// --------------------------------------------------------------- collision
// SRC/col_MC.F90:275-519.  force_mode 0: constant forcex/y/z (the native
// C-ABI contract, SRC/col_MC_gpu.hpp:237-255); force_mode 1: forcex = fx*rho
// etc. (the CHANNEL volume force of SRC/col_MC.F90:472-485).
template <class S, class C>
void col_mc(Ctx<S, C>& A, Ctx<S, C>& B, int l, int m, int n, C omega, C cte1, int force_mode,
            C fx, C fy, C fz, int nthreads) {
    const C cte0 = C(1) - cte1;
    const C p0 = (C)(1.0 / 3.0), p1 = (C)(1.0 / 18.0);
    const C p2 = (C)(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
    const C rf = C(3), qf = C(1.5), tre = C(3);
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int k = 1; k <= n; ++k) {
        for (int j = 1; j <= m; ++j) {
            for (int i = 1; i <= l; ++i) {
                const C x01 = A.ld(1, i - 1, j + 1, k);
                const C x02 = A.ld(2, i - 1, j, k + 1);
                const C x03 = A.ld(3, i - 1, j - 1, k);
                const C x04 = A.ld(4, i - 1, j, k - 1);
                const C x05 = A.ld(5, i - 1, j, k);
                const C x06 = A.ld(6, i, j, k - 1);
                const C x07 = A.ld(7, i, j - 1, k - 1);
                const C x08 = A.ld(8, i, j - 1, k);
                const C x09 = A.ld(9, i, j - 1, k + 1);
                const C x10 = A.ld(10, i + 1, j + 1, k);
                const C x11 = A.ld(11, i + 1, j, k + 1);
                const C x12 = A.ld(12, i + 1, j - 1, k);
                const C x13 = A.ld(13, i + 1, j, k - 1);
                const C x14 = A.ld(14, i + 1, j, k);
                const C x15 = A.ld(15, i, j, k + 1);
                const C x16 = A.ld(16, i, j + 1, k + 1);
                const C x17 = A.ld(17, i, j + 1, k);
                const C x18 = A.ld(18, i, j + 1, k - 1);
                const C x19 = A.ld(19, i, j, k);

                const C rho = x01 + x02 + x03 + x04 + x05 + x06 + x07 + x08 + x09 + x10 + x11 +
                              x12 + x13 + x14 + x15 + x16 + x17 + x18 + x19 + cte1;
                const C rhoinv = C(1) / rho;
                C vx = (x01 + x02 + x03 + x04 + x05 - x10 - x11 - x12 - x13 - x14) * rhoinv;
                C vy = (x03 + x07 + x08 + x09 + x12 - x01 - x10 - x16 - x17 - x18) * rhoinv;
                C vz = (x04 + x06 + x07 + x13 + x18 - x02 - x09 - x11 - x15 - x16) * rhoinv;

                const C vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
                const C vsq = vx2 + vy2 + vz2;
                C vxpy = vx + vy;
                const C qxpy = cte0 + qf * (tre * vxpy * vxpy - vsq);
                C vxmy = vx - vy;
                const C qxmy = cte0 + qf * (tre * vxmy * vxmy - vsq);
                C vxpz = vx + vz;
                const C qxpz = cte0 + qf * (tre * vxpz * vxpz - vsq);
                C vxmz = vx - vz;
                const C qxmz = cte0 + qf * (tre * vxmz * vxmz - vsq);
                C vypz = vy + vz;
                const C qypz = cte0 + qf * (tre * vypz * vypz - vsq);
                C vymz = vy - vz;
                const C qymz = cte0 + qf * (tre * vymz * vymz - vsq);
                const C qx = cte0 + qf * (tre * vx2 - vsq);
                const C qy = cte0 + qf * (tre * vy2 - vsq);
                const C qz = cte0 + qf * (tre * vz2 - vsq);
                const C q0 = cte0 + qf * (-vsq);

                vx = rf * vx; vy = rf * vy; vz = rf * vz;
                vxpy = rf * vxpy; vxmy = rf * vxmy; vxpz = rf * vxpz;
                vxmz = rf * vxmz; vypz = rf * vypz; vymz = rf * vymz;

                const C rp0 = rho * p0, rp1 = rho * p1, rp2 = rho * p2;
                const C e01 = rp2 * (+vxmy + qxmy) + cte1 * (rp2 - p2);
                const C e02 = rp2 * (+vxmz + qxmz) + cte1 * (rp2 - p2);
                const C e03 = rp2 * (+vxpy + qxpy) + cte1 * (rp2 - p2);
                const C e04 = rp2 * (+vxpz + qxpz) + cte1 * (rp2 - p2);
                const C e05 = rp1 * (+vx + qx) + cte1 * (rp1 - p1);
                const C e06 = rp1 * (+vz + qz) + cte1 * (rp1 - p1);
                const C e07 = rp2 * (+vypz + qypz) + cte1 * (rp2 - p2);
                const C e08 = rp1 * (+vy + qy) + cte1 * (rp1 - p1);
                const C e09 = rp2 * (+vymz + qymz) + cte1 * (rp2 - p2);
                const C e10 = rp2 * (-vxpy + qxpy) + cte1 * (rp2 - p2);
                const C e11 = rp2 * (-vxpz + qxpz) + cte1 * (rp2 - p2);
                const C e12 = rp2 * (-vxmy + qxmy) + cte1 * (rp2 - p2);
                const C e13 = rp2 * (-vxmz + qxmz) + cte1 * (rp2 - p2);
                const C e14 = rp1 * (-vx + qx) + cte1 * (rp1 - p1);
                const C e15 = rp1 * (-vz + qz) + cte1 * (rp1 - p1);
                const C e16 = rp2 * (-vypz + qypz) + cte1 * (rp2 - p2);
                const C e17 = rp1 * (-vy + qy) + cte1 * (rp1 - p1);
                const C e18 = rp2 * (-vymz + qymz) + cte1 * (rp2 - p2);
                const C e19 = rp0 * (+q0) + cte1 * (rp0 - p0);

                C forcex = fx, forcey = fy, forcez = fz;
                if (force_mode == 1) { forcex = fx * rho; forcey = fy * rho; forcez = fz * rho; }

                B.st(1, i, j, k, x01 - omega * (x01 - e01) + forcex - forcey);
                B.st(2, i, j, k, x02 - omega * (x02 - e02) + forcex - forcez);
                B.st(3, i, j, k, x03 - omega * (x03 - e03) + forcex + forcey);
                B.st(4, i, j, k, x04 - omega * (x04 - e04) + forcex + forcez);
                B.st(5, i, j, k, x05 - omega * (x05 - e05) + forcex);
                B.st(6, i, j, k, x06 - omega * (x06 - e06) + forcez);
                B.st(7, i, j, k, x07 - omega * (x07 - e07) + forcey + forcez);
                B.st(8, i, j, k, x08 - omega * (x08 - e08) + forcey);
                B.st(9, i, j, k, x09 - omega * (x09 - e09) + forcey - forcez);
                B.st(10, i, j, k, x10 - omega * (x10 - e10) - forcex - forcey);
                B.st(11, i, j, k, x11 - omega * (x11 - e11) - forcex - forcez);
                B.st(12, i, j, k, x12 - omega * (x12 - e12) - forcex + forcey);
                B.st(13, i, j, k, x13 - omega * (x13 - e13) - forcex + forcez);
                B.st(14, i, j, k, x14 - omega * (x14 - e14) - forcex);
                B.st(15, i, j, k, x15 - omega * (x15 - e15) - forcez);
                B.st(16, i, j, k, x16 - omega * (x16 - e16) - forcey - forcez);
                B.st(17, i, j, k, x17 - omega * (x17 - e17) - forcey);
                B.st(18, i, j, k, x18 - omega * (x18 - e18) - forcey + forcez);
                A.st(19, i, j, k, x19 - omega * (x19 - e19));
            }
        }
    }
}

// ------------------------------------------------------------- diagnostics
// SRC/diagno.F90:87-132: per-node rho and u in the compute type, sums in FP64.
// obs (optional): nodes with obs==1 are skipped.  out = {sum rho, sum ux,
// sum uy, sum uz, sum 0.5|u|^2}.
template <class S, class C>
void diagno(Ctx<S, C>& A, int l, int m, int n, const int32_t* obs, C cte1, double* out) {
    double rtot = 0, xtot = 0, ytot = 0, ztot = 0, stot = 0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                if (obs && obs[(long)(i - 1) + (long)l * (j - 1) + (long)l * m * (k - 1)] == 1) continue;
                C x[19];
                for (int p = 0; p < 19; ++p) x[p] = A.ld(p + 1, i, j, k);
                const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] +
                              x[10] + x[11] + x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + cte1;
                const C rhoinv = C(1) / rho;
                const C xj = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
                const C yj = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
                const C zj = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
                rtot += (double)rho;
                xtot += (double)xj;
                ytot += (double)yj;
                ztot += (double)zj;
                stot += (double)(C(0.5) * (xj * xj + yj * yj + zj * zj));
            }
    out[0] = rtot; out[1] = xtot; out[2] = ytot; out[3] = ztot; out[4] = stot;
}

// SRC/draglift.F90:77-176: out = {Fx, Fy, Fz} (unnormalised), FP64 sums of
// the per-node mykind terms 2*c_a*a_p(x)*obs(x+c_p) over fluid nodes in the box.
template <class S, class C>
void draglift(Ctx<S, C>& A, const int32_t* obs, int l, int m, int n, int is, int ie, int js,
              int je, int ks, int ke, double* out) {
    static const int cx[18] = {1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0};
    static const int cy[18] = {-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1};
    static const int cz[18] = {0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1};
    auto O = [&](int i, int j, int k) -> int {
        if (i < 1 || i > l || j < 1 || j > m || k < 1 || k > n) return 0;
        return obs[(long)(i - 1) + (long)l * (j - 1) + (long)l * m * (k - 1)];
    };
    double F[3] = {0, 0, 0};
    for (int ax = 0; ax < 3; ++ax) {
        const int* cc = ax == 0 ? cx : (ax == 1 ? cy : cz);
        for (int k = ks; k <= ke; ++k)
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i) {
                    if (O(i, j, k) != 0) continue;
                    C s = C(0);
                    for (int p = 0; p < 18; ++p) {
                        const C term = C(2.0) * (C)cc[p] * A.ld(p + 1, i, j, k) *
                                       (C)O(i + cx[p], j + cy[p], k + cz[p]);
                        s = (p == 0) ? term : s + term;
                    }
                    F[ax] += (double)s;
                }
    }
    out[0] = F[0]; out[1] = F[1]; out[2] = F[2];
}

// SRC/dissipation.F90:136-338 over fluid nodes (obs == 1 skipped): each
// population pulled from its upstream neighbour as stored (the caller fills
// the halo first, as the reference's boundary routines do), rho and u, the
// generic equilibrium e_p, n_p = x_p - e_p, the stress components and
// Ptotal, all in the compute type in source order.  out = {sum 0.5*vsq,
// sum 2*svisc*Ptotal, sum vx2, sum vy2, sum vz2} (FP64 sums).
template <class S, class C>
void dissipation(Ctx<S, C>& A, int l, int m, int n, const int32_t* obs, C svisc, C cte0, C cte1, C p0, C p1, C p2,
                 C rf, C qf, C tre, double* out) {
    const C due = C(2);
    double diss = 0, tke = 0, vx2m = 0, vy2m = 0, vz2m = 0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                if (obs && obs[(long)(i - 1) + (long)l * (j - 1) + (long)l * m * (k - 1)] == 1) continue;
                const C x01 = A.ld(1, i - 1, j + 1, k);
                const C x02 = A.ld(2, i - 1, j, k + 1);
                const C x03 = A.ld(3, i - 1, j - 1, k);
                const C x04 = A.ld(4, i - 1, j, k - 1);
                const C x05 = A.ld(5, i - 1, j, k);
                const C x06 = A.ld(6, i, j, k - 1);
                const C x07 = A.ld(7, i, j - 1, k - 1);
                const C x08 = A.ld(8, i, j - 1, k);
                const C x09 = A.ld(9, i, j - 1, k + 1);
                const C x10 = A.ld(10, i + 1, j + 1, k);
                const C x11 = A.ld(11, i + 1, j, k + 1);
                const C x12 = A.ld(12, i + 1, j - 1, k);
                const C x13 = A.ld(13, i + 1, j, k - 1);
                const C x14 = A.ld(14, i + 1, j, k);
                const C x15 = A.ld(15, i, j, k + 1);
                const C x16 = A.ld(16, i, j + 1, k + 1);
                const C x17 = A.ld(17, i, j + 1, k);
                const C x18 = A.ld(18, i, j + 1, k - 1);
                const C x19 = A.ld(19, i, j, k);
                const C rho = x01 + x02 + x03 + x04 + x05 + x06 + x07 + x08 + x09 + x10 + x11 + x12 + x13 + x14 +
                              x15 + x16 + x17 + x18 + x19 + cte1;
                const C rhoinv = C(1) / rho;
                C vx = (x01 + x02 + x03 + x04 + x05 - x10 - x11 - x12 - x13 - x14) * rhoinv;
                C vy = (x03 + x07 + x08 + x09 + x12 - x01 - x10 - x16 - x17 - x18) * rhoinv;
                C vz = (x04 + x06 + x07 + x13 + x18 - x02 - x09 - x11 - x15 - x16) * rhoinv;
                const C vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
                vx2m += (double)vx2;
                vy2m += (double)vy2;
                vz2m += (double)vz2;
                const C vsq = vx2 + vy2 + vz2;
                tke += (double)(C(0.5) * vsq);
                C vxpy = vx + vy;
                const C qxpy = cte0 + qf * (tre * vxpy * vxpy - vsq);
                C vxmy = vx - vy;
                const C qxmy = cte0 + qf * (tre * vxmy * vxmy - vsq);
                C vxpz = vx + vz;
                const C qxpz = cte0 + qf * (tre * vxpz * vxpz - vsq);
                C vxmz = vx - vz;
                const C qxmz = cte0 + qf * (tre * vxmz * vxmz - vsq);
                C vypz = vy + vz;
                const C qypz = cte0 + qf * (tre * vypz * vypz - vsq);
                C vymz = vy - vz;
                const C qymz = cte0 + qf * (tre * vymz * vymz - vsq);
                const C qx = cte0 + qf * (tre * vx2 - vsq);
                const C qy = cte0 + qf * (tre * vy2 - vsq);
                const C qz = cte0 + qf * (tre * vz2 - vsq);
                vx = rf * vx; vy = rf * vy; vz = rf * vz;
                vxpy = rf * vxpy; vxmy = rf * vxmy; vxpz = rf * vxpz;
                vxmz = rf * vxmz; vypz = rf * vypz; vymz = rf * vymz;
                const C rp1 = rho * p1, rp2 = rho * p2;
                (void)p0;   // e19 enters no stress component
                const C e01 = rp2 * (+vxmy + qxmy) + cte1 * (rp2 - p2);
                const C e02 = rp2 * (+vxmz + qxmz) + cte1 * (rp2 - p2);
                const C e03 = rp2 * (+vxpy + qxpy) + cte1 * (rp2 - p2);
                const C e04 = rp2 * (+vxpz + qxpz) + cte1 * (rp2 - p2);
                const C e05 = rp1 * (+vx + qx) + cte1 * (rp1 - p1);
                const C e06 = rp1 * (+vz + qz) + cte1 * (rp1 - p1);
                const C e07 = rp2 * (+vypz + qypz) + cte1 * (rp2 - p2);
                const C e08 = rp1 * (+vy + qy) + cte1 * (rp1 - p1);
                const C e09 = rp2 * (+vymz + qymz) + cte1 * (rp2 - p2);
                const C e10 = rp2 * (-vxpy + qxpy) + cte1 * (rp2 - p2);
                const C e11 = rp2 * (-vxpz + qxpz) + cte1 * (rp2 - p2);
                const C e12 = rp2 * (-vxmy + qxmy) + cte1 * (rp2 - p2);
                const C e13 = rp2 * (-vxmz + qxmz) + cte1 * (rp2 - p2);
                const C e14 = rp1 * (-vx + qx) + cte1 * (rp1 - p1);
                const C e15 = rp1 * (-vz + qz) + cte1 * (rp1 - p1);
                const C e16 = rp2 * (-vypz + qypz) + cte1 * (rp2 - p2);
                const C e17 = rp1 * (-vy + qy) + cte1 * (rp1 - p1);
                const C e18 = rp2 * (-vymz + qymz) + cte1 * (rp2 - p2);
                const C n01 = x01 - e01, n02 = x02 - e02, n03 = x03 - e03, n04 = x04 - e04, n05 = x05 - e05;
                const C n06 = x06 - e06, n07 = x07 - e07, n08 = x08 - e08, n09 = x09 - e09, n10 = x10 - e10;
                const C n11 = x11 - e11, n12 = x12 - e12, n13 = x13 - e13, n14 = x14 - e14, n15 = x15 - e15;
                const C n16 = x16 - e16, n17 = x17 - e17, n18 = x18 - e18;
                const C Pxx = n01 + n02 + n03 + n04 + n05 + n10 + n11 + n12 + n13 + n14;
                const C Pyy = n01 + n03 + n07 + n08 + n09 + n10 + n12 + n16 + n17 + n18;
                const C Pzz = n02 + n04 + n06 + n07 + n09 + n11 + n13 + n15 + n16 + n18;
                const C Pxz = -n02 + n04 + n11 - n13;
                const C Pxy = -n01 + n03 + n10 - n12;
                const C Pyz = +n07 - n09 + n16 - n18;
                const C Pyx = Pxy, Pzx = Pxz, Pzy = Pyz;
                const C Ptotal = (Pxx * Pxx) + (Pyy * Pyy) + (Pzz * Pzz) + (due * Pxy * Pyx) + (due * Pxz * Pzx) +
                                 (due * Pyz * Pzy);
                diss += (double)(due * svisc * Ptotal);
            }
    out[0] = tke; out[1] = diss; out[2] = vx2m; out[3] = vy2m; out[4] = vz2m;
}

// Enstrophy: node velocities of the stored state as SRC/vtk_om.xy.binary.F90
// :49-55 computes them (here in the compute type), central differences
// du_a/dx_b = 0.5 (u_a(x + e_b) - u_a(x - e_b)) as :79-84, w = curl u as
// :85-87, and the FP64 sum of 0.5 |w|^2.  Periodic axes (px, py, pz) wrap;
// along other axes the two face layers are left out; with obs, nodes that
// are solid or have a solid neighbour are left out.  out = {sum, nodes}.
template <class S, class C>
void enstrophy(Ctx<S, C>& A, int l, int m, int n, const int32_t* obs, C cte1, bool px, bool py, bool pz,
               double* out) {
    const long nn = (long)l * m * n;
    std::vector<C> u(nn), v(nn), w(nn);
    auto at = [&](int i, int j, int k) -> long { return (long)(i - 1) + (long)l * (j - 1) + (long)l * m * (k - 1); };
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                C x[19];
                for (int p = 0; p < 19; ++p) x[p] = A.ld(p + 1, i, j, k);
                const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] + x[11] +
                              x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + cte1;
                const C rhoinv = C(1) / rho;
                u[at(i, j, k)] = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
                v[at(i, j, k)] = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
                w[at(i, j, k)] = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
            }
    auto wrap = [](int c, int len) { return c < 1 ? c + len : (c > len ? c - len : c); };
    auto solid = [&](int i, int j, int k) { return obs && obs[at(i, j, k)] == 1; };
    double sum = 0, cnt = 0;
    const C h = C(0.5);
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                if (!px && (i < 2 || i > l - 1)) continue;
                if (!py && (j < 2 || j > m - 1)) continue;
                if (!pz && (k < 2 || k > n - 1)) continue;
                const int im = wrap(i - 1, l), ip = wrap(i + 1, l), jm = wrap(j - 1, m), jp = wrap(j + 1, m);
                const int km = wrap(k - 1, n), kp = wrap(k + 1, n);
                if (solid(i, j, k) || solid(im, j, k) || solid(ip, j, k) || solid(i, jm, k) || solid(i, jp, k) ||
                    solid(i, j, km) || solid(i, j, kp))
                    continue;
                const C dudy = h * (u[at(i, jp, k)] - u[at(i, jm, k)]);
                const C dudz = h * (u[at(i, j, kp)] - u[at(i, j, km)]);
                const C dvdx = h * (v[at(ip, j, k)] - v[at(im, j, k)]);
                const C dvdz = h * (v[at(i, j, kp)] - v[at(i, j, km)]);
                const C dwdx = h * (w[at(ip, j, k)] - w[at(im, j, k)]);
                const C dwdy = h * (w[at(i, jp, k)] - w[at(i, jm, k)]);
                const C ox = dvdz - dwdy, oy = dwdx - dudz, oz = dudy - dvdx;
                sum += (double)(h * (ox * ox + oy * oy + oz * oz));
                cnt += 1.0;
            }
    out[0] = sum; out[1] = cnt;
}

// ------------------------------------------------------- initial state
// Sine and cosine of the compute type as the reference calls them (sin/cos
// of real(8); for real(4) the correctly rounded single-precision value --
// libm's sinf/cosf, which the reference calls, agree with it except in rare
// last-bit cases).
inline float rsin(float a) { return (float)std::sin((double)a); }
inline double rsin(double a) { return std::sin(a); }
inline float rcos(float a) { return (float)std::cos((double)a); }
inline double rcos(double a) { return std::cos(a); }

// The 19 reference populations of SRC/init.F90:158-197 from (crho, xj, yj,
// zj) in the compute type, with cte1 = 0 (shifted storage: no NOSHIFT):
// f_p = crho * w_p * (cte1 + cx_p).
template <class C>
void init_pops_reference(C crho, C xj, C yj, C zj, C rf, C qf, C tre, C p0, C p1, C p2, C (&f)[19]) {
    const C cte1 = C(0);
    const C cvsq = xj * xj + yj * yj + zj * zj;
    const C cx01 = rf * (xj - yj) + qf * (tre * (xj - yj) * (xj - yj) - cvsq);
    const C cx02 = rf * (xj - zj) + qf * (tre * (xj - zj) * (xj - zj) - cvsq);
    const C cx03 = rf * (xj + yj) + qf * (tre * (xj + yj) * (xj + yj) - cvsq);
    const C cx04 = rf * (xj + zj) + qf * (tre * (xj + zj) * (xj + zj) - cvsq);
    const C cx05 = rf * (xj) + qf * (tre * (xj) * (xj) - cvsq);
    const C cx06 = rf * (zj) + qf * (tre * (zj) * (zj) - cvsq);
    const C cx07 = rf * (yj + zj) + qf * (tre * (yj + zj) * (yj + zj) - cvsq);
    const C cx08 = rf * (yj) + qf * (tre * (yj) * (yj) - cvsq);
    const C cx09 = rf * (yj - zj) + qf * (tre * (yj - zj) * (yj - zj) - cvsq);
    const C cx10 = rf * (-xj - yj) + qf * (tre * (xj + yj) * (xj + yj) - cvsq);
    const C cx11 = rf * (-xj - zj) + qf * (tre * (xj + zj) * (xj + zj) - cvsq);
    const C cx12 = rf * (-xj + yj) + qf * (tre * (xj - yj) * (xj - yj) - cvsq);
    const C cx13 = rf * (-xj + zj) + qf * (tre * (xj - zj) * (xj - zj) - cvsq);
    const C cx14 = rf * (-xj) + qf * (tre * (xj) * (xj) - cvsq);
    const C cx15 = rf * (-zj) + qf * (tre * (zj) * (zj) - cvsq);
    const C cx16 = rf * (-yj - zj) + qf * (tre * (yj + zj) * (yj + zj) - cvsq);
    const C cx17 = rf * (-yj) + qf * (tre * (yj) * (yj) - cvsq);
    const C cx18 = rf * (-yj + zj) + qf * (tre * (yj - zj) * (yj - zj) - cvsq);
    const C cx19 = rf * C(0) + qf * (tre * C(0) * C(0) - cvsq);
    const C cx[19] = {cx01, cx02, cx03, cx04, cx05, cx06, cx07, cx08, cx09, cx10,
                      cx11, cx12, cx13, cx14, cx15, cx16, cx17, cx18, cx19};
    for (int p = 0; p < 19; ++p) {
        const int ax = std::abs(cx_tab(p)) + std::abs(cy_tab(p)) + std::abs(cz_tab(p));
        const C w = ax == 0 ? p0 : (ax == 1 ? p1 : p2);
        f[p] = crho * w * (cte1 + cx[p]);
    }
}

// flow 0 uniform (prm = rho, ux, uy, uz), 1 Taylor-Green and 2 Kida at
// x = 2 pi (i-1)/l (prm[0] = u0): w (rho - 1) + w rho (3 c.u + 4.5 (c.u)^2 -
// 1.5 u^2) in double, rounded once to the storage kind.  flow 3: the
// reference's TGV3D form (SRC/init.F90:119-158, prm[0] = u00), flow 4: its
// default periodic 2-D Taylor-Green form (:125-130): x = (i - 0.5)/l in
// double rounded to mykind, the rest in mykind.  Every node of the box
// 0..l+1, 0..m+1, 0..n+1 is written.
template <class S, class C>
void init_state(Ctx<S, C>& A, int l, int m, int n, int flow, const double* prm, C rf, C qf, C tre, C p0, C p1,
                C p2) {
    const double tp = 6.283185307179586476925286766559;
    const C pi = C(3.14159265358979323846f);   // a default-real literal (SRC/init.F90:63)
    for (int k = 0; k <= n + 1; ++k)
        for (int j = 0; j <= m + 1; ++j)
            for (int i = 0; i <= l + 1; ++i) {
                if (flow <= 2) {
                    double rho = 1.0, ux = 0.0, uy = 0.0, uz = 0.0;
                    if (flow == 0) {
                        rho = prm[0]; ux = prm[1]; uy = prm[2]; uz = prm[3];
                    } else {
                        const double x = tp * (i - 1) / l, y = tp * (j - 1) / m, z = tp * (k - 1) / n;
                        const double u0 = prm[0];
                        if (flow == 1) {
                            ux = u0 * std::sin(x) * std::cos(y) * std::cos(z);
                            uy = -u0 * std::cos(x) * std::sin(y) * std::cos(z);
                            rho = 1.0 + 3.0 * (u0 * u0 / 16.0) * (std::cos(2.0 * x) + std::cos(2.0 * y)) *
                                            (std::cos(2.0 * z) + 2.0);
                        } else {
                            ux = u0 * std::sin(x) * (std::cos(3.0 * y) * std::cos(z) - std::cos(y) * std::cos(3.0 * z));
                            uy = u0 * std::sin(y) * (std::cos(3.0 * z) * std::cos(x) - std::cos(z) * std::cos(3.0 * x));
                            uz = u0 * std::sin(z) * (std::cos(3.0 * x) * std::cos(y) - std::cos(x) * std::cos(3.0 * y));
                        }
                    }
                    const double usq = ux * ux + uy * uy + uz * uz;
                    for (int p = 0; p < 19; ++p) {
                        const double cu = cx_tab(p) * ux + cy_tab(p) * uy + cz_tab(p) * uz;
                        const int ax = std::abs(cx_tab(p)) + std::abs(cy_tab(p)) + std::abs(cz_tab(p));
                        const double w = ax == 2 ? 1.0 / 36.0 : (ax == 1 ? 1.0 / 18.0 : 1.0 / 3.0);
                        const double v = w * (rho - 1.0) + w * rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
                        A.at(p + 1, i, j, k) = StoreD<S>::st(v, A.scl);
                    }
                    continue;
                }
                const C x = (C)(((double)i - 0.5) / (double)l);
                const C y = (C)(((double)j - 0.5) / (double)m);
                const C z = (C)(((double)k - 0.5) / (double)n);
                C xj, yj, zj, crho = C(1);
                if (flow == 3) {
                    const C u00 = (C)prm[0], due = C(2), qua = C(4);
                    xj = u00 * rsin(due * pi * x) * rcos(due * pi * y) * rcos(due * pi * z);
                    yj = -(u00 * rcos(due * pi * x) * rsin(due * pi * y) * rcos(due * pi * z));
                    zj = C(0);
                    crho = C(1) + ((u00 * u00) / (qua * qua * tre)) * (rcos(qua * pi * x) + rcos(qua * pi * y)) *
                                      (rcos(qua * pi * z) + due);
                } else {
                    const C two = C(2);
                    xj = (C)(0.1 * (double)rsin(two * pi * x) * (double)rcos(two * pi * z));
                    yj = C(0);
                    zj = (C)(-(0.1 * (double)rcos(two * pi * x) * (double)rsin(two * pi * z)));
                }
                C f[19];
                init_pops_reference<C>(crho, xj, yj, zj, rf, qf, tre, p0, p1, p2, f);
                for (int p = 0; p < 19; ++p) A.st(p + 1, i, j, k, f[p]);
            }
}

// ------------------------------------------------- profiles, probe, slices
// The storage arithmetic: the reference sums the storage arrays directly in
// these routines, so the arithmetic is the storage kind's (float for the
// 4-byte and, here, the 16-bit kinds, whose values are unscaled first).
template <class S> struct ArithOf { typedef float type; };
template <> struct ArithOf<double> { typedef double type; };

// SRC/prof_k.F90:47-77 (SRC/prof_i.F90:48-77, SRC/prof_j.F90:48-77 likewise):
// den = a01+...+a19 (storage arithmetic) + cte1 (compute type), u = (x
// momentum sum, storage arithmetic) / den in the compute type.  axis 0 runs
// i at (j, k) = (c1, c2), axis 1 runs j at (i, k) = (c1, c2), axis 2 runs k
// at (i, j) = (c1, c2).  out: 4 values per node (u_x, u_y, u_z, rho).
template <class S, class C>
void profile(Ctx<S, C>& A, int axis, int c1, int c2, int len, C cte1, double* out) {
    typedef typename ArithOf<S>::type R;
    for (int t = 1; t <= len; ++t) {
        const int i = axis == 0 ? t : c1, j = axis == 1 ? t : (axis == 0 ? c1 : c2), k = axis == 2 ? t : c2;
        R x[19];
        for (int p = 0; p < 19; ++p) x[p] = (R)A.ld(p + 1, i, j, k);
        const R s = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] + x[11] +
                    x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18];
        const C den = (C)s + cte1;
        const R sx = x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13];
        const R sy = x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17];
        const R sz = x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15];
        double* o = out + 4 * (long)(t - 1);
        o[0] = (double)((C)sx / den); o[1] = (double)((C)sy / den); o[2] = (double)((C)sz / den);
        o[3] = (double)den;
    }
}

// SRC/probe.F90:50-78: populations copied into compute-type variables first,
// rho and the momentum summed in the compute type.  out = (u_x, u_y, u_z, rho).
template <class S, class C>
void probe(Ctx<S, C>& A, int i, int j, int k, C cte1, double* out) {
    C x[19];
    for (int p = 0; p < 19; ++p) x[p] = A.ld(p + 1, i, j, k);
    const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] + x[11] + x[12] +
                  x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + cte1;
    const C xj = x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13];
    const C yj = x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17];
    const C zj = x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15];
    out[0] = (double)(xj / rho); out[1] = (double)(yj / rho); out[2] = (double)(zj / rho); out[3] = (double)rho;
}

// SRC/vtk_xy.binary.F90:78-97 (vtk_xz / vtk_yz likewise): u, den in single
// precision -- each sum in the storage arithmetic (den with cte1 = 1.0),
// rounded to float -- and u/den in float.  plane 0: xy at k = index (j, i
// loops), 1: xz at j = index (k, i), 2: yz at i = index (k, j); out: 3
// floats per node, inner index fastest.
template <class S, class C>
void slice(Ctx<S, C>& A, int plane, int index, int l, int m, int n, float* out) {
    typedef typename ArithOf<S>::type R;
    const int n1 = plane == 2 ? m : l, n2 = plane == 0 ? m : n;
    long o = 0;
    for (int b = 1; b <= n2; ++b)
        for (int a = 1; a <= n1; ++a) {
            const int i = plane == 2 ? index : a;
            const int j = plane == 0 ? b : (plane == 1 ? index : a);
            const int k = plane == 0 ? index : b;
            R x[19];
            for (int p = 0; p < 19; ++p) x[p] = (R)A.ld(p + 1, i, j, k);
            const float u = (float)(x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]);
            const float w = (float)(x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]);
            const float v = (float)(x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]);
            const float den = (float)(x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] +
                                      x[11] + x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + (R)1.0);
            out[o++] = u / den; out[o++] = w / den; out[o++] = v / den;
        }
}

template <class S, class C>
void make(Ctx<S, C>& c, void** a, int nx, int ny, const float* scale) {
    make_ctx_common(c, a, nx, ny, scale);
    SetSc<S, C>::set(c);
}

}  // namespace

// ============================================================== extern "C"
#define DISPATCH(kind, ...)                                                      \
    switch (kind) {                                                              \
    case 0: { typedef double S; typedef double C; __VA_ARGS__ } break;           \
    case 1: { typedef float S; typedef float C; __VA_ARGS__ } break;             \
    case 2: { typedef Half S; typedef float C; __VA_ARGS__ } break;              \
    case 3: { typedef BF16 S; typedef float C; __VA_ARGS__ } break;              \
    case 4: { typedef float S; typedef double C; __VA_ARGS__ } break;            \
    default: return -1;                                                          \
    }

extern "C" {

int orc_bcond(int kind, int bcase, void** a, int l, int m, int n, int nx, int ny,
              double force, double u_inflow, double inflow_cte1, const float* scale) {
    // bcase: 0 driven, 1 periodic, 2 channel, 3 inflow
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        if (bcase == 0) bc_driven(A, l, m, n, (C)force);
        else if (bcase == 1) bc_periodic(A, l, m, n);
        else if (bcase == 2) { bc_xy_periodic(A, l, m, n); bc_z_walls(A, l, m, n, false, C(0)); }
        else if (bcase == 3) bc_inflow(A, l, m, n, (C)u_inflow, (C)inflow_cte1);
        else return -2;
    });
    return 0;
}

int orc_bcond_obs(int kind, void** a, const int32_t* obs, int l, int m, int n, int nx, int ny,
                  int imin, int imax, int jmin, int jmax, int kmin, int kmax, const float* scale) {
    (void)n;
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        bc_obs(A, obs, l, m, imin, imax, jmin, jmax, kmin, kmax);
    });
    return 0;
}

int orc_col_mc(int kind, void** a, void** b, int l, int m, int n, int nx, int ny, double omega,
               double cte1, int force_mode, double fx, double fy, double fz, const float* scale,
               int nthreads) {
    if (nthreads < 1) nthreads = 1;
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        Ctx<S, C> B; make(B, b, nx, ny, scale);
        col_mc(A, B, l, m, n, (C)omega, (C)cte1, force_mode, (C)fx, (C)fy, (C)fz, nthreads);
    });
    return 0;
}

int orc_diagno(int kind, void** a, int l, int m, int n, int nx, int ny, const int32_t* obs,
               double cte1, const float* scale, double* out) {
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        diagno(A, l, m, n, obs, (C)cte1, out);
    });
    return 0;
}

int orc_draglift(int kind, void** a, const int32_t* obs, int l, int m, int n, int nx, int ny,
                 int is, int ie, int js, int je, int ks, int ke, const float* scale, double* out) {
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        draglift(A, obs, l, m, n, is, ie, js, je, ks, ke, out);
    });
    return 0;
}

int orc_profile(int kind, void** a, int l, int m, int n, int nx, int ny, int axis, int c1, int c2,
                double cte1, const float* scale, double* out) {
    const int len = axis == 0 ? l : (axis == 1 ? m : n);
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        profile(A, axis, c1, c2, len, (C)cte1, out);
    });
    return 0;
}

int orc_probe(int kind, void** a, int nx, int ny, int i, int j, int k, double cte1, const float* scale,
              double* out) {
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        probe(A, i, j, k, (C)cte1, out);
    });
    return 0;
}

int orc_slice(int kind, void** a, int l, int m, int n, int nx, int ny, int plane, int index,
              const float* scale, float* out) {
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        slice(A, plane, index, l, m, n, out);
    });
    return 0;
}

// out[0..4]: dissipation sums (see dissipation above); the halo as stored.
int orc_dissipation(int kind, void** a, int l, int m, int n, int nx, int ny, const int32_t* obs, double svisc,
                    double cte0, double cte1, double p0, double p1, double p2, double rf, double qf, double tre,
                    const float* scale, double* out) {
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        dissipation(A, l, m, n, obs, (C)svisc, (C)cte0, (C)cte1, (C)p0, (C)p1, (C)p2, (C)rf, (C)qf, (C)tre, out);
    });
    return 0;
}

// out[0..1]: enstrophy sum and node count; periodic: bit 0 x, bit 1 y, bit 2 z.
int orc_enstrophy(int kind, void** a, int l, int m, int n, int nx, int ny, const int32_t* obs, double cte1,
                  int periodic, const float* scale, double* out) {
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        enstrophy(A, l, m, n, obs, (C)cte1, (periodic & 1) != 0, (periodic & 2) != 0, (periodic & 4) != 0, out);
    });
    return 0;
}

// The initial state of `flow` (see init_state) over the whole box.
int orc_init(int kind, void** a, int l, int m, int n, int nx, int ny, int flow, const double* prm, double rf,
             double qf, double tre, double p0, double p1, double p2, const float* scale) {
    if (flow < 0 || flow > 4) return -2;
    DISPATCH(kind, {
        Ctx<S, C> A; make(A, a, nx, ny, scale);
        init_state(A, l, m, n, flow, prm, (C)rf, (C)qf, (C)tre, (C)p0, (C)p1, (C)p2);
    });
    return 0;
}

// 16-bit conversions exposed for tests of the oracle itself.
uint16_t orc_float_to_half(float f) { return float_to_half(f); }
float orc_half_to_float(uint16_t h) { return half_to_float(h); }
uint16_t orc_float_to_bf16(float f) { return float_to_bf16(f); }
float orc_bf16_to_float(uint16_t b) { return bf16_to_float(b); }

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
