// Host-side construction of kernel arguments, shared by the library's
// translation units (typed ABI and library-owned lattices).
#pragma once
#include <cmath>
#include <cstdint>
#include "bgk3d_b200.h"
#include "bgk_internal.h"
#include "sweep_ab.cuh"
#include "reduce.cuh"

namespace bgk {

// Storage scale of the 16-bit kinds (1 otherwise).
inline double storage_scale(const bgk_sweep_params* p) {
    return (p->kind == K_F16 || p->kind == K_BF16) ? (double)p->scale : 1.0;
}

// Collision constants in the compute type; with sc != 1 the weights and the
// forces are in storage units.  Each constant is rounded to C first and then
// scaled (exact for power-of-two scales), so the products equal the
// physical constants times the scale.
template <class C>
ColConst<C> col_const(const bgk_sweep_params* p, double sc = 1.0) {
    ColConst<C> k;
    k.omega = (C)p->omega; k.cte0 = (C)p->cte0; k.cte1 = (C)p->cte1;
    k.p0 = (C)p->p0 * (C)sc; k.p1 = (C)p->p1 * (C)sc; k.p2 = (C)p->p2 * (C)sc;
    k.rf = (C)p->rf; k.qf = (C)p->qf; k.tre = (C)p->tre;
    k.force_mode = p->force_mode;
    k.fx = (C)p->fx * (C)sc; k.fy = (C)p->fy * (C)sc; k.fz = (C)p->fz * (C)sc;
    return k;
}

// v rounded to `bits` significant bits.
inline double round_to_bits(double v, int bits) {
    int e;
    const double m = std::frexp(v, &e);
    return std::ldexp(std::nearbyint(std::ldexp(m, bits)), e - bits);
}

// Constants of the fused-multiply-add collision (d3q19.cuh), in storage units.
// Momentum is conserved only if (1 - omega) + (2 r1 + 8 r2) = 1 in the
// arithmetic that runs: rounded independently, the two parts miss 1 by a few
// 1e-8, and the momentum drifts by that factor every step (measured: 4e-5
// kinetic-energy error after 400 steps).  So r2 is rounded to two bits fewer
// than C holds, r1 = 2 r2 (p1 = 2 p2), 2 r1 + 8 r2 = 12 r2 and 1 - 12 r2 are
// then exact in C, and the other constants use that omega' = 12 r2 / rf / 3.
template <class C>
FastConst<C> fast_const(const bgk_sweep_params* p, double sc) {
    FastConst<C> f;
    const int bits = sizeof(C) == 4 ? 22 : 51;
    const double k2 = round_to_bits(p->omega * p->rf * p->p2, bits);
    const double k1 = (p->p1 == 2.0 * p->p2) ? 2.0 * k2 : round_to_bits(p->omega * p->rf * p->p1, bits);
    const double om = 2.0 * k1 + 8.0 * k2;   // omega' (= omega (1 + O(1e-7)) for the reference weights)
    f.omc = (C)(1.0 - om);
    f.r1 = (C)(k1 * sc);
    f.r2 = (C)(k2 * sc);
    f.a1 = (C)(om * p->qf * p->tre * p->p1 * sc);
    f.a2 = (C)(om * p->qf * p->tre * p->p2 * sc);
    f.b0 = (C)(om * p->p0 * sc);
    f.b1 = (C)(om * p->p1 * sc);
    f.b2 = (C)(om * p->p2 * sc);
    f.qf = (C)p->qf; f.cte0 = (C)p->cte0; f.cte1 = (C)p->cte1;
    f.force_mode = p->force_mode;
    f.fx = (C)(p->fx * sc); f.fy = (C)(p->fy * sc); f.fz = (C)(p->fz * sc);
    return f;
}

// A compute value rounded to storage kind S on the host, as Conv<S, C>::pack
// rounds it on the device (round to nearest even).
template <class S, class C> inline S host_pack(C v);
template <> inline double host_pack<double, double>(double v) { return v; }
template <> inline float host_pack<float, float>(float v) { return v; }
template <> inline float host_pack<float, double>(double v) { return (float)v; }
template <> inline __half host_pack<__half, float>(float v) { return __float2half_rn(v); }
template <> inline __nv_bfloat16 host_pack<__nv_bfloat16, float>(float v) { return __float2bfloat16_rn(v); }

template <class S, class C>
SweepArgs<S, C> sweep_args(const bgk_sweep_params* p, void* const* a, void* const* b) {
    SweepArgs<S, C> A;
    for (int d = 0; d < 19; ++d) {
        A.a[d] = (const S*)a[d];
        A.b[d] = (d < 18) ? (S*)b[d] : (S*)a[18];
    }
    A.nx = p->nx; A.nxy = p->nx * p->ny;
    A.l = p->l; A.m = p->m; A.n = p->n;
    const double sc = storage_scale(p);
    A.col = col_const<C>(p, sc);
    A.fc = fast_const<C>(p, sc);
    A.lid_force = (C)p->lid_force * (C)sc;
    A.u_inflow = (C)p->u_inflow;
    A.inflow_cte1 = (C)p->inflow_cte1;
    // the inflow face's five equilibria are constants of the lattice: the
    // same operations in the same type as inflow_eq runs on the device
    // (separate IEEE roundings on both sides), rounded to storage once here
    for (int d = 0; d < 5; ++d) A.inflow_s[d] = host_pack<S, C>(inflow_eq<C>(d, A.u_inflow, A.inflow_cte1, A.col));
    A.scale = (p->kind == K_F16 || p->kind == K_BF16) ? p->scale : 1.0f;
    A.inv_scale = 1.0f / A.scale;
    const bool has_obs = p->obs && p->imin <= p->imax && p->jmin <= p->jmax && p->kmin <= p->kmax;
    A.obs = has_obs ? p->obs : nullptr;
    A.obs_nx = p->obs_nx; A.obs_nxy = (long long)p->obs_nx * p->obs_ny;
    A.imin = p->imin; A.imax = p->imax; A.jmin = p->jmin; A.jmax = p->jmax;
    A.kmin = p->kmin; A.kmax = p->kmax;
    A.mom = nullptr;
    A.mom_span = 8;
    A.mom_out = nullptr;
    A.mom_ticket = nullptr;
    A.bcase = p->bcase;
    A.generic = !(p->cte1 == 1.0 && p->cte0 == 0.0 && p->fx == 0.0 && p->fy == 0.0 && p->fz == 0.0);
    A.fast = (p->fast != 0 && sizeof(C) == 4) ? 1 : 0;
    A.zhalo = p->zhalo & 3;
    A.outflow_next = 0;
    return A;
}

// Warp-segment launch geometry of sweep_ab_kernel (see sweep_ab.cuh);
// allow_flat: the launch is the one-node AB sweep, which also knows the
// plane mapping.
template <class S, class C>
void segment_geometry(SweepArgs<S, C>& A, const void* a0, bool allow_flat = false) {
    const long long elem = (long long)((uintptr_t)a0 / sizeof(S));
    A.align_base = elem & 31;
    const SegPlan s = seg_plan(A.l, A.m, A.n, A.nx, A.align_base, allow_flat);
    A.nseg_aligned = s.aligned ? 1 : 0;
    A.nseg = (int)s.nseg;
    A.nrows = (uint32_t)((long long)A.m * A.n);
    A.nwarps = (uint32_t)s.warps;
    A.div_seg.init((uint32_t)A.nseg);
    A.div_m.init((uint32_t)A.m);
    A.flat = s.flat ? 1 : 0;
    A.fwpp = (uint32_t)s.wpp;
    A.div_fw.init(A.fwpp);
    A.div_nx.init((uint32_t)(A.nx < (1LL << 31) ? A.nx : 1));
}

// True unless the collision can use the shifted, force-free specialisation.
inline bool generic_collision(const bgk_sweep_params* p) {
    return !(p->cte1 == 1.0 && p->cte0 == 0.0 && p->fx == 0.0 && p->fy == 0.0 && p->fz == 0.0);
}

template <class S, class C>
FieldArgs<S, C> field_args(const bgk_sweep_params* p, void* const* a) {
    FieldArgs<S, C> F;
    for (int d = 0; d < 19; ++d) F.a[d] = (const S*)a[d];
    F.nx = p->nx; F.nxy = p->nx * p->ny;
    F.l = p->l; F.m = p->m; F.n = p->n;
    F.cte1 = (C)p->cte1;
    F.inv_scale = (p->kind == K_F16 || p->kind == K_BF16) ? 1.0f / p->scale : 1.0f;
    const bool has_obs = p->obs && p->imin <= p->imax && p->jmin <= p->jmax && p->kmin <= p->kmax;
    F.obs = has_obs ? p->obs : nullptr;
    F.obs_nx = p->obs_nx; F.obs_nxy = (long long)p->obs_nx * p->obs_ny;
    F.imin = p->imin; F.imax = p->imax; F.jmin = p->jmin; F.jmax = p->jmax;
    F.kmin = p->kmin; F.kmax = p->kmax;
    return F;
}

}  // namespace bgk
