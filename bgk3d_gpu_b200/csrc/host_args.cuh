// Host-side construction of kernel arguments, shared by the library's
// translation units (typed ABI and library-owned lattices).
#pragma once
#include <cstdint>
#include "bgk3d_b200.h"
#include "sweep_ab.cuh"
#include "reduce.cuh"

namespace bgk {

template <class C>
ColConst<C> col_const(const bgk_sweep_params* p) {
    ColConst<C> k;
    k.omega = (C)p->omega; k.cte0 = (C)p->cte0; k.cte1 = (C)p->cte1;
    k.p0 = (C)p->p0; k.p1 = (C)p->p1; k.p2 = (C)p->p2;
    k.rf = (C)p->rf; k.qf = (C)p->qf; k.tre = (C)p->tre;
    k.force_mode = p->force_mode;
    k.fx = (C)p->fx; k.fy = (C)p->fy; k.fz = (C)p->fz;
    return k;
}

template <class S, class C>
SweepArgs<S, C> sweep_args(const bgk_sweep_params* p, void* const* a, void* const* b) {
    SweepArgs<S, C> A;
    for (int d = 0; d < 19; ++d) {
        A.a[d] = (const S*)a[d];
        A.b[d] = (d < 18) ? (S*)b[d] : (S*)a[18];
    }
    A.nx = p->nx; A.nxy = p->nx * p->ny;
    A.l = p->l; A.m = p->m; A.n = p->n;
    A.col = col_const<C>(p);
    A.lid_force = (C)p->lid_force;
    A.u_inflow = (C)p->u_inflow;
    A.inflow_cte1 = (C)p->inflow_cte1;
    A.scale = (p->kind == K_F16 || p->kind == K_BF16) ? p->scale : 1.0f;
    A.inv_scale = 1.0f / A.scale;
    const bool has_obs = p->obs && p->imin <= p->imax && p->jmin <= p->jmax && p->kmin <= p->kmax;
    A.obs = has_obs ? p->obs : nullptr;
    A.obs_nx = p->obs_nx; A.obs_nxy = (long long)p->obs_nx * p->obs_ny;
    A.imin = p->imin; A.imax = p->imax; A.jmin = p->jmin; A.jmax = p->jmax;
    A.kmin = p->kmin; A.kmax = p->kmax;
    A.mom = nullptr;
    A.bcase = p->bcase;
    A.generic = !(p->cte1 == 1.0 && p->cte0 == 0.0 && p->fx == 0.0 && p->fy == 0.0 && p->fz == 0.0);
    return A;
}

// Warp-segment launch geometry of sweep_ab_kernel (see sweep_ab.cuh).
template <class S, class C>
void segment_geometry(SweepArgs<S, C>& A, const void* a0) {
    const long long elem = (long long)((uintptr_t)a0 / sizeof(S));
    A.align_base = elem & 31;
    const bool aligned = ((A.align_base + 1) % 32 == 0) && (A.nx % 32 == 0);
    A.nseg_aligned = aligned ? 1 : 0;
    A.nseg = aligned ? (A.l + 31) / 32 : (A.l + 62) / 32;
    A.nrows = (uint32_t)((long long)A.m * A.n);
    A.div_seg.init((uint32_t)A.nseg);
    A.div_m.init((uint32_t)A.m);
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
