// Launch wrappers (templates) of every kernel, instantiated once per storage
// kind by the inst_*.cu translation units; declared in kernels.h.
#pragma once
#include <algorithm>
#include <cuda_runtime.h>
#include "bgk3d_b200.h"
#include "bgk_internal.h"
#include "host_args.cuh"
#include "sweep_ab.cuh"
#include "sweep_aa.cuh"
#include "sweep_tma.cuh"
#include "reduce.cuh"
#include "batch.cuh"
#include "init.cuh"
#include "dissipation.cuh"

namespace bgk {

// Kernel variants: collision mode CM (fused-multiply-add modes for float
// compute only) and obstacle logic OBS, for 32-bit offsets; lattices of 2^31
// elements or more take 64-bit offsets with the generic collision and the
// obstacle logic compiled in.
template <template <class, class, int, class, int, bool> class L, class S, class C, int BC, class... A>
void by_variant(long long nelem, int cm, bool obs, A... args) {
    constexpr bool FLOAT = sizeof(C) == 4;
    if (nelem >= (1LL << 31)) {
        if constexpr (FLOAT) {
            if (cm_fast(cm)) { L<S, C, BC, long long, CM_FAST_GENERIC, true>::go(args...); return; }
        }
        L<S, C, BC, long long, CM_STRICT_GENERIC, true>::go(args...);
        return;
    }
    switch (cm) {
        case CM_STRICT:
            if (obs) L<S, C, BC, int, CM_STRICT, true>::go(args...);
            else L<S, C, BC, int, CM_STRICT, false>::go(args...);
            break;
        case CM_STRICT_GENERIC:
            if (obs) L<S, C, BC, int, CM_STRICT_GENERIC, true>::go(args...);
            else L<S, C, BC, int, CM_STRICT_GENERIC, false>::go(args...);
            break;
        case CM_FAST:
            if constexpr (FLOAT) {
                if (obs) L<S, C, BC, int, CM_FAST, true>::go(args...);
                else L<S, C, BC, int, CM_FAST, false>::go(args...);
            }
            break;
        default:
            if constexpr (FLOAT) {
                if (obs) L<S, C, BC, int, CM_FAST_GENERIC, true>::go(args...);
                else L<S, C, BC, int, CM_FAST_GENERIC, false>::go(args...);
            }
            break;
    }
}

template <class S, class C, int BC, class IDX, int CM, bool OBS> struct AbLaunch {
    static void go(const SweepArgs<S, C>& A, unsigned blocks, cudaStream_t st) {
        if (A.mom) {
            if (A.flat) sweep_ab_kernel<S, C, BC, IDX, CM, OBS, true, true><<<blocks, 256, 0, st>>>(A);
            else sweep_ab_kernel<S, C, BC, IDX, CM, OBS, false, true><<<blocks, 256, 0, st>>>(A);
        } else {
            if (A.flat) sweep_ab_kernel<S, C, BC, IDX, CM, OBS, true, false><<<blocks, 256, 0, st>>>(A);
            else sweep_ab_kernel<S, C, BC, IDX, CM, OBS, false, false><<<blocks, 256, 0, st>>>(A);
        }
    }
};
// The obstacle's grown box (sweep_box_kernel, obstacle logic compiled in);
// instantiated through by_variant with OBS = false only.
template <class S, class C, int BC, class IDX, int CM, bool OBS> struct BoxLaunch {
    static void go(const SweepArgs<S, C>& A, unsigned blocks, cudaStream_t st) {
        if constexpr (!OBS) sweep_box_kernel<S, C, BC, IDX, CM><<<blocks, 256, 0, st>>>(A);
    }
};
template <class S, class C, int BC, class IDX, int CM, bool OBS> struct Ab2Launch {
    static void go(const SweepArgs<S, C>& A, unsigned blocks, cudaStream_t st) {
        if constexpr (sizeof(S) == 2 && sizeof(C) == 4 && !OBS)
            sweep_ab2_kernel<S, C, BC, IDX, CM><<<blocks, 256, 0, st>>>(A);
    }
};
template <class S, class C, int BC, class IDX, int CM, bool OBS> struct AbpLaunch {
    static void go(const SweepArgs<S, C>& A, unsigned blocks, cudaStream_t st) {
        if constexpr (sizeof(S) == 2 && sizeof(C) == 4 && sizeof(IDX) == 4)
            sweep_abp_kernel<S, C, BC, CM, OBS><<<blocks, kPairThreads, 0, st>>>(A);
    }
};
// True when every node pair (i, i + 1), i odd, is one aligned 32-bit word in
// every population plane of a and b: even row pitches and each plane's base
// at 2 mod 4 bytes (then element 1 of every row starts a word).
template <class S>
bool pairs_aligned(const bgk_sweep_params* p, void* const* a, void* const* b) {
    if (sizeof(S) != 2 || (p->l & 1) || (p->nx & 1) || ((p->nx * p->ny) & 1)) return false;
    for (int d = 0; d < 19; ++d)
        if (((uintptr_t)a[d] & 3u) != 2u) return false;
    for (int d = 0; d < 18; ++d)
        if (((uintptr_t)b[d] & 3u) != 2u) return false;
    return true;
}
template <class S, class C, int BC, class IDX, int CM, bool OBS> struct AaEvenLaunch {
    static void go(const SweepArgs<S, C>& A, unsigned blocks, cudaStream_t st) {
        if (A.mom) aa_even_kernel<S, C, BC, IDX, CM, OBS, true><<<blocks, 256, 0, st>>>(A);
        else aa_even_kernel<S, C, BC, IDX, CM, OBS, false><<<blocks, 256, 0, st>>>(A);
    }
};
template <class S, class C, int BC, class IDX, int CM, bool OBS> struct AaOddLaunch {
    static void go(const SweepArgs<S, C>& A, unsigned blocks, cudaStream_t st) {
        if (A.mom) aa_odd_kernel<S, C, BC, IDX, CM, OBS, true><<<blocks, 256, 0, st>>>(A);
        else aa_odd_kernel<S, C, BC, IDX, CM, OBS, false><<<blocks, 256, 0, st>>>(A);
    }
};

// Collision mode of the arguments (fast modes need float compute).
template <class S, class C> int coll_mode(const SweepArgs<S, C>& A) {
    return A.generic + ((sizeof(C) == 4 && A.fast) ? 2 : 0);
}

// halo (inflow, nullable): on entry nonzero when a's outflow plane already
// holds the equilibria of a's state at x = l (the previous launch wrote it),
// so the pre-pass is skipped; on return nonzero when this launch wrote the
// next state's outflow plane into b (the one-node sweep does, the pair
// sweeps do not).
template <class S, class C>
int launch_sweep(const bgk_sweep_params* p, void* const* a, void* const* b, double* mom, cudaStream_t st,
                 int* halo, double* mom_out, unsigned* mom_ticket) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, a, b);
    segment_geometry(A, a[0], true);
    A.mom = mom;
    const bool fresh = halo && *halo;
    if (halo) *halo = 0;
    // the one-node and the adjacent-pair sweeps write the next outflow plane
    // when asked (outflow_next); the i / i + 32 sweep (sweep_ab2_kernel) does not
    bool writes_next = true;
    if constexpr (sizeof(S) == 2 && sizeof(C) == 4) {
        const long long ne = p->nx * p->ny * ((long long)p->n + 2) + 64;
        if (g_pair_kernels && mom == nullptr && ne < (1LL << 31) && !pairs_aligned<S>(p, a, b) &&
            cm_fast(coll_mode(A)) && A.obs == nullptr)
            writes_next = false;
    }
    if (p->bcase == BC_INFLOW) {
        if (!fresh || !writes_next) {
            dim3 blk(128), grd((p->m + 127) / 128, p->n);
            outflow_halo_kernel<S, C><<<grd, blk, 0, st>>>(A);
            if (int e = check_launch("outflow_halo_kernel")) return e;
        }
        if (halo && writes_next) {
            A.outflow_next = 1;
            *halo = 1;
        }
    }
    const long long warps = seg_plan(p->l, p->m, p->n, p->nx, A.align_base, true).warps;
    const long long blocks = (warps + 7) / 8;
    if (warps >= (1LL << 32) - 8) return set_error(BGK_ERR_ARG, "lattice too large for one launch");
    const long long nelem = p->nx * p->ny * ((long long)p->n + 2) + 64;
    const int cm = coll_mode(A);
    const bool obs = A.obs != nullptr;
    const MomPlan mp = mom_plan(warps);
    A.mom_span = (uint32_t)mp.span;
    if (mom && (!mom_out || !mom_ticket)) return set_error(BGK_ERR_ARG, "moments need their output and counters");
    A.mom_out = mom_out;
    A.mom_ticket = mom_ticket;
    const unsigned nb = (unsigned)(mom ? mp.blocks : blocks);
    if constexpr (sizeof(S) == 2 && sizeof(C) == 4) {
        if (g_pair_kernels && mom == nullptr && nelem < (1LL << 31) && pairs_aligned<S>(p, a, b)) {
            // adjacent node pairs: 64-node segments from i = 1
            SweepArgs<S, C> A2 = A;
            A2.nseg = (p->l + 63) / 64;
            A2.div_seg.init((uint32_t)A2.nseg);
            const long long w2 = (long long)A2.nseg * p->m * p->n;
            constexpr int wpb = kPairThreads / 32;
            const unsigned nb2 = (unsigned)((w2 + wpb - 1) / wpb);
            switch (p->bcase) {
                case BC_NONE: by_variant<AbpLaunch, S, C, BC_NONE>(nelem, cm, obs, A2, nb2, st); break;
                case BC_DRIVEN: by_variant<AbpLaunch, S, C, BC_DRIVEN>(nelem, cm, obs, A2, nb2, st); break;
                case BC_PERIODIC: by_variant<AbpLaunch, S, C, BC_PERIODIC>(nelem, cm, obs, A2, nb2, st); break;
                case BC_CHANNEL: by_variant<AbpLaunch, S, C, BC_CHANNEL>(nelem, cm, obs, A2, nb2, st); break;
                case BC_INFLOW: by_variant<AbpLaunch, S, C, BC_INFLOW>(nelem, cm, obs, A2, nb2, st); break;
            }
            return check_launch("sweep_abp_kernel");
        }
        if (g_pair_kernels && cm_fast(cm) && !obs && mom == nullptr && nelem < (1LL << 31)) {
            // two nodes per thread: 64-element segments (fused collision only:
            // with the reference-order collision the kernel spills and is
            // slower than the one-node sweep)
            SweepArgs<S, C> A2 = A;
            A2.nseg = (A.nseg + 1) / 2;
            A2.div_seg.init((uint32_t)A2.nseg);
            const long long w2 = (long long)A2.nseg * p->m * p->n;
            const unsigned nb2 = (unsigned)((w2 + 7) / 8);
            switch (p->bcase) {
                case BC_NONE: by_variant<Ab2Launch, S, C, BC_NONE>(nelem, cm, false, A2, nb2, st); break;
                case BC_DRIVEN: by_variant<Ab2Launch, S, C, BC_DRIVEN>(nelem, cm, false, A2, nb2, st); break;
                case BC_PERIODIC: by_variant<Ab2Launch, S, C, BC_PERIODIC>(nelem, cm, false, A2, nb2, st); break;
                case BC_CHANNEL: by_variant<Ab2Launch, S, C, BC_CHANNEL>(nelem, cm, false, A2, nb2, st); break;
                case BC_INFLOW: by_variant<Ab2Launch, S, C, BC_INFLOW>(nelem, cm, false, A2, nb2, st); break;
            }
            return check_launch("sweep_ab2_kernel");
        }
    }
    if (obs && g_obstacle_split && mom == nullptr && nelem < (1LL << 31)) {
        // the obstacle-free variant over every node outside the obstacle's
        // grown box, then that box with the obstacle logic: the obstacle's
        // per-link tests cost every node about 20 % more instructions
        switch (p->bcase) {
            case BC_NONE: by_variant<AbLaunch, S, C, BC_NONE>(nelem, cm, false, A, nb, st); break;
            case BC_DRIVEN: by_variant<AbLaunch, S, C, BC_DRIVEN>(nelem, cm, false, A, nb, st); break;
            case BC_PERIODIC: by_variant<AbLaunch, S, C, BC_PERIODIC>(nelem, cm, false, A, nb, st); break;
            case BC_CHANNEL: by_variant<AbLaunch, S, C, BC_CHANNEL>(nelem, cm, false, A, nb, st); break;
            case BC_INFLOW: by_variant<AbLaunch, S, C, BC_INFLOW>(nelem, cm, false, A, nb, st); break;
        }
        if (int e = check_launch("sweep_ab_kernel")) return e;
        const long long box = (long long)(A.imax - A.imin + 3) * (A.jmax - A.jmin + 3) * (A.kmax - A.kmin + 3);
        const unsigned nbb = (unsigned)((box + 255) / 256);
        switch (p->bcase) {
            case BC_NONE: by_variant<BoxLaunch, S, C, BC_NONE>(nelem, cm, false, A, nbb, st); break;
            case BC_DRIVEN: by_variant<BoxLaunch, S, C, BC_DRIVEN>(nelem, cm, false, A, nbb, st); break;
            case BC_PERIODIC: by_variant<BoxLaunch, S, C, BC_PERIODIC>(nelem, cm, false, A, nbb, st); break;
            case BC_CHANNEL: by_variant<BoxLaunch, S, C, BC_CHANNEL>(nelem, cm, false, A, nbb, st); break;
            case BC_INFLOW: by_variant<BoxLaunch, S, C, BC_INFLOW>(nelem, cm, false, A, nbb, st); break;
        }
        return check_launch("sweep_box_kernel");
    }
    switch (p->bcase) {
        case BC_NONE: by_variant<AbLaunch, S, C, BC_NONE>(nelem, cm, obs, A, nb, st); break;
        case BC_DRIVEN: by_variant<AbLaunch, S, C, BC_DRIVEN>(nelem, cm, obs, A, nb, st); break;
        case BC_PERIODIC: by_variant<AbLaunch, S, C, BC_PERIODIC>(nelem, cm, obs, A, nb, st); break;
        case BC_CHANNEL: by_variant<AbLaunch, S, C, BC_CHANNEL>(nelem, cm, obs, A, nb, st); break;
        case BC_INFLOW: by_variant<AbLaunch, S, C, BC_INFLOW>(nelem, cm, obs, A, nb, st); break;
    }
    return check_launch("sweep_ab_kernel");
}

// TMA-staged sweep (sweep_tma.cuh) for library-owned AB lattices without
// obstacle; map is the lattice's tensor map, pa[d] the plane of a[d].

template <class S, class C, int BC, int CM>
int launch_tma_variant(const SweepArgs<S, C>& A, const TmaSched& T, const CUtensorMap& map, cudaStream_t st) {
    auto kern = sweep_tma_kernel<S, C, BC, CM>;
    const size_t smem = TmaBox<S>::SMEM;
    static int grid_per_sm = 0;   // per instantiation, set up on the first launch
    if (grid_per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "tma smem attribute: %s", cudaGetErrorString(e));
        int per = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kTmaThreads, smem);
        if (e != cudaSuccess || per < 1) return set_error(BGK_ERR_CUDA, "tma occupancy: %s", cudaGetErrorString(e));
        grid_per_sm = per;
    }
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long grid = std::min<long long>((long long)nsm * grid_per_sm, (long long)T.ntiles);
    kern<<<(unsigned)std::max<long long>(grid, 1), kTmaThreads, smem, st>>>(A, T, map);
    if (int e = check_launch("sweep_tma_kernel")) return e;
    const long long l = A.l, m = A.m, n = A.n;
    const long long faces = (n > 1 ? 2 : 1) * l * m + (m > 1 ? 2 : 1) * l * std::max(n - 2, 0LL) +
                            (l > 1 ? 2 : 1) * std::max(m - 2, 0LL) * std::max(n - 2, 0LL);
    sweep_faces_kernel<S, C, BC, CM><<<(unsigned)((faces + 255) / 256), 256, 0, st>>>(A);
    return check_launch("sweep_faces_kernel");
}

template <class S, class C, int BC>
int launch_tma_bc(const SweepArgs<S, C>& A, const TmaSched& T, const CUtensorMap& map, int cm, cudaStream_t st) {
    switch (cm) {
        case CM_STRICT: return launch_tma_variant<S, C, BC, CM_STRICT>(A, T, map, st);
        case CM_STRICT_GENERIC: return launch_tma_variant<S, C, BC, CM_STRICT_GENERIC>(A, T, map, st);
        case CM_FAST:
            if constexpr (sizeof(C) == 4) return launch_tma_variant<S, C, BC, CM_FAST>(A, T, map, st);
            break;
        default:
            if constexpr (sizeof(C) == 4) return launch_tma_variant<S, C, BC, CM_FAST_GENERIC>(A, T, map, st);
            break;
    }
    return set_error(BGK_ERR_ARG, "collision mode %d", cm);
}

template <class S, class C>
int launch_sweep_tma(const bgk_sweep_params* p, void* const* a, void* const* b, const void* tmap, const int* pa,
                     int* err, cudaStream_t st) {
    if constexpr (sizeof(C) != 4 || sizeof(S) > 4) {
        return set_error(BGK_ERR_UNSUPPORTED, "the TMA sweep serves float compute");
    } else {
    SweepArgs<S, C> A = sweep_args<S, C>(p, a, b);
    segment_geometry(A, a[0]);
    A.mom = nullptr;
    if (p->bcase == BC_INFLOW) {
        dim3 blk(128), grd((p->m + 127) / 128, p->n);
        outflow_halo_kernel<S, C><<<grd, blk, 0, st>>>(A);
        if (int e = check_launch("outflow_halo_kernel")) return e;
    }
    TmaSched T;
    for (int d = 0; d < 19; ++d) T.pa[d] = pa[d];
    T.ntx = (p->l + 63) / 64;
    T.nty = (p->m + kTmaRows - 1) / kTmaRows;
    T.ntiles = (uint32_t)((long long)T.ntx * T.nty * p->n);
    T.err = err;
    const CUtensorMap& map = *static_cast<const CUtensorMap*>(tmap);
    const int cm = coll_mode(A);
    switch (p->bcase) {
        case BC_DRIVEN: return launch_tma_bc<S, C, BC_DRIVEN>(A, T, map, cm, st);
        case BC_PERIODIC: return launch_tma_bc<S, C, BC_PERIODIC>(A, T, map, cm, st);
        case BC_CHANNEL: return launch_tma_bc<S, C, BC_CHANNEL>(A, T, map, cm, st);
        case BC_INFLOW: return launch_tma_bc<S, C, BC_INFLOW>(A, T, map, cm, st);
        default: return set_error(BGK_ERR_ARG, "the TMA sweep needs a boundary case");
    }
    }
}

template <class S, class C>
int launch_moments(const bgk_sweep_params* p, void* const* a, double* out, double* ws, cudaStream_t st) {
    FieldArgs<S, C> F = field_args<S, C>(p, a);
    dim3 grd, blk;
    moments_grid(p->l, p->m, p->n, grd, blk);
    moments_partial_kernel<S, C><<<grd, blk, 0, st>>>(F, ws);
    if (int e = check_launch("moments_partial_kernel")) return e;
    const long long nparts = (long long)grd.x * grd.y * grd.z;
    finalize_partials_kernel<5><<<1, kFinalizeThreads, 0, st>>>(ws, nparts, out);
    return check_launch("finalize_partials_kernel");
}

template <class S, class C, int BC>
int launch_dissipation_bc(const bgk_sweep_params* p, const SweepArgs<S, C>& A, const FieldArgs<S, C>& F, C two_nu,
                          double* out, double* ws, cudaStream_t st) {
    dim3 grd, blk;
    moments_grid(p->l, p->m, p->n, grd, blk);
    const long long nb1 = (long long)grd.x * grd.y * grd.z;
    const ColConst<C> K = col_const<C>(p, 1.0);
    const long long nelem = p->nx * p->ny * ((long long)p->n + 2) + 64;
    if (nelem >= (1LL << 31))
        dissipation_partial_kernel<S, C, BC, long long><<<grd, blk, 0, st>>>(A, K, two_nu, ws);
    else
        dissipation_partial_kernel<S, C, BC, int><<<grd, blk, 0, st>>>(A, K, two_nu, ws);
    if (int e = check_launch("dissipation_partial_kernel")) return e;
    finalize_partials_kernel<5><<<1, kFinalizeThreads, 0, st>>>(ws, nb1, out);
    if (int e = check_launch("finalize_partials_kernel")) return e;
    const dim3 eg = enstrophy_grid(p->l, p->m, p->n);
    const long long nb2 = (long long)eg.x * eg.y * eg.z;
    double* ws2 = ws + 5 * nb1;
    enstrophy_partial_kernel<S, C, BC><<<eg, dim3(kEnsTX, kEnsTY), 0, st>>>(F, p->zhalo, ws2);
    if (int e = check_launch("enstrophy_partial_kernel")) return e;
    finalize_partials_kernel<2><<<1, kFinalizeThreads, 0, st>>>(ws2, nb2, out + 5);
    return check_launch("finalize_partials_kernel");
}

// TKE, dissipation, mean squares and enstrophy (dissipation.cuh) into
// out[0..6]; ws holds bgk_dissipation_workspace_bytes(l, m, n) bytes.  The
// inflow case first writes the outflow halo plane of the current state, as
// the reference's boundary routine does before its pull.
template <class S, class C>
int launch_dissipation(const bgk_sweep_params* p, void* const* a, double nu, double* out, double* ws,
                       cudaStream_t st) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, a, a);
    const FieldArgs<S, C> F = field_args<S, C>(p, a);
    const C two_nu = C(2) * (C)nu;
    switch (p->bcase) {
        case BC_NONE: return launch_dissipation_bc<S, C, BC_NONE>(p, A, F, two_nu, out, ws, st);
        case BC_DRIVEN: return launch_dissipation_bc<S, C, BC_DRIVEN>(p, A, F, two_nu, out, ws, st);
        case BC_PERIODIC: return launch_dissipation_bc<S, C, BC_PERIODIC>(p, A, F, two_nu, out, ws, st);
        case BC_CHANNEL: return launch_dissipation_bc<S, C, BC_CHANNEL>(p, A, F, two_nu, out, ws, st);
        case BC_INFLOW: {
            dim3 blk(128), grd((p->m + 127) / 128, p->n);
            outflow_halo_kernel<S, C><<<grd, blk, 0, st>>>(A);
            if (int e = check_launch("outflow_halo_kernel")) return e;
            return launch_dissipation_bc<S, C, BC_INFLOW>(p, A, F, two_nu, out, ws, st);
        }
    }
    return set_error(BGK_ERR_ARG, "bcase %d", p->bcase);
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
    finalize_partials_kernel<3><<<1, kFinalizeThreads, 0, st>>>(ws, nb, out);
    return check_launch("finalize_partials_kernel");
}

template <class S, class C, int BC>
void launch_aa_bc(const SweepArgs<S, C>& A, bool odd, long long nelem, unsigned blocks, cudaStream_t st) {
    const int cm = coll_mode(A);
    const bool obs = A.obs != nullptr;
    if (odd) by_variant<AaOddLaunch, S, C, BC>(nelem, cm, obs, A, blocks, st);
    else by_variant<AaEvenLaunch, S, C, BC>(nelem, cm, obs, A, blocks, st);
}

template <class S, class C, int BC, bool OBS>
void launch_aa_odd_pair_obs(const SweepArgs<S, C>& A, int cm, unsigned blocks, cudaStream_t st) {
    switch (cm) {
        case CM_STRICT: aa_odd_pair_kernel<S, C, BC, CM_STRICT, OBS><<<blocks, kPairThreads, 0, st>>>(A); break;
        case CM_STRICT_GENERIC:
            aa_odd_pair_kernel<S, C, BC, CM_STRICT_GENERIC, OBS><<<blocks, kPairThreads, 0, st>>>(A);
            break;
        case CM_FAST: aa_odd_pair_kernel<S, C, BC, CM_FAST, OBS><<<blocks, kPairThreads, 0, st>>>(A); break;
        default: aa_odd_pair_kernel<S, C, BC, CM_FAST_GENERIC, OBS><<<blocks, kPairThreads, 0, st>>>(A); break;
    }
}
template <class S, class C, int BC>
void launch_aa_odd_pair(const SweepArgs<S, C>& A, int cm, bool obs, unsigned blocks, cudaStream_t st) {
    if constexpr (sizeof(S) == 2 && sizeof(C) == 4) {
        if (obs) launch_aa_odd_pair_obs<S, C, BC, true>(A, cm, blocks, st);
        else launch_aa_odd_pair_obs<S, C, BC, false>(A, cm, blocks, st);
    }
}
template <class S, class C, bool INFLOW, bool OBS>
void launch_aa_even_pair(const SweepArgs<S, C>& A, int cm, unsigned blocks, cudaStream_t st) {
    switch (cm) {
        case CM_STRICT: aa_even_pair_kernel<S, C, CM_STRICT, INFLOW, OBS><<<blocks, kPairThreads, 0, st>>>(A); break;
        case CM_STRICT_GENERIC:
            aa_even_pair_kernel<S, C, CM_STRICT_GENERIC, INFLOW, OBS><<<blocks, kPairThreads, 0, st>>>(A);
            break;
        case CM_FAST: aa_even_pair_kernel<S, C, CM_FAST, INFLOW, OBS><<<blocks, kPairThreads, 0, st>>>(A); break;
        default: aa_even_pair_kernel<S, C, CM_FAST_GENERIC, INFLOW, OBS><<<blocks, kPairThreads, 0, st>>>(A); break;
    }
}

template <class S, class C>
int launch_aa(const bgk_sweep_params* p, void* const* slots, bool odd, double* mom, cudaStream_t st,
              double* mom_out, unsigned* mom_ticket) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, slots, slots);
    A.b[18] = (S*)slots[18];
    segment_geometry(A, slots[0]);
    A.mom = mom;
    const long long warps = (long long)A.nseg * p->m * p->n;
    if (warps >= (1LL << 32) - 8) return set_error(BGK_ERR_ARG, "lattice too large for one launch");
    const MomPlan mp = mom_plan(warps);
    A.mom_span = (uint32_t)mp.span;
    if (mom && (!mom_out || !mom_ticket)) return set_error(BGK_ERR_ARG, "moments need their output and counters");
    A.mom_out = mom_out;
    A.mom_ticket = mom_ticket;
    const unsigned blocks = (unsigned)(mom ? mp.blocks : (warps + 7) / 8);
    const long long nelem = p->nx * p->ny * ((long long)p->n + 2) + 64;
    if constexpr (sizeof(S) == 2 && sizeof(C) == 4) {
        const int cm = coll_mode(A);
        if (g_pair_kernels && mom == nullptr && p->bcase != BC_NONE && nelem < (1LL << 31) &&
            pairs_aligned<S>(p, slots, slots)) {
            SweepArgs<S, C> A2 = A;
            A2.nseg = (p->l + 63) / 64;
            A2.div_seg.init((uint32_t)A2.nseg);
            constexpr int wpb = kPairThreads / 32;
            const unsigned nb2 = (unsigned)(((long long)A2.nseg * p->m * p->n + wpb - 1) / wpb);
            const bool obs = A.obs != nullptr, inflow = p->bcase == BC_INFLOW;
            if (!odd) {
                if (inflow) {
                    if (obs) launch_aa_even_pair<S, C, true, true>(A2, cm, nb2, st);
                    else launch_aa_even_pair<S, C, true, false>(A2, cm, nb2, st);
                } else {
                    if (obs) launch_aa_even_pair<S, C, false, true>(A2, cm, nb2, st);
                    else launch_aa_even_pair<S, C, false, false>(A2, cm, nb2, st);
                }
                return check_launch("aa_even_pair_kernel");
            }
            switch (p->bcase) {
                case BC_DRIVEN: launch_aa_odd_pair<S, C, BC_DRIVEN>(A2, cm, obs, nb2, st); break;
                case BC_PERIODIC: launch_aa_odd_pair<S, C, BC_PERIODIC>(A2, cm, obs, nb2, st); break;
                case BC_CHANNEL: launch_aa_odd_pair<S, C, BC_CHANNEL>(A2, cm, obs, nb2, st); break;
                case BC_INFLOW: launch_aa_odd_pair<S, C, BC_INFLOW>(A2, cm, obs, nb2, st); break;
                default: return set_error(BGK_ERR_ARG, "AA lattices need a boundary case");
            }
            return check_launch("aa_odd_pair_kernel");
        }
    }
    switch (p->bcase) {
        case BC_DRIVEN: launch_aa_bc<S, C, BC_DRIVEN>(A, odd, nelem, blocks, st); break;
        case BC_PERIODIC: launch_aa_bc<S, C, BC_PERIODIC>(A, odd, nelem, blocks, st); break;
        case BC_CHANNEL: launch_aa_bc<S, C, BC_CHANNEL>(A, odd, nelem, blocks, st); break;
        case BC_INFLOW: launch_aa_bc<S, C, BC_INFLOW>(A, odd, nelem, blocks, st); break;
        default: return set_error(BGK_ERR_ARG, "AA lattices need a boundary case");
    }
    return check_launch(odd ? "aa_odd_kernel" : "aa_even_kernel");
}

template <class S, class C>
int launch_aa_prepass(const bgk_sweep_params* p, void* const* slots, cudaStream_t st) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, slots, slots);
    dim3 blk(128), grd((p->m + 127) / 128, p->n);
    aa_outflow_prepass_kernel<S, C><<<grd, blk, 0, st>>>(A);
    return check_launch("aa_outflow_prepass_kernel");
}

// Batched stepping (batch.cuh): the two kernel-argument records of one
// lattice (parity 0: current a/b, parity 1: swapped) and its tile count.
template <class S, class C>
size_t fill_batch_desc(const bgk_sweep_params* p, void* const* a, void* const* b, void* out, uint32_t* tiles) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, a, b);
    segment_geometry(A, a[0]);
    if (p->bcase == BC_INFLOW) {
        // write the next state's outflow plane exactly when the member's own
        // step (launch_sweep) does: unless it takes the i / i + 32 sweep
        bool writes_next = true;
        if constexpr (sizeof(S) == 2 && sizeof(C) == 4) {
            const long long ne = p->nx * p->ny * ((long long)p->n + 2) + 64;
            if (g_pair_kernels && ne < (1LL << 31) && !pairs_aligned<S>(p, a, b) && cm_fast(coll_mode(A)) &&
                A.obs == nullptr)
                writes_next = false;
        }
        A.outflow_next = writes_next ? 1 : 0;
    }
    SweepArgs<S, C> B = A;
    for (int d = 0; d < 18; ++d) {
        B.a[d] = (const S*)b[d];
        B.b[d] = (S*)a[d];
    }
    SweepArgs<S, C>* o = static_cast<SweepArgs<S, C>*>(out);
    o[0] = A;
    o[1] = B;
    *tiles = (uint32_t)(((long long)A.nseg * p->m * p->n + 7) / 8);
    return 2 * sizeof(SweepArgs<S, C>);
}

template <class S, class C>
int launch_batch(const void* desc, const uint32_t* tile_begin, int nlat, uint32_t ntiles, unsigned* counter,
                 int parity, int sub, int grid, cudaStream_t st) {
    BatchView<S, C> V;
    V.desc = static_cast<const SweepArgs<S, C>*>(desc);
    V.tile_begin = tile_begin;
    V.nlat = nlat;
    V.ntiles = ntiles;
    V.counter = counter;
    V.parity = parity;
    V.sub = sub;
    if (grid <= 0) {   // one block per tile
        batch_grid_kernel<S, C><<<ntiles, 256, 0, st>>>(V);
        return check_launch("batch_grid_kernel");
    }
    batch_sweep_kernel<S, C><<<grid, 256, 0, st>>>(V);
    return check_launch("batch_sweep_kernel");
}

template <class S, class C, int BC, int CM>
void launch_group_bc_cm(const BatchGroupView<S, C>& V, uint32_t nchunks, bool obs, cudaStream_t st) {
    if (obs) batch_chunk_kernel<S, C, BC, CM, true><<<nchunks, 256, 0, st>>>(V);
    else batch_chunk_kernel<S, C, BC, CM, false><<<nchunks, 256, 0, st>>>(V);
}

template <class S, class C, int BC>
void launch_group_bc(const BatchGroupView<S, C>& V, uint32_t nchunks, int cm, bool obs, cudaStream_t st) {
    switch (cm) {
        case CM_STRICT: launch_group_bc_cm<S, C, BC, CM_STRICT>(V, nchunks, obs, st); break;
        case CM_STRICT_GENERIC: launch_group_bc_cm<S, C, BC, CM_STRICT_GENERIC>(V, nchunks, obs, st); break;
        case CM_FAST:
            if constexpr (sizeof(C) == 4) launch_group_bc_cm<S, C, BC, CM_FAST>(V, nchunks, obs, st);
            break;
        default:
            if constexpr (sizeof(C) == 4) launch_group_bc_cm<S, C, BC, CM_FAST_GENERIC>(V, nchunks, obs, st);
            break;
    }
}

// One group of a batch step (batch.cuh, grouped form): nchunks blocks over
// the group's chunk table.
template <class S, class C>
int launch_batch_group(const void* desc, const void* chunks, uint32_t nchunks, uint32_t chunk_warps, int parity,
                       int bcase, int cm, bool obs, cudaStream_t st) {
    if (nchunks == 0) return BGK_OK;
    BatchGroupView<S, C> V;
    V.desc = static_cast<const SweepArgs<S, C>*>(desc);
    V.chunks = static_cast<const uint2*>(chunks);
    V.parity = parity;
    V.chunk_warps = chunk_warps;
    switch (bcase) {
        case BC_DRIVEN: launch_group_bc<S, C, BC_DRIVEN>(V, nchunks, cm, obs, st); break;
        case BC_PERIODIC: launch_group_bc<S, C, BC_PERIODIC>(V, nchunks, cm, obs, st); break;
        case BC_CHANNEL: launch_group_bc<S, C, BC_CHANNEL>(V, nchunks, cm, obs, st); break;
        case BC_INFLOW: launch_group_bc<S, C, BC_INFLOW>(V, nchunks, cm, obs, st); break;
        default: return set_error(BGK_ERR_ARG, "batch members need a boundary case");
    }
    return check_launch("batch_chunk_kernel");
}

template <class S, class C>
int launch_outflow(const bgk_sweep_params* p, void* const* a, cudaStream_t st) {
    SweepArgs<S, C> A = sweep_args<S, C>(p, a, a);
    dim3 blk(128), grd((p->m + 127) / 128, p->n);
    outflow_halo_kernel<S, C><<<grd, blk, 0, st>>>(A);
    return check_launch("outflow_halo_kernel");
}

template <class S, class C>
int launch_init(void* const* f, long long nx, long long ny, int l, int m, int n, int flow, const double* prm,
                float scale, const bgk_sweep_params* p, cudaStream_t st) {
    if (flow == INIT_TGV_REF || flow == INIT_TG2D_REF) {
        InitRefArgs<S, C> R;
        for (int d = 0; d < 19; ++d) R.f[d] = (S*)f[d];
        R.nx = nx; R.nxy = nx * ny;
        R.l = l; R.m = m; R.n = n;
        R.flow = flow;
        R.u00 = (C)(prm ? prm[0] : 0.0);
        R.rf = (C)p->rf; R.qf = (C)p->qf; R.tre = (C)p->tre;
        R.p0 = (C)p->p0; R.p1 = (C)p->p1; R.p2 = (C)p->p2;
        R.scale = scale;
        const long long nodes = (long long)(l + 2) * (m + 2) * (n + 2);
        init_reference_kernel<S, C><<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(R);
        return check_launch("init_reference_kernel");
    }
    InitArgs<S> A;
    for (int d = 0; d < 19; ++d) A.f[d] = (S*)f[d];
    A.nx = nx; A.nxy = nx * ny;
    A.l = l; A.m = m; A.n = n;
    A.flow = flow;
    for (int q = 0; q < 4; ++q) A.p[q] = prm ? prm[q] : 0.0;
    A.scale = scale;
    const long long nodes = (long long)(l + 2) * (m + 2) * (n + 2);
    init_equilibrium_kernel<S><<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(A);
    return check_launch("init_equilibrium_kernel");
}

}  // namespace bgk

// Explicit instantiations, split so that the kernel variants of one storage
// kind compile in parallel translation units.
#define BGK_INSTANTIATE_AB(S, C)                                                                   \
    namespace bgk {                                                                                \
    template int launch_sweep<S, C>(const bgk_sweep_params*, void* const*, void* const*, double*,  \
                                    cudaStream_t, int*, double*, unsigned*);                       \
    template int launch_sweep_tma<S, C>(const bgk_sweep_params*, void* const*, void* const*,        \
                                        const void*, const int*, int*, cudaStream_t);              \
    }
#define BGK_INSTANTIATE_AA(S, C)                                                                   \
    namespace bgk {                                                                                \
    template int launch_aa<S, C>(const bgk_sweep_params*, void* const*, bool, double*,             \
                                 cudaStream_t, double*, unsigned*);                                \
    }
#define BGK_INSTANTIATE_BATCH(S, C)                                                                \
    namespace bgk {                                                                                \
    template size_t fill_batch_desc<S, C>(const bgk_sweep_params*, void* const*, void* const*,     \
                                          void*, uint32_t*);                                       \
    template int launch_batch<S, C>(const void*, const uint32_t*, int, uint32_t, unsigned*, int,   \
                                    int, int, cudaStream_t);                                       \
    template int launch_batch_group<S, C>(const void*, const void*, uint32_t, uint32_t, int, int,   \
                                          int, bool, cudaStream_t);                                \
    }
#define BGK_INSTANTIATE_MISC(S, C)                                                                 \
    namespace bgk {                                                                                \
    template int launch_moments<S, C>(const bgk_sweep_params*, void* const*, double*, double*,     \
                                      cudaStream_t);                                               \
    template int launch_draglift<S, C>(const bgk_sweep_params*, void* const*, int, int, int, int,  \
                                       int, int, double*, double*, size_t, cudaStream_t);          \
    template int launch_aa_prepass<S, C>(const bgk_sweep_params*, void* const*, cudaStream_t);     \
    template int launch_outflow<S, C>(const bgk_sweep_params*, void* const*, cudaStream_t);        \
    template int launch_init<S, C>(void* const*, long long, long long, int, int, int, int,          \
                                   const double*, float, const bgk_sweep_params*, cudaStream_t);   \
    template int launch_dissipation<S, C>(const bgk_sweep_params*, void* const*, double, double*,  \
                                          double*, cudaStream_t);                                  \
    }
