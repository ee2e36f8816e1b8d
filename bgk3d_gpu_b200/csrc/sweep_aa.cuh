// In-place AA-pattern time step: one population set, half the footprint of
// the two-lattice scheme, same arithmetic and the same boundary semantics as
// sweep_ab_kernel (so the results are bit-identical to the reference's).
//
// Slot convention.  "Layout E" (after the even kernel): slot opp(p) of node x
// holds the post-collision population p of x.  The odd kernel reads every
// incoming population from its source node's slot opp(p) (or resolves it by
// the boundary rules), collides, and pushes each outgoing population p to
// slot p of its target node x + c_p ("Layout O": slot p of x then holds the
// value x pulls in the next step).  The even kernel reads slot p of its own
// node, collides, and writes population p into slot opp(p): purely local.
// A thread's reads and writes touch the same memory locations, so neither
// kernel has an inter-thread hazard.
//
// Boundaries in the odd kernel, link by link (same precedence as the AB sweep):
//   * wall / solid source        -> read own slot p (= own post-collision opp(p));
//     the mirrored outgoing link writes own slot opp(p) (lid: +-force, rounded
//     through storage, on pops 02/11 at the top face);
//   * periodic axes              -> read/push the wrapped node;
//   * inflow face (x = 0)        -> constant equilibrium in; the node also
//     writes that constant into its own slots 01..05 for the next even step;
//     outgoing populations leaving through x = 0 are dropped;
//   * outflow face (x = l+1)     -> read the halo cell's slot opp(p), which the
//     even kernel (or the upload prepass) filled with the outflow equilibrium
//     of node (l, j, k); the odd kernel of node (l, j, k) pushes the new
//     outflow equilibrium into slots 10..14 of (l, j+c_y, k+c_z) (y/z wrapped).
// Solid nodes are skipped by both kernels.  The observable (post-collision)
// state exists only in Layout E, i.e. after an even number of steps.
#pragma once
#include "sweep_ab.cuh"

namespace bgk {

// Node of this thread under the warp-segment mapping of sweep_ab_kernel;
// returns false for idle lanes.
template <class S, class C, class IDX>
__device__ __forceinline__ bool aa_node(const SweepArgs<S, C>& P, uint32_t gw, int& i, int& j, int& k, IDX& c) {
    const int lane = threadIdx.x & 31;
    const uint32_t row = P.div_seg.div(gw);
    if (row >= P.nrows) return false;
    const int seg = (int)(gw - row * (uint32_t)P.nseg);
    const uint32_t kk = P.div_m.div(row);
    j = (int)(row - kk * (uint32_t)P.m) + 1;
    k = (int)kk + 1;
    const IDX rowoff = (IDX)P.nx * (IDX)j + (IDX)P.nxy * (IDX)k;
    const int sh = (int)((P.align_base + (long long)rowoff + 1) & 31);
    i = seg * 32 + lane + 1 - (P.nseg_aligned ? 0 : sh);
    if (i < 1 || i > P.l) return false;
    c = rowoff + (IDX)i;
    return true;
}

// Even (local) step of node (i, j, k) at element c.  P.a and P.b both name
// the slot arrays.  Arithmetic in storage units, as in sweep_node.
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM>
__device__ __forceinline__ void aa_even_at(const SweepArgs<S, C>& P, int i, int j, int k, IDX c, double (&m5)[5]) {
    if (OBS && P.obs != nullptr && i >= P.imin && i <= P.imax && j >= P.jmin && j <= P.jmax &&
        k >= P.kmin && k <= P.kmax && (obstacle_links(P, i, j, k) & 0x80000000u))
        return;
    // the slot arrays: read through P.a, written through P.b (the same arrays;
    // indexing the kernel parameters directly keeps them out of local memory)
    const float inv = P.inv_scale;
    C x[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) x[d] = Conv<S, C>::raw(P.a[d][c]);
    C y[19];
    collide_cm<S, C, CM>(x, y, P.col, P.fc, inv);
    S st[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) st[d] = Conv<S, C>::pack(y[d]);
#pragma unroll
    for (int d = 0; d < 19; ++d) P.b[opp_of(d)][c] = st[d];
    if (BC == BC_INFLOW && i == P.l) {
        C s[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) s[d] = Conv<S, C>::raw(st[d]);
        C eq[5];
        outflow_eq<C, Scaled<S>::value>(s, P.inflow_cte1, P.col, inv, eq);
#pragma unroll
        for (int e = 0; e < 5; ++e) P.b[opp_of(9 + e)][c + 1] = Conv<S, C>::pack(eq[e]);
    }
    if constexpr (MOM) {
        C s[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) s[d] = Conv<S, C>::ld(st[d], inv);
        diagno_node<C>(s, P.col.cte1, m5);
    }
}

// Even step of this lane's node.
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM>
__device__ __forceinline__ void aa_even_node(const SweepArgs<S, C>& P, uint32_t gw, double (&m5)[5]) {
    int i, j, k;
    IDX c;
    if (!aa_node<S, C, IDX>(P, gw, i, j, k, c)) return;
    aa_even_at<S, C, BC, IDX, CM, OBS, MOM>(P, i, j, k, c, m5);
}

template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 3 : 4) aa_even_kernel(const SweepArgs<S, C> P) {
    double m5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if constexpr (!MOM) {
        aa_even_node<S, C, BC, IDX, CM, OBS, false>(P, blockIdx.x * 8u + (threadIdx.x >> 5), m5);
    } else {
        const SegRun r = block_segments(P.nwarps, P.mom_span);
        for (uint32_t gw = r.beg + (threadIdx.x >> 5); gw < r.end; gw += 8u)
            aa_even_node<S, C, BC, IDX, CM, OBS, true>(P, gw, m5);
        block_reduce_store<5>(m5, P.mom);
        finalize_by_tickets<5>(P.mom, P.mom_out, P.mom_ticket);
    }
}

// Even step of the 16-bit kinds on aligned pairs
// (the adjacent-pair layout of sweep_abp_kernel): thread t reads the 19 slot
// words of its pair (i, i + 1), runs the two collisions as one on packed
// FP32 pairs and writes population p of both nodes as one word into slot
// opp(p); bit-identical to aa_even_kernel, in either collision mode.  Purely
// local, so no shuffles.  INFLOW: node l also writes the outflow halo
// (aa_even_at's rule) from its values just stored.  OBS: a warp whose 64
// nodes touch the obstacle's box grown by one node advances them node by
// node with the one-node rules (solid nodes are not updated).  No fused
// moments.
template <class S, class C, int CM, bool INFLOW, bool OBS>
__global__ void __launch_bounds__(kPairThreads, kPairBlocks) aa_even_pair_kernel(const SweepArgs<S, C> P) {
    static_assert(sizeof(S) == 2 && sizeof(C) == 4, "pair step: 16-bit storage, float compute");
    const uint32_t gw = blockIdx.x * (uint32_t)(kPairThreads / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const uint32_t row = P.div_seg.div(gw);
    if (row >= P.nrows) return;
    const int seg = (int)(gw - row * (uint32_t)P.nseg);
    const uint32_t kk = P.div_m.div(row);
    const int j = (int)(row - kk * (uint32_t)P.m) + 1;
    const int k = (int)kk + 1;
    const int i0 = seg * 64 + 2 * lane + 1;
    if (i0 >= P.l) return;                            // l even: the pair (i0, i0 + 1) is inside
    const int c = (int)P.nx * j + (int)P.nxy * k + i0;
    if (OBS && P.obs != nullptr && j >= P.jmin - 1 && j <= P.jmax + 1 && k >= P.kmin - 1 && k <= P.kmax + 1 &&
        seg * 64 + 64 >= P.imin - 1 && seg * 64 + 1 <= P.imax + 1) {
        double m5[5];
        aa_even_at<S, C, INFLOW ? BC_INFLOW : BC_NONE, int, CM, true, false>(P, i0, j, k, c, m5);
        aa_even_at<S, C, INFLOW ? BC_INFLOW : BC_NONE, int, CM, true, false>(P, i0 + 1, j, k, c + 1, m5);
        return;
    }
    // P.a and P.b name the same slot arrays (P.b[18] too)
    uint32_t wv[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) wv[d] = *reinterpret_cast<const unsigned*>(P.a[d] + c);   // all reads first
    auto xs = [&](int d) { return raw_bits<S>(wv[d]); };
    auto xp = [&](int d) { return raw_bits_again<S>(wv[d]); };
    auto ys = [&](int d, F2 y) { *reinterpret_cast<unsigned*>(P.b[opp_of(d)] + c) = pack_bits<S>(y); };
    if constexpr (cm_fast(CM))
        bgk_collide_fast_f<F2, float, cm_generic(CM), Scaled<S>::value>(xs, xp, ys, P.fc, P.inv_scale);
    else
        bgk_collide_f<F2, float, cm_generic(CM), Scaled<S>::value>(xs, xp, ys, P.col, P.inv_scale);
    if (INFLOW && i0 + 1 == P.l) {
        // node l is the high half: its populations as just stored (slot
        // opp(d), this thread's own stores), the outflow equilibria into the
        // halo cell l + 1, as aa_even_at writes them
        const int cl = c + 1;
        C r[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) r[d] = Conv<S, C>::raw(P.b[opp_of(d)][cl]);
        C eq[5];
        outflow_eq<C, Scaled<S>::value>(r, P.inflow_cte1, P.col, P.inv_scale, eq);
#pragma unroll
        for (int e = 0; e < 5; ++e) P.b[opp_of(9 + e)][cl + 1] = Conv<S, C>::pack(eq[e]);
    }
}

// Odd (pull + push) step of node (i, j, k) at element c.  YZW = false: the
// node's row lies on no y or z wall (and so not on the driven lid); that
// logic is compiled out.
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM, bool YZW = true>
__device__ __forceinline__ void aa_odd_at(const SweepArgs<S, C>& P, int i, int j, int k, IDX c, double (&m5)[5]) {
    typedef Faces<BC> F;
    uint32_t sl = 0;
    if (OBS && P.obs != nullptr && i >= P.imin - 1 && i <= P.imax + 1 && j >= P.jmin - 1 &&
        j <= P.jmax + 1 && k >= P.kmin - 1 && k <= P.kmax + 1) {
        sl = obstacle_links(P, i, j, k);
        if (sl & 0x80000000u) return;
    }
    // the slot arrays: read through P.a, written through P.b (the same arrays;
    // indexing the kernel parameters directly keeps them out of local memory)
    const IDX nx = (IDX)P.nx, nxy = (IDX)P.nxy;
    // offset of the neighbour at -1 / +1 along each axis (periodic axes wrap)
    const IDX oxm = (F::PX && i == 1) ? (IDX)(P.l - 1) : (IDX)(-1);
    const IDX oxp = (F::PX && i == P.l) ? (IDX)(1 - P.l) : (IDX)1;
    const IDX oym = (F::PY && j == 1) ? (IDX)(P.m - 1) * nx : -nx;
    const IDX oyp = (F::PY && j == P.m) ? (IDX)(1 - P.m) * nx : nx;
    const IDX ozm = (F::PZ && k == 1) ? (IDX)(P.n - 1) * nxy : -nxy;
    const IDX ozp = (F::PZ && k == P.n) ? (IDX)(1 - P.n) * nxy : nxy;
    // the -1 / +1 neighbour lies behind a wall
    const bool wxm = F::WX && i == 1, wxp = F::WX && i == P.l;
    const bool wym = YZW && F::WY && j == 1, wyp = YZW && F::WY && j == P.m;
    const bool wzm = YZW && F::WZ && k == 1, wzp = YZW && F::WZ && k == P.n;
    const float inv = P.inv_scale;
    C x[19];
#pragma unroll
    for (int d = 0; d < 18; ++d) {
        const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
        // source x - c_d
        IDX off = c;
        if (cx == 1) off += oxm; else if (cx == -1) off += oxp;
        if (cy == 1) off += oym; else if (cy == -1) off += oyp;
        if (cz == 1) off += ozm; else if (cz == -1) off += ozp;
        bool bounce = OBS && ((sl >> d) & 1u) != 0;
        if (cx == 1) bounce |= wxm; else if (cx == -1) bounce |= wxp;
        if (cy == 1) bounce |= wym; else if (cy == -1) bounce |= wyp;
        if (cz == 1) bounce |= wzm; else if (cz == -1) bounce |= wzp;
        C v = Conv<S, C>::raw(bounce ? P.a[d][c] : P.a[opp_of(d)][off]);
        if (YZW && BC == BC_DRIVEN && (d == 1 || d == 10) && k == P.n)
            v = roundtrip<S, C>(d == 1 ? v + P.lid_force : v - P.lid_force);
        if (BC == BC_INFLOW && cx == 1 && i == 1)
            v = Conv<S, C>::raw(P.inflow_s[d]);
        x[d] = v;
    }
    x[18] = Conv<S, C>::raw(P.a[18][c]);
    C y[19];
    collide_cm<S, C, CM>(x, y, P.col, P.fc, inv);
    S sv[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) sv[d] = Conv<S, C>::pack(y[d]);
#pragma unroll
    for (int d = 0; d < 18; ++d) {
        const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d), od = opp_of(d);
        // target x + c_d
        IDX off = c;
        if (cx == 1) off += oxp; else if (cx == -1) off += oxm;
        if (cy == 1) off += oyp; else if (cy == -1) off += oym;
        if (cz == 1) off += ozp; else if (cz == -1) off += ozm;
        bool bounce = OBS && ((sl >> od) & 1u) != 0;
        if (cx == 1) bounce |= wxp; else if (cx == -1) bounce |= wxm;
        if (cy == 1) bounce |= wyp; else if (cy == -1) bounce |= wym;
        if (cz == 1) bounce |= wzp; else if (cz == -1) bounce |= wzm;
        if (bounce) {
            S bv = sv[d];
            if (YZW && BC == BC_DRIVEN && (od == 1 || od == 10) && k == P.n) {
                const C r = Conv<S, C>::raw(sv[d]);
                bv = Conv<S, C>::pack(od == 1 ? r + P.lid_force : r - P.lid_force);
            }
            P.b[od][c] = bv;
        } else {
            const bool gone = BC == BC_INFLOW && ((cx == -1 && i == 1) || (cx == 1 && i == P.l));
            if (!gone) P.b[d][off] = sv[d];
        }
    }
    P.b[18][c] = sv[18];
    if constexpr (MOM) {
        C s[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) s[d] = Conv<S, C>::ld(sv[d], inv);
        diagno_node<C>(s, P.col.cte1, m5);
    }
    if (BC == BC_INFLOW && i == 1) {
#pragma unroll
        for (int d = 0; d < 5; ++d)
            P.b[d][c] = P.inflow_s[d];
    }
    if (BC == BC_INFLOW && i == P.l) {
        C s[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) s[d] = Conv<S, C>::raw(sv[d]);
        C eq[5];
        outflow_eq<C, Scaled<S>::value>(s, P.inflow_cte1, P.col, inv, eq);
#pragma unroll
        for (int e = 0; e < 5; ++e) {
            const int d = 9 + e, cy = cy_of(d), cz = cz_of(d);
            IDX off = c;   // (l+1, j, k) + c_d = (l, j + c_y, k + c_z)
            if (cy == 1) off += oyp; else if (cy == -1) off += oym;
            if (cz == 1) off += ozp; else if (cz == -1) off += ozm;
            P.b[d][off] = Conv<S, C>::pack(eq[e]);
        }
    }
}

// Odd step of this lane's node.
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM>
__device__ __forceinline__ void aa_odd_node(const SweepArgs<S, C>& P, uint32_t gw, double (&m5)[5]) {
    int i, j, k;
    IDX c;
    if (!aa_node<S, C, IDX>(P, gw, i, j, k, c)) return;
    // the driven cavity's rows inside its y and z walls (the same for the
    // whole warp) run without the wall and lid logic
    if (BC == BC_DRIVEN && j > 1 && j < P.m && k > 1 && k < P.n)
        aa_odd_at<S, C, BC, IDX, CM, OBS, MOM, false>(P, i, j, k, c, m5);
    else
        aa_odd_at<S, C, BC, IDX, CM, OBS, MOM, true>(P, i, j, k, c, m5);
}

template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 3 : 4) aa_odd_kernel(const SweepArgs<S, C> P) {
    double m5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if constexpr (!MOM) {
        aa_odd_node<S, C, BC, IDX, CM, OBS, false>(P, blockIdx.x * 8u + (threadIdx.x >> 5), m5);
    } else {
        const SegRun r = block_segments(P.nwarps, P.mom_span);
        for (uint32_t gw = r.beg + (threadIdx.x >> 5); gw < r.end; gw += 8u)
            aa_odd_node<S, C, BC, IDX, CM, OBS, true>(P, gw, m5);
        block_reduce_store<5>(m5, P.mom);
        finalize_by_tickets<5>(P.mom, P.mom_out, P.mom_ticket);
    }
}

// The pairs of one warp of aa_odd_pair_kernel in row (j, k), lane's pair at
// node ia (element c).  WALLS = false: the row lies on no y or z wall (the
// driven cavity's inner rows), whose tests and lid term are compiled out.
template <class S, class C, int BC, int CM, bool WALLS>
__device__ __forceinline__ void aa_odd_pair_row(const SweepArgs<S, C>& P, int j, int k, int lane, int ia, bool valid,
                                                int c) {
    typedef Faces<BC> F;
    const int nx = (int)P.nx, nxy = (int)P.nxy;
    const bool at_lo = ia == 1, at_hi = ia + 1 == P.l;
    const bool edge_lo = lane == 0 || at_lo, edge_hi = lane == 31 || at_hi;
    const int oym = (F::PY && j == 1) ? (P.m - 1) * nx : -nx;
    const int oyp = (F::PY && j == P.m) ? (1 - P.m) * nx : nx;
    const int ozm = (F::PZ && k == 1) ? (P.n - 1) * nxy : -nxy;
    const int ozp = (F::PZ && k == P.n) ? (1 - P.n) * nxy : nxy;
    const bool wym = WALLS && F::WY && j == 1, wyp = WALLS && F::WY && j == P.m;
    const bool wzm = WALLS && F::WZ && k == 1, wzp = WALLS && F::WZ && k == P.n;
    // ---- pull (all loads first)
    uint32_t w[18], e[18];
    bool wall[18];
#pragma unroll
    for (int d = 0; d < 18; ++d) {
        const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
        bool wl = false;
        int off = c;
        if (cy == 1) { off += oym; wl |= wym; } else if (cy == -1) { off += oyp; wl |= wyp; }
        if (cz == 1) { off += ozm; wl |= wzm; } else if (cz == -1) { off += ozp; wl |= wzp; }
        wall[d] = wl;
        const S* src = wl ? P.a[d] + c : P.a[opp_of(d)] + off;
        w[d] = *reinterpret_cast<const unsigned*>(src);
        if (cx == 1) {
            const S* ep = (F::WX && at_lo) ? P.a[d] + c
                                           : P.a[opp_of(d)] + off + ((F::PX && at_lo) ? P.l - 1 : -1);
            e[d] = s_bits(*ep);
        } else if (cx == -1) {
            const S* ep = (F::WX && at_hi) ? P.a[d] + c + 1
                                           : P.a[opp_of(d)] + off + ((F::PX && at_hi) ? 2 - P.l : 2);
            e[d] = s_bits(*ep);
        }
    }
    uint32_t wv[19];
#pragma unroll
    for (int d = 0; d < 18; ++d) {
        const int cx = cx_of(d);
        uint32_t v = w[d];
        if (cx == 1) {
            const uint32_t left = __shfl_up_sync(0xffffffffu, v, 1) >> 16;
            uint32_t lo = edge_lo ? e[d] : left;
            if (BC == BC_INFLOW && at_lo) lo = s_bits(P.inflow_s[d]);   // the inflow face x = 0
            if (!wall[d]) v = __byte_perm(lo, v, 0x5410);
        } else if (cx == -1) {
            const uint32_t right = __shfl_down_sync(0xffffffffu, v, 1) & 0xffffu;
            const uint32_t hi = edge_hi ? e[d] : right;
            if (!wall[d]) v = __byte_perm(v, hi, 0x5432);
        }
        if (WALLS && BC == BC_DRIVEN && (d == 1 || d == 10) && k == P.n) {
            F2 f = raw_bits<S>(v);
            f.v.x = roundtrip<S, C>(d == 1 ? f.v.x + P.lid_force : f.v.x - P.lid_force);
            f.v.y = roundtrip<S, C>(d == 1 ? f.v.y + P.lid_force : f.v.y - P.lid_force);
            v = pack_bits<S>(f);
        }
        wv[d] = v;
    }
    wv[18] = *reinterpret_cast<const unsigned*>(P.a[18] + c);
    // ---- collision, and the push of each population as soon as it is known
    auto bounce_bits = [&](int od, uint32_t bits) -> uint32_t {   // lid on a wall-reflected value
        if (WALLS && BC == BC_DRIVEN && (od == 1 || od == 10) && k == P.n) {
            const C r = Conv<S, C>::raw(bits_s<S>(bits));
            return s_bits(Conv<S, C>::pack(od == 1 ? r + P.lid_force : r - P.lid_force));
        }
        return bits;
    };
    auto st16 = [&](int arr, int at, uint32_t bits) { *reinterpret_cast<unsigned short*>(P.b[arr] + at) = (unsigned short)bits; };
    auto st32 = [&](int arr, int at, uint32_t word) { *reinterpret_cast<unsigned*>(P.b[arr] + at) = word; };
    auto xs = [&](int d) { return raw_bits<S>(wv[d]); };
    auto xp = [&](int d) { return raw_bits_again<S>(wv[d]); };
    auto ys = [&](int d, F2 y) {
        const uint32_t pk = pack_bits<S>(y);                  // lo: node ia, hi: node ia + 1
        if (d == 18) {
            if (valid) st32(18, c, pk);
            return;
        }
        const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d), od = opp_of(d);
        bool wl = false;
        int off = c;                                          // target row: x + c_d in y and z
        if (cy == 1) { off += oyp; wl |= wyp; } else if (cy == -1) { off += oym; wl |= wym; }
        if (cz == 1) { off += ozp; wl |= wzp; } else if (cz == -1) { off += ozm; wl |= wzm; }
        if (cx == 1) {
            const uint32_t prev_b = __shfl_up_sync(0xffffffffu, pk, 1) >> 16;     // lane t-1's node ia+1
            if (!valid) return;
            if (wl) { st32(od, c, bounce_bits(od, pk & 0xffffu) | (bounce_bits(od, pk >> 16) << 16)); return; }
            if (edge_lo) st16(d, off + 1, pk & 0xffffu);      // node ia -> ia + 1 (hi half only)
            else st32(d, off, __byte_perm(prev_b, pk, 0x5410));
            if (edge_hi) {                                    // node ia + 1 -> ia + 2 leaves the lane's word
                if (at_hi && F::WX) st16(od, c + 1, bounce_bits(od, pk >> 16));
                else st16(d, off + ((F::PX && at_hi) ? 2 - P.l : 2), pk >> 16);
            }
        } else if (cx == -1) {
            const uint32_t next_a = __shfl_down_sync(0xffffffffu, pk, 1) & 0xffffu;  // lane t+1's node ia
            if (!valid) return;
            if (wl) { st32(od, c, bounce_bits(od, pk & 0xffffu) | (bounce_bits(od, pk >> 16) << 16)); return; }
            if (edge_hi) st16(d, off, pk >> 16);              // node ia + 1 -> ia (lo half only)
            else st32(d, off, __byte_perm(pk, next_a, 0x5432));
            if (edge_lo) {                                    // node ia -> ia - 1 leaves the lane's word
                if (at_lo && F::WX) st16(od, c, bounce_bits(od, pk & 0xffffu));
                else if (!(BC == BC_INFLOW && at_lo))         // through the inflow face: gone
                    st16(d, off + ((F::PX && at_lo) ? P.l - 1 : -1), pk & 0xffffu);
            }
        } else {
            if (!valid) return;
            if (wl) st32(od, c, bounce_bits(od, pk & 0xffffu) | (bounce_bits(od, pk >> 16) << 16));
            else st32(d, off, pk);
        }
    };
    if constexpr (cm_fast(CM))
        bgk_collide_fast_f<F2, float, cm_generic(CM), Scaled<S>::value>(xs, xp, ys, P.fc, P.inv_scale);
    else
        bgk_collide_f<F2, float, cm_generic(CM), Scaled<S>::value>(xs, xp, ys, P.col, P.inv_scale);
    if (BC == BC_INFLOW && valid && at_lo) {
        // node 1: the inflow equilibrium into its own slots 01..05 (no node
        // pushes into them), as aa_odd_at writes it
#pragma unroll
        for (int d = 0; d < 5; ++d) st16(d, c, s_bits(P.inflow_s[d]));
    }
    if (BC == BC_INFLOW && valid && at_hi) {
        // node l is the high half: its populations where this thread has
        // just pushed them (c_x = 0: the high half of the target word; c_x =
        // +1: the halo cell l + 1, which the next even step rewrites; c_x =
        // -1: node l - 1), then the outflow equilibria into slots 10..14 of
        // (l, j + c_y, k + c_z), as aa_odd_at writes them
        auto target = [&](int d) {
            const int cy = cy_of(d), cz = cz_of(d);
            int off = c;
            if (cy == 1) off += oyp; else if (cy == -1) off += oym;
            if (cz == 1) off += ozp; else if (cz == -1) off += ozm;
            return off;
        };
        C r[19];
#pragma unroll
        for (int d = 0; d < 18; ++d) {
            const int cx = cx_of(d);
            r[d] = Conv<S, C>::raw(P.b[d][target(d) + (cx == 1 ? 2 : (cx == -1 ? 0 : 1))]);
        }
        r[18] = Conv<S, C>::raw(P.b[18][c + 1]);
        C eq[5];
        outflow_eq<C, Scaled<S>::value>(r, P.inflow_cte1, P.col, P.inv_scale, eq);
#pragma unroll
        for (int e = 0; e < 5; ++e) P.b[9 + e][target(9 + e) + 1] = Conv<S, C>::pack(eq[e]);
    }
}

// Odd step of the 16-bit kinds on aligned pairs (the layout of
// aa_even_pair_kernel; every boundary case; no fused moments).  Inflow:
// node 1 pulls the inflow equilibrium across x = 0 and writes it into its
// own slots 01..05, its populations leaving through x = 0 are dropped, and
// node l writes the outflow equilibria of its new state (aa_odd_at's rules).
// OBS: a warp whose 64 nodes touch the obstacle's box grown by one node
// advances them node by node with the one-node rules.  Pull: population d of the pair's nodes comes
// from slot opp(d) of the source row as one 32-bit word, the x-shifted half
// through a lane shuffle as in sweep_abp_kernel (behind a wall: own slot d).
// Push: population d of both nodes goes to slot d of the target row; for
// c_x = +-1 the word at the lane's own pair position holds one value of this
// lane and one of its neighbour lane (a shuffle), and the value that leaves
// the warp (or crosses an x face: wrap, bounce-back into own slot opp(d))
// is stored as a 16-bit value.  Every slot is written once, by the node that
// read it (or, within a warp, after the neighbour lane's read through the
// shuffled data), so the in-place update has no hazard.  Bit-identical to
// aa_odd_kernel.
template <class S, class C, int BC, int CM, bool OBS>
__global__ void __launch_bounds__(kPairThreads, kPairBlocks) aa_odd_pair_kernel(const SweepArgs<S, C> P) {
    static_assert(sizeof(S) == 2 && sizeof(C) == 4, "pair step: 16-bit storage, float compute");
    static_assert(BC == BC_DRIVEN || BC == BC_PERIODIC || BC == BC_CHANNEL || BC == BC_INFLOW,
                  "pair odd step: a boundary case");
    typedef Faces<BC> F;
    const uint32_t gw = blockIdx.x * (uint32_t)(kPairThreads / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const uint32_t row = P.div_seg.div(gw);
    if (row >= P.nrows) return;                       // whole warp
    const int seg = (int)(gw - row * (uint32_t)P.nseg);
    const uint32_t kk = P.div_m.div(row);
    const int j = (int)(row - kk * (uint32_t)P.m) + 1;
    const int k = (int)kk + 1;
    const int i0 = seg * 64 + 2 * lane + 1;
    const bool valid = i0 < P.l;                      // l even: the pair (i0, i0 + 1) is inside
    const int ia = valid ? i0 : P.l - 1;              // other lanes read a valid pair, store nothing
    const int nx = (int)P.nx, nxy = (int)P.nxy;
    const int c = nx * j + nxy * k + ia;
    if (OBS && P.obs != nullptr && j >= P.jmin - 1 && j <= P.jmax + 1 && k >= P.kmin - 1 && k <= P.kmax + 1 &&
        seg * 64 + 64 >= P.imin - 1 && seg * 64 + 1 <= P.imax + 1) {
        // the warp's 64 nodes touch the obstacle's box grown by one node:
        // node by node with the one-node rules (each node reads and writes
        // only slots no other node touches, so the order does not matter)
        double m5[5];
        if (valid) {
            aa_odd_at<S, C, BC, int, CM, true, false>(P, ia, j, k, c, m5);
            aa_odd_at<S, C, BC, int, CM, true, false>(P, ia + 1, j, k, c + 1, m5);
        }
        return;
    }
    if (BC != BC_DRIVEN || j == 1 || j == P.m || k == 1 || k == P.n)
        aa_odd_pair_row<S, C, BC, CM, true>(P, j, k, lane, ia, valid, c);
    else
        aa_odd_pair_row<S, C, BC, CM, false>(P, j, k, lane, ia, valid, c);
}

// Outflow halo in slot form for a freshly loaded Layout E state: halo cell
// (l+1, j, k) slot opp(p), p = 10..14, from the populations of (l, j, k).
template <class S, class C>
__global__ void aa_outflow_prepass_kernel(const SweepArgs<S, C> P) {
    const int j = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int k = 1 + (int)blockIdx.y;
    if (j > P.m) return;
    // the slot arrays: read through P.a, written through P.b (the same arrays;
    // indexing the kernel parameters directly keeps them out of local memory)
    const long long c = (long long)P.l + P.nx * (long long)j + P.nxy * (long long)k;
    C s[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) s[d] = Conv<S, C>::raw(P.a[opp_of(d)][c]);
    C eq[5];
    outflow_eq<C, Scaled<S>::value>(s, P.inflow_cte1, P.col, P.inv_scale, eq);
#pragma unroll
    for (int e = 0; e < 5; ++e) P.b[opp_of(9 + e)][c + 1] = Conv<S, C>::pack(eq[e]);
}

}  // namespace bgk
