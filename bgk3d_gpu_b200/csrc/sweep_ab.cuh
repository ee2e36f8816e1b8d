// Fused boundary + pull-stream + BGK collide sweep, two-lattice (A -> B)
// pattern, on the reference's structure-of-arrays layout.
//
// What one launch computes is what the reference computes with
//   bcond_<case> (SRC/bcond.<case>.F90, x -> y -> z halo writes)
//   bcond_obs    (SRC/bcond.obs.F90:103-122, writes into solid nodes)
//   col_MC       (SRC/col_MC.F90:255-536, pull from a, write b / a19)
// for every fluid node, without materialising the halo: each link whose
// source x - c_p lies outside the lattice (or in a solid node) is resolved in
// registers by the rule the reference's halo writes produce:
//   * a wall face (driven: all six, channel: z) -> the node's own opposite
//     population (half-way bounce-back), plus the lid term on pops 02/11 at
//     the top face (SRC/bcond.driven.F90:243-246; the z loop runs last, so it
//     wins at every edge);
//   * periodic axes -> the wrapped node (the full-range x, y, z copies of
//     SRC/bcond.periodic.F90 make every edge and corner a double/triple wrap);
//   * inflow face x=0 -> the equilibrium at rho=1, u=(u_in,0,0)
//     (SRC/bcond.inflow.F90:165-181), rounded to storage precision;
//   * outflow face x=l+1 -> the halo plane written by outflow_halo_kernel
//     (SRC/bcond.inflow.F90:135-162), read at the y/z-wrapped position;
//   * a solid neighbour (obs==1) -> own opposite population.
// Values that the reference constructs arithmetically before storing them in
// the halo (lid, inflow) are rounded through the storage type, so 16-bit and
// mixed kinds see exactly the reference's stored value.  All arithmetic is in
// storage units (Conv::raw / Conv::pack; the constants carry the scale).
//
// Solid nodes are not updated (their reference values are racy garbage: see
// SRC/bcond_gpu.hpp:438-455).  An obstacle must keep one node away from the
// faces (validated by the host), because the reference's periodic and outflow
// copies would otherwise read solid-node garbage.
#pragma once
#include "d3q19.cuh"
#include "f2.cuh"
#include "reduce.cuh"

namespace bgk {

template <class S, class C> struct SweepArgs {
    const S* a[19];   // current populations (a[18] is also written: in place)
    S* b[19];         // next populations; b[18] is ignored (pop 19 stays in a)
    long long nx, nxy;
    int l, m, n;
    ColConst<C> col;  // storage units: p0, p1, p2, fx, fy, fz carry the scale
    FastConst<C> fc;  // constants of the fused-multiply-add collision
    C lid_force;      // driven, storage units: added to pop 02 / subtracted from pop 11 at z = n+1
    C u_inflow;       // inflow: prescribed x velocity at x = 0
    C inflow_cte1;    // inflow equilibrium constant (0 for shifted storage)
    S inflow_s[5];    // inflow: pops 01..05 of the x = 0 face, inflow_eq rounded to storage (host-computed)
    float scale, inv_scale;
    const int* obs;   // optional: obstacle mask, Fortran layout (1:l,1:m,1:n)
    long long obs_nx, obs_nxy;
    int imin, imax, jmin, jmax, kmin, kmax;
    // launch geometry of the warp-segment mapping
    long long align_base;  // (address of a[0]) / sizeof(S), mod 32
    int nseg;              // 32-node segments per row
    int nseg_aligned;      // 1 when every row starts on a segment boundary
    uint32_t nrows;        // m * n
    uint32_t nwarps;       // the warps of one step: nseg * nrows, or fwpp * n when flat
    FastDiv div_seg, div_m;
    // plane mapping of the one-node AB sweep for rows that start mid-segment
    // (the reference's own nx = l + 2 layout): flat = 1 when in use
    int flat;
    uint32_t fwpp;         // warps per z plane
    FastDiv div_fw, div_nx;
    double* mom;           // optional: per-block FP64 moment records of the new state (finalize_by_tickets)
    uint32_t mom_span;     // with mom: segments per block (mom_plan), a multiple of 8
    double* mom_out;       // with mom: the launch's finalized sums, mom_out[0..4]
    unsigned* mom_ticket;  // with mom: the ticket counters
    int bcase;             // BC_* (used by the batched kernel, which dispatches per tile)
    int generic;           // 1 unless the force-free shifted collision applies
    int fast;              // 1: fused-multiply-add collision (float compute only)
    int zhalo;             // bit 0 / bit 1: the face k = 1 / k = n reads the halo plane as stored
    int outflow_next;      // inflow: nodes i = l also write the next state's outflow plane into b
};

// Equilibrium population p (0..4 -> 01..05) of the inflow face
// (SRC/bcond.inflow.F90:165-181), in the compute type (storage units when K
// carries the scale).
template <class C>
__host__ __device__ __forceinline__ C inflow_eq(int p, C u_in, C cte1, const ColConst<C>& K) {
    const C rf = K.rf, qf = K.qf, three = C(3), crho = C(1);
    const C xj = u_in, yj = C(0), zj = C(0);
    const C cvsq = xj * xj + yj * yj + zj * zj;
    C cxp;
    switch (p) {
        case 0: cxp = rf * (xj - yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq); break;
        case 1: cxp = rf * (xj - zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq); break;
        case 2: cxp = rf * (xj + yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq); break;
        case 3: cxp = rf * (xj + zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq); break;
        default: cxp = rf * (xj) + qf * (three * (xj) * (xj) - cvsq); break;
    }
    const C w = (p == 4) ? K.p1 : K.p2;
    return crho * w * (cte1 + cxp);
}

// A value rounded to storage precision, as the reference's halo store rounds it.
template <class S, class C>
__device__ __forceinline__ C roundtrip(C v) {
    return Conv<S, C>::raw(Conv<S, C>::pack(v));
}

// Outflow equilibria e = 9..13 (pops 10..14) from the stored populations
// a[] (storage units) of node (l, j, k) at rho = 1
// (SRC/bcond.inflow.F90:135-162).
template <class C, bool SCALED>
__device__ __forceinline__ void outflow_eq(const C (&a)[19], C cte1, const ColConst<C>& K, float inv,
                                           C (&eq)[5]) {
    const C rhoinv = C(1), crho = C(1), rf = K.rf, qf = K.qf, three = C(3), p1 = K.p1, p2 = K.p2;
    C mx = a[0] + a[1] + a[2] + a[3] + a[4] - a[9] - a[10] - a[11] - a[12] - a[13];
    C my = a[2] + a[6] + a[7] + a[8] + a[11] - a[0] - a[9] - a[15] - a[16] - a[17];
    C mz = a[3] + a[5] + a[6] + a[12] + a[17] - a[1] - a[8] - a[10] - a[14] - a[15];
    if (SCALED) { mx = mx * (C)inv; my = my * (C)inv; mz = mz * (C)inv; }
    const C xj = mx * rhoinv, yj = my * rhoinv, zj = mz * rhoinv;
    const C cvsq = xj * xj + yj * yj + zj * zj;
    const C cx10 = rf * (-xj - yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
    const C cx11 = rf * (-xj - zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
    const C cx12 = rf * (-xj + yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
    const C cx13 = rf * (-xj + zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
    const C cx14 = rf * (-xj) + qf * (three * (xj) * (xj) - cvsq);
    eq[0] = crho * p2 * (cte1 + cx10);
    eq[1] = crho * p2 * (cte1 + cx11);
    eq[2] = crho * p2 * (cte1 + cx12);
    eq[3] = crho * p2 * (cte1 + cx13);
    eq[4] = crho * p1 * (cte1 + cx14);
}

// Compile-time description of the six faces of a boundary case.
template <int BC> struct Faces {
    // periodic axes wrap; wall axes bounce back
    static constexpr bool PX = (BC == BC_PERIODIC || BC == BC_CHANNEL);
    static constexpr bool PY = (BC == BC_PERIODIC || BC == BC_CHANNEL || BC == BC_INFLOW);
    static constexpr bool PZ = (BC == BC_PERIODIC || BC == BC_INFLOW);
    static constexpr bool WX = (BC == BC_DRIVEN);
    static constexpr bool WY = (BC == BC_DRIVEN);
    static constexpr bool WZ = (BC == BC_DRIVEN || BC == BC_CHANNEL);
};

// Bit D set when the source x - c_D of node (i,j,k) is a solid node; bit 31
// when the node itself is solid.
template <class S, class C>
__device__ __forceinline__ uint32_t obstacle_links(const SweepArgs<S, C>& P, int i, int j, int k) {
    uint32_t bits = 0;
    auto solid = [&](int si, int sj, int sk) -> bool {
        if (si < P.imin || si > P.imax || sj < P.jmin || sj > P.jmax || sk < P.kmin || sk > P.kmax)
            return false;
        const long long o = (long long)(si - 1) + P.obs_nx * (long long)(sj - 1) +
                            P.obs_nxy * (long long)(sk - 1);
        return __ldg(P.obs + o) == 1;
    };
    if (solid(i, j, k)) return 0x80000000u;
#pragma unroll
    for (int d = 0; d < 18; ++d)
        if (solid(i - cx_of(d), j - cy_of(d), k - cz_of(d))) bits |= 1u << d;
    return bits;
}

// Warp-segment mapping: every warp owns 32 consecutive elements of one
// (j, k) row whose first element is 32-element aligned in memory, whatever
// the row's own alignment (P.align_base = (address of a[0]) / sizeof(S) mod
// 32; a row starting mid-segment simply leaves lanes idle).  Aligned warps
// make every store and every c_x = 0 load a whole number of 32-byte sectors.
// One thread per node; blocks of 256 threads = 8 row segments.
// gw: this warp's global segment index within the lattice.
// CM: collision mode; OBS: the lattice may have an obstacle (P.obs is then
// tested at run time; OBS = false compiles the obstacle logic out).
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM = false>
__device__ __forceinline__ void sweep_at(const SweepArgs<S, C>& P, int i, int j, int k, double (&m5)[5]);

// Collision of the gathered values x[] (storage units) of the node at element
// c, the store of the new populations (b[0..17], pop 19 in place) and, with
// MOM (the launch sums moments into P.mom), the node's moments of the stored
// state.
// outflow: the node is at i = l of an inflow lattice whose launch writes
// the next state's outflow plane (P.outflow_next): the equilibria that
// outflow_halo_kernel would compute from this node's stored state at the
// next step are written to b[9..13] at (l + 1, j, k) right away.
template <class S, class C, class IDX, int CM, bool MOM>
__device__ __forceinline__ void collide_store(const SweepArgs<S, C>& P, const C (&x)[19], IDX c, double (&m5)[5],
                                              bool outflow = false) {
    const float inv = P.inv_scale;
    C y[19];
    collide_cm<S, C, CM>(x, y, P.col, P.fc, inv);
    S sv[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) sv[d] = Conv<S, C>::pack(y[d]);
#pragma unroll
    for (int d = 0; d < 18; ++d) P.b[d][c] = sv[d];
    const_cast<S*>(P.a[18])[c] = sv[18];
    if (outflow) {
        C r[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) r[d] = Conv<S, C>::raw(sv[d]);
        C eq[5];
        outflow_eq<C, Scaled<S>::value>(r, P.inflow_cte1, P.col, P.inv_scale, eq);
#pragma unroll
        for (int e = 0; e < 5; ++e) P.b[9 + e][c + 1] = Conv<S, C>::pack(eq[e]);
    }
    if constexpr (MOM) {
        C s[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) s[d] = Conv<S, C>::ld(sv[d], inv);
        diagno_node<C>(s, P.col.cte1, m5);
    }
}

// True when node (i, j, k) lies in the obstacle's box grown by one node and
// the launch leaves that box to sweep_box_kernel: with P.obs set, an
// obstacle-free variant (OBS = false) skips exactly the nodes whose links
// may touch a solid node, and every other node's result is the same as with
// the obstacle logic compiled in.
template <class S, class C>
__device__ __forceinline__ bool in_obstacle_box(const SweepArgs<S, C>& P, int i, int j, int k) {
    return P.obs != nullptr && i >= P.imin - 1 && i <= P.imax + 1 && j >= P.jmin - 1 && j <= P.jmax + 1 &&
           k >= P.kmin - 1 && k <= P.kmax + 1;
}

// Plane mapping (P.flat): a warp owns 32 consecutive, 32-element aligned
// elements of the range that runs from node (1, 1, k) to node (l, m, k) of
// one z plane, rows back to back.  Lanes that land on a halo column (i = 0 or
// i > l) idle: 2 of every nx lanes on the reference's nx = l + 2 layout,
// where whole rows would cost one extra warp per row (9 warps for 256 nodes).
// Row mapping (otherwise): a warp owns 32 elements of one (j, k) row.
// Returns false for a lane without a node.  FLAT selects the plane mapping
// at compile time (a run-time choice between the two made the compiler lay
// out some variants of the sweep 12 % slower).
template <class S, class C, class IDX, bool FLAT>
__device__ __forceinline__ bool warp_node(const SweepArgs<S, C>& P, uint32_t gw, int& i, int& j, int& k) {
    const int lane = threadIdx.x & 31;
    const IDX nx = (IDX)P.nx, nxy = (IDX)P.nxy;
    if constexpr (FLAT) {
        const uint32_t kk = P.div_fw.div(gw);
        if (kk >= (uint32_t)P.n) return false;
        const int s = (int)(gw - kk * P.fwpp);
        k = (int)kk + 1;
        const IDX first = nx + nxy * (IDX)k + 1;            // element of node (1, 1, k)
        const int sh = (int)((P.align_base + (long long)first) & 31);
        const int r = s * 32 + lane - sh;                    // element offset from node (1, 1, k)
        if (r < 0) return false;
        const uint32_t jj = P.div_nx.div((uint32_t)r);
        i = r - (int)jj * (int)P.nx + 1;
        j = (int)jj + 1;
        return i <= P.l && j <= P.m;
    }
    const uint32_t row = P.div_seg.div(gw);
    if (row >= P.nrows) return false;
    const int seg = (int)(gw - row * (uint32_t)P.nseg);
    const uint32_t kk = P.div_m.div(row);
    j = (int)(row - kk * (uint32_t)P.m) + 1;
    k = (int)kk + 1;
    const IDX rowoff = nx * (IDX)j + nxy * (IDX)k;
    const int sh = (int)((P.align_base + (long long)rowoff + 1) & 31);
    i = seg * 32 + lane + 1 - (P.nseg_aligned ? 0 : sh);
    return i >= 1 && i <= P.l;
}

// The node of this lane under the warp-segment mapping (FLAT: the plane
// mapping, which the launch selects when P.flat is set), and its time step
// (MOM: with the node's moments added to m5).
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool FLAT = false, bool MOM = false>
__device__ __forceinline__ void sweep_node(const SweepArgs<S, C>& P, uint32_t gw, double (&m5)[5]) {
    int i, j, k;
    if (!warp_node<S, C, IDX, FLAT>(P, gw, i, j, k)) return;
    if (!OBS && in_obstacle_box(P, i, j, k)) return;
    sweep_at<S, C, BC, IDX, CM, OBS, MOM>(P, i, j, k, m5);
}

// The 19 pulled values (storage units) of interior node (i, j, k), 1 <= i <= l
// etc., with every boundary link resolved; false for a solid node.
template <class S, class C, int BC, class IDX, bool OBS>
__device__ __forceinline__ bool gather_at(const SweepArgs<S, C>& P, int i, int j, int k, C (&x)[19]) {
    typedef Faces<BC> F;
    const IDX nx = (IDX)P.nx, nxy = (IDX)P.nxy;
    const IDX c = nx * (IDX)j + nxy * (IDX)k + (IDX)i;

    uint32_t sl = 0;
    if (OBS && P.obs != nullptr && i >= P.imin - 1 && i <= P.imax + 1 && j >= P.jmin - 1 &&
        j <= P.jmax + 1 && k >= P.kmin - 1 && k <= P.kmax + 1) {
        sl = obstacle_links(P, i, j, k);
        if (sl & 0x80000000u) return false;   // solid node: not updated
    }
    // source offsets for c = +1 (source at -1) and c = -1 (source at +1) on
    // each axis; periodic axes wrap, others step into the halo (those links
    // are then resolved below, never read from the halo)
    const IDX oxm = (F::PX && i == 1) ? (IDX)(P.l - 1) : (IDX)(-1);
    const IDX oxp = (F::PX && i == P.l) ? (IDX)(1 - P.l) : (IDX)1;
    const IDX oym = (F::PY && j == 1) ? (IDX)(P.m - 1) * nx : -nx;
    const IDX oyp = (F::PY && j == P.m) ? (IDX)(1 - P.m) * nx : nx;
    // a z face of a slab (P.zhalo) reads the halo plane as stored: no wrap, no wall, no lid
    const bool zlo = k == 1 && !(P.zhalo & 1), zhi = k == P.n && !(P.zhalo & 2);
    const IDX ozm = (F::PZ && zlo) ? (IDX)(P.n - 1) * nxy : -nxy;
    const IDX ozp = (F::PZ && zhi) ? (IDX)(1 - P.n) * nxy : nxy;
    const bool wxm = F::WX && i == 1, wxp = F::WX && i == P.l;
    const bool wym = F::WY && j == 1, wyp = F::WY && j == P.m;
    const bool wzm = F::WZ && zlo, wzp = F::WZ && zhi;
#pragma unroll
    for (int d = 0; d < 18; ++d) {
        const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
        IDX off = c;
        if (cx == 1) off += oxm; else if (cx == -1) off += oxp;
        if (cy == 1) off += oym; else if (cy == -1) off += oyp;
        if (cz == 1) off += ozm; else if (cz == -1) off += ozp;
        bool bounce = OBS && ((sl >> d) & 1u) != 0;
        if (cx == 1) bounce |= wxm; else if (cx == -1) bounce |= wxp;
        if (cy == 1) bounce |= wym; else if (cy == -1) bounce |= wyp;
        if (cz == 1) bounce |= wzm; else if (cz == -1) bounce |= wzp;
        const S* src = bounce ? P.a[opp_of(d)] : P.a[d];
        C v = Conv<S, C>::raw(ldro<S>(src + (bounce ? c : off)));
        if (BC == BC_DRIVEN && (d == 1 || d == 10) && zhi)
            v = roundtrip<S, C>(d == 1 ? v + P.lid_force : v - P.lid_force);
        if (BC == BC_INFLOW && cx == 1 && i == 1) v = Conv<S, C>::raw(P.inflow_s[d]);
        x[d] = v;
    }
    x[18] = Conv<S, C>::raw(P.a[18][c]);
    return true;
}

// The time step of interior node (i, j, k): gather, collision, store and
// (MOM) the node's moments.
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool MOM>
__device__ __forceinline__ void sweep_at(const SweepArgs<S, C>& P, int i, int j, int k, double (&m5)[5]) {
    C x[19];
    if (!gather_at<S, C, BC, IDX, OBS>(P, i, j, k, x)) return;
    collide_store<S, C, IDX, CM, MOM>(P, x, (IDX)P.nx * (IDX)j + (IDX)P.nxy * (IDX)k + (IDX)i, m5,
                                 BC == BC_INFLOW && P.outflow_next && i == P.l);
}

// One launch = one time step.  MOM (the launch has P.mom set and the grid of
// mom_plan, each block advancing one contiguous run of segments): the launch
// also sums SRC/diagno.F90's per-node moments of the state it produced
// (fluid nodes) in FP64 into P.mom_out[0..4] (finalize_by_tickets).  The two
// forms are separate kernels: as one kernel with a run-time branch, changes
// to either path moved the other's speed by up to 9 % (code layout).
template <class S, class C, int BC, class IDX, int CM, bool OBS, bool FLAT, bool MOM>
__global__ void __launch_bounds__(256, (SweepBlocks<S, C>::value)) sweep_ab_kernel(const SweepArgs<S, C> P) {
    double m5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if constexpr (!MOM) {
        sweep_node<S, C, BC, IDX, CM, OBS, FLAT, false>(P, blockIdx.x * 8u + (threadIdx.x >> 5), m5);
    } else {
        // several nodes per thread and one block reduction per run (once per
        // 256 nodes it had cost as many instructions as the sums)
        const SegRun r = block_segments(P.nwarps, P.mom_span);
        for (uint32_t gw = r.beg + (threadIdx.x >> 5); gw < r.end; gw += 8u)
            sweep_node<S, C, BC, IDX, CM, OBS, FLAT, true>(P, gw, m5);
        block_reduce_store<5>(m5, P.mom);
        finalize_by_tickets<5>(P.mom, P.mom_out, P.mom_ticket);
    }
}

// The nodes of the obstacle's box grown by one node (the box the
// obstacle-free variant of sweep_ab_kernel skips), one per thread, i
// fastest, with the obstacle logic compiled in.  No fused moments.
template <class S, class C, int BC, class IDX, int CM>
__global__ void __launch_bounds__(256, (SweepBlocks<S, C>::value)) sweep_box_kernel(const SweepArgs<S, C> P) {
    const int i0 = P.imin - 1, j0 = P.jmin - 1, k0 = P.kmin - 1;
    const int ni = P.imax - P.imin + 3, nj = P.jmax - P.jmin + 3, nk = P.kmax - P.kmin + 3;
    const long long t = blockIdx.x * 256LL + threadIdx.x;
    if (t >= (long long)ni * nj * nk) return;
    const int i = i0 + (int)(t % ni), j = j0 + (int)((t / ni) % nj), k = k0 + (int)(t / ((long long)ni * nj));
    double m5[5];
    sweep_at<S, C, BC, IDX, CM, true>(P, i, j, k, m5);
}

// Two nodes per thread for the 16-bit kinds: a warp owns 64 consecutive
// elements of one row (two 32-element segments, P.nseg counting 64-element
// segments), lane t the nodes at t and t + 32.  Each node is gathered by the
// one-node rules (gather_at); the two collisions run as one on packed FP32
// pairs (FADD2 / FFMA2, lane-wise the same roundings, so the result is
// bit-identical to the one-node sweep) and the stores stay 16-bit and
// coalesced.  Per node this halves the collision's instructions and shares
// the row/segment arithmetic.  No obstacle and no fused moments (the host
// takes the one-node kernel for those).
template <class S, class C, int BC, class IDX, int CM>
__global__ void __launch_bounds__(256, 4) sweep_ab2_kernel(const SweepArgs<S, C> P) {
    static_assert(sizeof(S) == 2 && sizeof(C) == 4, "two-node sweep: 16-bit storage, float compute");
    const uint32_t gw = blockIdx.x * 8u + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const uint32_t row = P.div_seg.div(gw);
    if (row >= P.nrows) return;
    const int seg = (int)(gw - row * (uint32_t)P.nseg);
    const uint32_t kk = P.div_m.div(row);
    const int j = (int)(row - kk * (uint32_t)P.m) + 1;
    const int k = (int)kk + 1;
    const IDX nx = (IDX)P.nx, nxy = (IDX)P.nxy;
    const IDX rowoff = nx * (IDX)j + nxy * (IDX)k;
    const int sh = (int)((P.align_base + (long long)rowoff + 1) & 31);
    int ia = seg * 64 + lane + 1 - (P.nseg_aligned ? 0 : sh);
    int ib = ia + 32;
    const bool va = ia >= 1 && ia <= P.l, vb = ib >= 1 && ib <= P.l;
    if (!va && !vb) return;
    if (!va) ia = ib;          // compute the valid node twice, store it once
    if (!vb) ib = ia;
    C xa[19], xb[19];
    gather_at<S, C, BC, IDX, false>(P, ia, j, k, xa);
    gather_at<S, C, BC, IDX, false>(P, ib, j, k, xb);
    F2 x[19], y[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) x[d] = F2(xa[d], xb[d]);
    if constexpr (cm_fast(CM))
        bgk_collide_fast_v<F2, float, cm_generic(CM), Scaled<S>::value>(x, y, P.fc, P.inv_scale);
    else
        bgk_collide_v<F2, float, cm_generic(CM), Scaled<S>::value>(x, y, P.col, P.inv_scale);
    typedef Pack2<S> PK;
    const IDX ca = rowoff + (IDX)ia, cb = rowoff + (IDX)ib;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
        const typename PK::V w = PK::pack(y[d]);
        S* dst = d < 18 ? P.b[d] : const_cast<S*>(P.a[18]);
        if (va) dst[ca] = PK::lo(w);
        if (vb) dst[cb] = PK::hi(w);
    }
}

// Adjacent node pairs for the 16-bit kinds on aligned rows of even length:
// a warp owns 64 consecutive nodes of one row, lane t the pair (i, i + 1)
// with i = 64 seg + 2t + 1 (i odd, so the pair is one aligned 32-bit word in
// every plane).  Per population one 32-bit load fetches the pair at the
// source row (y/z offsets and their wraps are the same for the whole warp):
//   c_x =  0: both values;
//   c_x = +1: node i + 1 takes the low half, node i the high half of lane
//             t - 1's word (a shuffle);
//   c_x = -1: node i takes the high half, node i + 1 the low half of lane
//             t + 1's word.
// The value the warp does not hold (lane 0's left, lane 31's right
// neighbour) and the x faces (i = 1, i + 1 = l) are resolved per node by the
// one-node rules (gather_at): wrap, bounce-back, inflow equilibrium, outflow
// halo.  A y/z wall bounces both nodes to their own opposite populations
// (one aligned load).  The two collisions run as one on packed FP32 pairs
// (bit-identical to the one-node sweep) and every store is one aligned
// 32-bit word.  Warps whose nodes touch an obstacle's box (grown by one
// node) take the one-node rules node by node.  No fused moments, 32-bit
// element offsets.
constexpr int kPairThreads = 128;   // threads per block of sweep_abp_kernel
constexpr int kPairBlocks = 7;      // resident blocks per SM it is compiled for (72 registers)

// The pairs of one warp in row (j, k): lane's pair starts at node ia; WALLS:
// the row lies on a y or z wall of the case (compiled separately, so that
// the rows inside carry no wall logic).
template <class S, class C, int BC, int CM, bool WALLS>
__device__ __forceinline__ void abp_row(const SweepArgs<S, C>& P, int j, int k, int lane, int ia, bool valid) {
    typedef Faces<BC> F;
    const int nx = (int)P.nx, nxy = (int)P.nxy;
    const int c = nx * j + nxy * k + ia;
    const bool at_lo = ia == 1, at_hi = ia + 1 == P.l;
    const bool edge_lo = lane == 0 || at_lo, edge_hi = lane == 31 || at_hi;
    const int oym = (F::PY && j == 1) ? (P.m - 1) * nx : -nx;
    const int oyp = (F::PY && j == P.m) ? (1 - P.m) * nx : nx;
    const bool zlo = k == 1 && !(P.zhalo & 1), zhi = k == P.n && !(P.zhalo & 2);   // slab faces: halo
    const int ozm = (F::PZ && zlo) ? (P.n - 1) * nxy : -nxy;
    const int ozp = (F::PZ && zhi) ? (1 - P.n) * nxy : nxy;
    const bool wym = WALLS && F::WY && j == 1, wyp = WALLS && F::WY && j == P.m;
    const bool wzm = WALLS && F::WZ && zlo, wzp = WALLS && F::WZ && zhi;
    // all loads first (no branch between them, so they are in flight
    // together): the pair word of every population and, for c_x != 0, the
    // one element the lane may need from outside its warp or across a face
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
        // a y/z wall (same for the whole warp): both nodes bounce back
        const S* src = wl ? P.a[opp_of(d)] + c : P.a[d] + off;
        w[d] = __ldg(reinterpret_cast<const unsigned*>(src));
        if (cx == 1) {
            const S* ep = (F::WX && at_lo) ? P.a[opp_of(d)] + c
                                           : P.a[d] + off + ((F::PX && at_lo) ? P.l - 1 : -1);
            e[d] = s_bits(ldro<S>(ep));
        } else if (cx == -1) {
            const S* ep = (F::WX && at_hi) ? P.a[opp_of(d)] + c + 1
                                           : P.a[d] + off + ((F::PX && at_hi) ? 2 - P.l : 2);
            e[d] = s_bits(ldro<S>(ep));
        }
    }
    // the final pair word of every population (storage representation)
    uint32_t wv[19];
#pragma unroll
    for (int d = 0; d < 18; ++d) {
        const int cx = cx_of(d);
        uint32_t v = w[d];
        if (cx == 1) {
            // node i + 1: low half; node i: lane t - 1's high half, or the edge value
            const uint32_t left = __shfl_up_sync(0xffffffffu, v, 1) >> 16;
            uint32_t lo = edge_lo ? e[d] : left;
            if (BC == BC_INFLOW && at_lo)
                lo = s_bits(P.inflow_s[d]);
            if (!wall[d]) v = __byte_perm(lo, v, 0x5410);
        } else if (cx == -1) {
            // node i: high half; node i + 1: lane t + 1's low half, or the edge value
            const uint32_t right = __shfl_down_sync(0xffffffffu, v, 1) & 0xffffu;
            const uint32_t hi = edge_hi ? e[d] : right;
            if (!wall[d]) v = __byte_perm(v, hi, 0x5432);
        }
        if (WALLS && BC == BC_DRIVEN && (d == 1 || d == 10) && zhi) {
            // lid term, rounded to storage: the packed word holds it exactly
            F2 f = raw_bits<S>(v);
            f.v.x = roundtrip<S, C>(d == 1 ? f.v.x + P.lid_force : f.v.x - P.lid_force);
            f.v.y = roundtrip<S, C>(d == 1 ? f.v.y + P.lid_force : f.v.y - P.lid_force);
            v = pack_bits<S>(f);
        }
        wv[d] = v;
    }
    wv[18] = *reinterpret_cast<const unsigned*>(P.a[18] + c);
    // collision on packed FP32 pairs; the words stay packed (converted for
    // the moments and again for the relaxation) and each result is stored
    // as soon as it is known
    auto xs = [&](int d) { return raw_bits<S>(wv[d]); };
    auto xp = [&](int d) { return raw_bits_again<S>(wv[d]); };
    auto ys = [&](int d, F2 y) {
        if (valid) *reinterpret_cast<unsigned*>((d < 18 ? P.b[d] : const_cast<S*>(P.a[18])) + c) = pack_bits<S>(y);
    };
    if constexpr (cm_fast(CM))
        bgk_collide_fast_f<F2, float, cm_generic(CM), Scaled<S>::value>(xs, xp, ys, P.fc, P.inv_scale);
    else
        bgk_collide_f<F2, float, cm_generic(CM), Scaled<S>::value>(xs, xp, ys, P.col, P.inv_scale);
    if (BC == BC_INFLOW && P.outflow_next && valid && at_hi) {
        // node l is the high half of this lane's pair: the next state's
        // outflow plane from the values just stored (plain loads: this
        // thread's own stores of this launch), as outflow_halo_kernel would
        // compute it at the next step
        const int cl = c + 1;
        C r[19];
#pragma unroll
        for (int d = 0; d < 18; ++d) r[d] = Conv<S, C>::raw(P.b[d][cl]);
        r[18] = Conv<S, C>::raw(P.a[18][cl]);
        C eq[5];
        outflow_eq<C, Scaled<S>::value>(r, P.inflow_cte1, P.col, P.inv_scale, eq);
#pragma unroll
        for (int e = 0; e < 5; ++e) P.b[9 + e][cl + 1] = Conv<S, C>::pack(eq[e]);
    }
}

template <class S, class C, int BC, int CM, bool OBS>
__global__ void __launch_bounds__(kPairThreads, kPairBlocks) sweep_abp_kernel(const SweepArgs<S, C> P) {
    static_assert(sizeof(S) == 2 && sizeof(C) == 4, "pair sweep: 16-bit storage, float compute");
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
    if (OBS && P.obs != nullptr && j >= P.jmin - 1 && j <= P.jmax + 1 && k >= P.kmin - 1 && k <= P.kmax + 1 &&
        seg * 64 + 64 >= P.imin - 1 && seg * 64 + 1 <= P.imax + 1) {
        // the warp's 64 nodes touch the obstacle's box grown by one node:
        // the one-node rules (solid nodes skipped, links into solids bounced)
        double m5[5];
        if (valid) {
            sweep_at<S, C, BC, int, CM, true>(P, ia, j, k, m5);
            sweep_at<S, C, BC, int, CM, true>(P, ia + 1, j, k, m5);
        }
        return;
    }
    // the driven cavity's rows inside its walls run without wall logic
    // (measured +12 % at 256^3); for the channel the split costs registers
    // (spills) and runs slower, so every channel row takes the wall path
    const bool wall_row = (F::WY && (j == 1 || j == P.m)) ||
                          (F::WZ && ((k == 1 && !(P.zhalo & 1)) || (k == P.n && !(P.zhalo & 2))));
    if (BC != BC_DRIVEN || wall_row) abp_row<S, C, BC, CM, true>(P, j, k, lane, ia, valid);
    else abp_row<S, C, BC, CM, false>(P, j, k, lane, ia, valid);
}

// Outflow halo plane for the inflow case: a10..a14(l+1, j, k) from the
// moments of node (l, j, k) at rho = 1 (SRC/bcond.inflow.F90:135-162), over
// j = 1..m, k = 1..n (the sweep reads the y/z-wrapped position, which is
// always one of these).
template <class S, class C>
__global__ void outflow_halo_kernel(const SweepArgs<S, C> P) {
    const int j = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int k = 1 + (int)blockIdx.y;
    if (j > P.m) return;
    const long long c = (long long)P.l + P.nx * (long long)j + P.nxy * (long long)k;
    C a[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) a[d] = Conv<S, C>::raw(P.a[d][c]);
    C eq[5];
    outflow_eq<C, Scaled<S>::value>(a, P.inflow_cte1, P.col, P.inv_scale, eq);
    const long long h = c + 1;
    S** A = const_cast<S**>(P.a);
#pragma unroll
    for (int e = 0; e < 5; ++e) A[9 + e][h] = Conv<S, C>::pack(eq[e]);
}

}  // namespace bgk
