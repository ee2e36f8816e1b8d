// FP64 global reductions over a lattice: per-node quantities in the compute
// type (as the reference computes them), accumulated in double with warp
// shuffles, a shared-memory block stage and a deterministic second pass over
// the per-block partials (fixed order, so repeated calls give identical bits).
#pragma once
#include "d3q19.cuh"

namespace bgk {

template <class S, class C> struct FieldArgs {
    const S* a[19];
    long long nx, nxy;
    int l, m, n;
    C cte1;
    float inv_scale;
    const int* obs;      // optional: nodes with obs==1 are skipped
    long long obs_nx, obs_nxy;
    int imin, imax, jmin, jmax, kmin, kmax;   // obstacle bbox
};

template <int NQ>
__device__ __forceinline__ void block_reduce_store(double (&v)[NQ], double* partial) {
    __shared__ double sm[32][NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nw = (nthr + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) sm[warp][q] = v[q];
    __syncthreads();
    if (tid == 0) {
        const long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
        for (int q = 0; q < NQ; ++q) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += sm[w][q];
            partial[bid * NQ + q] = s;
        }
    }
}

// Fused second pass of a time-step launch with moments (1-D blocks): every
// block writes one record of NQ sums (block_reduce_store, thread 0), then
// the last block of each group of kTicketGroup consecutive blocks to finish
// (one ticket counter per group) sums its group's records in index order into
// a group record, and the last group to finish sums the group records in
// index order into out[0..NQ-1].  Which block finishes last changes
// nothing: every sum has a fixed order.  It saves the separate finalize
// launch (about 7 us per 256^3 step).  One record per warp instead, with a
// ticket per warp and three levels, measured 8 % slower: each warp's fence
// and atomic delayed its exit.
// Workspace (fused_ws): the counters first, sized for the largest launch of
// the lattice's shape (a launch's own block count follows the arrays'
// alignment), then the block and group records.  The counters are zero
// before a launch, and every completed launch leaves them zero.
constexpr unsigned kTicketGroup = 64;
__host__ __device__ inline long long fused_groups(long long nblocks) {
    return (nblocks + kTicketGroup - 1) / kTicketGroup;
}
struct FusedWs {
    unsigned* tickets;
    double* records;
};
inline size_t fused_ticket_bytes(long long nb_max) {
    return (size_t)((fused_groups(nb_max) + 1) * sizeof(unsigned) + 7) / 8 * 8;
}
inline size_t fused_workspace_bytes(long long nb_max, int nq) {
    return fused_ticket_bytes(nb_max) + (size_t)(nb_max + fused_groups(nb_max)) * nq * sizeof(double);
}
inline FusedWs fused_ws(void* ws, long long nb_max) {
    FusedWs f;
    f.tickets = static_cast<unsigned*>(ws);
    f.records = reinterpret_cast<double*>(static_cast<char*>(ws) + fused_ticket_bytes(nb_max));
    return f;
}
template <int NQ>
__device__ __forceinline__ void finalize_by_tickets(double* partial, double* out, unsigned* tickets) {
    if (threadIdx.x >= 32) return;   // warp 0; its thread 0 wrote this block's record
    const unsigned lane = threadIdx.x;
    const unsigned nb = gridDim.x, g = blockIdx.x / kTicketGroup, ng = (nb + kTicketGroup - 1) / kTicketGroup;
    const unsigned g0 = g * kTicketGroup, gn = min(nb - g0, kTicketGroup);
    unsigned last = 0;
    if (lane == 0) {
        __threadfence();   // the record before the ticket
        last = atomicAdd(&tickets[g], 1u) == gn - 1 ? 1u : 0u;
    }
    if (!__shfl_sync(0xffffffffu, last, 0)) return;
    __threadfence();
    double v[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    // the group: lane t adds records g0 + t and g0 + t + 32, then a shuffle tree
    if (lane < gn)
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] = __ldcg(partial + (size_t)(g0 + lane) * NQ + q);
    if (lane + 32 < gn)
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] += __ldcg(partial + (size_t)(g0 + lane + 32) * NQ + q);
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partial[(size_t)(nb + g) * NQ + q] = v[q];
        tickets[g] = 0;    // every block of the group has taken its ticket
        __threadfence();   // the group record before the ticket
        last = atomicAdd(&tickets[ng], 1u) == ng - 1 ? 1u : 0u;
    }
    if (!__shfl_sync(0xffffffffu, last, 0)) return;
    __threadfence();
    // all groups: lane t adds group records t, t + 32, ... in order, then the tree
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    for (unsigned r = lane; r < ng; r += 32)
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] += __ldcg(partial + (size_t)(nb + r) * NQ + q);
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) out[q] = v[q];
        tickets[ng] = 0;
    }
}

// The warp segments [beg, end) that block blockIdx.x of a time-step launch
// that also sums moments advances (the grid of mom_plan): the contiguous run
// of span segments from blockIdx.x * span.  The block's warps interleave
// (warp w takes beg + w, beg + w + 8, ...), so neighbouring segments, which
// share the DRAM sectors of their c_x = +-1 links, run at about the same
// time.  (A grid stride over the whole lattice let the warps drift apart:
// measured 13 % slower than the step without moments at 256^3 FP32.)
struct SegRun {
    uint32_t beg, end;
};
__device__ __forceinline__ SegRun block_segments(uint32_t nwarps, uint32_t span) {
    const unsigned long long beg = (unsigned long long)span * blockIdx.x, end = beg + span;
    SegRun r;
    r.beg = (uint32_t)(beg < nwarps ? beg : nwarps);
    r.end = (uint32_t)(end < nwarps ? end : nwarps);
    return r;
}

// Per-node diagnostics of SRC/diagno.F90:112-127 (rho, u in the compute
// type) accumulated into FP64: v += {rho, u_x, u_y, u_z, 0.5|u|^2}.
template <class C>
__device__ __forceinline__ void diagno_node(const C (&x)[19], C cte1, double (&v)[5]) {
    const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] +
                  x[11] + x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + cte1;
    const C rhoinv = C(1) / rho;
    const C xj = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
    const C yj = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
    const C zj = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
    v[0] += (double)rho;
    v[1] += (double)xj;
    v[2] += (double)yj;
    v[3] += (double)zj;
    v[4] += (double)(C(0.5) * (xj * xj + yj * yj + zj * zj));
}

template <class S, class C>
__device__ __forceinline__ bool is_solid(const FieldArgs<S, C>& P, int i, int j, int k) {
    if (P.obs == nullptr || i < P.imin || i > P.imax || j < P.jmin || j > P.jmax || k < P.kmin ||
        k > P.kmax)
        return false;
    return P.obs[(long long)(i - 1) + P.obs_nx * (j - 1) + P.obs_nxy * (k - 1)] == 1;
}

// Per-node rho, u and 0.5|u|^2 of the stored (post-collision) state, the
// arithmetic of SRC/diagno.F90:112-127.  Sums over fluid nodes.
// grid = (ceil(l/TX), ceil(m/TY), KB); blocks stride over k.
template <class S, class C>
__global__ void __launch_bounds__(256) moments_partial_kernel(const FieldArgs<S, C> P, double* partial) {
    const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    double v[5] = {0, 0, 0, 0, 0};
    if (i <= P.l && j <= P.m) {
        for (int k = 1 + (int)blockIdx.z; k <= P.n; k += (int)gridDim.z) {
            if (is_solid(P, i, j, k)) continue;
            const long long c = (long long)i + P.nx * (long long)j + P.nxy * (long long)k;
            C x[19];
#pragma unroll
            for (int d = 0; d < 19; ++d) x[d] = Conv<S, C>::ld(P.a[d][c], P.inv_scale);
            diagno_node<C>(x, P.cte1, v);
        }
    }
    block_reduce_store<5>(v, partial);
}

// Momentum-exchange force on the obstacle, SRC/draglift.F90:77-176:
// F_a = sum over fluid nodes x in the box of sum_p 2 c_pa a_p(x) obs(x + c_p).
// grid covers the box; one node per thread.
template <class S, class C>
__global__ void __launch_bounds__(256) draglift_partial_kernel(const FieldArgs<S, C> P, int is, int js,
                                                               int ks, int ni, int nj, int nk,
                                                               double* partial) {
    double v[3] = {0, 0, 0};
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long tot = (long long)ni * nj * nk;
    if (t < tot) {
        const int i = is + (int)(t % ni);
        const int j = js + (int)((t / ni) % nj);
        const int k = ks + (int)(t / ((long long)ni * nj));
        if (i >= 1 && i <= P.l && j >= 1 && j <= P.m && k >= 1 && k <= P.n && !is_solid(P, i, j, k)) {
            const long long c = (long long)i + P.nx * (long long)j + P.nxy * (long long)k;
            C ap[18];
            C ob[18];
#pragma unroll
            for (int d = 0; d < 18; ++d) {
                ap[d] = Conv<S, C>::ld(P.a[d][c], P.inv_scale);
                ob[d] = is_solid(P, i + cx_of(d), j + cy_of(d), k + cz_of(d)) ? C(1) : C(0);
            }
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                C s = C(0);
#pragma unroll
                for (int d = 0; d < 18; ++d) {
                    const int cc = ax == 0 ? cx_of(d) : (ax == 1 ? cy_of(d) : cz_of(d));
                    const C term = C(2.0) * (C)cc * ap[d] * ob[d];
                    s = (d == 0) ? term : s + term;
                }
                v[ax] = (double)s;
            }
        }
    }
    block_reduce_store<3>(v, partial);
}

// Second pass: one block sums nparts partials of NQ values in a fixed order.
// Thread t adds partials t, t + T, t + 2T, ... in that order (T = 512, so
// that the eight records in flight fit in registers), eight records in
// flight at a time (the fused-moments sweep at 256^3 leaves ~8 K records:
// this pass is a few microseconds of latency, two rounds of loads); then the
// threads' sums are combined by a fixed shuffle tree and the warps' in warp
// order.
constexpr int kFinalizeThreads = 512;
template <int NQ>
__global__ void __launch_bounds__(kFinalizeThreads) finalize_partials_kernel(const double* partial, long long nparts,
                                                                             double* out) {
    constexpr int T = kFinalizeThreads, U = 8;
    __shared__ double sm[T / 32][NQ];
    double v[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    long long p = threadIdx.x;
    for (; p + (U - 1) * (long long)T < nparts; p += U * (long long)T) {
        double t[U][NQ];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < NQ; ++q) t[u][q] = partial[(p + u * (long long)T) * NQ + q];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < NQ; ++q) v[q] += t[u][q];
    }
    for (; p < nparts; p += T)
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] += partial[p * NQ + q];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) sm[warp][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double s2 = 0.0;
            for (int w = 0; w < T / 32; ++w) s2 += sm[w][q];
            out[q] = s2;
        }
}

}  // namespace bgk
