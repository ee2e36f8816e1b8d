// TMA-staged, warp-specialised AB time step for library-owned lattices.
//
// The one-node kernel (sweep_ab_kernel) issues its 19 loads from registers:
// with the 16-bit kinds it runs out of issue slots and of loads in flight
// long before HBM does.  Here a persistent grid moves the populations with
// the Tensor Memory Accelerator instead: per tile of 64 x 8 nodes (one x
// segment of eight rows of one z plane) one producer thread issues 19 tiled
// bulk copies -- for population p the eight source rows j - c_y(p) of plane
// k - c_z(p), x from 16 bytes left of the tile to 16 bytes right of it --
// into a ring of shared-memory stages, and eight consumer warps (one per
// row) read the pulled values from shared memory at the x offset -c_x(p).  Each
// consumer thread advances two adjacent nodes with the packed FP32
// arithmetic of sm_100 (f2.cuh), which halves the collision's instructions
// per node; no register holds a load in flight, so the copies in flight are
// set by the ring depth, not by the occupancy that the wider registers cost.
// Float compute only (storage float, half, bfloat16); FP64 runs at the HBM
// roofline with the one-node kernel.
//
// Every tile is staged (box rows beyond the halo box read the fill value);
// the consumers advance the interior nodes, and the nodes on the six faces
// of the lattice -- the only ones with links through a face -- are advanced
// by sweep_faces_kernel, one thread each, by the one-node rules (periodic
// wrap, wall bounce, lid, inflow equilibrium, outflow halo), so every result
// is bit-identical to sweep_ab_kernel's.  Lattices with an
// obstacle, and steps with fused moments, use sweep_ab_kernel.
//
// Tensor map: the whole allocation as a 4-D array (x: row pitch nx, y: m + 2,
// z: n + 2, w: population plane), so one map serves both arrangements of the
// AB ping-pong; node (i, j, k) of plane q is at (31 + i, j, k, q).  Every box
// starts at an x coordinate that is a multiple of 16 bytes, as TMA requires.
// Waits on the pipeline barriers are bounded: a wait that gives up sets
// *err and the kernel returns.
#pragma once
#include <cuda.h>
#include "f2.cuh"
#include "sweep_ab.cuh"

namespace bgk {

constexpr int kTmaRows = 8;      // rows per tile (one consumer warp per row)
constexpr int kTmaConsumers = 8; // consumer warps (two nodes per thread)
constexpr int kTmaThreads = 32 * (1 + kTmaConsumers);
constexpr int kTmaOrigin = 31;   // x coordinate of node 0 (library layout)

template <class S> struct TmaBox {
    static constexpr int A = 16 / (int)sizeof(S);                 // 16-byte margin, elements
    static constexpr int W = 64 + 2 * A;                          // box width, elements
    static constexpr int BYTES = W * kTmaRows * (int)sizeof(S);   // one population's box
    // ring depth and resident blocks per SM: under 100 KB of stages per
    // block, two blocks (16 consumer warps) per SM
    static constexpr int STAGES = sizeof(S) == 2 ? 4 : 2;
    static constexpr int MIN_BLOCKS = 2;
    static constexpr size_t SMEM = (size_t)STAGES * 19 * BYTES + 2 * STAGES * sizeof(uint64_t) + 128;
};

struct TmaSched {
    int pa[19];          // tensor-map plane of a[d] in this step's arrangement
    int ntx, nty;        // tiles along x (64 nodes) and y (kTmaRows rows)
    uint32_t ntiles;     // ntx * nty * n
    int* err;            // set to 1 by a wait that gives up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the completion of the barrier phase with the given
// parity: try_wait suspends the thread for up to about a microsecond per
// attempt; after about a second in all, *err = 1 and false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t n = 0; n < (1u << 20); ++n) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(1000u)
            : "memory");
        if (done) return true;
    }
    atomicExch(err, 1);
    return false;
}

// Tiled bulk copy of one box into shared memory, completion counted on bar.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

// Tile t -> x segment start x0 (0, 64, ...), first row j0, plane k.  Every
// tile is staged: box rows outside the halo box read the fill value, and the
// consumers take a face node's links from global memory.
__device__ __forceinline__ void tma_tile(const TmaSched& T, uint32_t t, int& x0, int& j0, int& k) {
    const uint32_t tx = t % (uint32_t)T.ntx, r = t / (uint32_t)T.ntx;
    const uint32_t ty = r % (uint32_t)T.nty;
    x0 = (int)tx * 64;
    j0 = (int)ty * kTmaRows + 1;
    k = (int)(r / (uint32_t)T.nty) + 1;
}

template <class S, class C, int BC, int CM>
__global__ void __launch_bounds__(kTmaThreads, TmaBox<S>::MIN_BLOCKS)
sweep_tma_kernel(const SweepArgs<S, C> P, const TmaSched T, const __grid_constant__ CUtensorMap map) {
    static_assert(sizeof(C) == 4 && sizeof(S) <= 4, "the TMA sweep serves float compute");
    typedef TmaBox<S> B;
    typedef Faces<BC> F;
    constexpr int kTmaStages = B::STAGES;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // ring of stages, each 19 boxes; 128-byte aligned
    unsigned char* ring = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)kTmaStages * 19 * B::BYTES);
    uint64_t* empty = full + kTmaStages;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTmaStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTmaConsumers);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == 0) {
        // producer: one thread issues the copies of the staged tiles
        if (lane != 0) return;
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
        uint32_t it = 0;
        for (uint32_t t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
            int x0, j0, k;
            tma_tile(T, t, x0, j0, k);
            const int s = (int)(it % kTmaStages);
            const uint32_t use = it / kTmaStages;
            if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1u, T.err)) return;
            mbar_expect_tx(&full[s], 19u * B::BYTES);
            unsigned char* st = ring + (size_t)s * 19 * B::BYTES;
#pragma unroll
            for (int d = 0; d < 19; ++d)
                tma_load_4d(st + (size_t)d * B::BYTES, &map, kTmaOrigin + 1 + x0 - B::A, j0 - cy_of(d),
                            k - cz_of(d), T.pa[d], &full[s]);
            ++it;
        }
        // the last copies issued have been consumed before the consumers
        // finish; wait for them (bounded) so that none is in flight at exit
        for (uint32_t q = it > kTmaStages ? it - kTmaStages : 0; q < it; ++q)
            if (!mbar_wait(&full[q % kTmaStages], (q / kTmaStages) & 1u, T.err)) return;
        return;
    }

    // consumers: nodes (x0 + 1 + 2q, x0 + 2 + 2q) of row j0 + r, plane k
    typedef Pack2<S> PK;
    typedef Conv<S, float> CV;
    const int tid = threadIdx.x - 32;
    const int r = tid >> 5, lx0 = 2 * (tid & 31);
    constexpr int BOXE = B::BYTES / (int)sizeof(S);
    uint32_t it = 0;
    for (uint32_t t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
        int x0, j0, k;
        tma_tile(T, t, x0, j0, k);
        const int i0 = x0 + 1 + lx0, i1 = i0 + 1, j = j0 + r;
        const int s = (int)(it % kTmaStages);
        if (!mbar_wait(&full[s], (it / kTmaStages) & 1u, T.err)) return;
        // element of node i0's own position in population 0's box (even: the
        // 2-element reads of c_x = 0 populations are aligned)
        const S* base = reinterpret_cast<const S*>(ring + (size_t)s * 19 * B::BYTES) + r * B::W + B::A + lx0;
        F2 x[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) {
            const S* q = base + d * BOXE - cx_of(d);
            if (cx_of(d) == 0) x[d] = PK::raw(*reinterpret_cast<const typename PK::V*>(q));
            else x[d] = F2(CV::raw(q[0]), CV::raw(q[1]));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        ++it;
        if (i0 > P.l || j > P.m || j == 1 || j == P.m || k == 1 || k == P.n) continue;
        // nodes on a face of the lattice are advanced by sweep_faces_kernel
        const bool f0 = i0 == 1 || i0 == P.l, f1 = i1 > P.l || i1 == P.l;
        if (f0 && f1) continue;
        F2 y[19];
        if constexpr (cm_fast(CM))
            bgk_collide_fast_v<F2, float, cm_generic(CM), Scaled<S>::value>(x, y, P.fc, P.inv_scale);
        else
            bgk_collide_v<F2, float, cm_generic(CM), Scaled<S>::value>(x, y, P.col, P.inv_scale);
        const int c0 = i0 + (int)P.nx * j + (int)P.nxy * k;
        if (!f0 && !f1) {
#pragma unroll
            for (int d = 0; d < 18; ++d) *reinterpret_cast<typename PK::V*>(P.b[d] + c0) = PK::pack(y[d]);
            *reinterpret_cast<typename PK::V*>(const_cast<S*>(P.a[18]) + c0) = PK::pack(y[18]);
        } else {
            // one node of the pair lies on an x face: store the other one
            const int c = f0 ? c0 + 1 : c0;
#pragma unroll
            for (int d = 0; d < 18; ++d) P.b[d][c] = f0 ? PK::hi(PK::pack(y[d])) : PK::lo(PK::pack(y[d]));
            const_cast<S*>(P.a[18])[c] = f0 ? PK::hi(PK::pack(y[18])) : PK::lo(PK::pack(y[18]));
        }
    }
}

// The nodes on the six faces of the lattice (i in {1, l}, j in {1, m} or k in
// {1, n}), one thread each, by the one-node rules; with sweep_tma_kernel this
// completes a time step.  Order: the planes k = 1 and k = n, then the rows
// j = 1 and j = m of the other planes, then the nodes i = 1 and i = l of the
// remaining rows.
template <class S, class C, int BC, int CM>
__global__ void __launch_bounds__(256) sweep_faces_kernel(const SweepArgs<S, C> P) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long l = P.l, m = P.m, n = P.n;
    const long long nk = (n > 1 ? 2 : 1) * l * m;                 // planes k = 1, n
    const long long ni = n > 2 ? n - 2 : 0;                      // inner planes
    const long long nj = (m > 1 ? 2 : 1) * l * ni;                // rows j = 1, m
    const long long mj = m > 2 ? m - 2 : 0;
    const long long nx = (l > 1 ? 2 : 1) * mj * ni;               // nodes i = 1, l
    int i, j, k;
    if (t < nk) {
        const long long q = t % (l * m);
        i = (int)(q % l) + 1; j = (int)(q / l) + 1; k = t < l * m ? 1 : (int)n;
    } else if (t < nk + nj) {
        const long long u = t - nk, q = u % (l * ni);
        i = (int)(q % l) + 1; k = (int)(q / l) + 2; j = u < l * ni ? 1 : (int)m;
    } else if (t < nk + nj + nx) {
        const long long u = t - nk - nj, q = u % (mj * ni);
        j = (int)(q % mj) + 2; k = (int)(q / mj) + 2; i = u < mj * ni ? 1 : (int)l;
    } else {
        return;
    }
    double m5[5];
    sweep_at<S, C, BC, int, CM, false>(P, i, j, k, m5);
}

}  // namespace bgk
