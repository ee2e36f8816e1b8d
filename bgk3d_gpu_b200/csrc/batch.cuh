// Batched time step: many independent lattices of different extents,
// boundary cases and collision parameters advanced by ONE persistent launch.
//
// Work is cut into tiles of 8 row segments (256 nodes, one block's worth in
// the single-lattice sweep).  Tiles of all lattices are numbered
// consecutively (tile_begin[L] is lattice L's first tile); a persistent grid
// of blocks takes `sub` consecutive tiles at a time from a device counter
// (the tile queue), finds the tile's lattice by binary search, stages that
// lattice's kernel arguments in shared memory, and runs the same per-node
// code as sweep_ab_kernel for the lattice's boundary case.  The last block
// to finish resets the counter, so the next launch (or graph replay) starts
// from an empty queue with no host intervention.
#pragma once
#include "sweep_ab.cuh"

namespace bgk {

template <class S, class C> struct BatchView {
    const SweepArgs<S, C>* desc;   // 2 per lattice: [2 L + parity], parity 1 = a/b swapped
    const uint32_t* tile_begin;    // nlat + 1 entries
    int nlat;
    uint32_t ntiles;
    unsigned* counter;             // [0] next tile, [1] blocks finished
    int parity;
    int sub;                       // tiles taken per queue access
};

// One node of the tile's lattice: boundary case and collision mode chosen at
// run time (the obstacle test is always compiled in, P.obs decides).
template <class S, class C, int BC>
__device__ __forceinline__ void batch_node_bc(const SweepArgs<S, C>& P, uint32_t gw, double (&m5)[5]) {
    const int cm = P.generic + (sizeof(C) == 4 ? 2 * P.fast : 0);
    switch (cm) {
        case CM_STRICT: sweep_node<S, C, BC, int, CM_STRICT, true>(P, gw, m5); break;
        case CM_STRICT_GENERIC: sweep_node<S, C, BC, int, CM_STRICT_GENERIC, true>(P, gw, m5); break;
        case CM_FAST:
            if constexpr (sizeof(C) == 4) sweep_node<S, C, BC, int, CM_FAST, true>(P, gw, m5);
            break;
        default:
            if constexpr (sizeof(C) == 4) sweep_node<S, C, BC, int, CM_FAST_GENERIC, true>(P, gw, m5);
            break;
    }
}

template <class S, class C>
__device__ __forceinline__ void batch_node(const SweepArgs<S, C>& P, uint32_t gw) {
    double m5[5];
    switch (P.bcase) {
        case BC_DRIVEN: batch_node_bc<S, C, BC_DRIVEN>(P, gw, m5); break;
        case BC_PERIODIC: batch_node_bc<S, C, BC_PERIODIC>(P, gw, m5); break;
        case BC_CHANNEL: batch_node_bc<S, C, BC_CHANNEL>(P, gw, m5); break;
        case BC_INFLOW: batch_node_bc<S, C, BC_INFLOW>(P, gw, m5); break;
        default: break;
    }
}

template <class S, class C>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 3 : 4) batch_sweep_kernel(const BatchView<S, C> V) {
    __shared__ __align__(16) SweepArgs<S, C> sd;
    __shared__ uint32_t s_tile;
    __shared__ int s_lat;
    int cur = -1;
    const uint32_t warp = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(V.counter, (unsigned)V.sub);
        __syncthreads();
        const uint32_t t0 = s_tile;
        if (t0 >= V.ntiles) break;
        const uint32_t t1 = min(t0 + (uint32_t)V.sub, V.ntiles);
        for (uint32_t t = t0; t < t1; ++t) {
            if (threadIdx.x == 0) {
                int lo = 0, hi = V.nlat - 1;   // last L with tile_begin[L] <= t
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldg(V.tile_begin + mid) <= t) lo = mid; else hi = mid - 1;
                }
                s_lat = lo;
            }
            __syncthreads();
            const int L = s_lat;
            if (L != cur) {
                const uint32_t* src = reinterpret_cast<const uint32_t*>(V.desc + 2 * L + V.parity);
                uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
                for (uint32_t w = threadIdx.x; w < sizeof(SweepArgs<S, C>) / 4; w += blockDim.x) dst[w] = __ldg(src + w);
                cur = L;
                __syncthreads();
            }
            batch_node<S, C>(sd, (t - __ldg(V.tile_begin + L)) * 8u + warp);
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned done = atomicAdd(V.counter + 1, 1u);
        if (done == gridDim.x - 1) {   // every block has left the queue
            V.counter[0] = 0u;
            V.counter[1] = 0u;
            __threadfence();
        }
    }
}

// Non-persistent variant: one block per tile (the hardware block scheduler is
// the queue); the tile's lattice is found by every thread, and its kernel
// arguments are read through the L1 cache.
template <class S, class C>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 3 : 4) batch_grid_kernel(const BatchView<S, C> V) {
    const uint32_t t = blockIdx.x;
    int lo = 0, hi = V.nlat - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(V.tile_begin + mid) <= t) lo = mid; else hi = mid - 1;
    }
    const SweepArgs<S, C>& P = V.desc[2 * lo + V.parity];
    batch_node<S, C>(P, (t - __ldg(V.tile_begin + lo)) * 8u + (threadIdx.x >> 5));
}

// Grouped form (the default): the members that share a boundary case,
// collision mode and obstacle logic form a group, and each group is one
// launch of a kernel compiled for exactly that variant -- no run-time
// dispatch, no obstacle code in obstacle-free groups.  The host cuts every
// member's step into chunks of chunk_warps consecutive warp segments and
// lists them (member, first warp) in a table, so a block finds its work with
// one load: it stages the member's kernel arguments in shared memory (the
// block's only barrier) and its 8 warps then stride through the chunk's warp
// segments with the per-node code of sweep_ab_kernel.  The hardware block
// scheduler is the queue.
template <class S, class C> struct BatchGroupView {
    const SweepArgs<S, C>* desc;   // 2 per member of the batch: [2 member + parity]
    const uint2* chunks;           // (member, first warp segment) per chunk of this group
    int parity;
    uint32_t chunk_warps;          // warp segments per chunk
};

template <class S, class C, int BC, int CM, bool OBS>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 3 : 4) batch_chunk_kernel(const BatchGroupView<S, C> V) {
    __shared__ __align__(16) SweepArgs<S, C> sd;
    const uint2 ch = V.chunks[blockIdx.x];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(V.desc + 2 * ch.x + V.parity);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
    for (uint32_t w = threadIdx.x; w < sizeof(SweepArgs<S, C>) / 4; w += blockDim.x) dst[w] = __ldg(src + w);
    __syncthreads();
    double m5[5];
    const uint32_t end = min(ch.y + V.chunk_warps, sd.nwarps);
    for (uint32_t gw = ch.y + (threadIdx.x >> 5); gw < end; gw += 8u) sweep_node<S, C, BC, int, CM, OBS>(sd, gw, m5);
}

}  // namespace bgk
