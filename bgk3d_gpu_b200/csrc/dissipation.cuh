// FP64 reductions of the turbulence diagnostics: turbulent kinetic energy,
// the 2 nu Pi:Pi dissipation of the non-equilibrium stress, the mean squared
// velocity components (SRC/dissipation.F90:136-338) and the enstrophy
// 0.5 |curl u|^2 with central differences of the node velocities
// (SRC/vtk_om.xy.binary.F90:27-87 computes the vorticity this way).
//
// Per-node values are in the compute type, in the reference's operation
// order (the library is built with --fmad=false); the sums are FP64 (the
// reference accumulates these in mykind), per block and then over the
// blocks in a fixed order (finalize_partials_kernel), so repeated calls give
// identical bits.
#pragma once
#include "sweep_ab.cuh"
#include "reduce.cuh"

namespace bgk {

// Per-node terms of SRC/dissipation.F90:155-338 from the 19 pulled values
// x[] (physical units, compute type): v += {0.5 |u|^2, 2 nu Pi:Pi, u_x^2,
// u_y^2, u_z^2}.  The equilibrium is the generic form (cte0, cte1), exactly
// as the routine writes it.
template <class C>
__device__ __forceinline__ void dissipation_node(const C (&x)[19], const ColConst<C>& K, C two_nu,
                                                 double (&v)[5]) {
    const C cte0 = K.cte0, cte1 = K.cte1, qf = K.qf, tre = K.tre, rf = K.rf;
    const C p0 = K.p0, p1 = K.p1, p2 = K.p2;
    const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] + x[11] + x[12] +
                  x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + cte1;
    const C rhoinv = C(1) / rho;
    C vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
    C vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
    C vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
    const C vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    v[2] += (double)vx2;
    v[3] += (double)vy2;
    v[4] += (double)vz2;
    const C vsq = vx2 + vy2 + vz2;
    v[0] += (double)(C(0.5) * vsq);
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
    const C s2 = cte1 * (rp2 - p2), s1 = cte1 * (rp1 - p1), s0 = cte1 * (rp0 - p0);
    // non-equilibrium parts n_p = x_p - e_p, p = 01..18
    const C n01 = x[0] - (rp2 * (+vxmy + qxmy) + s2);
    const C n02 = x[1] - (rp2 * (+vxmz + qxmz) + s2);
    const C n03 = x[2] - (rp2 * (+vxpy + qxpy) + s2);
    const C n04 = x[3] - (rp2 * (+vxpz + qxpz) + s2);
    const C n05 = x[4] - (rp1 * (+vx + qx) + s1);
    const C n06 = x[5] - (rp1 * (+vz + qz) + s1);
    const C n07 = x[6] - (rp2 * (+vypz + qypz) + s2);
    const C n08 = x[7] - (rp1 * (+vy + qy) + s1);
    const C n09 = x[8] - (rp2 * (+vymz + qymz) + s2);
    const C n10 = x[9] - (rp2 * (-vxpy + qxpy) + s2);
    const C n11 = x[10] - (rp2 * (-vxpz + qxpz) + s2);
    const C n12 = x[11] - (rp2 * (-vxmy + qxmy) + s2);
    const C n13 = x[12] - (rp2 * (-vxmz + qxmz) + s2);
    const C n14 = x[13] - (rp1 * (-vx + qx) + s1);
    const C n15 = x[14] - (rp1 * (-vz + qz) + s1);
    const C n16 = x[15] - (rp2 * (-vypz + qypz) + s2);
    const C n17 = x[16] - (rp1 * (-vy + qy) + s1);
    const C n18 = x[17] - (rp2 * (-vymz + qymz) + s2);
    (void)q0; (void)s0;   // e19 enters no stress component
    const C Pxx = n01 + n02 + n03 + n04 + n05 + n10 + n11 + n12 + n13 + n14;
    const C Pyy = n01 + n03 + n07 + n08 + n09 + n10 + n12 + n16 + n17 + n18;
    const C Pzz = n02 + n04 + n06 + n07 + n09 + n11 + n13 + n15 + n16 + n18;
    const C Pxz = -n02 + n04 + n11 - n13;
    const C Pxy = -n01 + n03 + n10 - n12;
    const C Pyz = +n07 - n09 + n16 - n18;
    const C two = C(2);
    const C Ptotal = Pxx * Pxx + Pyy * Pyy + Pzz * Pzz + (two * Pxy * Pxy) + (two * Pxz * Pxz) + (two * Pyz * Pyz);
    v[1] += (double)(two_nu * Ptotal);
}

// One node per thread over (i, j) rows, blocks striding k (the moments
// grid): every fluid node pulls its 19 populations by the sweep's rules
// (gather_at: periodic wrap, wall bounce-back with the lid, inflow
// equilibrium, outflow halo, obstacle links), which is what the reference's
// pull reads after its boundary routines filled the halo; with BC_NONE the
// halo is read as stored.  Partial sums: 5 doubles per block.
// K: the collision constants in physical units (P.col carries the storage
// scale of the 16-bit kinds, which the pulled values lose first).
template <class S, class C, int BC, class IDX>
__global__ void __launch_bounds__(256) dissipation_partial_kernel(const SweepArgs<S, C> P, const ColConst<C> K,
                                                                  C two_nu, double* partial) {
    const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    double v[5] = {0, 0, 0, 0, 0};
    if (i <= P.l && j <= P.m) {
        for (int k = 1 + (int)blockIdx.z; k <= P.n; k += (int)gridDim.z) {
            C x[19];
            if (!gather_at<S, C, BC, IDX, true>(P, i, j, k, x)) continue;
            if (Scaled<S>::value) {
#pragma unroll
                for (int d = 0; d < 19; ++d) x[d] = x[d] * (C)P.inv_scale;
            }
            dissipation_node<C>(x, K, two_nu, v);
        }
    }
    block_reduce_store<5>(v, partial);
}

// Enstrophy: 0.5 |w|^2 summed over the nodes where the central differences
// exist, w = curl u with du_a/dx_b = 0.5 (u_a(x + e_b) - u_a(x - e_b)) and u
// the node velocity of the stored state (SRC/vtk_om.xy.binary.F90:49-87, in
// the compute type).  Periodic axes of the case wrap; along other axes the
// two face layers are left out (the reference's vorticity slices cover
// 2..l-1 and 2..m-1 only); nodes that are solid or have a solid neighbour
// are left out.  Tiles of 32 x 8 nodes march along k over chunks of
// kEnsChunk planes with the velocities of three planes (tile plus a one-node
// rim) in shared memory, so each population is read about 1.3 times.
// Partial sums per block: {sum 0.5 |w|^2, nodes counted}.
constexpr int kEnsTX = 32, kEnsTY = 8, kEnsChunk = 16;
constexpr int kEnsW = kEnsTX + 2, kEnsH = kEnsTY + 2;

// Grid of the enstrophy pass: tiles of kEnsTX x kEnsTY nodes, chunks of
// kEnsChunk planes.
inline dim3 enstrophy_grid(int l, int m, int n) {
    return dim3((l + kEnsTX - 1) / kEnsTX, (m + kEnsTY - 1) / kEnsTY, (n + kEnsChunk - 1) / kEnsChunk);
}

template <class S, class C, int BC>
__global__ void __launch_bounds__(kEnsTX * kEnsTY) enstrophy_partial_kernel(const FieldArgs<S, C> P, int zhalo,
                                                                            double* partial) {
    typedef Faces<BC> F;
    __shared__ C U[3][3][kEnsH][kEnsW];   // [component][plane slot][j][i]
    const int tid = threadIdx.x + kEnsTX * threadIdx.y;
    const int i0 = 1 + (int)blockIdx.x * kEnsTX, j0 = 1 + (int)blockIdx.y * kEnsTY;
    const int k0 = 1 + (int)blockIdx.z * kEnsChunk;
    const int k1 = min(k0 + kEnsChunk - 1, P.n);
    const bool pz = F::PZ && zhalo == 0;
    auto wrap = [](int c, int len, bool per) -> int {
        if (per) { if (c < 1) return c + len; if (c > len) return c - len; }
        return (c >= 1 && c <= len) ? c : 0;   // 0: outside, not needed by any counted node
    };
    auto load_plane = [&](int kp) {
        const int kk = wrap(kp, P.n, pz);
        const int slot = (kp + 3) % 3;
        for (int t = tid; t < kEnsW * kEnsH; t += kEnsTX * kEnsTY) {
            const int ii = t % kEnsW, jj = t / kEnsW;
            const int i = wrap(i0 - 1 + ii, P.l, F::PX), j = wrap(j0 - 1 + jj, P.m, F::PY);
            C u = C(0), v = C(0), w = C(0);
            if (i && j && kk && i0 - 1 + ii <= P.l + 1 && j0 - 1 + jj <= P.m + 1) {
                const long long c = (long long)i + P.nx * (long long)j + P.nxy * (long long)kk;
                C x[19];
#pragma unroll
                for (int d = 0; d < 19; ++d) x[d] = Conv<S, C>::ld(P.a[d][c], P.inv_scale);
                const C rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] +
                              x[11] + x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + P.cte1;
                const C rhoinv = C(1) / rho;
                u = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
                v = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
                w = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
            }
            U[0][slot][jj][ii] = u;
            U[1][slot][jj][ii] = v;
            U[2][slot][jj][ii] = w;
        }
    };
    const int ti = threadIdx.x, tj = threadIdx.y;
    const int i = i0 + ti, j = j0 + tj;
    const bool in_ij = i <= P.l && j <= P.m && (F::PX || (i >= 2 && i <= P.l - 1)) &&
                       (F::PY || (j >= 2 && j <= P.m - 1));
    double s[2] = {0.0, 0.0};
    if (k0 <= P.n) {
        load_plane(k0 - 1);
        load_plane(k0);
        for (int k = k0; k <= k1; ++k) {
            load_plane(k + 1);
            __syncthreads();
            bool in = in_ij && (pz || (k >= 2 && k <= P.n - 1));
            if (in && P.obs != nullptr) {
                const int im = wrap(i - 1, P.l, F::PX), ip = wrap(i + 1, P.l, F::PX);
                const int jm = wrap(j - 1, P.m, F::PY), jp = wrap(j + 1, P.m, F::PY);
                const int km = wrap(k - 1, P.n, pz), kp = wrap(k + 1, P.n, pz);
                in = !is_solid(P, i, j, k) && !is_solid(P, im, j, k) && !is_solid(P, ip, j, k) &&
                     !is_solid(P, i, jm, k) && !is_solid(P, i, jp, k) && !is_solid(P, i, j, km) &&
                     !is_solid(P, i, j, kp);
            }
            if (in) {
                const int sm = (k - 1 + 3) % 3, s0 = k % 3, sp = (k + 1) % 3;
                const int a = ti + 1, b = tj + 1;
                const C h = C(0.5);
                const C dudy = h * (U[0][s0][b + 1][a] - U[0][s0][b - 1][a]);
                const C dudz = h * (U[0][sp][b][a] - U[0][sm][b][a]);
                const C dvdx = h * (U[1][s0][b][a + 1] - U[1][s0][b][a - 1]);
                const C dvdz = h * (U[1][sp][b][a] - U[1][sm][b][a]);
                const C dwdx = h * (U[2][s0][b][a + 1] - U[2][s0][b][a - 1]);
                const C dwdy = h * (U[2][s0][b + 1][a] - U[2][s0][b - 1][a]);
                const C ox = dvdz - dwdy, oy = dwdx - dudz, oz = dudy - dvdx;
                s[0] += (double)(h * (ox * ox + oy * oy + oz * oz));
                s[1] += 1.0;
            }
            __syncthreads();
        }
    }
    block_reduce_store<2>(s, partial);
}

}  // namespace bgk
