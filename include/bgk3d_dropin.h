/*
 * bgk3d_dropin.h -- the reference's own native C ABI, re-implemented on the
 * B200 library.  libbgk3d_dropin_sp.so exports these symbols with
 * real_t = float, libbgk3d_dropin_dp.so (built with -DDOUBLE_P) with
 * real_t = double, exactly as SRC/col_MC_gpu.hpp:78-82 selects real_t.
 * A Fortran build links one of them in place of col_MC_cuda.o + bcond_cuda.o
 * (SRC/Makefile:587-595); the Fortran interfaces stay unchanged
 * (SRC/col_MC.F90:101-123, SRC/bcond_gpu_mod.F90:30-77).
 *
 * Semantics differ from the reference in HOW, not WHAT:
 *   * bcond_*_gpu records the boundary case and its parameters for the next
 *     col_mc_gpu call on the same host thread (no launch); col_mc_gpu then
 *     runs ONE fused launch (boundaries + stream + collide).  The fluid-node
 *     results are those of the reference's halo writes followed by its pull.
 *     The halo cells themselves are not written (except the outflow plane
 *     a10..a14(l+1,1..m,1..n) of the inflow case).
 *   * bcond_obs_gpu records the obstacle mask pointer and box; solid nodes
 *     are not updated (the reference writes racy values there).
 *   * col_mc_gpu checks that the recorded arrays are its a01..a19; on a
 *     mismatch it reports an error on stderr and applies no boundary.
 * All launches go to the legacy default stream, asynchronously, as in the
 * reference (SRC/col_MC_gpu.hpp:261-280).
 */
#ifndef BGK3D_DROPIN_H
#define BGK3D_DROPIN_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(DOUBLE_P) || defined(GPU_DOUBLE)
typedef double real_t;
#else
typedef float real_t;
#endif

/* SRC/col_MC_cuda.cu:16-29 */
void col_mc_gpu(const real_t* a01, const real_t* a02, const real_t* a03, const real_t* a04,
                const real_t* a05, const real_t* a06, const real_t* a07, const real_t* a08,
                const real_t* a09, const real_t* a10, const real_t* a11, const real_t* a12,
                const real_t* a13, const real_t* a14, const real_t* a15, const real_t* a16,
                const real_t* a17, const real_t* a18, const real_t* a19, real_t* b01, real_t* b02,
                real_t* b03, real_t* b04, real_t* b05, real_t* b06, real_t* b07, real_t* b08,
                real_t* b09, real_t* b10, real_t* b11, real_t* b12, real_t* b13, real_t* b14,
                real_t* b15, real_t* b16, real_t* b17, real_t* b18, int l, int m, int n, int nx,
                int ny, real_t omega, real_t cte0, real_t cte1, real_t p0, real_t p1, real_t p2,
                real_t rf, real_t qf, real_t tre, real_t forcex, real_t forcey, real_t forcez);

/* SRC/bcond_gpu.hpp:499-504 */
void bcond_periodic_gpu(real_t** a, int l, int m, int n, int nx, int ny);
/* SRC/bcond_gpu.hpp:506-511 */
void bcond_channel_gpu(real_t** a, int l, int m, int n, int nx, int ny);
/* SRC/bcond_gpu.hpp:513-519 */
void bcond_driven_gpu(real_t** a, int l, int m, int n, int nx, int ny, real_t force);
/* SRC/bcond_gpu.hpp:521-531 */
void bcond_inflow_gpu(real_t** a, int l, int m, int n, int nx, int ny, real_t u_inflow, real_t rf,
                      real_t qf, real_t tre, real_t p1, real_t p2, real_t cte1);
/* SRC/bcond_gpu.hpp:533-544 */
void bcond_obs_gpu(real_t** a, const int* obs, int l, int m, int n, int nx, int ny, int imin,
                   int imax, int jmin, int jmax, int kmin, int kmax, int obs_nx, int obs_ny);
/* SRC/bcond_gpu.hpp:548-571: device barrier, abort() on a device error */
void gpu_device_sync(void);

/* Not in the reference: drop any recorded boundary/obstacle state of the
   calling thread (e.g. after the caller re-allocates its arrays). */
void bgk_dropin_reset(void);

/* Not in the reference: with tracking on, every col_mc_gpu also sums the
   FP64 moments of the state it writes (rho, u_x, u_y, u_z, 0.5|u|^2 over
   the fluid nodes, the per-node arithmetic of SRC/diagno.F90), in the same
   launch; bgk_dropin_moments then copies the last call's sums to
   out_dev[0..4] (device memory, stream-ordered on `stream`) without reading
   the lattice again.  Returns 0, or BGK_ERR_STATE (-5) when the last
   col_mc_gpu was not a tracked step.  bgk_dropin_moments_ptr gives the
   device address of those five sums instead (NULL when there are none):
   they stay there until the next tracked col_mc_gpu of the calling thread,
   so a copy from it enqueued on the default stream before that call reads
   this step's values.  bgk_dropin_moments_to(dst) makes the next tracked
   col_mc_gpu of the calling thread write its five sums to dst[0..4]
   instead: device memory, or page-locked host memory (cudaHostAlloc /
   cudaMallocHost), which the launch writes directly, so a host-side series
   of per-step sums needs no copy at all (read it after the step completes);
   bgk_dropin_moments_ptr then returns dst. */
void bgk_dropin_track_moments(int on);
int bgk_dropin_moments(double* out_dev, void* stream);
const double* bgk_dropin_moments_ptr(void);
void bgk_dropin_moments_to(double* dst);

#ifdef __cplusplus
}
#endif
#endif /* BGK3D_DROPIN_H */
