/*
 * bgk3d_b200.h -- C ABI of the B200 D3Q19 BGK time-step library
 * (libbgk3d_b200.so).  Plain pointers and sizes only; all array arguments are
 * DEVICE pointers unless a parameter name ends in _host.
 *
 * Layout contract (the reference's, SRC/alloca.F90:153-191): every population
 * p = 01..19 is its own array (0:l+1+ipad, 0:m+1+jpad, 0:n+1) with i fastest;
 * element (i,j,k) is at i + nx*j + nx*ny*k, nx = l+2+ipad, ny = m+2+jpad.
 * Populations are stored shifted by their weight (f_p - w_p) when cte1 = 1.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   bgk_sweep      <- col_mc_gpu        SRC/col_MC_cuda.cu:16-53 together with
 *                     bcond_*_gpu       SRC/bcond_gpu.hpp:499-544 (boundaries
 *                                       fused into the same launch)
 *   bgk_moments    <- diagno            SRC/diagno.F90:87-138 (host/OpenACC
 *                                       reduction in the reference)
 *   bgk_draglift   <- draglift          SRC/draglift.F90:77-181
 *   bgk_dissipation<- dissipation       SRC/dissipation.F90:25-350 (TKE and
 *                                       2 nu Pi:Pi), plus the enstrophy of
 *                                       the vorticity of SRC/vtk_om.xy.binary.F90
 *   bgk_profile    <- prof_i/_j/_k      SRC/prof_k.F90:47-87 (host loops
 *                                       after a full-state copy in the reference)
 *   bgk_probe      <- probe             SRC/probe.F90:50-78
 *   bgk_slice      <- vtk_xy/xz/yz_bin  SRC/vtk_xy.binary.F90:78-97
 *   bgk_device_sync<- gpu_device_sync   SRC/bcond_gpu.hpp:548-571
 * The reference-named drop-in symbols themselves are declared in
 * bgk3d_dropin.h.
 *
 * Every function returns BGK_OK (0) or a negative status; bgk_last_error()
 * returns a message for the calling thread's last failure.
 */
#ifndef BGK3D_B200_H
#define BGK3D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#include <stddef.h>
#include <stdint.h>

#define BGK_OK 0
#define BGK_ERR_ARG (-1)
#define BGK_ERR_CUDA (-2)
#define BGK_ERR_UNSUPPORTED (-3)
#define BGK_ERR_NOMEM (-4)
#define BGK_ERR_STATE (-5)

/* storage / compute precision (SRC/precision.F90:14-47) */
#define BGK_KIND_F64 0     /* DOUBLE: f64 storage, f64 collision               */
#define BGK_KIND_F32 1     /* SINGLE: f32 storage, f32 collision               */
#define BGK_KIND_F16 2     /* f - w stored as binary16 (x scale), f32 collision */
#define BGK_KIND_BF16 3    /* f - w stored as bfloat16 (x scale), f32 collision */
#define BGK_KIND_F32_F64 4 /* MIXED2: f32 storage, f64 collision               */

/* boundary case (SRC/boundaries.F90:31-43) */
#define BGK_BC_NONE (-1)   /* halos are left as the caller prepared them */
#define BGK_BC_DRIVEN 0    /* six bounce-back walls, moving lid at z = n+1 */
#define BGK_BC_PERIODIC 1
#define BGK_BC_CHANNEL 2   /* x, y periodic; z no-slip walls */
#define BGK_BC_INFLOW 3    /* x: inflow at 0 / outflow at l+1; y, z periodic */

typedef struct bgk_sweep_params {
    int kind;                 /* BGK_KIND_* */
    int bcase;                /* BGK_BC_* */
    int l, m, n;              /* interior extents */
    long long nx, ny;         /* leading dimensions of each population array */
    /* collision constants, SRC/col_MC_gpu.hpp:86-94 (bgk_sweep_params_init
       fills the reference's values) */
    double omega, cte0, cte1, p0, p1, p2, rf, qf, tre;
    int force_mode;           /* 0: constant forces (native ABI); 1: force*rho (CHANNEL) */
    double fx, fy, fz;
    double lid_force;         /* DRIVEN: u00/6 (SRC/bcond.driven.F90:61) */
    double u_inflow;          /* INFLOW: prescribed u_x at x = 0 */
    double inflow_cte1;       /* INFLOW equilibrium constant: 0 for shifted storage */
    float scale;              /* 16-bit kinds: power-of-two storage scale */
    const int32_t* obs;       /* optional obstacle mask (1:l,1:m,1:n), obs==1 solid */
    int obs_nx, obs_ny;       /* its leading dimensions (normally l, m) */
    int imin, imax, jmin, jmax, kmin, kmax;  /* bounding box of the solid nodes */
    int fast;                 /* 0: the reference's operation order, bit-exact (default);
                                 1: fused multiply-adds and a regrouped equilibrium for
                                 float compute (kinds F32, F16, BF16): fewer instructions,
                                 results within a few units in the last place per step.
                                 Ignored for double compute. */
    int zhalo;                /* z faces that read the halo plane as stored (a slab of a
                                 lattice split along z; the planes k = 0 / n+1 hold the
                                 neighbour slab's populations): bit 0 the face k = 1, bit 1
                                 the face k = n.  Such a face has no wrap, wall or lid.
                                 0 (default): the case's own z rule at both faces. */
} bgk_sweep_params;

/* Fill *p with the reference's constants (p0 = 1/3, p1 = 1/18, p2 = 1/36,
   rf = tre = 3, qf = 1.5, cte1 = 1, cte0 = 0), no force, no obstacle,
   bcase NONE, scale 1, nx = l+2, ny = m+2, fast 0, zhalo 0. */
void bgk_sweep_params_init(bgk_sweep_params* p, int kind, int l, int m, int n, double omega);

/* One fused time step: boundary rules + pull-stream + BGK collision from the
   19 arrays a[] into b[0..17] and (in place) a[18].  b[18] is ignored.
   Stream-ordered, no synchronisation.  For BGK_BC_INFLOW it also writes the
   outflow halo plane a[9..13](l+1, 1..m, 1..n). */
int bgk_sweep(const bgk_sweep_params* p, void* const* a, void* const* b, void* stream);

/* bgk_sweep plus, in the same launch, the FP64 moments of the state it
   writes (the sums bgk_moments would return on that state, up to FP64
   summation order; the same bits on every run) into out_dev[0..4].
   Workspace: bgk_sweep_moments_workspace_bytes(p) bytes of device memory,
   no initialisation needed (per-block partial sums and the counters of
   their in-launch summation, which the call clears first); one workspace
   per stream of calls. */
size_t bgk_sweep_moments_workspace_bytes(const bgk_sweep_params* p);
int bgk_sweep_moments(const bgk_sweep_params* p, void* const* a, void* const* b, double* out_dev,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Bytes of device workspace bgk_moments / bgk_draglift need for a lattice of
   these extents (per-block FP64 partial sums). */
size_t bgk_reduce_workspace_bytes(int l, int m, int n);

/* FP64 sums over fluid nodes of rho, u_x, u_y, u_z, 0.5|u|^2 (per-node values
   computed as SRC/diagno.F90:112-127) into out_dev[0..4] (device memory).
   Uses p->kind, l, m, n, nx, ny, cte1, scale, obs/bbox.  Deterministic. */
int bgk_moments(const bgk_sweep_params* p, void* const* a, double* out_dev, void* workspace,
                size_t workspace_bytes, void* stream);

/* Allocation-free variant of bgk_moments.  No counterpart in the reference:
   for callers that cannot allocate device memory where they need the
   diagnostic (a Fortran/OpenACC driver whose device memory is owned by the
   directive runtime, a solver or server that reserves its whole memory budget
   up front and forbids allocation in its time loop).  The per-block partial
   sums live in a 2 MiB device array inside the library (bgk_moments_noalloc_
   max_bytes()), held on every GPU that loads the library until exit; the
   device address is looked up on the first call on each device (make that
   call before any stream capture) and kept until exit, so the entry point
   must not be used on a device after a cudaDeviceReset of it.  Lattices
   whose reduction needs more than 2 MiB (bgk_reduce_workspace_bytes(l, m, n)
   = 40 B x ceil(l/tx) x ceil(m/ty) x min(n, 64) blocks, tx x ty = 256, tx the
   smallest power of two >= l in 32..256: at most 52428 blocks, so 256^3 is
   served and 512^3 is not) are rejected with BGK_ERR_ARG.  Calls share the
   array: calls that overlap on the GPU race.  Results are identical to
   bgk_moments bit for bit (the same launches with the same grid). */
int bgk_moments_noalloc(const bgk_sweep_params* p, void* const* a, double* out_dev, void* stream);
size_t bgk_moments_noalloc_max_bytes(void);

/* FP64 turbulence diagnostics of the state in a (the routine dissipation of
   SRC/dissipation.F90:25-350, called by SRC/diagnostic.F90:103), into
   out_dev[0..6]:
     [0] sum 0.5 |u|^2           (tke,  :177)
     [1] sum 2 nu Pi:Pi          (diss, :338; Pi the non-equilibrium stress of
                                  the pulled populations, :180-335)
     [2..4] sum u_x^2, u_y^2, u_z^2   (vx2m, vy2m, vz2m, :172-174)
     [5] sum 0.5 |w|^2, w = curl u by central differences of the node
         velocities (the vorticity of SRC/vtk_om.xy.binary.F90:49-87)
     [6] number of nodes in [5]
   Sums over fluid nodes, per-node values in the compute type and the
   reference's operation order, accumulated in FP64 (the reference
   accumulates in mykind).  [0..4] pull every population from its upstream
   neighbour as the reference does (:136-154), with the boundary case of p
   resolved as bgk_sweep resolves it -- what the reference's pull reads
   right after its boundary routines -- or, for BGK_BC_NONE, the halo as
   stored; the inflow case writes the outflow halo plane first.  [5, 6]:
   periodic axes of the case wrap; along other axes the two face layers are
   left out; nodes that are solid or next to a solid are left out.  nu is
   the kinematic viscosity (svisc); the caller normalises as the reference
   writes dissipation.dat (divide by l m n u0^2).  Workspace:
   bgk_dissipation_workspace_bytes(l, m, n) bytes. */
size_t bgk_dissipation_workspace_bytes(int l, int m, int n);
int bgk_dissipation(const bgk_sweep_params* p, void* const* a, double nu, double* out_dev, void* workspace,
                    size_t workspace_bytes, void* stream);

/* FP64 momentum-exchange force (Fx, Fy, Fz, unnormalised) on the obstacle,
   summed over fluid nodes in the box [is..ie]x[js..je]x[ks..ke]
   (SRC/draglift.F90:77-176) into out_dev[0..2]. */
int bgk_draglift(const bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks,
                 int ke, double* out_dev, void* workspace, size_t workspace_bytes, void* stream);

/* Velocity and density along a grid line, computed on the device with the
   arithmetic of SRC/prof_k.F90:47-77 (prof_i, prof_j likewise): density =
   sum of the 19 stored values (storage arithmetic) + cte1 (1, compute type),
   velocity = momentum sum (storage arithmetic) / density (compute type).
   axis 0 runs i = 1..l at (j, k) = (c1, c2) (prof_i), 1 runs j = 1..m at
   (i, k) = (c1, c2) (prof_j), 2 runs k = 1..n at (i, j) = (c1, c2) (prof_k).
   out_dev: 4 doubles per node (u_x, u_y, u_z, rho); the reference writes
   them as (position, u_x, u_y, u_z, rho) with u_y its "w" and u_z its "v". */
int bgk_profile(const bgk_sweep_params* p, void* const* a, int axis, int c1, int c2, double* out_dev,
                void* stream);

/* Velocity and density at node (i, j, k) with the arithmetic of
   SRC/probe.F90:50-78 (all in the compute type): out_dev = (u_x, u_y, u_z, rho). */
int bgk_probe(const bgk_sweep_params* p, void* const* a, int i, int j, int k, double* out_dev, void* stream);

/* Velocity over a plane in single precision, SRC/vtk_xy.binary.F90:78-97:
   plane 0 = xy at k = index (out[j][i]), 1 = xz at j = index (out[k][i]),
   2 = yz at i = index (out[k][j]); 3 floats (u_x, u_y, u_z) per node, the
   order the reference's VTK writers emit. */
int bgk_slice(const bgk_sweep_params* p, void* const* a, int plane, int index, float* out_dev, void* stream);

/* Helpers of the drop-in library's tracked moments (bgk3d_dropin.h):
   bgk_dropin_sweep_tracked is bgk_sweep that also sums, in the same launch,
   the FP64 moments of the state it writes (rho, u_x, u_y, u_z, 0.5|u|^2 over
   the fluid nodes, the per-node arithmetic of SRC/diagno.F90:112-127) into
   out_dev[0..4]: the blocks' partial sums are added in a fixed order by the
   last blocks to finish, so the bits do not depend on timing.  workspace:
   bgk_dropin_tracked_workspace_bytes(p) bytes of device memory, zeroed once
   before its first use with p's lattice shape (it holds counters that every
   completed call leaves at zero); one workspace per stream of calls.
   Returns BGK_ERR_ARG when the workspace is too small. */
size_t bgk_dropin_tracked_workspace_bytes(const bgk_sweep_params* p);
int bgk_dropin_sweep_tracked(const bgk_sweep_params* p, void* const* a, void* const* b, void* workspace,
                             size_t bytes, double* out_dev);

/* cudaDeviceSynchronize; returns BGK_ERR_CUDA (does not abort) on failure. */
int bgk_device_sync(void);

/* Message describing the calling thread's last error ("" if none). */
const char* bgk_last_error(void);

/* Library version string. */
const char* bgk_version(void);

/* Size in bytes of the library's structs as compiled: 0 bgk_sweep_params,
   1 bgk_lattice_desc (bgk3d_lattice.h); 0 for anything else.  A binding in
   another language (Fortran bind(C) types, Python ctypes) checks its mirror
   against it.  No counterpart in the reference. */
size_t bgk_abi_struct_size(int which);
/* Byte offset of field number `field` (declaration order, from 0) of the
   same structs, or -1 past the last field: a mirror checks every field's
   place, not only the total size.  No counterpart in the reference. */
long long bgk_abi_field_offset(int which, int field);

/* One-node AB sweep of a lattice with an obstacle, without fused moments:
   1 runs the obstacle-free kernel variant over every node outside the
   obstacle's box grown by one node and a second launch over that box with
   the obstacle logic compiled in (bit-identical: only nodes in the grown box
   can link to a solid node); 0 (default; measured 4-7 % faster on the
   sphere case) runs one launch with the obstacle logic for every node.
   Returns the previous setting.  No counterpart in the reference. */
int bgk_set_obstacle_split(int enable);

/* Two-node sweeps for the 16-bit kinds (FP16 / BF16 storage, FP32 compute)
   without fused moments (warps next to an obstacle advance their nodes one
   by one): every thread advances two
   nodes and the two collisions run as one on packed FP32 pairs (lane-wise the
   same roundings: results are bit-identical to the one-node sweep).  Where
   every node pair (i, i + 1), i odd, is one aligned 32-bit word (library-owned
   lattices of even l) the pair is adjacent and each population moves as one
   word, in either collision mode (and both steps of the AA pattern run in
   pairs); otherwise, with the fused collision (fast = 1), the thread takes
   nodes i and i + 32.  Used by bgk_sweep and lattice steps.  On by default;
   0 selects the one-node sweep.  Returns the previous setting (not
   thread-safe against concurrent launches).  No counterpart in the
   reference. */
int bgk_set_pair_kernels(int enable);

#ifdef __cplusplus
}
#endif
#endif /* BGK3D_B200_H */
