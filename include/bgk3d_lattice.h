/*
 * bgk3d_lattice.h -- library-owned lattices (part of libbgk3d_b200.so).
 *
 * A bgk_lattice holds its populations in device memory in a padded layout
 * (row pitch a multiple of 32 elements, node (1,j,k) on a 128-byte boundary)
 * and advances them with the fused sweep, either as two lattices (AB, the
 * reference's ping-pong, SRC/col_MC.F90:539-596) or in place (AA: one
 * population set, half the memory).  Host transfers use the reference's own
 * layout: 19 consecutive arrays (0:l+1, 0:m+1, 0:n+1), i fastest, in the
 * storage kind's representation (raw 16-bit words for the 16-bit kinds),
 * which is the record layout of SRC/restore_raw.F90:43-61 without markers.
 *
 * Reference counterparts: the Fortran driver's allocation and time loop
 * (SRC/alloca.F90:150-191, SRC/bgk3d.F90:169-196) for one case.
 */
#ifndef BGK3D_LATTICE_H
#define BGK3D_LATTICE_H

#include "bgk3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define BGK_PATTERN_AB 0   /* two population sets, pointer swap (reference scheme) */
#define BGK_PATTERN_AA 1   /* one population set, in place                        */

typedef struct bgk_lattice bgk_lattice;

typedef struct bgk_lattice_desc {
    int kind;              /* BGK_KIND_* */
    int bcase;             /* BGK_BC_DRIVEN / PERIODIC / CHANNEL / INFLOW */
    int pattern;           /* BGK_PATTERN_AB or BGK_PATTERN_AA */
    int l, m, n;           /* interior extents */
    double omega;          /* BGK relaxation frequency */
    int force_mode;        /* 0: constant per-population force; 1: force * rho */
    double fx, fy, fz;
    double lid_force;      /* DRIVEN: u_lid / 6 */
    double u_inflow;       /* INFLOW */
    float scale;           /* 16-bit kinds: power-of-two storage scale */
    int fast;              /* bgk_sweep_params.fast: 1 = fused-multiply-add collision */
} bgk_lattice_desc;

/* Defaults: AB pattern, no force, lid 0, inflow 0, scale 1, fast 0. */
void bgk_lattice_desc_init(bgk_lattice_desc* d, int kind, int bcase, int l, int m, int n, double omega);

/* Device bytes a lattice with this description occupies (admission control). */
size_t bgk_lattice_device_bytes(const bgk_lattice_desc* d);

/* Allocate the lattice on the current device.  Lattices, batches and their
   masks and workspaces come from one stream-ordered memory pool per device;
   creation zeroes the populations on a private stream, so it does not wait
   for kernels in flight on other streams.  Destruction waits for the device,
   like cudaFree. */
int bgk_lattice_create(const bgk_lattice_desc* d, bgk_lattice** out);
int bgk_lattice_destroy(bgk_lattice* lat);
/* Destroy without waiting for the device: the lattice's memory goes back to
   the pool ordered after the work queued on `stream`.  Every launch and copy
   that used the lattice must be on that stream or ordered before the call
   (a server that steps each solve on its own stream retires it this way
   while the other solves keep running).  No counterpart in the reference. */
int bgk_lattice_destroy_async(bgk_lattice* lat, void* stream);

/* Bytes of freed lattice memory the current device's pool keeps for reuse
   (default 0: freed memory goes back to the device at once).  A server that
   creates and destroys many lattices sets its budget here, so that creation
   reuses memory instead of mapping it anew. */
int bgk_set_retained_bytes(size_t bytes);
/* Give every unused block of the current device's pool back to the device. */
int bgk_trim_memory(void);

/* Obstacle mask obs_host[l*m*n] (i fastest, 1 = solid, SRC/build.obs.F90
   convention); copied to the device, bounding box computed here.  Must stay
   one node inside the lattice.  NULL removes the obstacle. */
int bgk_lattice_set_obstacle(bgk_lattice* lat, const int32_t* obs_host);

/* Solid sphere obstacle built on the device: nodes with (i - cx)^2 +
   (j - cy)^2 + (k - cz)^2 <= r2 are solid (the mask bgk_lattice_set_obstacle
   would get from the same rule on the host; bounding box gathered on the
   device).  Same validation; synchronous.  No counterpart in the reference
   (SRC/build.obs.F90 builds a shell on the host). */
int bgk_lattice_set_sphere(bgk_lattice* lat, double cx, double cy, double cz, double r2);

/* Load / store the post-collision state in the reference layout (see top).
   Stream-ordered; host memory should be pinned for asynchrony.  store needs
   an even number of AA steps since the last load (BGK_ERR_STATE otherwise). */
int bgk_lattice_load(bgk_lattice* lat, const void* host, void* stream);
int bgk_lattice_store(const bgk_lattice* lat, void* host, void* stream);

/* Equilibrium initial state of an analytic flow computed on the device
   (SRC/init.F90:113-201 without the host): flow 0 uniform (params = rho,
   u_x, u_y, u_z; rest = 1,0,0,0), 1 Taylor-Green vortex (params[0] = u0;
   x = 2 pi (i-1)/l, ...), 2 Kida vortex (params[0] = u0, rho = 1) -- these
   three in double, rounded once, keeping w_p (rho - 1) -- and the
   reference's own forms in its arithmetic (compute type, its literals,
   w_p (rho - 1) dropped as its shifted storage drops it): 3 the TGV3D form
   (SRC/init.F90:141-148, x = (i - 0.5)/l, params[0] = u00), 4 the default
   periodic 2-D Taylor-Green form (:125-130).  Resets the step count like
   bgk_lattice_load. */
int bgk_lattice_init(bgk_lattice* lat, int flow, const double* params, void* stream);

/* Restart files in the reference's record format (SRC/save_raw.F90:37-69,
   SRC/restore_raw.F90:35-61): a Fortran sequential unformatted file of 20
   records framed by 4-byte length markers -- the time step (4-byte
   integer), then populations 01..19 over the full halo box (0..l+1, 0..m+1,
   0..n+1), i fastest.  Records over 2147483639 bytes are split into
   subrecords the gfortran way (negative leading marker: more follows;
   negative trailing marker: continues an earlier subrecord).
   save: file_bytes 0 writes the stored elements as they are (16-bit kinds:
   the scaled 16-bit patterns); 4 or 8 converts on the device to real*4 /
   real*8 (16-bit kinds unscaled), what a reference build of that precision
   restores.  AA lattices must be at an even step.  The file name is the
   caller's (the reference writes save.<itime, 8 digits>.bin and restores
   from restore.bin).
   restore: the element size is taken from the record lengths; 2-byte values
   go as they are into a 16-bit lattice and are read as IEEE half values into
   a 4- or 8-byte one (the reference's HALF storage); other sizes are
   converted on the device.  The file's box must be this lattice's; the
   framing of all records is checked before the lattice is touched.  Sets
   *itime (if not null) to the file's time step and resets the step count
   like bgk_lattice_load.  Both return after the data is written/read. */
int bgk_lattice_save(const bgk_lattice* lat, const char* path, int itime, int file_bytes, void* stream);
int bgk_lattice_restore(bgk_lattice* lat, const char* path, int* itime, void* stream);
/* Largest subrecord bgk_lattice_save writes (default and maximum 2147483639
   bytes; values outside 4..2147483639 are ignored); returns the previous
   limit.  Lowering it exercises the subrecord framing with small lattices.
   No counterpart in the reference. */
long long bgk_io_set_subrecord_limit(long long bytes);

/* Advance nsteps time steps (boundaries + stream + collide), stream-ordered.
   Runs of 32 or more steps replay a captured 16-step CUDA graph (captured on
   the first such run unless bgk_lattice_prepare captured it before). */
int bgk_lattice_step(bgk_lattice* lat, int nsteps, void* stream);

/* Capture the 16-step CUDA graph of bgk_lattice_step now, without running
   it (no kernel executes and the state is untouched), so that the first long
   step run launches at once.  A no-op when the graph exists.  No counterpart
   in the reference. */
int bgk_lattice_prepare(bgk_lattice* lat);

/* Advance nsteps steps and record the FP64 moments (as bgk_moments) of the
   state after every `every`-th step, computed in the same pass as that step:
   sample s (0 <= s < nsteps / every) goes to out_dev[5 s .. 5 s + 4]. */
int bgk_lattice_step_moments(bgk_lattice* lat, int nsteps, int every, double* out_dev, void* stream);

/* Change the relaxation frequency / force of an existing lattice. */
int bgk_lattice_set_omega(bgk_lattice* lat, double omega);

/* FP64 moments (as bgk_moments) of the current state into out_dev[0..4];
   AA lattices need an even step count. */
int bgk_lattice_moments(const bgk_lattice* lat, double* out_dev, void* stream);

/* FP64 turbulence diagnostics (as bgk_dissipation) of the current state into
   out_dev[0..6], with the lattice's boundary case; AA lattices need an even
   step count. */
int bgk_lattice_dissipation(const bgk_lattice* lat, double nu, double* out_dev, void* stream);

/* FP64 drag/lift (as bgk_draglift) over the box into out_dev[0..2]. */
int bgk_lattice_draglift(const bgk_lattice* lat, int is, int ie, int js, int je, int ks, int ke,
                         double* out_dev, void* stream);

/* bgk_profile / bgk_probe / bgk_slice on the lattice's current state (AA
   lattices: at an even step). */
int bgk_lattice_profile(const bgk_lattice* lat, int axis, int c1, int c2, double* out_dev, void* stream);
int bgk_lattice_probe(const bgk_lattice* lat, int i, int j, int k, double* out_dev, void* stream);
int bgk_lattice_slice(const bgk_lattice* lat, int plane, int index, float* out_dev, void* stream);

/* Optional TMA-staged sweep for AB lattices with float compute (F32, F16,
   BF16) and no obstacle: a persistent grid in which one producer thread per
   block copies, for each tile of 64 x 8 nodes, the 19 source row blocks into
   a ring of shared-memory stages (tiled bulk copies through a tensor map of
   the allocation) and eight consumer warps advance two nodes per thread with
   packed FP32 arithmetic; a second launch advances the nodes on the faces.
   Results are bit-identical to the one-node sweep.  Off by default: on a
   B200 it issues 280 instead of 408 instructions per FP16 node but runs at
   about half the one-node sweep's rate at 256^3.  Steps with fused moments
   always use the one-node sweep.
   bgk_lattice_uses_tma: 1 when the next plain step of this lattice takes the
   TMA path.  bgk_set_tma_kernels: switch for all lattices (default off),
   returns the previous setting (not thread-safe against concurrent launches).
   bgk_lattice_status: BGK_ERR_CUDA when a TMA sweep gave up waiting for its
   copies (about one second; the kernel then returns and the state is
   undefined), else BGK_OK; synchronous.  No counterpart in the reference. */
int bgk_lattice_uses_tma(const bgk_lattice* lat);
int bgk_set_tma_kernels(int enable);
int bgk_lattice_status(const bgk_lattice* lat);

/* z-slab decomposition (a lattice split along z over several devices or
   processes, one slab each).  bgk_lattice_set_zhalo(lat, flags): the faces
   in flags (bit 0: k = 1, bit 1: k = n) read the populations that enter
   through them from the halo planes k = 0 / n+1 as stored, with no wrap,
   wall or lid there; the caller fills those planes from the neighbour slabs
   before every step.  AB pattern only; not with the inflow case or an
   obstacle (both would need the neighbour's outflow plane or mask).
   bgk_lattice_plane(lat, pop, k, &ptr, &bytes): device address and size of
   plane k (0..n+1) of population pop (0..18) of the current state, the
   (nx * ny)-element region that holds its nodes (1..l, 1..m) contiguously:
   what a halo exchange sends (planes 1 and n) and receives (planes 0 and
   n+1).  Valid until the next step (the two population sets swap).  No
   counterpart in the reference (which runs on one GPU). */
int bgk_lattice_set_zhalo(bgk_lattice* lat, int flags);
int bgk_lattice_plane(const bgk_lattice* lat, int pop, int k, void** ptr, size_t* bytes);

/* Steps advanced since the last load. */
long long bgk_lattice_steps(const bgk_lattice* lat);

/* Current population pointers (device) and the layout, for callers that
   run their own kernels on the state: a[19] in reference population order
   (AA: valid after an even step count), nx/ny leading dimensions. */
int bgk_lattice_arrays(const bgk_lattice* lat, void** a19, long long* nx, long long* ny);

#ifdef __cplusplus
}
#endif
#endif /* BGK3D_LATTICE_H */
