/*
 * bgk3d_batch.h -- many independent lattices advanced together by one
 * persistent launch per time step (part of libbgk3d_b200.so).
 *
 * No counterpart in the reference, which runs one lattice per process; the
 * reference's size sweeps (UTIL/run_sweep.sh) run lattices one after another.
 *
 * A batch groups existing AB-pattern lattices (bgk3d_lattice.h) of one
 * storage kind; any extents, boundary cases, obstacles, relaxation
 * frequencies and forces may be mixed.  Stepping the batch advances every
 * member exactly as bgk_lattice_step would (bit-identical results); the
 * members stay usable individually (load/store/moments) between batch steps.
 * The work of a step is cut into 256-node tiles taken from a device queue by
 * a persistent grid (tile shape and grid size chosen by bgk_batch_tune), and
 * runs of steps replay a captured CUDA graph.
 */
#ifndef BGK3D_BATCH_H
#define BGK3D_BATCH_H

#include "bgk3d_lattice.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bgk_batch bgk_batch;

/* Group count lattices (same kind, AB pattern).  The batch keeps pointers
   to them: destroy the batch before any of its lattices. */
int bgk_batch_create(bgk_lattice* const* lattices, int count, bgk_batch** out);
int bgk_batch_destroy(bgk_batch* batch);

/* Advance every member nsteps steps, stream-ordered.  BGK_ERR_STATE if a
   member was stepped or reloaded on its own since the batch last ran. */
int bgk_batch_step(bgk_batch* batch, int nsteps, void* stream);

/* Accept the members' current states after they were loaded or stepped on
   their own (rebuilds the batch's kernel arguments). */
int bgk_batch_resync(bgk_batch* batch);

/* Tile queue parameters: tiles taken per queue access (1..16) and resident
   blocks per SM of the persistent grid (1..8); blocks_per_sm = 0 selects the
   non-persistent form, one block per tile. */
int bgk_batch_set_config(bgk_batch* batch, int tiles_per_grab, int blocks_per_sm);
int bgk_batch_get_config(const bgk_batch* batch, int* tiles_per_grab, int* blocks_per_sm);

/* Autotuner: times `trial_steps` steps (rounded up to even) of each
   candidate configuration on this batch and keeps the fastest.  The trial
   steps advance the lattices like bgk_batch_step; *steps_used reports how
   many.  Synchronises the stream. */
int bgk_batch_tune(bgk_batch* batch, int trial_steps, void* stream, int* steps_used);

/* Total interior nodes of the batch and its tile count. */
long long bgk_batch_nodes(const bgk_batch* batch);
long long bgk_batch_tiles(const bgk_batch* batch);

#ifdef __cplusplus
}
#endif
#endif /* BGK3D_BATCH_H */
