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
 * Two forms cut the work of a step, chosen by bgk_batch_tune:
 *   grouped (the default): members that share boundary case, collision mode
 *     and obstacle logic form a group; each group is one launch of a kernel
 *     compiled for that variant, whose blocks each take one chunk of
 *     consecutive 32-node warp segments of one member from a table built on
 *     the host (bgk_batch_set_chunk);
 *   tile queue: one persistent launch over all members, 256-node tiles taken
 *     from a device counter (bgk_batch_set_config).
 * Runs of steps replay a captured CUDA graph.
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

/* Grouped form: warp segments per chunk (a multiple of 8, 8..4096; default
   32 = 1024 nodes); 0 selects the tile-queue form below.
   Members of min_nodes interior nodes or more step solo, with their own
   single-lattice launch (kernel arguments in the constant bank), instead of
   through a group launch; 0 (the default) runs every member in groups.
   In a captured run of steps the work items (groups and solo members) are
   spread over up to 8 graph branches by node count, each branch running its
   items' chains of steps.  bgk_batch_groups returns the number of launches
   per step (groups + solo members; 1 in the tile-queue form). */
int bgk_batch_set_chunk(bgk_batch* batch, int warps_per_chunk);
int bgk_batch_get_chunk(const bgk_batch* batch, int* warps_per_chunk);
int bgk_batch_set_solo(bgk_batch* batch, long long min_nodes);
long long bgk_batch_get_solo(const bgk_batch* batch);
int bgk_batch_groups(const bgk_batch* batch);

/* Tile queue parameters: tiles taken per queue access (1..16) and resident
   blocks per SM of the persistent grid (1..8); blocks_per_sm = 0 selects the
   non-persistent form, one block per tile.  Used when the chunk size is 0. */
int bgk_batch_set_config(bgk_batch* batch, int tiles_per_grab, int blocks_per_sm);
int bgk_batch_get_config(const bgk_batch* batch, int* tiles_per_grab, int* blocks_per_sm);

/* Autotuner: times `trial_steps` steps (rounded up to even, at least 16,
   after as many untimed steps that capture the step graph) of each
   candidate configuration (grouped form with 8..128 warp segments per
   chunk, then solo thresholds of 2^21 and 2^19 nodes; tile-queue forms) on
   this batch and keeps the fastest.  The trial
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
