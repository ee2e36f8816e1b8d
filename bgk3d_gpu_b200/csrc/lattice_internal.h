// Definition of the library-owned lattice object, shared by lattice.cu and
// the batched stepper (batch.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <vector>
#include "bgk3d_b200.h"
#include "bgk3d_lattice.h"

struct bgk_lattice {
    bgk_lattice_desc desc;
    bgk_sweep_params p;          // sweep parameters (kind, case, constants, layout, obstacle)
    int es;                      // bytes per stored value
    long long nx, ny, nz, origin, plane;   // elements
    long long shift = 0;                   // elements before the first plane's origin (128-byte row starts)
    char* base = nullptr;
    size_t bytes = 0;
    std::vector<void*> planes;   // plane pointers at element (0,0,0)
    void* a[19];                 // AB: current populations; AA: slot arrays
    void* b[19];                 // AB: next populations (b[18] = a[18])
    int32_t* obs_dev = nullptr;
    long long steps = 0;
    double* ws = nullptr;
    size_t ws_bytes = 0;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    double* mom = nullptr;       // per-block partial moments of fused steps
    size_t mom_bytes = 0;
    alignas(64) CUtensorMap tmap; // the allocation as x, y, z, plane (sweep_tma.cuh)
    bool tma_ok = false;         // tmap is valid (AB pattern, driver support)
    int* err = nullptr;          // device flag set by a TMA kernel wait that gave up
    // inflow, AB: the current a arrays' outflow plane holds the equilibria of
    // the current state (the last step wrote it), so the next step needs no
    // pre-pass; graph_fresh: the same after a replay of the step graph
    bool outflow_fresh = false;
    bool graph_fresh = false;
};

// Shared by the lattice's host-transfer paths (lattice.cu, lattice_io.cu).
namespace bgk_lat {
// Device arrays holding populations 01..19 of the observable state.
void observable(const bgk_lattice* L, void** out);
// Reset the pointer arrangement to the base planes and return the arrays a
// new state of populations 01..19 is written to (AA: slot opp(d)).
void begin_load(bgk_lattice* L, void** out);
// After a new state is written: step count 0, AA outflow pre-pass.
int end_load(bgk_lattice* L, cudaStream_t st);
}  // namespace bgk_lat
