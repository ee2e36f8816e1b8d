// Definition of the library-owned lattice object, shared by lattice.cu and
// the batched stepper (batch.cu).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "bgk3d_b200.h"
#include "bgk3d_lattice.h"

struct bgk_lattice {
    bgk_lattice_desc desc;
    bgk_sweep_params p;          // sweep parameters (kind, case, constants, layout, obstacle)
    int es;                      // bytes per stored value
    long long nx, ny, nz, origin, plane;   // elements
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
};
