// Declarations of the per-kind launch wrappers (definitions in launch.cuh,
// instantiated in inst_*.cu) and the kind dispatch used by the C ABI.
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "bgk3d_b200.h"
#include "bgk_internal.h"

namespace bgk {
template <class S, class C>
int launch_sweep(const bgk_sweep_params* p, void* const* a, void* const* b, double* mom, cudaStream_t st,
                 int* halo = nullptr, double* mom_out = nullptr, unsigned* mom_ticket = nullptr);
template <class S, class C>
int launch_sweep_tma(const bgk_sweep_params* p, void* const* a, void* const* b, const void* tmap, const int* pa,
                     int* err, cudaStream_t st);
template <class S, class C>
int launch_moments(const bgk_sweep_params* p, void* const* a, double* out, double* ws, cudaStream_t st);
template <class S, class C>
int launch_draglift(const bgk_sweep_params* p, void* const* a, int is, int ie, int js, int je, int ks, int ke,
                    double* out, double* ws, size_t ws_bytes, cudaStream_t st);
template <class S, class C>
int launch_aa(const bgk_sweep_params* p, void* const* slots, bool odd, double* mom, cudaStream_t st,
              double* mom_out = nullptr, unsigned* mom_ticket = nullptr);
template <class S, class C>
int launch_aa_prepass(const bgk_sweep_params* p, void* const* slots, cudaStream_t st);
template <class S, class C>
size_t fill_batch_desc(const bgk_sweep_params* p, void* const* a, void* const* b, void* out, uint32_t* tiles);
template <class S, class C>
int launch_batch(const void* desc, const uint32_t* tile_begin, int nlat, uint32_t ntiles, unsigned* counter,
                 int parity, int sub, int grid, cudaStream_t st);
template <class S, class C>
int launch_dissipation(const bgk_sweep_params* p, void* const* a, double nu, double* out, double* ws,
                       cudaStream_t st);
template <class S, class C>
int launch_batch_group(const void* desc, const void* chunks, uint32_t nchunks, uint32_t chunk_warps, int parity,
                       int bcase, int cm, bool obs, cudaStream_t st);
template <class S, class C>
int launch_outflow(const bgk_sweep_params* p, void* const* a, cudaStream_t st);
template <class S, class C>
int launch_init(void* const* f, long long nx, long long ny, int l, int m, int n, int flow, const double* prm,
                float scale, const bgk_sweep_params* p, cudaStream_t st);
}  // namespace bgk

// storage kinds: 0 f64/f64, 1 f32/f32, 2 f16/f32, 3 bf16/f32, 4 f32/f64
#define KIND_DISPATCH(kind, CALL)                                                     \
    switch (kind) {                                                                   \
        case 0: { typedef double S; typedef double C; return CALL; }                  \
        case 1: { typedef float S; typedef float C; return CALL; }                    \
        case 2: { typedef __half S; typedef float C; return CALL; }                   \
        case 3: { typedef __nv_bfloat16 S; typedef float C; return CALL; }            \
        case 4: { typedef float S; typedef double C; return CALL; }                   \
    }                                                                                 \
    return set_error(BGK_ERR_ARG, "bad kind");
