// Library-owned lattices (include/bgk3d_lattice.h): padded aligned layout,
// AB and in-place AA time steps, CUDA-graph replay of long step runs,
// host transfers in the reference layout, FP64 diagnostics.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>
#include "bgk3d_b200.h"
#include "bgk3d_lattice.h"
#include "bgk_internal.h"
#include "kernels.h"
#include "d3q19.cuh"
#include "lattice_internal.h"
#include "sweep_tma.cuh"

using namespace bgk;



namespace {

constexpr int kGraphSteps = 16;

int elem_bytes(int kind) {
    switch (kind) {
        case K_F64: return 8;
        case K_F32: case K_F32_F64: return 4;
        default: return 2;
    }
}

struct Geometry { long long nx, ny, nz, origin, shift, plane; };

Geometry geometry(const bgk_lattice_desc* d) {
    Geometry g;
    const long long es = elem_bytes(d->kind);
    // Node (1, j, k) of every row starts a 128-byte line: rows are whole
    // lines, so a row's interior values fill whole lines of DRAM bursts (a
    // row of 16-bit values at a 64-byte offset in its line cost 12.5 % more
    // DRAM reads, measured).  Row pitch: whole 32-element segments and whole
    // 128-byte lines, with room for nodes 0..l at elements 31..l+31 of their
    // own row (the TMA sweep's tensor map sees a row as nx elements; the halo
    // node l+1 may spill into the next row's unused first element).
    const long long seg = std::max<long long>(32, 128 / es);
    g.nx = ((long long)d->l + 32 + seg - 1) / seg * seg;
    g.ny = (long long)d->m + 2;
    g.nz = (long long)d->n + 2;
    g.origin = 31;                                   // node (1, j, k) on a segment boundary
    // elements before the origin that put node 1 on a 128-byte boundary
    // (plane starts are 256-byte aligned): 0 for 4- and 8-byte kinds
    g.shift = (128 / es - (g.origin + 1) % (128 / es)) % (128 / es);
    const long long raw = g.nx * g.ny * g.nz + g.shift + g.origin + 32;
    const long long unit = 256 / es;                 // plane starts on 256-byte boundaries
    g.plane = (raw + unit - 1) / unit * unit;
    return g;
}

int nplanes(const bgk_lattice_desc* d) { return d->pattern == BGK_PATTERN_AA ? 19 : 37; }

void drop_graph(bgk_lattice* L) {
    if (L->graph) cudaGraphExecDestroy(L->graph);
    L->graph = nullptr;
    L->graph_steps = 0;
}

int aa_step(const bgk_sweep_params* p, void* const* slots, bool odd, double* mom, cudaStream_t st,
            double* mom_out = nullptr, unsigned* mom_ticket = nullptr) {
    KIND_DISPATCH(p->kind, (launch_aa<S, C>(p, slots, odd, mom, st, mom_out, mom_ticket)));
}

int aa_prepass(const bgk_sweep_params* p, void* const* slots, cudaStream_t st) {
    KIND_DISPATCH(p->kind, (launch_aa_prepass<S, C>(p, slots, st)));
}

// AA: population p of the observable state lives in slot opp(p).
// One time step on stream st (no graph); with mom, the FP64 partial moments
// of the new state go to mom (one slot of 5 doubles per block).
int tma_step(bgk_lattice* L, cudaStream_t st);

// mom (nullable): per-block moment partials of the new state; mom_out
// (nullable, with mom): their sums, finalized in the same launch with the
// ticket counters mom_ticket.
int one_step(bgk_lattice* L, cudaStream_t st, double* mom = nullptr, double* mom_out = nullptr,
             unsigned* mom_ticket = nullptr) {
    if (L->desc.pattern == BGK_PATTERN_AA) {
        const bool odd = (L->steps % 2) == 0;   // Layout E -> odd kernel
        if (int e = aa_step(&L->p, L->a, odd, mom, st, mom_out, mom_ticket)) return e;
    } else {
        const bool has_obs = L->p.obs && L->p.imin <= L->p.imax;
        if (!mom && L->tma_ok && g_tma_kernels && !has_obs && !L->p.zhalo) {
            if (int e = tma_step(L, st)) return e;
            L->outflow_fresh = false;
        } else {
            int halo = L->outflow_fresh ? 1 : 0;
            if (int e = sweep_launch_mom(&L->p, L->a, L->b, mom, st, &halo, mom_out, mom_ticket)) return e;
            L->outflow_fresh = halo != 0;
        }
        for (int d = 0; d < 18; ++d) std::swap(L->a[d], L->b[d]);
    }
    ++L->steps;
    return BGK_OK;
}

// Capture kGraphSteps steps (starting from an even step count, so the
// pointer arrangement / slot layout after the graph equals the one before).
int build_graph(bgk_lattice* L) {
    if (!L->cap_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&L->cap_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "stream create: %s", cudaGetErrorString(e));
    }
    const long long saved = L->steps;
    void* a0[19]; void* b0[19];
    std::memcpy(a0, L->a, sizeof a0); std::memcpy(b0, L->b, sizeof b0);
    const bool fresh0 = L->outflow_fresh;
    // a replay may follow a load: the graph's first step recomputes the
    // outflow plane (inflow case), its later steps take it from the step before
    L->outflow_fresh = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(L->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { L->outflow_fresh = fresh0; return set_error(BGK_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e)); }
    int rc = BGK_OK;
    for (int s = 0; s < kGraphSteps && rc == BGK_OK; ++s) rc = one_step(L, L->cap_stream);
    e = cudaStreamEndCapture(L->cap_stream, &g);
    L->graph_fresh = L->outflow_fresh;
    L->outflow_fresh = fresh0;
    L->steps = saved;
    std::memcpy(L->a, a0, sizeof a0); std::memcpy(L->b, b0, sizeof b0);
    if (rc != BGK_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&L->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { L->graph = nullptr; return set_error(BGK_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    L->graph_steps = kGraphSteps;
    return BGK_OK;
}

int ensure_workspace(const bgk_lattice* Lc) {
    bgk_lattice* L = const_cast<bgk_lattice*>(Lc);
    const size_t need = std::max<size_t>({bgk_reduce_workspace_bytes(L->desc.l, L->desc.m, L->desc.n),
                                          dissipation_workspace(L->desc.l, L->desc.m, L->desc.n), size_t(1) << 16});
    if (L->ws && L->ws_bytes >= need) return BGK_OK;
    dev_free(L->ws);
    L->ws = nullptr;
    if (int rc = dev_alloc(reinterpret_cast<void**>(&L->ws), need, false, "workspace")) return rc;
    L->ws_bytes = need;
    return BGK_OK;
}

// Solid sphere mask on the device: obs[(i-1) + l (j-1) + l m (k-1)] = 1 where
// (i - cx)^2 + (j - cy)^2 + (k - cz)^2 <= r2, with the bounding box of the
// solid nodes gathered by atomics into box[0..5] (min i, max i, min j, ...).
__global__ void sphere_mask_kernel(int32_t* obs, int l, int m, int n, double cx, double cy, double cz, double r2,
                                   int* box) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)l * m * n) return;
    const int i = (int)(t % l) + 1, j = (int)((t / l) % m) + 1, k = (int)(t / ((long long)l * m)) + 1;
    const double dx = i - cx, dy = j - cy, dz = k - cz;
    const int solid = (dx * dx + dy * dy + dz * dz <= r2) ? 1 : 0;
    obs[t] = solid;
    if (solid) {
        atomicMin(&box[0], i); atomicMax(&box[1], i);
        atomicMin(&box[2], j); atomicMax(&box[3], j);
        atomicMin(&box[4], k); atomicMax(&box[5], k);
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda); null when the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

// The 4-D tensor map of an AB lattice's allocation for the TMA sweep: x over
// the row pitch, y over m + 2 rows, z over n + 2 planes, w over the 37
// population planes; box = (64 nodes + 16 bytes each side) x kTmaRows rows.
void make_tensor_map(bgk_lattice* L) {
    L->tma_ok = false;
    if (L->desc.pattern != BGK_PATTERN_AB) return;
    // float compute only (FP64 compute already reaches the HBM roofline)
    if (L->desc.kind != K_F32 && L->desc.kind != K_F16 && L->desc.kind != K_BF16) return;
    if (L->nx * L->ny * L->nz + 64 >= (1LL << 31)) return;   // the TMA kernel uses 32-bit offsets
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return;
    CUtensorMapDataType dt;
    int box_x;
    switch (L->desc.kind) {
        case K_F64: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64; box_x = TmaBox<double>::W; break;
        case K_F16: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; box_x = TmaBox<__half>::W; break;
        case K_BF16: dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; box_x = TmaBox<__nv_bfloat16>::W; break;
        default: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; box_x = TmaBox<float>::W; break;
    }
    const cuuint64_t es = (cuuint64_t)L->es;
    const cuuint64_t dims[4] = {(cuuint64_t)L->nx, (cuuint64_t)L->ny, (cuuint64_t)L->nz, (cuuint64_t)L->planes.size()};
    const cuuint64_t strides[3] = {(cuuint64_t)L->nx * es, (cuuint64_t)(L->nx * L->ny) * es,
                                   (cuuint64_t)L->plane * es};
    const cuuint32_t box[4] = {(cuuint32_t)box_x, (cuuint32_t)kTmaRows, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(&L->tmap, dt, 4, L->base + L->shift * L->es, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    L->tma_ok = (r == CUDA_SUCCESS) && L->origin == kTmaOrigin;
}

// Tensor-map plane of each current population array.
void plane_indices(const bgk_lattice* L, int* pa) {
    for (int d = 0; d < 19; ++d)
        pa[d] = (int)(((char*)L->a[d] - L->base) / ((long long)L->plane * L->es));
}

int tma_step(bgk_lattice* L, cudaStream_t st) {
    int pa[19];
    plane_indices(L, pa);
    KIND_DISPATCH(L->p.kind, (launch_sweep_tma<S, C>(&L->p, L->a, L->b, &L->tmap, pa, L->err, st)));
}

}  // namespace

namespace bgk_lat {
void observable(const bgk_lattice* L, void** out) {
    if (L->desc.pattern == BGK_PATTERN_AA)
        for (int d = 0; d < 19; ++d) out[d] = L->a[opp_of(d)];
    else
        for (int d = 0; d < 19; ++d) out[d] = L->a[d];
}

void begin_load(bgk_lattice* L, void** out) {
    for (int q = 0; q < 19; ++q) L->a[q] = L->planes[q];
    if (L->desc.pattern == BGK_PATTERN_AB) {
        for (int q = 0; q < 18; ++q) L->b[q] = L->planes[19 + q];
        L->b[18] = L->a[18];
    }
    observable(L, out);
}

int end_load(bgk_lattice* L, cudaStream_t st) {
    L->steps = 0;
    L->outflow_fresh = false;
    if (L->desc.pattern == BGK_PATTERN_AA && L->desc.bcase == BC_INFLOW)
        if (int e = aa_prepass(&L->p, L->a, st)) return e;
    return BGK_OK;
}
}  // namespace bgk_lat

using bgk_lat::observable;

extern "C" {

void bgk_lattice_desc_init(bgk_lattice_desc* d, int kind, int bcase, int l, int m, int n, double omega) {
    std::memset(d, 0, sizeof *d);
    d->kind = kind; d->bcase = bcase; d->pattern = BGK_PATTERN_AB;
    d->l = l; d->m = m; d->n = n; d->omega = omega;
    d->scale = 1.0f;
}

size_t bgk_lattice_device_bytes(const bgk_lattice_desc* d) {
    const Geometry g = geometry(d);
    return (size_t)g.plane * nplanes(d) * elem_bytes(d->kind);
}

int bgk_lattice_create(const bgk_lattice_desc* d, bgk_lattice** out) {
    if (!d || !out) return set_error(BGK_ERR_ARG, "null argument");
    *out = nullptr;
    if (d->bcase < BC_DRIVEN || d->bcase > BC_INFLOW) return set_error(BGK_ERR_ARG, "lattices need a boundary case");
    if (d->pattern != BGK_PATTERN_AB && d->pattern != BGK_PATTERN_AA) return set_error(BGK_ERR_ARG, "bad pattern");
    bgk_lattice* L = new (std::nothrow) bgk_lattice;
    if (!L) return set_error(BGK_ERR_NOMEM, "host allocation");
    L->desc = *d;
    const Geometry g = geometry(d);
    L->nx = g.nx; L->ny = g.ny; L->nz = g.nz; L->origin = g.origin; L->shift = g.shift; L->plane = g.plane;
    L->es = elem_bytes(d->kind);
    bgk_sweep_params_init(&L->p, d->kind, d->l, d->m, d->n, d->omega);
    L->p.bcase = d->bcase;
    L->p.nx = g.nx; L->p.ny = g.ny;
    L->p.force_mode = d->force_mode; L->p.fx = d->fx; L->p.fy = d->fy; L->p.fz = d->fz;
    L->p.lid_force = d->lid_force; L->p.u_inflow = d->u_inflow; L->p.inflow_cte1 = 0.0;
    L->p.scale = d->scale;
    L->p.fast = d->fast;
    if (int e = validate(&L->p)) { delete L; return e; }
    L->bytes = bgk_lattice_device_bytes(d);
    if (int rc = dev_alloc(reinterpret_cast<void**>(&L->base), L->bytes, true, "lattice")) {
        delete L;
        return rc;
    }
    const int np = nplanes(d);
    L->planes.resize(np);
    for (int q = 0; q < np; ++q) L->planes[q] = L->base + ((size_t)q * L->plane + L->shift + L->origin) * L->es;
    for (int q = 0; q < 19; ++q) L->a[q] = L->planes[q];
    if (d->pattern == BGK_PATTERN_AB) {
        for (int q = 0; q < 18; ++q) L->b[q] = L->planes[19 + q];
        L->b[18] = L->a[18];
    } else {
        for (int q = 0; q < 19; ++q) L->b[q] = L->a[q];
    }
    if (int rc = dev_alloc(reinterpret_cast<void**>(&L->err), sizeof(int), true, "status flag")) {
        dev_free(L->base);
        delete L;
        return rc;
    }
    make_tensor_map(L);
    *out = L;
    return BGK_OK;
}

int bgk_lattice_status(const bgk_lattice* L) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    int flag = 0;
    const cudaError_t e = cudaMemcpy(&flag, L->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "status: %s", cudaGetErrorString(e));
    if (flag) return set_error(BGK_ERR_CUDA, "a TMA sweep gave up waiting for its copies; the state is undefined");
    return BGK_OK;
}

int bgk_lattice_uses_tma(const bgk_lattice* L) {
    if (!L) return 0;
    const bool has_obs = L->p.obs && L->p.imin <= L->p.imax;
    return (L->tma_ok && g_tma_kernels && !has_obs && !L->p.zhalo) ? 1 : 0;
}

int bgk_lattice_set_zhalo(bgk_lattice* L, int flags) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    if (flags && L->desc.pattern != BGK_PATTERN_AB)
        return set_error(BGK_ERR_UNSUPPORTED, "z-slab faces need the AB pattern");
    bgk_sweep_params q = L->p;
    q.zhalo = flags;
    if (int e = validate(&q)) return e;
    drop_graph(L);
    L->p.zhalo = flags;
    return BGK_OK;
}

int bgk_lattice_plane(const bgk_lattice* L, int pop, int k, void** ptr, size_t* bytes) {
    if (!L || !ptr || !bytes) return set_error(BGK_ERR_ARG, "null argument");
    if (L->desc.pattern != BGK_PATTERN_AB) return set_error(BGK_ERR_UNSUPPORTED, "planes of AB lattices only");
    if (pop < 0 || pop > 18 || k < 0 || k > L->desc.n + 1)
        return set_error(BGK_ERR_ARG, "plane %d of population %d out of range", k, pop);
    const long long nxy = (long long)L->nx * L->ny;
    *ptr = static_cast<char*>(L->a[pop]) + (nxy * k - L->origin) * (long long)L->es;
    *bytes = (size_t)nxy * L->es;
    return BGK_OK;
}

int bgk_set_tma_kernels(int enable) {
    const int prev = g_tma_kernels ? 1 : 0;
    g_tma_kernels = enable != 0;
    return prev;
}

int bgk_lattice_destroy_async(bgk_lattice* L, void* stream) {
    if (!L) return BGK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    // an executable graph or a stream still in flight is released when its
    // work completes
    drop_graph(L);
    if (L->cap_stream) cudaStreamDestroy(L->cap_stream);
    dev_free_async(L->base, st);
    dev_free_async(L->obs_dev, st);
    dev_free_async(L->ws, st);
    dev_free_async(L->mom, st);
    dev_free_async(L->err, st);
    delete L;
    return BGK_OK;
}

int bgk_lattice_destroy(bgk_lattice* L) {
    if (!L) return BGK_OK;
    drop_graph(L);
    if (L->cap_stream) cudaStreamDestroy(L->cap_stream);
    dev_free(L->base);
    dev_free(L->obs_dev);
    dev_free(L->ws);
    dev_free(L->mom);
    dev_free(L->err);
    delete L;
    return BGK_OK;
}

int bgk_lattice_set_sphere(bgk_lattice* L, double cx, double cy, double cz, double r2) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    drop_graph(L);
    dev_free(L->obs_dev);
    L->obs_dev = nullptr;
    L->p.obs = nullptr;
    L->p.imin = 1; L->p.imax = 0; L->p.jmin = 1; L->p.jmax = 0; L->p.kmin = 1; L->p.kmax = 0;
    const int l = L->desc.l, m = L->desc.m, n = L->desc.n;
    const long long nodes = (long long)l * m * n;
    int32_t* obs = nullptr;
    int* box = nullptr;
    if (int rc = dev_alloc(reinterpret_cast<void**>(&obs), (size_t)nodes * sizeof(int32_t), false, "obstacle mask"))
        return rc;
    if (int rc = dev_alloc(reinterpret_cast<void**>(&box), 6 * sizeof(int), false, "bbox")) { dev_free(obs); return rc; }
    int hb[6] = {l + 1, 0, m + 1, 0, n + 1, 0};
    cudaStream_t s = setup_stream();
    cudaError_t e = cudaMemcpyAsync(box, hb, sizeof hb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        sphere_mask_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(obs, l, m, n, cx, cy, cz, r2, box);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hb, box, sizeof hb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(box);
    if (e != cudaSuccess) { dev_free(obs); return set_error(BGK_ERR_CUDA, "sphere mask: %s", cudaGetErrorString(e)); }
    if (hb[1] == 0) { dev_free(obs); return BGK_OK; }   // no solid node
    bgk_sweep_params q = L->p;
    q.obs = obs; q.obs_nx = l; q.obs_ny = m;
    q.imin = hb[0]; q.imax = hb[1]; q.jmin = hb[2]; q.jmax = hb[3]; q.kmin = hb[4]; q.kmax = hb[5];
    if (int err = validate(&q)) { dev_free(obs); return err; }
    L->obs_dev = obs;
    L->p = q;
    return BGK_OK;
}

int bgk_lattice_set_obstacle(bgk_lattice* L, const int32_t* obs) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    drop_graph(L);
    dev_free(L->obs_dev);
    L->obs_dev = nullptr;
    L->p.obs = nullptr;
    L->p.imin = 1; L->p.imax = 0; L->p.jmin = 1; L->p.jmax = 0; L->p.kmin = 1; L->p.kmax = 0;
    if (!obs) return BGK_OK;
    const int l = L->desc.l, m = L->desc.m, n = L->desc.n;
    int b[6] = {l + 1, 0, m + 1, 0, n + 1, 0};
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i)
                if (obs[(size_t)(i - 1) + (size_t)l * (j - 1) + (size_t)l * m * (k - 1)] == 1) {
                    b[0] = std::min(b[0], i); b[1] = std::max(b[1], i);
                    b[2] = std::min(b[2], j); b[3] = std::max(b[3], j);
                    b[4] = std::min(b[4], k); b[5] = std::max(b[5], k);
                }
    if (b[1] == 0) return BGK_OK;   // no solid node
    bgk_sweep_params q = L->p;
    q.obs = obs; q.obs_nx = l; q.obs_ny = m;
    q.imin = b[0]; q.imax = b[1]; q.jmin = b[2]; q.jmax = b[3]; q.kmin = b[4]; q.kmax = b[5];
    if (int e = validate(&q)) return e;
    const size_t nb = (size_t)l * m * n * sizeof(int32_t);
    if (int rc = dev_alloc(reinterpret_cast<void**>(&L->obs_dev), nb, false, "obstacle mask")) return rc;
    cudaStream_t s = setup_stream();
    cudaError_t e = cudaMemcpyAsync(L->obs_dev, obs, nb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dev_free(L->obs_dev);
        L->obs_dev = nullptr;
        return set_error(BGK_ERR_CUDA, "obstacle copy: %s", cudaGetErrorString(e));
    }
    q.obs = L->obs_dev;
    L->p = q;
    return BGK_OK;
}

int bgk_lattice_load(bgk_lattice* L, const void* host, void* stream) {
    if (!L || !host) return set_error(BGK_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int l = L->desc.l, m = L->desc.m, n = L->desc.n;
    const size_t es = L->es, row = (size_t)(l + 2) * es, rows = (size_t)(m + 2) * (n + 2);
    void* f[19];
    bgk_lat::begin_load(L, f);
    for (int d = 0; d < 19; ++d) {
        void* dst = f[d];
        const char* src = (const char*)host + (size_t)d * row * rows;
        cudaError_t e = cudaMemcpy2DAsync(dst, (size_t)L->nx * es, src, row, row, rows, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "load: %s", cudaGetErrorString(e));
    }
    return bgk_lat::end_load(L, st);
}

int bgk_lattice_init(bgk_lattice* L, int flow, const double* params, void* stream) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    if (flow < 0 || flow > 4) return set_error(BGK_ERR_ARG, "unknown flow %d", flow);
    cudaStream_t st = (cudaStream_t)stream;
    void* f[19];
    bgk_lat::begin_load(L, f);
    const float scale = (L->desc.kind == K_F16 || L->desc.kind == K_BF16) ? L->desc.scale : 1.0f;
    int rc;
    {
        const bgk_sweep_params* p = &L->p;
        switch (L->desc.kind) {
            case K_F64: rc = launch_init<double, double>(f, L->nx, L->ny, p->l, p->m, p->n, flow, params, scale, p, st); break;
            case K_F32: rc = launch_init<float, float>(f, L->nx, L->ny, p->l, p->m, p->n, flow, params, scale, p, st); break;
            case K_F16: rc = launch_init<__half, float>(f, L->nx, L->ny, p->l, p->m, p->n, flow, params, scale, p, st); break;
            case K_BF16: rc = launch_init<__nv_bfloat16, float>(f, L->nx, L->ny, p->l, p->m, p->n, flow, params, scale, p, st); break;
            default: rc = launch_init<float, double>(f, L->nx, L->ny, p->l, p->m, p->n, flow, params, scale, p, st); break;
        }
    }
    if (rc) return rc;
    return bgk_lat::end_load(L, st);
}

int bgk_lattice_store(const bgk_lattice* L, void* host, void* stream) {
    if (!L || !host) return set_error(BGK_ERR_ARG, "null argument");
    if (L->desc.pattern == BGK_PATTERN_AA && (L->steps % 2) != 0)
        return set_error(BGK_ERR_STATE, "AA lattice after an odd number of steps holds no observable state");
    cudaStream_t st = (cudaStream_t)stream;
    const int l = L->desc.l, m = L->desc.m, n = L->desc.n;
    const size_t es = L->es, row = (size_t)(l + 2) * es, rows = (size_t)(m + 2) * (n + 2);
    void* obsv[19];
    observable(L, obsv);
    for (int d = 0; d < 19; ++d) {
        char* dst = (char*)host + (size_t)d * row * rows;
        cudaError_t e = cudaMemcpy2DAsync(dst, row, obsv[d], (size_t)L->nx * es, row, rows, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "store: %s", cudaGetErrorString(e));
    }
    return BGK_OK;
}

int bgk_lattice_prepare(bgk_lattice* L) {
    if (!L) return set_error(BGK_ERR_ARG, "bad argument");
    if (L->graph) return BGK_OK;
    // the graph starts from the arrangement of an even step count
    const long long saved = L->steps;
    void* a0[19]; void* b0[19];
    std::memcpy(a0, L->a, sizeof a0); std::memcpy(b0, L->b, sizeof b0);
    if (L->steps % 2) {
        if (L->desc.pattern == BGK_PATTERN_AB)
            for (int d = 0; d < 18; ++d) std::swap(L->a[d], L->b[d]);
        L->steps -= 1;
    }
    const int rc = build_graph(L);
    L->steps = saved;
    std::memcpy(L->a, a0, sizeof a0); std::memcpy(L->b, b0, sizeof b0);
    return rc;
}

int bgk_lattice_step(bgk_lattice* L, int nsteps, void* stream) {
    if (!L || nsteps < 0) return set_error(BGK_ERR_ARG, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    int left = nsteps;
    if (left >= 2 * kGraphSteps) {
        if ((L->steps % 2) != 0) {   // reach the base arrangement first
            if (int e = one_step(L, st)) return e;
            --left;
        }
        if (!L->graph)
            if (int e = build_graph(L)) return e;
        while (left >= L->graph_steps) {
            cudaError_t e = cudaGraphLaunch(L->graph, st);
            if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
            L->steps += L->graph_steps;
            left -= L->graph_steps;
            L->outflow_fresh = L->graph_fresh;
        }
    }
    while (left-- > 0)
        if (int e = one_step(L, st)) return e;
    return BGK_OK;
}

int bgk_lattice_step_moments(bgk_lattice* L, int nsteps, int every, double* out_dev, void* stream) {
    if (!L || nsteps < 0 || every < 1 || !out_dev) return set_error(BGK_ERR_ARG, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    // ticket counters and moment records of the launches that sum their own
    // moments (finalize_by_tickets), laid out for the largest block count
    // of this lattice's shape; the counters start at zero and every launch
    // leaves them so
    const long long nb_max = sweep_blocks(&L->p, nullptr);
    const size_t need = fused_workspace_bytes(nb_max, 5);
    if (L->mom_bytes < need) {
        dev_free(L->mom);
        L->mom = nullptr; L->mom_bytes = 0;
        if (int rc = dev_alloc(reinterpret_cast<void**>(&L->mom), need, false, "moment partials")) return rc;
        L->mom_bytes = need;
        cudaError_t e = cudaMemsetAsync(L->mom, 0, need, st);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    }
    const FusedWs fw = fused_ws(L->mom, nb_max);
    const int samples = nsteps / every;
    for (int s = 0; s < samples; ++s) {
        if (every > 1)
            if (int e = bgk_lattice_step(L, every - 1, stream)) return e;
        if (int e = one_step(L, st, fw.records, out_dev + 5 * (size_t)s, fw.tickets)) return e;
    }
    return bgk_lattice_step(L, nsteps - samples * every, stream);
}

int bgk_lattice_set_omega(bgk_lattice* L, double omega) {
    if (!L) return set_error(BGK_ERR_ARG, "null lattice");
    drop_graph(L);
    L->p.omega = omega;
    L->desc.omega = omega;
    return BGK_OK;
}

int bgk_lattice_dissipation(const bgk_lattice* L, double nu, double* out_dev, void* stream) {
    if (!L || !out_dev) return set_error(BGK_ERR_ARG, "null argument");
    if (!(nu >= 0.0)) return set_error(BGK_ERR_ARG, "viscosity must be >= 0");
    if (L->desc.pattern == BGK_PATTERN_AA && (L->steps % 2) != 0)
        return set_error(BGK_ERR_STATE, "AA lattice after an odd number of steps holds no observable state");
    if (int e = ensure_workspace(L)) return e;
    void* obsv[19];
    observable(L, obsv);
    return dissipation_launch(&L->p, obsv, nu, out_dev, L->ws, (cudaStream_t)stream);
}

int bgk_lattice_moments(const bgk_lattice* L, double* out_dev, void* stream) {
    if (!L || !out_dev) return set_error(BGK_ERR_ARG, "null argument");
    if (L->desc.pattern == BGK_PATTERN_AA && (L->steps % 2) != 0)
        return set_error(BGK_ERR_STATE, "AA lattice after an odd number of steps holds no observable state");
    if (int e = ensure_workspace(L)) return e;
    void* obsv[19];
    observable(L, obsv);
    return moments_launch(&L->p, obsv, out_dev, L->ws, (cudaStream_t)stream);
}

int bgk_lattice_draglift(const bgk_lattice* L, int is, int ie, int js, int je, int ks, int ke, double* out_dev,
                         void* stream) {
    if (!L || !out_dev) return set_error(BGK_ERR_ARG, "null argument");
    if (L->desc.pattern == BGK_PATTERN_AA && (L->steps % 2) != 0)
        return set_error(BGK_ERR_STATE, "AA lattice after an odd number of steps holds no observable state");
    if (ie < is || je < js || ke < ks) return set_error(BGK_ERR_ARG, "empty draglift box");
    if (int e = ensure_workspace(L)) return e;
    void* obsv[19];
    observable(L, obsv);
    return draglift_launch(&L->p, obsv, is, ie, js, je, ks, ke, out_dev, L->ws, L->ws_bytes, (cudaStream_t)stream);
}

long long bgk_lattice_steps(const bgk_lattice* L) { return L ? L->steps : -1; }

int bgk_lattice_arrays(const bgk_lattice* L, void** a19, long long* nx, long long* ny) {
    if (!L || !a19) return set_error(BGK_ERR_ARG, "null argument");
    observable(L, a19);
    if (nx) *nx = L->nx;
    if (ny) *ny = L->ny;
    return BGK_OK;
}

}  // extern "C"
