// Batched stepping of many lattices (include/bgk3d_batch.h): descriptors,
// tile queue, persistent launches, graph replay and the autotuner.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>
#include "bgk3d_b200.h"
#include "bgk3d_batch.h"
#include "bgk_internal.h"
#include "kernels.h"
#include "lattice_internal.h"

using namespace bgk;

struct bgk_batch {
    int kind = 0;
    std::vector<bgk_lattice*> lats;
    std::vector<int> inflow;              // members that need the outflow-plane launch
    char* desc = nullptr;                 // device: 2 kernel-argument records per member
    size_t rec = 0;                       // bytes of one record pair
    uint32_t* tile_begin = nullptr;       // device prefix of tiles
    unsigned* counter = nullptr;          // device queue counter + finished blocks
    uint32_t ntiles = 0;
    long long nodes = 0;
    int sub = 2, bpsm = 4, nsm = 148;
    long long steps = 0;                  // steps since the descriptors were built
    std::vector<long long> expect;        // each member's step count as the batch left it
    std::vector<void*> base_a, base_b;    // members' a/b arrays when the descriptors were built (19 each)
    cudaStream_t cap = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
};

namespace {

constexpr int kBatchGraphSteps = 8;

int fill_desc(int kind, const bgk_sweep_params* p, void* const* a, void* const* b, void* out, uint32_t* tiles,
              size_t* rec) {
    auto run = [&](auto sz) -> int { *rec = sz; return BGK_OK; };
    switch (kind) {
        case 0: return run(fill_batch_desc<double, double>(p, a, b, out, tiles));
        case 1: return run(fill_batch_desc<float, float>(p, a, b, out, tiles));
        case 2: return run(fill_batch_desc<__half, float>(p, a, b, out, tiles));
        case 3: return run(fill_batch_desc<__nv_bfloat16, float>(p, a, b, out, tiles));
        case 4: return run(fill_batch_desc<float, double>(p, a, b, out, tiles));
    }
    return set_error(BGK_ERR_ARG, "bad kind");
}

int batch_launch(const bgk_batch* B, int parity, cudaStream_t st) {
    const int grid = B->nsm * B->bpsm;   // 0: one block per tile
    switch (B->kind) {
        case 0: return launch_batch<double, double>(B->desc, B->tile_begin, (int)B->lats.size(), B->ntiles, B->counter, parity, B->sub, grid, st);
        case 1: return launch_batch<float, float>(B->desc, B->tile_begin, (int)B->lats.size(), B->ntiles, B->counter, parity, B->sub, grid, st);
        case 2: return launch_batch<__half, float>(B->desc, B->tile_begin, (int)B->lats.size(), B->ntiles, B->counter, parity, B->sub, grid, st);
        case 3: return launch_batch<__nv_bfloat16, float>(B->desc, B->tile_begin, (int)B->lats.size(), B->ntiles, B->counter, parity, B->sub, grid, st);
        case 4: return launch_batch<float, double>(B->desc, B->tile_begin, (int)B->lats.size(), B->ntiles, B->counter, parity, B->sub, grid, st);
    }
    return set_error(BGK_ERR_ARG, "bad kind");
}

int outflow_launch(int kind, const bgk_sweep_params* p, void* const* a, cudaStream_t st) {
    KIND_DISPATCH(kind, (launch_outflow<S, C>(p, a, st)));
}

// Member idx's `a` arrays at batch parity `par` (relative to the arrangement
// the descriptors were built from).
void member_arrays(const bgk_batch* B, size_t idx, int par, void** a) {
    const void* const* a0 = &B->base_a[19 * idx];
    const void* const* b0 = &B->base_b[19 * idx];
    for (int d = 0; d < 19; ++d) a[d] = const_cast<void*>((par && d < 18) ? b0[d] : a0[d]);
}

void record_base(bgk_batch* B) {
    B->base_a.assign(19 * B->lats.size(), nullptr);
    B->base_b.assign(19 * B->lats.size(), nullptr);
    for (size_t i = 0; i < B->lats.size(); ++i)
        for (int d = 0; d < 19; ++d) {
            B->base_a[19 * i + d] = B->lats[i]->a[d];
            B->base_b[19 * i + d] = B->lats[i]->b[d];
        }
}

// One batch step: outflow planes of the inflow members, then the persistent launch.
int batch_one(bgk_batch* B, cudaStream_t st) {
    const int par = (int)(B->steps & 1);
    for (int idx : B->inflow) {
        void* a[19];
        member_arrays(B, (size_t)idx, par, a);
        if (int e = outflow_launch(B->kind, &B->lats[idx]->p, a, st)) return e;
    }
    if (int e = batch_launch(B, par, st)) return e;
    ++B->steps;
    return BGK_OK;
}

// Hand the advanced state back to the members (pointer arrangement, step count).
void sync_members(bgk_batch* B, long long nsteps) {
    if (nsteps & 1)
        for (bgk_lattice* L : B->lats)
            for (int d = 0; d < 18; ++d) std::swap(L->a[d], L->b[d]);
    for (size_t i = 0; i < B->lats.size(); ++i) {
        B->lats[i]->steps += nsteps;
        B->expect[i] = B->lats[i]->steps;
    }
}

void drop_graph(bgk_batch* B) {
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    B->graph_steps = 0;
}

int build_graph(bgk_batch* B) {
    if (!B->cap) {
        cudaError_t e = cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "stream create: %s", cudaGetErrorString(e));
    }
    const long long saved = B->steps;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    int rc = BGK_OK;
    for (int s = 0; s < kBatchGraphSteps && rc == BGK_OK; ++s) rc = batch_one(B, B->cap);
    e = cudaStreamEndCapture(B->cap, &g);
    B->steps = saved;
    if (rc != BGK_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&B->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { B->graph = nullptr; return set_error(BGK_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    B->graph_steps = kBatchGraphSteps;
    return BGK_OK;
}

// Steps without handing the state back (the caller does it once).
int run_steps(bgk_batch* B, int nsteps, cudaStream_t st) {
    int left = nsteps;
    if (left >= 2 * kBatchGraphSteps) {
        if (B->steps & 1) {
            if (int e = batch_one(B, st)) return e;
            --left;
        }
        if (!B->graph)
            if (int e = build_graph(B)) return e;
        while (left >= B->graph_steps) {
            cudaError_t e = cudaGraphLaunch(B->graph, st);
            if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
            B->steps += B->graph_steps;
            left -= B->graph_steps;
        }
    }
    while (left-- > 0)
        if (int e = batch_one(B, st)) return e;
    return BGK_OK;
}

}  // namespace

extern "C" {

int bgk_batch_create(bgk_lattice* const* lats, int count, bgk_batch** out) {
    if (!lats || count < 1 || !out) return set_error(BGK_ERR_ARG, "bad argument");
    *out = nullptr;
    const int kind = lats[0]->desc.kind;
    for (int i = 0; i < count; ++i) {
        if (!lats[i]) return set_error(BGK_ERR_ARG, "null lattice %d", i);
        if (lats[i]->desc.kind != kind) return set_error(BGK_ERR_ARG, "batch members must share one storage kind");
        if (lats[i]->desc.pattern != BGK_PATTERN_AB) return set_error(BGK_ERR_UNSUPPORTED, "batch members use the AB pattern");
        for (int j = 0; j < i; ++j)
            if (lats[j] == lats[i]) return set_error(BGK_ERR_ARG, "lattice %d appears twice", i);
    }
    bgk_batch* B = new (std::nothrow) bgk_batch;
    if (!B) return set_error(BGK_ERR_NOMEM, "host allocation");
    B->kind = kind;
    B->lats.assign(lats, lats + count);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&B->nsm, cudaDevAttrMultiProcessorCount, dev);
    std::vector<char> host;
    std::vector<uint32_t> begin(count + 1, 0);
    for (int i = 0; i < count; ++i) {
        bgk_lattice* L = lats[i];
        alignas(16) char tmp[4096];
        uint32_t tiles = 0;
        size_t rec = 0;
        if (int e = fill_desc(kind, &L->p, L->a, L->b, tmp, &tiles, &rec)) { delete B; return e; }
        if (rec > sizeof tmp) { delete B; return set_error(BGK_ERR_UNSUPPORTED, "descriptor too large"); }
        B->rec = rec;
        host.insert(host.end(), tmp, tmp + rec);
        if ((unsigned long long)begin[i] + tiles > 0xffffffffull) { delete B; return set_error(BGK_ERR_ARG, "batch too large"); }
        begin[i + 1] = begin[i] + tiles;
        B->nodes += (long long)L->desc.l * L->desc.m * L->desc.n;
        if (L->desc.bcase == BGK_BC_INFLOW) B->inflow.push_back(i);
    }
    B->ntiles = begin[count];
    for (int i = 0; i < count; ++i) B->expect.push_back(lats[i]->steps);
    record_base(B);
    int rc = dev_alloc(reinterpret_cast<void**>(&B->desc), host.size(), false, "batch descriptors");
    if (!rc) rc = dev_alloc(reinterpret_cast<void**>(&B->tile_begin), begin.size() * sizeof(uint32_t), false, "tile table");
    if (!rc) rc = dev_alloc(reinterpret_cast<void**>(&B->counter), 2 * sizeof(unsigned), true, "tile counter");
    if (rc) { bgk_batch_destroy(B); return rc; }
    cudaStream_t s = setup_stream();
    cudaError_t e = cudaMemcpyAsync(B->desc, host.data(), host.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->tile_begin, begin.data(), begin.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { bgk_batch_destroy(B); return set_error(BGK_ERR_CUDA, "batch tables: %s", cudaGetErrorString(e)); }
    *out = B;
    return BGK_OK;
}

int bgk_batch_resync(bgk_batch* B) {
    if (!B) return set_error(BGK_ERR_ARG, "null batch");
    drop_graph(B);
    std::vector<char> host;
    for (size_t i = 0; i < B->lats.size(); ++i) {
        bgk_lattice* L = B->lats[i];
        alignas(16) char tmp[4096];
        uint32_t tiles = 0;
        size_t rec = 0;
        if (int e = fill_desc(B->kind, &L->p, L->a, L->b, tmp, &tiles, &rec)) return e;
        host.insert(host.end(), tmp, tmp + rec);
        B->expect[i] = L->steps;
    }
    cudaError_t e = cudaMemcpy(B->desc, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "resync: %s", cudaGetErrorString(e));
    record_base(B);
    B->steps = 0;
    return BGK_OK;
}

int bgk_batch_destroy(bgk_batch* B) {
    if (!B) return BGK_OK;
    drop_graph(B);
    if (B->cap) cudaStreamDestroy(B->cap);
    dev_free(B->desc);
    dev_free(B->tile_begin);
    dev_free(B->counter);
    delete B;
    return BGK_OK;
}

int bgk_batch_step(bgk_batch* B, int nsteps, void* stream) {
    if (!B || nsteps < 0) return set_error(BGK_ERR_ARG, "bad argument");
    for (size_t i = 0; i < B->lats.size(); ++i)
        if (B->lats[i]->steps != B->expect[i])
            return set_error(BGK_ERR_STATE, "member %zu was stepped or reloaded outside the batch; create the batch again", i);
    const long long before = B->steps;
    const int rc = run_steps(B, nsteps, (cudaStream_t)stream);
    sync_members(B, B->steps - before);
    return rc;
}

int bgk_batch_set_config(bgk_batch* B, int sub, int bpsm) {
    if (!B || sub < 1 || sub > 16 || bpsm < 0 || bpsm > 8) return set_error(BGK_ERR_ARG, "bad configuration");
    if (sub != B->sub || bpsm != B->bpsm) drop_graph(B);
    B->sub = sub;
    B->bpsm = bpsm;
    return BGK_OK;
}

int bgk_batch_get_config(const bgk_batch* B, int* sub, int* bpsm) {
    if (!B) return set_error(BGK_ERR_ARG, "null batch");
    if (sub) *sub = B->sub;
    if (bpsm) *bpsm = B->bpsm;
    return BGK_OK;
}

int bgk_batch_tune(bgk_batch* B, int trial_steps, void* stream, int* steps_used) {
    if (!B) return set_error(BGK_ERR_ARG, "null batch");
    cudaStream_t st = (cudaStream_t)stream;
    const int n = std::max(2, (trial_steps + 1) / 2 * 2);
    const int subs[] = {1, 2, 4, 8};
    const int bpsms[] = {0, 2, 3, 4};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bsub = B->sub, bb = B->bpsm;
    long long used = 0;
    for (int s : subs)
        for (int b : bpsms) {
            if (b == 0 && s != 1) continue;   // one block per tile has no queue grab size
            bgk_batch_set_config(B, s, b);
            if (int e = bgk_batch_step(B, 2, st)) return e;   // warm
            cudaEventRecord(e0, st);
            if (int e = bgk_batch_step(B, n, st)) return e;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            used += n + 2;
            if (ms < best) { best = ms; bsub = s; bb = b; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    bgk_batch_set_config(B, bsub, bb);
    if (steps_used) *steps_used = (int)used;
    return BGK_OK;
}

long long bgk_batch_nodes(const bgk_batch* B) { return B ? B->nodes : -1; }
long long bgk_batch_tiles(const bgk_batch* B) { return B ? (long long)B->ntiles : -1; }

}  // extern "C"
