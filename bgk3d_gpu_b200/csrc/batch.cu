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
#include "host_args.cuh"
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
    // grouped form: members grouped by (boundary case, collision mode,
    // obstacle), one launch per group over a chunk table
    struct Group {
        int bcase = 0, cm = 0;
        bool obs = false;
        std::vector<int> members;
        size_t first = 0;      // offset of the group's chunks in the chunk table
        uint32_t nchunks = 0;
    };
    std::vector<Group> groups;
    int chunk = 32;                       // warp segments per chunk; 0: tile-queue forms
    uint2* chunks = nullptr;              // device chunk table of all groups
    size_t chunk_cap = 0;                 // entries allocated
    // members of at least solo_nodes nodes (0: none) step with their own
    // single-lattice launch instead of a group launch
    long long solo_nodes = 0;
    std::vector<int> solo;
    // graph branches of the grouped form: work items (solo member: its index;
    // group g: -1 - g) spread over up to kBranches branches
    std::vector<std::vector<int>> branches;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;          // fork + one join per branch
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

int group_launch(const bgk_batch* B, const bgk_batch::Group& g, int parity, cudaStream_t st) {
    const uint2* ch = B->chunks + g.first;
    const uint32_t cw = (uint32_t)B->chunk;
    switch (B->kind) {
        case 0: return launch_batch_group<double, double>(B->desc, ch, g.nchunks, cw, parity, g.bcase, g.cm, g.obs, st);
        case 1: return launch_batch_group<float, float>(B->desc, ch, g.nchunks, cw, parity, g.bcase, g.cm, g.obs, st);
        case 2: return launch_batch_group<__half, float>(B->desc, ch, g.nchunks, cw, parity, g.bcase, g.cm, g.obs, st);
        case 3: return launch_batch_group<__nv_bfloat16, float>(B->desc, ch, g.nchunks, cw, parity, g.bcase, g.cm, g.obs, st);
        case 4: return launch_batch_group<float, double>(B->desc, ch, g.nchunks, cw, parity, g.bcase, g.cm, g.obs, st);
    }
    return set_error(BGK_ERR_ARG, "bad kind");
}

int batch_launch(const bgk_batch* B, int parity, cudaStream_t st) {
    if (B->chunk > 0) {   // grouped form (batch_one runs the solo members)
        for (const bgk_batch::Group& g : B->groups)
            if (int e = group_launch(B, g, parity, st)) return e;
        return BGK_OK;
    }
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

// Warp segments of one step of member L (the row mapping of its padded layout).
long long member_warps(const bgk_lattice* L) {
    const int kind = L->desc.kind;
    const size_t es = kind == 0 ? 8 : (kind == 2 || kind == 3) ? 2 : 4;
    const long long align = (long long)(((uintptr_t)L->a[0] / es) & 31);
    return seg_plan(L->p.l, L->p.m, L->p.n, L->p.nx, align, false).warps;
}

// Collision mode of member L's kernel (bgk_sweep_params -> CollMode).
int member_mode(const bgk_lattice* L) {
    const bool float_compute = L->desc.kind == 1 || L->desc.kind == 2 || L->desc.kind == 3;
    return (generic_collision(&L->p) ? 1 : 0) + ((L->p.fast && float_compute) ? 2 : 0);
}

// Branches of the captured step graph of the grouped form.
constexpr int kBranches = 8;

long long member_nodes(const bgk_batch* B, int i) {
    return B->lats[i]->desc.l * (long long)B->lats[i]->desc.m * B->lats[i]->desc.n;
}

// Groups, solo members, graph branches and the chunk table of the grouped
// form for the current chunk size and solo threshold.
int build_groups(bgk_batch* B) {
    B->groups.clear();
    B->solo.clear();
    B->branches.clear();
    for (size_t i = 0; i < B->lats.size(); ++i) {
        const bgk_lattice* L = B->lats[i];
        if (B->chunk > 0 && B->solo_nodes > 0 && member_nodes(B, (int)i) >= B->solo_nodes) {
            B->solo.push_back((int)i);
            continue;
        }
        const int bc = L->p.bcase, cm = member_mode(L);
        const bool obs = L->p.obs && L->p.imin <= L->p.imax && L->p.jmin <= L->p.jmax && L->p.kmin <= L->p.kmax;
        bgk_batch::Group* g = nullptr;
        for (bgk_batch::Group& h : B->groups)
            if (h.bcase == bc && h.cm == cm && h.obs == obs) g = &h;
        if (!g) {
            B->groups.emplace_back();
            g = &B->groups.back();
            g->bcase = bc; g->cm = cm; g->obs = obs;
        }
        g->members.push_back((int)i);
    }
    // work items, largest first, each onto the branch with the fewest nodes
    std::vector<std::pair<long long, int>> items;
    for (int i : B->solo) items.push_back({member_nodes(B, i), i});
    for (size_t g = 0; g < B->groups.size(); ++g) {
        long long nodes = 0;
        for (int i : B->groups[g].members) nodes += member_nodes(B, i);
        items.push_back({nodes, -1 - (int)g});
    }
    std::stable_sort(items.begin(), items.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    const size_t nb = std::min<size_t>(kBranches, items.size());
    B->branches.assign(nb, {});
    std::vector<long long> load(nb, 0);
    for (const auto& it : items) {
        const size_t t = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        B->branches[t].push_back(it.second);
        load[t] += it.first;
    }
    if (B->chunk <= 0) return BGK_OK;
    // launches of earlier steps may still read the current table (they run
    // asynchronously on the caller's stream): wait for them before the table
    // is rewritten in place
    if (B->chunks) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "chunk table: %s", cudaGetErrorString(e));
    }
    std::vector<uint2> table;
    for (bgk_batch::Group& g : B->groups) {
        g.first = table.size();
        for (int i : g.members) {
            const long long w = member_warps(B->lats[i]);
            for (long long c = 0; c < w; c += B->chunk) table.push_back(make_uint2((unsigned)i, (unsigned)c));
        }
        g.nchunks = (uint32_t)(table.size() - g.first);
    }
    if (table.size() > B->chunk_cap) {
        dev_free(B->chunks);
        B->chunks = nullptr;
        B->chunk_cap = 0;
        if (int rc = dev_alloc(reinterpret_cast<void**>(&B->chunks), table.size() * sizeof(uint2), false, "chunk table"))
            return rc;
        B->chunk_cap = table.size();
    }
    cudaStream_t s = setup_stream();
    cudaError_t e = cudaMemcpyAsync(B->chunks, table.data(), table.size() * sizeof(uint2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "chunk table: %s", cudaGetErrorString(e));
    return BGK_OK;
}

// One step of one group (grouped form): the outflow planes of its inflow
// members, then its launch.
int group_step(bgk_batch* B, const bgk_batch::Group& g, int par, cudaStream_t st) {
    for (int idx : g.members) {
        if (B->lats[idx]->desc.bcase != BGK_BC_INFLOW) continue;
        void* a[19];
        member_arrays(B, (size_t)idx, par, a);
        if (int e = outflow_launch(B->kind, &B->lats[idx]->p, a, st)) return e;
    }
    return group_launch(B, g, par, st);
}

// One step of solo member idx: its own single-lattice launch (outflow plane
// included), with the member's arrays at batch parity par.
int member_step(bgk_batch* B, int idx, int par, cudaStream_t st) {
    void* a[19];
    void* b[19];
    member_arrays(B, (size_t)idx, par, a);
    member_arrays(B, (size_t)idx, par ^ 1, b);
    b[18] = a[18];
    int halo = 0;   // pre-pass, and the next outflow plane written like the member's own step
    return sweep_launch_mom(&B->lats[idx]->p, a, b, nullptr, st, &halo);
}

// One step of a work item (solo member idx >= 0, or group -1 - idx).
int item_step(bgk_batch* B, int item, int par, cudaStream_t st) {
    if (item >= 0) return member_step(B, item, par, st);
    return group_step(B, B->groups[(size_t)(-1 - item)], par, st);
}

// Graph of kBatchGraphSteps steps of the grouped form: the work items are
// independent lattices, so each branch runs its items' chains of steps
// (fork / join), and one item's last wave overlaps the others' work.
int capture_branches(bgk_batch* B) {
    const size_t G = B->branches.size();
    while (B->side.size() < G) {
        cudaStream_t s = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "stream create: %s", cudaGetErrorString(e));
        B->side.push_back(s);
    }
    while (B->ev.size() < G + 1) {
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "event create: %s", cudaGetErrorString(e));
        B->ev.push_back(ev);
    }
    if (cudaEventRecord(B->ev[0], B->cap) != cudaSuccess) return set_error(BGK_ERR_CUDA, "fork record");
    for (size_t g = 0; g < G; ++g) {
        if (cudaStreamWaitEvent(B->side[g], B->ev[0], 0) != cudaSuccess) return set_error(BGK_ERR_CUDA, "fork wait");
        for (int s = 0; s < kBatchGraphSteps; ++s)
            for (int item : B->branches[g])
                if (int e = item_step(B, item, s & 1, B->side[g])) return e;
        if (cudaEventRecord(B->ev[g + 1], B->side[g]) != cudaSuccess) return set_error(BGK_ERR_CUDA, "join record");
        if (cudaStreamWaitEvent(B->cap, B->ev[g + 1], 0) != cudaSuccess) return set_error(BGK_ERR_CUDA, "join wait");
    }
    return BGK_OK;
}

// One batch step: outflow planes of the inflow members, then the persistent launch.
int batch_one(bgk_batch* B, cudaStream_t st) {
    const int par = (int)(B->steps & 1);
    if (B->chunk > 0) {
        for (const std::vector<int>& br : B->branches)
            for (int item : br)
                if (int e = item_step(B, item, par, st)) return e;
    } else {
        for (int idx : B->inflow) {
            void* a[19];
            member_arrays(B, (size_t)idx, par, a);
            if (int e = outflow_launch(B->kind, &B->lats[idx]->p, a, st)) return e;
        }
        if (int e = batch_launch(B, par, st)) return e;
    }
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
        if (nsteps) B->lats[i]->outflow_fresh = false;   // batched steps do not write the next outflow plane
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
    if (B->chunk > 0 && B->branches.size() > 1) rc = capture_branches(B);
    else
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
    if (int rc2 = build_groups(B)) { bgk_batch_destroy(B); return rc2; }
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
    return build_groups(B);
}

int bgk_batch_destroy(bgk_batch* B) {
    if (!B) return BGK_OK;
    drop_graph(B);
    if (B->cap) cudaStreamDestroy(B->cap);
    for (cudaStream_t s : B->side) cudaStreamDestroy(s);
    for (cudaEvent_t ev : B->ev) cudaEventDestroy(ev);
    dev_free(B->desc);
    dev_free(B->tile_begin);
    dev_free(B->counter);
    dev_free(B->chunks);
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

int bgk_batch_set_chunk(bgk_batch* B, int warps) {
    if (!B || warps < 0 || warps > 4096 || (warps % 8) != 0) return set_error(BGK_ERR_ARG, "bad chunk size");
    if (warps == B->chunk) return BGK_OK;
    drop_graph(B);
    B->chunk = warps;
    return build_groups(B);
}

int bgk_batch_set_solo(bgk_batch* B, long long min_nodes) {
    if (!B || min_nodes < 0) return set_error(BGK_ERR_ARG, "bad solo threshold");
    if (min_nodes == B->solo_nodes) return BGK_OK;
    drop_graph(B);
    B->solo_nodes = min_nodes;
    return build_groups(B);
}

long long bgk_batch_get_solo(const bgk_batch* B) { return B ? B->solo_nodes : -1; }

int bgk_batch_get_chunk(const bgk_batch* B, int* warps) {
    if (!B) return set_error(BGK_ERR_ARG, "null batch");
    if (warps) *warps = B->chunk;
    return BGK_OK;
}

int bgk_batch_groups(const bgk_batch* B) {
    return B ? (int)(B->chunk > 0 ? B->groups.size() + B->solo.size() : 1) : -1;
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
    // long enough for the graph path (runs of 2 kBatchGraphSteps or more):
    // the warm-up run captures the graph, the timed run replays it
    const int n = std::max(2 * kBatchGraphSteps, (trial_steps + 1) / 2 * 2);
    const int subs[] = {1, 2, 4, 8};
    const int bpsms[] = {0, 2, 3, 4};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bsub = B->sub, bb = B->bpsm, bchunk = B->chunk;
    long long bsolo = B->solo_nodes, solo = 0;
    long long used = 0;
    auto trial = [&](int chunk, int s, int b) -> int {
        if (int e = bgk_batch_set_solo(B, solo)) return e;
        if (int e = bgk_batch_set_chunk(B, chunk)) return e;
        if (chunk == 0)
            if (int e = bgk_batch_set_config(B, s, b)) return e;
        if (int e = bgk_batch_step(B, n, st)) return e;   // warm, graph capture
        cudaEventRecord(e0, st);
        if (int e = bgk_batch_step(B, n, st)) return e;
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        used += 2 * n;
        if (ms < best) { best = ms; bsub = s; bb = b; bchunk = chunk; bsolo = solo; }
        return BGK_OK;
    };
    // grouped form: chunk sizes, then members of 2^21 / 2^19 nodes or more
    // stepping solo with the best chunk size; tile-queue forms: grab size x
    // blocks per SM
    for (int c : {8, 16, 32, 64, 128})
        if (int e = trial(c, B->sub, B->bpsm)) return e;
    const int cbest = bchunk > 0 ? bchunk : 32;
    for (long long t : {1LL << 21, 1LL << 19}) {
        solo = t;
        if (int e = trial(cbest, B->sub, B->bpsm)) return e;
    }
    solo = 0;
    for (int s : subs)
        for (int b : bpsms) {
            if (b == 0 && s != 1) continue;   // one block per tile has no queue grab size
            if (int e = trial(0, s, b)) return e;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    bgk_batch_set_config(B, bsub, bb);
    bgk_batch_set_solo(B, bsolo);
    bgk_batch_set_chunk(B, bchunk);
    if (steps_used) *steps_used = (int)used;
    return BGK_OK;
}

long long bgk_batch_nodes(const bgk_batch* B) { return B ? B->nodes : -1; }
long long bgk_batch_tiles(const bgk_batch* B) { return B ? (long long)B->ntiles : -1; }

}  // extern "C"
