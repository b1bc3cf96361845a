// sph_api.cu — C-ABI implementation: handle, device buffers, step orchestration.
//
// Replaces the reference's SPHSystem constructor allocations
// (SPH-3D-2/sph_system.cpp:34-47,95-101), its per-step launch sequence
// (animation(), SPH-3D-2/sph_system.cpp:302-404; animate(), SPH-2D/sph_system.cpp:190-264)
// and its launch wrappers (SPH-3D-2/sph_system.cuh).  Differences by design:
// one stream per handle, no host synchronisation inside a step (the particle
// count lives on the device), state in SoA float4 arrays, every CUDA status
// checked and reported through the int return codes.
#include "../../include/sph/sph.h"
#include "sph_kernels.cuh"
#include "sph_scan.cuh"
#include "sph_mc.cuh"
#include "sph_persistent.cuh"

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

using namespace sph;

struct Rollout;   // differentiable rollout state (sph_rollout_impl.cuh)

struct sph_handle {
    sph_config cfg;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;        // where the handle's work runs
    cudaStream_t own_stream = nullptr;    // the handle's own stream (destroyed with it)
    uint32_t cap = 0, ncells = 0;
    CanonPtrs buf[2];
    int cur = 0;
    Counters *cnt = nullptr;       // [2], one per parity
    WorkPtrs w;
    uint32_t *scan_blocks = nullptr;  // kScanBlocks * 2 u32
    uint32_t *scan_grand = nullptr;   // scratch total
    uint32_t *stat_buf = nullptr;     // sph_last_step_stats: level-2 count
    uint32_t n_ub = 0;                // host upper bound of the live count
    uint32_t n_last_sorted = 0;       // count the last step started with (host copy)
    bool have_step = false;
    bool debug = false;
    uint32_t last_launches = 0;
    std::vector<void *> allocs;
    std::string err;
    // density grid + marching cubes
    McBuffers mc;
    bool grid_valid = false;
    uint64_t step_index = 0;
    // reference-layout staging buffer (allocated on first use)
    float *aos = nullptr;
    // per-stage profiling
    static constexpr int kMaxStages = 24;
    bool profiling = false;
    cudaEvent_t ev[kMaxStages + 1] = {};
    const char *stage_name[kMaxStages] = {};
    int nstages = 0;
    // asynchronous readback: side stream, per-parity completion events
    cudaStream_t rb_stream = nullptr;
    cudaEvent_t rb_ready = nullptr;
    cudaEvent_t rb_done[2] = {nullptr, nullptr};
    bool rb_pending[2] = {false, false};
    // CUDA graphs of one step, one per buffer parity
    bool use_graph = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_grid[2] = {0, 0};   // launch_key at capture
    uint32_t graph_launches[2] = {0, 0};
    // batched scenes: device table of 2 float4 per scene (own allocation,
    // replaced by sph_set_scenes)
    float4 *scene_tab = nullptr;
    uint32_t scene_tab_cap = 0;
    // differentiable rollout; state_gen counts state and config changes made
    // outside of steps, so a rollout can tell it still describes the state
    Rollout *ro = nullptr;
    uint64_t state_gen = 0;
    // launch shape per tuned stage (sph_set_tuning / sph_autotune)
    double *cons = nullptr;   // conserved-quantity partial sums (allocated on first use)
    // defaults: the streaming stages at full occupancy with grid-stride loops;
    // density, force, energy and write one particle per thread in 128-thread
    // blocks (many more blocks than fit at once, so the block scheduler evens
    // out warps of unequal work), the autotuner's usual choice on 1M particles
    uint32_t tune_bs[SPH_TUNE_STAGES] = {256, 256, 256, 128, 128, 128, 256, 128};
    uint32_t tune_bpsm[SPH_TUNE_STAGES] = {8, 8, 8, 64, 64, 64, 8, 64};
    uint32_t tune_minb[SPH_TUNE_STAGES] = {0, 0, 0, 0, 0, 0, 0, 0};   // 1: register-capped variant
    // persistent step: the whole step as one cooperative launch
    bool persistent = false;
    uint32_t spin_limit = SPH_PERSISTENT_SPIN_DEFAULT;
    GridSync *gsync = nullptr;               // [2]: persistent launches alternate between them
    uint32_t persist_launch = 0;             // persistent launches so far (picks the barrier state)
    bool counts_zero = false;                // the cell counts are zero (left so by a persistent step)
    // a persistent step without split and merge leaves the next step's hash
    // (keys, slots, counts) of the state it wrote; valid while the state, the
    // config and the step index are the ones it saw
    bool counts_hashed = false;
    uint64_t hashed_gen = 0, hashed_step = 0;
    // the current state's acc, dens, press, energy and surface are still to be
    // written from the last step's sorted arrays (k_materialize)
    bool outputs_pending = false;
    int persist_blocks_per_sm[2][2] = {};    // resident blocks of k_step_persistent<2|3, 64|256> (0: not queried)
    int persist_cluster_ok[2] = {0, 0};      // one-cluster launches: 1 possible, -1 not, 0 not queried
    bool persist_use_cluster = true;         // off: always the polled barriers
};

namespace {

const char *kNoHandle = "null handle";
void rollout_free(Rollout *r);

template <typename T> int dalloc(sph_handle *h, T **p, size_t count)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (count ? count : 1));
    if (e != cudaSuccess) {
        h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return SPH_ERR_CUDA;
    }
    cudaMemset(q, 0, sizeof(T) * (count ? count : 1));
    h->allocs.push_back(q);
    *p = (T *)q;
    return SPH_OK;
}

int cuda_check(sph_handle *h, const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        h->err = std::string(what) + ": " + cudaGetErrorString(e);
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

uint32_t total_cells(const sph_config &c) { return c.ncell[0] * c.ncell[1] * (c.dim == 3 ? c.ncell[2] : 1u); }

int validate(const sph_config *c, std::string &why)
{
    if (!c) { why = "null config"; return SPH_ERR_INVALID; }
    if (c->dim != 2 && c->dim != 3) { why = "dim must be 2 or 3"; return SPH_ERR_INVALID; }
    if (c->max_particle == 0 || c->max_particle > (1u << 30)) { why = "max_particle out of range"; return SPH_ERR_INVALID; }
    if (!(c->cell_size > 0.0f)) { why = "cell_size must be > 0"; return SPH_ERR_INVALID; }
    for (uint32_t a = 0; a < c->dim; ++a)
        if (c->ncell[a] == 0) { why = "empty cell grid"; return SPH_ERR_INVALID; }
    uint64_t C = (uint64_t)c->ncell[0] * c->ncell[1] * (c->dim == 3 ? c->ncell[2] : 1u);
    if (C >= (1ull << 31)) { why = "cell grid too large"; return SPH_ERR_INVALID; }
    if (c->split_ways != 2 && c->split_ways != 4) { why = "split_ways must be 2 or 4"; return SPH_ERR_INVALID; }
    if (c->kernel[0] > c->cell_size * 1.0000001f || c->kernel[1] > c->cell_size * 1.0000001f) {
        why = "kernel length exceeds the cell size (neighbour stencil would miss pairs)";
        return SPH_ERR_INVALID;
    }
    return SPH_OK;
}

uint32_t grid_for(const sph_handle *h, uint32_t work)
{
    uint32_t b = (work + kThreads - 1) / kThreads;
    uint32_t cap = (uint32_t)h->num_sms * 8u;
    return std::max(1u, std::min(b, cap));
}

// Grid of a tuned stage: blocks of tune_bs threads, capped at tune_bpsm
// blocks per SM; the kernels loop grid-stride over the rest.
uint32_t grid_st(const sph_handle *h, uint32_t work, int stage)
{
    const uint32_t bs = h->tune_bs[stage];
    const uint32_t b = (work + bs - 1) / bs;
    const uint32_t cap = (uint32_t)h->num_sms * h->tune_bpsm[stage];
    return std::max(1u, std::min(b, cap));
}

// Launch key of the step: every stage's grid and block size (a captured
// graph is valid while it is unchanged).
uint64_t launch_key(const sph_handle *h)
{
    uint64_t k = 1469598103934665603ull;
    for (int st = 0; st < SPH_TUNE_STAGES; ++st) {
        const uint32_t work = st == SPH_TUNE_MERGE ? h->ncells : h->n_ub;
        k = (k ^ grid_st(h, work, st)) * 1099511628211ull;
        k = (k ^ (h->tune_bs[st] * 2u + (h->tune_minb[st] ? 1u : 0u))) * 1099511628211ull;
    }
    return k;
}

// Instantiates a launch for the stage's block size B (128, 256 or 512; the
// SWITCH2 kernels hold a 48 KB shared list at 256 threads and stop at 256).
#define SPH_BS_SWITCH(bs, ...)                                   \
    switch (bs) {                                                \
    case 128: { constexpr int B = 128; __VA_ARGS__; } break;     \
    case 512: { constexpr int B = 512; __VA_ARGS__; } break;     \
    default: { constexpr int B = 256; __VA_ARGS__; } break;      \
    }
// SWITCH2 also sets the occupancy target M (minimum resident blocks per SM
// handed to __launch_bounds__, i.e. the register budget the compiler works
// to): 6 blocks of 128 / 3 of 256 (85 registers) by default, 8 / 4 (64
// registers) for the register-capped build.
#define SPH_BS_SWITCH2(bs, cap, ...)                                                    \
    switch ((bs) * 16 + ((cap) ? 1 : 0)) {                                              \
    case 128 * 16 + 1: { constexpr int B = 128, M = 8; __VA_ARGS__; } break;            \
    case 128 * 16: { constexpr int B = 128, M = 6; __VA_ARGS__; } break;                \
    case 256 * 16 + 1: { constexpr int B = 256, M = 4; __VA_ARGS__; } break;            \
    default: { constexpr int B = 256, M = 3; __VA_ARGS__; } break;                      \
    }

// Exclusive scan of u32 `in` -> `out`; length from len_ptr (device) or
// len_const.  skip_if_zero: a device count of the nonzero inputs (0: the
// output is all zeros and is written without a scan).
void scan_u32(sph_handle *h, const uint32_t *in, uint32_t *out, const uint32_t *len_ptr, uint32_t len_const,
              uint32_t *grand, int total_at_len, uint32_t *list, const uint32_t *skip_if_zero = nullptr)
{
    scan_phase1<uint32_t><<<kScanBlocks, kScanThreads, 0, h->stream>>>(in, len_ptr, len_const, h->scan_blocks,
                                                                       skip_if_zero);
    scan_phase23<uint32_t><<<kScanBlocks, kScanThreads, 0, h->stream>>>(in, out, len_ptr, len_const, h->scan_blocks,
                                                                        grand, total_at_len, list, skip_if_zero);
    h->last_launches += 2;
}

// Marching cubes over the current device grid: classify, scan, emit.
void run_mc(sph_handle *h)
{
    McBuffers &mc = h->mc;
    // one thread per cube: every thread's corner loads are in flight at once
    const uint32_t GQ = (mc.cubes + kThreads - 1) / kThreads;
    k_mc_count<<<GQ, kThreads, 0, h->stream>>>(h->cfg, mc.dens, mc.cube_cnt);
    scan_u32(h, mc.cube_cnt, mc.cube_off, nullptr, mc.cubes, mc.num_tri, 0, nullptr);
    k_mc_emit<<<GQ, kThreads, 0, h->stream>>>(h->cfg, mc.dens, mc.normal, mc.cube_cnt, mc.cube_off, mc.max_tri,
                                               mc.tri);
    h->last_launches += 2;
}

// Records the end of a named stage when profiling (event 0 marks the start).
void stage(sph_handle *h, const char *name)
{
    if (!h->profiling || h->nstages >= sph_handle::kMaxStages) return;
    h->stage_name[h->nstages] = name;
    cudaEventRecord(h->ev[++h->nstages], h->stream);
}

// Deferred outputs: the ordinary launches record where each output comes
// from instead of writing acc, dens, press, energy and surface, except under
// the 2D cell merge rule, whose criterion reads the previous state's energy
// and surface (beyond the live count too) at merge time.
static bool defer_outputs(const sph_handle *h)
{
    return h->cfg.merge_rule != SPH_MERGE_WAVELET_CELL && h->cap <= kOutSlot;
}

// Writes the current state's deferred outputs (before anything reads the
// whole state).
void ensure_outputs(sph_handle *h)
{
    if (!h->outputs_pending) return;
    const uint32_t G = grid_for(h, h->n_ub);
    if (h->cfg.dim == 3) k_materialize<3><<<G, kThreads, 0, h->stream>>>(h->cfg, h->cnt + h->cur, h->buf[h->cur], h->w);
    else k_materialize<2><<<G, kThreads, 0, h->stream>>>(h->cfg, h->cnt + h->cur, h->buf[h->cur], h->w);
    h->outputs_pending = false;
}

// The cell counts, keys and slots hold the hash of the current state: the
// step that wrote it hashed it (its write-out), and nothing has changed the
// state, the config or the counts since.
static bool hash_ready(const sph_handle *h)
{
    return h->counts_hashed && h->hashed_gen == h->state_gen && h->hashed_step == h->step_index;
}

// Clears the cell counts and hashes the current state (the first stage of a
// step whose state no step has hashed).
template <int DIM> void hash_prologue(sph_handle *h)
{
    const sph_config &c = h->cfg;
    const int p = h->cur;
    WorkPtrs w = h->w;
    cudaStream_t s = h->stream;
    cudaMemsetAsync(w.cell_count, 0, sizeof(uint32_t) * h->ncells, s);
    SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_HASH],
                  k_hash<DIM, B><<<grid_st(h, h->n_ub, SPH_TUNE_HASH), B, 0, s>>>(c, h->cnt + p, h->buf[p], w));
    h->last_launches += 1;
}

// One step as separate launches.  prologue = false leaves out the hash of a
// state no step has hashed (a captured graph: the replay runs it when needed).
template <int DIM> int run_step(sph_handle *h, bool prologue = true)
{
    const sph_config &c = h->cfg;
    const int p = h->cur;
    Counters *cin = h->cnt + p, *cout = h->cnt + (p ^ 1);
    CanonPtrs in = h->buf[p], out = h->buf[p ^ 1];
    h->w.pos_comp = c.compensated_positions ? 1u : 0u;
    WorkPtrs w = h->w;
    if (c.walk_only) {   // the same pairs found by the stencil walks
        w.nlist = w.ncnt = nullptr;
    }
    if (!defer_outputs(h)) w.out_src = nullptr;
    cudaStream_t s = h->stream;
    h->nstages = 0;
    if (h->profiling) cudaEventRecord(h->ev[0], s);

    const uint32_t nub = h->n_ub;
    if (prologue && !hash_ready(h)) {
        hash_prologue<DIM>(h);
        stage(h, "hash");
    }
    scan_u32(h, w.cell_count, w.cell_off, nullptr, h->ncells, h->scan_grand, 1, nullptr);
    // the scan has read the counts: cleared for the write-out's hash of the next state
    cudaMemsetAsync(w.cell_count, 0, sizeof(uint32_t) * h->ncells, s);
    h->counts_zero = false;
    stage(h, "scan_cells");
    SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_SCATTER], k_scatter<B><<<grid_st(h, nub, SPH_TUNE_SCATTER), B, 0, s>>>(cin, w));
    stage(h, "scatter");
    SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_REORDER],
                  k_reorder<B><<<grid_st(h, nub, SPH_TUNE_REORDER), B, 0, s>>>(cin, in, w));
    stage(h, "reorder");
    const uint32_t gd = grid_st(h, nub, SPH_TUNE_DENSITY);
    if (c.density_skip_r2 == 0.0f) {
        SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_DENSITY], k_density<DIM, B, false><<<gd, B, 0, s>>>(c, cin, w));
    } else {
        SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_DENSITY], k_density<DIM, B, true><<<gd, B, 0, s>>>(c, cin, w));
    }
    stage(h, "density");
    SPH_BS_SWITCH2(h->tune_bs[SPH_TUNE_FORCE], h->tune_minb[SPH_TUNE_FORCE],
                   k_force_integrate<DIM, B, M><<<grid_st(h, nub, SPH_TUNE_FORCE), B, 0, s>>>(c, cin, w));
    stage(h, "force_integrate");
    // density grid + surface mid-step: stale cell lists, integrated positions
    // (SPH-3D-2/sph_system.cpp:336-362)
    if (DIM == 3 && c.grid_every && h->mc.nodes && h->step_index % c.grid_every == 0) {
        // one thread per node pair, uncapped: the block scheduler spreads the
        // heavy pairs (cells of split particles hold four times the candidates)
        k_splat<<<(h->mc.nodes / 2 + kThreads) / kThreads, kThreads, 0, s>>>(c, w.cell_off, w.spos_n, h->mc.dens);
        k_grid_normals<<<(h->mc.nodes + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, h->mc.dens, h->mc.normal);
        h->last_launches += 2;
        run_mc(h);
        h->grid_valid = true;
        stage(h, "surface");
    }
    SPH_BS_SWITCH2(h->tune_bs[SPH_TUNE_ENERGY], h->tune_minb[SPH_TUNE_ENERGY],
                   k_energy_split<DIM, B, M><<<grid_st(h, nub, SPH_TUNE_ENERGY), B, 0, s>>>(c, cin, in, w,
                                                                                          h->debug ? 1 : 0));
    stage(h, "energy_split");
    h->last_launches += 6;
    scan_u32(h, w.split_c, w.split_rank, &cin->n, 0, &cin->n_split, 0, w.split_list, &cin->split_flags);
    k_split_guard<<<1, 1, 0, s>>>(c, cin, h->cap);
    h->last_launches += 1;
    stage(h, "scan_split");
    if (c.use_merge) {   // one lane per cell, a warp scans 32 cells at a time
        SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_MERGE],
                      k_merge<DIM, B><<<grid_st(h, h->ncells, SPH_TUNE_MERGE), B, 0, s>>>(c, cin, in, w, h->ncells,
                                                                                          h->cap));
        h->last_launches += 1;
        stage(h, "merge");
    }
    scan_u32(h, w.removed_c, w.removed_rank, &cin->n, 0, &cin->n_removed, 0, nullptr, &cin->removed_flags);
    stage(h, "scan_removed");
    SPH_BS_SWITCH(h->tune_bs[SPH_TUNE_WRITE],
                  k_write<DIM, B><<<grid_st(h, nub, SPH_TUNE_WRITE), B, 0, s>>>(c, cin, cout, in, out, w, 1));
    h->last_launches += 1;
    stage(h, "write");
    h->cur = p ^ 1;
    h->step_index++;
    h->counts_hashed = true;   // the write-out hashed the new state
    h->hashed_gen = h->state_gen;
    h->hashed_step = h->step_index;
    h->outputs_pending = w.out_src != nullptr;
    uint64_t ub = h->n_ub;
    if (c.use_split) ub *= (c.split_ways == 4 ? 4u : 2u);
    h->n_ub = (uint32_t)std::min<uint64_t>(ub, h->cap);
    return cuda_check(h, "sph_step launch");
}

// The step as one cooperative launch of k_step_persistent (sph_persistent.cuh):
// same stages, same arithmetic, grid-wide barriers instead of launch
// boundaries.  One thread per particle of the live-count bound: up to 4,096
// particles one cluster of 256-thread blocks (hardware cluster barriers),
// up to 16K blocks of 64 threads (a small scene's stages spread over more
// SMs), above that blocks of 256; the grid is capped at what fits resident.
constexpr uint32_t kPersistSmallN = 16384;
constexpr uint32_t kPersistMaxBlocks = 1024;

// A grid of at most kPersistMaxCluster blocks of 256 threads is launched as
// one cluster when the device can hold it; -1 in cluster_ok: it cannot.
constexpr uint32_t kPersistMaxCluster = 16;

template <int DIM> int launch_persistent_cluster(sph_handle *h, int &cluster_ok, uint32_t G, int nsteps)
{
    const sph_config &c = h->cfg;
    const int p = h->cur;
    auto kern = k_step_persistent<DIM, 256>;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(G);
    lc.blockDim = dim3(256);
    lc.dynamicSmemBytes = 0;
    lc.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    if (cluster_ok == 0) {
        int n = 0;
        cluster_ok = -1;
        if (cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveClusters(&n, (const void *)kern, &lc) == cudaSuccess && n >= 1)
            cluster_ok = 1;
        cudaGetLastError();
        if (cluster_ok < 0) return SPH_ERR_INVALID;
    }
    const CanonPair buf = {{h->buf[0], h->buf[1]}};
    h->w.pos_comp = c.compensated_positions ? 1u : 0u;
    WorkPtrs w = h->w;
    if (c.walk_only) w.nlist = w.ncnt = nullptr;
    w.out_src = nullptr;   // the persistent step writes every output
    // the polled barriers' state is not used; the one due next is left as it
    // is (clean), so polled launches that follow keep alternating correctly
    PersistArgs a = {};
    a.gs = a.gs_next = h->gsync + (h->persist_launch & 1u);
    a.spin_limit = h->spin_limit;
    a.ncells = h->ncells;
    a.cap = h->cap;
    a.scan_blocks = h->scan_blocks;
    a.scan_grand = h->scan_grand;
    a.want_tv = h->debug ? 1 : 0;
    a.ranks = (c.use_split || c.use_merge) ? 1 : 0;
    a.cluster = 1;
    a.hash_ready = hash_ready(h) ? 1 : 0;
    a.parity = p;
    a.nsteps = nsteps;
    if (!a.hash_ready && !h->counts_zero) cudaMemsetAsync(w.cell_count, 0, sizeof(uint32_t) * h->ncells, h->stream);
    if (cudaLaunchKernelEx(&lc, kern, c, h->cnt, buf, w, a) != cudaSuccess)
        return cuda_check(h, "persistent step cluster launch");
    return SPH_OK;
}

template <int DIM, int BS> int launch_persistent(sph_handle *h, int &per_sm, uint32_t G_want, int nsteps)
{
    const sph_config &c = h->cfg;
    const int p = h->cur;
    Counters *cnt = h->cnt;
    CanonPair buf = {{h->buf[0], h->buf[1]}};
    h->w.pos_comp = c.compensated_positions ? 1u : 0u;
    WorkPtrs w = h->w;
    if (c.walk_only) w.nlist = w.ncnt = nullptr;
    w.out_src = nullptr;   // the persistent step writes every output
    auto kern = k_step_persistent<DIM, BS>;
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BS, 0) != cudaSuccess || per_sm < 1) {
            per_sm = 0;
            return cuda_check(h, "persistent step occupancy");
        }
    }
    const uint32_t G = std::min<uint32_t>({G_want, (uint32_t)(per_sm * h->num_sms), kPersistMaxBlocks,
                                           (uint32_t)kScanBlocks});
    PersistArgs a;
    const uint32_t q = h->persist_launch & 1u;
    a.gs = h->gsync + q;
    a.gs_next = h->gsync + (q ^ 1u);
    a.spin_limit = h->spin_limit;
    a.ncells = h->ncells;
    a.cap = h->cap;
    a.scan_blocks = h->scan_blocks;
    a.scan_grand = h->scan_grand;
    a.want_tv = h->debug ? 1 : 0;
    a.ranks = (c.use_split || c.use_merge) ? 1 : 0;
    a.cluster = 0;
    a.hash_ready = hash_ready(h) ? 1 : 0;
    a.parity = p;
    a.nsteps = nsteps;
    sph_config cc = c;
    void *args[] = {&cc, &cnt, &buf, &w, &a};
    if (!a.hash_ready && !h->counts_zero) cudaMemsetAsync(w.cell_count, 0, sizeof(uint32_t) * h->ncells, h->stream);
    if (cudaLaunchCooperativeKernel((void *)kern, dim3(G), dim3(BS), args, 0, h->stream) != cudaSuccess)
        return cuda_check(h, "persistent step launch");
    return SPH_OK;
}

// Steps one persistent launch runs at most.  Only steps whose particle count
// cannot grow (no splits) share a launch: the grid is sized for the count
// the first step starts from.
constexpr int kPersistMaxSteps = 256;

template <int DIM> int run_step_persistent(sph_handle *h, int nsteps)
{
    const sph_config &c = h->cfg;
    const int p = h->cur;
    int rc = SPH_ERR_INVALID;
    const uint32_t g256 = std::max<uint32_t>(1u, (h->n_ub + 255) / 256);
    if (g256 <= kPersistMaxCluster && h->persist_cluster_ok[DIM - 2] >= 0 && h->persist_use_cluster)
        rc = launch_persistent_cluster<DIM>(h, h->persist_cluster_ok[DIM - 2], g256, nsteps);
    if (rc != SPH_OK) {
        if (h->n_ub <= kPersistSmallN)
            rc = launch_persistent<DIM, 64>(h, h->persist_blocks_per_sm[DIM - 2][0], (h->n_ub + 63) / 64, nsteps);
        else
            rc = launch_persistent<DIM, 256>(h, h->persist_blocks_per_sm[DIM - 2][1], (h->n_ub + 255) / 256,
                                             nsteps);
        if (rc) return rc;
        h->persist_launch++;   // the polled barriers alternate between their two states
    }
    // the scatter stage cleared the counts and the write-out hashed the new
    // state into them
    h->counts_zero = false;
    h->counts_hashed = true;
    h->outputs_pending = false;
    h->last_launches += 1;
    h->cur = (p + nsteps) & 1;
    h->step_index += (uint64_t)nsteps;
    h->hashed_gen = h->state_gen;
    h->hashed_step = h->step_index;
    uint64_t ub = h->n_ub;
    if (c.use_split) ub *= (c.split_ways == 4 ? 4u : 2u);   // one step per launch then
    h->n_ub = (uint32_t)std::min<uint64_t>(ub, h->cap);
    return cuda_check(h, "sph_step persistent");
}

void pack4(const float *src, int dim, uint32_t n, std::vector<float4> &dst, const uint32_t *level)
{
    dst.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (src) {
            v.x = src[(size_t)i * dim];
            v.y = src[(size_t)i * dim + 1];
            if (dim == 3) v.z = src[(size_t)i * dim + 2];
        }
        if (level) v.w = (float)level[i];
        dst[i] = v;
    }
}

void unpack4(const std::vector<float4> &src, int dim, uint32_t n, float *dst)
{
    if (!dst) return;
    for (uint32_t i = 0; i < n; ++i) {
        dst[(size_t)i * dim] = src[i].x;
        dst[(size_t)i * dim + 1] = src[i].y;
        if (dim == 3) dst[(size_t)i * dim + 2] = src[i].z;
    }
}

uint32_t read_n(sph_handle *h)
{
    uint32_t n = 0;
    cudaMemcpyAsync(&n, &h->cnt[h->cur].n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    return n;
}

void write_n(sph_handle *h, uint32_t n)
{
    Counters c0;
    std::memset(&c0, 0, sizeof(c0));
    cudaMemcpyAsync(&c0, &h->cnt[h->cur], sizeof(Counters), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    c0.n = n;
    c0.error &= ~(1u << SPH_ERR_TIMEOUT);   // a new state: steps may run again after a timeout
    cudaMemcpyAsync(&h->cnt[h->cur], &c0, sizeof(Counters), cudaMemcpyHostToDevice, h->stream);
    // a new state: the persistent step's barrier states start clean (a
    // timeout leaves its abort flag set) and the cell counts are cleared
    // before its next launch
    cudaMemsetAsync(h->gsync, 0, sizeof(GridSync) * 2, h->stream);
    h->counts_zero = false;
    h->counts_hashed = false;
    h->outputs_pending = false;   // the caller wrote every field
    cudaStreamSynchronize(h->stream);
}

}  // namespace

extern "C" {

int sph_create(const sph_config *cfg, sph_handle **out)
{
    if (!out) return SPH_ERR_INVALID;
    *out = nullptr;
    std::string why;
    int rc = validate(cfg, why);
    if (rc) { fprintf(stderr, "sph_create: %s\n", why.c_str()); return rc; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SPH_ERR_NO_DEVICE;
    sph_handle *h = new sph_handle();
    h->cfg = *cfg;
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return SPH_ERR_CUDA;
    }
    h->own_stream = h->stream;
    h->cap = cfg->max_particle;
    h->ncells = total_cells(*cfg);
    const size_t cap = h->cap, C = h->ncells;
    rc = SPH_OK;
    for (int b = 0; b < 2 && !rc; ++b) {
        CanonPtrs &q = h->buf[b];
        rc |= dalloc(h, &q.pos, cap); rc |= dalloc(h, &q.vel, cap);
        rc |= dalloc(h, &q.ev, cap); rc |= dalloc(h, &q.acc, cap);
        rc |= dalloc(h, &q.dens, cap); rc |= dalloc(h, &q.press, cap);
        rc |= dalloc(h, &q.energy, cap); rc |= dalloc(h, &q.surface, cap);
        rc |= dalloc(h, &q.interior, cap); rc |= dalloc(h, &q.scene, cap); rc |= dalloc(h, &q.pos_lo, cap);
        rc |= dalloc(h, &q.sibling, cap);
        if (!rc) cudaMemset(q.sibling, 0xff, sizeof(uint32_t) * cap);   // no split groups
    }
    WorkPtrs &w = h->w;
    rc |= dalloc(h, &h->cnt, 2);
    rc |= dalloc(h, &w.key, cap); rc |= dalloc(h, &w.slot, cap); rc |= dalloc(h, &w.tmp, cap);
    rc |= dalloc(h, &w.cell_count, C); rc |= dalloc(h, &w.cell_off, C + 1);
    rc |= dalloc(h, &w.sidx, cap); rc |= dalloc(h, &w.skey, cap); rc |= dalloc(h, &w.inv, cap);
    rc |= dalloc(h, &w.spos, cap); rc |= dalloc(h, &w.svel, cap); rc |= dalloc(h, &w.sev, cap);
    rc |= dalloc(h, &w.saux, cap);
    rc |= dalloc(h, &w.spos_n, cap); rc |= dalloc(h, &w.svel_n, cap); rc |= dalloc(h, &w.sev_n, cap);
    rc |= dalloc(h, &w.sacc_n, cap);
    rc |= dalloc(h, &w.ssurf, cap); rc |= dalloc(h, &w.senergy, cap);
    rc |= dalloc(h, &w.snbr, cap); rc |= dalloc(h, &w.sinter, cap);
    rc |= dalloc(h, &w.stv, cap); rc |= dalloc(h, &w.sscene, cap);
    rc |= dalloc(h, &w.spos_lo, cap); rc |= dalloc(h, &w.spos_lo_n, cap);
    rc |= dalloc(h, &w.fnb_a, cap); rc |= dalloc(h, &w.fnb_b, cap);
    rc |= dalloc(h, &w.out_src, cap);
    // neighbour candidate lists (512 B per particle of capacity); without
    // them (very large capacities) the force and energy kernels walk the
    // stencil themselves
    w.nlist = nullptr;
    w.ncnt = nullptr;
    w.nl_stride = (uint32_t)cap;
    if ((uint64_t)cap * kNbrListCap * sizeof(uint32_t) <= (12ull << 30)) {
        rc |= dalloc(h, &w.nlist, cap * kNbrListCap);
        rc |= dalloc(h, &w.ncnt, cap);
    }
    w.pos_comp = cfg->compensated_positions ? 1u : 0u;
    w.scene_tab = nullptr;
    w.nscenes = 0;
    w.merge_to = nullptr;
    w.mvs = nullptr;
    w.wall = nullptr;
    rc |= dalloc(h, &w.split_c, cap); rc |= dalloc(h, &w.removed_c, cap);
    rc |= dalloc(h, &w.split_rank, cap); rc |= dalloc(h, &w.removed_rank, cap);
    rc |= dalloc(h, &w.split_list, cap); rc |= dalloc(h, &w.leader, cap);
    rc |= dalloc(h, &w.mpos, cap); rc |= dalloc(h, &w.mvel, cap); rc |= dalloc(h, &w.mev, cap);
    rc |= dalloc(h, &w.macc, cap); rc |= dalloc(h, &w.menergy, cap);
    rc |= dalloc(h, &h->scan_blocks, (size_t)kScanBlocks * 2);
    rc |= dalloc(h, &h->scan_grand, 4);
    rc |= dalloc(h, &h->stat_buf, 4);
    rc |= dalloc(h, &h->gsync, 2);
    if (!rc) rc = mc_alloc(h->mc, *cfg, h->allocs);
    if (rc) {
        fprintf(stderr, "sph_create: %s\n", h->err.c_str());
        sph_destroy(h);
        return rc ? rc : SPH_ERR_CUDA;
    }
    cudaDeviceSynchronize();
    *out = h;
    return SPH_OK;
}

int sph_destroy(sph_handle *h)
{
    if (!h) return SPH_ERR_INVALID;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int k = 0; k <= sph_handle::kMaxStages; ++k)
        if (h->ev[k]) cudaEventDestroy(h->ev[k]);
    for (int p = 0; p < 2; ++p)
        if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
    if (h->rb_stream) {
        cudaStreamSynchronize(h->rb_stream);
        cudaStreamDestroy(h->rb_stream);
        cudaEventDestroy(h->rb_ready);
        cudaEventDestroy(h->rb_done[0]);
        cudaEventDestroy(h->rb_done[1]);
    }
    rollout_free(h->ro);
    for (void *p : h->allocs) cudaFree(p);
    if (h->scene_tab) cudaFree(h->scene_tab);
    if (h->cons) cudaFree(h->cons);
    if (h->stream && h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return SPH_OK;
}

int sph_set_config(sph_handle *h, const sph_config *cfg)
{
    if (!h || !cfg) return SPH_ERR_INVALID;
    std::string why;
    if (validate(cfg, why)) { h->err = why; return SPH_ERR_INVALID; }
    if (cfg->dim != h->cfg.dim || cfg->max_particle != h->cfg.max_particle ||
        total_cells(*cfg) != h->ncells || cfg->ncell[0] != h->cfg.ncell[0] || cfg->ncell[1] != h->cfg.ncell[1]) {
        h->err = "sph_set_config: dimension, capacity and cell grid are fixed at creation";
        return SPH_ERR_INVALID;
    }
    if (cfg->ndens[0] != h->cfg.ndens[0] || cfg->ndens[1] != h->cfg.ndens[1] || cfg->ndens[2] != h->cfg.ndens[2]) {
        h->err = "sph_set_config: density grid is fixed at creation";
        return SPH_ERR_INVALID;
    }
    ensure_outputs(h);   // the last step's outputs, under the config it ran with
    if (cfg->compensated_positions && !h->cfg.compensated_positions) {
        // the low parts start from zero when compensation is switched on
        sph_readback_wait(h);
        for (int b = 0; b < 2; ++b) cudaMemsetAsync(h->buf[b].pos_lo, 0, sizeof(float4) * h->cap, h->stream);
        cudaStreamSynchronize(h->stream);
    }
    h->cfg = *cfg;
    h->state_gen++;
    // captured steps hold the old constants as kernel arguments
    for (int p = 0; p < 2; ++p) {
        if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
        h->graph[p] = nullptr;
    }
    return SPH_OK;
}

int sph_get_config(const sph_handle *h, sph_config *cfg)
{
    if (!h || !cfg) return SPH_ERR_INVALID;
    *cfg = h->cfg;
    return SPH_OK;
}

int sph_add_particles(sph_handle *h, uint32_t n, const float *pos, const float *vel, const uint32_t *level)
{
    if (!h || (n && (!pos || !level))) return SPH_ERR_INVALID;
    sph_readback_wait(h);   // the current buffer may still be read back
    ensure_outputs(h);      // the particles already there keep their outputs
    const int dim = (int)h->cfg.dim;
    uint32_t n0 = read_n(h);
    if ((uint64_t)n0 + n > h->cap) { h->err = "sph_add_particles: capacity exceeded"; return SPH_ERR_CAPACITY; }
    for (uint32_t i = 0; i < n; ++i)
        if (level[i] != 1u && level[i] != 2u) { h->err = "level must be 1 or 2"; return SPH_ERR_INVALID; }
    std::vector<float4> p4, v4, z4(n, make_float4(0.f, 0.f, 0.f, 0.f));
    pack4(pos, dim, n, p4, level);
    pack4(vel, dim, n, v4, nullptr);
    std::vector<float> zf(n, 0.0f);
    std::vector<uint32_t> zu(n, 0u);
    const CanonPtrs &b = h->buf[h->cur];
    cudaStream_t s = h->stream;
    cudaMemcpyAsync(b.pos + n0, p4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.vel + n0, v4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.ev + n0, z4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.acc + n0, z4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.dens + n0, zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.press + n0, zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.energy + n0, zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.surface + n0, zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.interior + n0, zu.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.scene + n0, zu.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(b.sibling + n0, 0xff, sizeof(uint32_t) * n, s);
    cudaMemsetAsync(b.pos_lo + n0, 0, sizeof(float4) * n, s);
    cudaStreamSynchronize(s);
    write_n(h, n0 + n);
    h->n_ub = n0 + n;
    h->state_gen++;
    return cuda_check(h, "sph_add_particles");
}

int sph_set_state(sph_handle *h, const sph_state_view *st)
{
    if (!h || !st) return SPH_ERR_INVALID;
    sph_readback_wait(h);
    const uint32_t n = st->n;
    if (n > h->cap) { h->err = "sph_set_state: capacity exceeded"; return SPH_ERR_CAPACITY; }
    if (n && (!st->pos || !st->level)) return SPH_ERR_INVALID;
    if (st->scene && h->w.nscenes)
        for (uint32_t i = 0; i < n; ++i)
            if (st->scene[i] >= h->w.nscenes) { h->err = "sph_set_state: scene index out of range"; return SPH_ERR_RANGE; }
    const int dim = (int)h->cfg.dim;
    std::vector<float4> p4, v4, e4, a4;
    pack4(st->pos, dim, n, p4, st->level);
    pack4(st->vel, dim, n, v4, nullptr);
    pack4(st->ev, dim, n, e4, nullptr);
    pack4(st->acc, dim, n, a4, nullptr);
    std::vector<float> zf(n, 0.0f);
    std::vector<uint32_t> zu(n, 0u);
    const CanonPtrs &b = h->buf[h->cur];
    cudaStream_t s = h->stream;
    cudaMemcpyAsync(b.pos, p4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.vel, v4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.ev, e4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.acc, a4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.dens, st->dens ? st->dens : zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.press, st->press ? st->press : zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.energy, st->energy ? st->energy : zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.surface, st->surface ? st->surface : zf.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.interior, st->interior ? st->interior : zu.data(), sizeof(uint32_t) * n,
                    cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b.scene, st->scene ? st->scene : zu.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s);
    if (st->sibling) cudaMemcpyAsync(b.sibling, st->sibling, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s);
    else cudaMemsetAsync(b.sibling, 0xff, sizeof(uint32_t) * (n ? n : 1), s);
    cudaMemsetAsync(b.pos_lo, 0, sizeof(float4) * (n ? n : 1), s);
    cudaStreamSynchronize(s);
    write_n(h, n);
    h->n_ub = n;
    h->have_step = false;
    h->state_gen++;
    return cuda_check(h, "sph_set_state");
}

static void drop_graphs(sph_handle *h)
{
    for (int p = 0; p < 2; ++p) {
        if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
        h->graph[p] = nullptr;
        h->graph_grid[p] = 0;
    }
}

// Records one step for the current parity into a graph (nothing executes
// during capture), restoring the host-side bookkeeping the recording moved.
static int capture_step(sph_handle *h)
{
    const int p = h->cur;
    const uint64_t step_index = h->step_index;
    const uint32_t n_ub = h->n_ub, launches = h->last_launches;
    const bool counts_zero = h->counts_zero, counts_hashed = h->counts_hashed, pending = h->outputs_pending;
    const uint64_t hashed_gen = h->hashed_gen, hashed_step = h->hashed_step;
    cudaGraph_t g = nullptr;
    h->last_launches = 0;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return cuda_check(h, "cudaStreamBeginCapture");
    int rc = h->cfg.dim == 3 ? run_step<3>(h, false) : run_step<2>(h, false);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->graph_launches[p] = h->last_launches;
    h->cur = p;
    h->step_index = step_index;
    h->n_ub = n_ub;
    h->last_launches = launches;
    h->counts_zero = counts_zero;
    h->counts_hashed = counts_hashed;
    h->outputs_pending = pending;
    h->hashed_gen = hashed_gen;
    h->hashed_step = hashed_step;
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_check(h, "cudaStreamEndCapture");
    if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
    h->graph[p] = nullptr;
    e = cudaGraphInstantiate(&h->graph[p], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_check(h, "cudaGraphInstantiate");
    h->graph_grid[p] = launch_key(h);
    return SPH_OK;
}

int sph_step(sph_handle *h, int nsteps)
{
    if (!h || nsteps < 0) return SPH_ERR_INVALID;
    h->last_launches = 0;
    auto surface_due = [h](uint64_t step) {
        return h->cfg.dim == 3 && h->cfg.grid_every && h->mc.nodes && step % h->cfg.grid_every == 0;
    };
    for (int k = 0; k < nsteps; ++k) {
        if (h->n_ub == 0) break;
        h->n_last_sorted = 0;   // resolved lazily by sph_get_debug
        // this step writes the other state buffer: wait for a readback of it
        if (h->rb_pending[h->cur ^ 1]) {
            cudaStreamWaitEvent(h->stream, h->rb_done[h->cur ^ 1], 0);
            h->rb_pending[h->cur ^ 1] = false;
        }
        int rc;
        if (h->persistent && !h->profiling && !surface_due(h->step_index)) {
            // the steps up to the next surface step in one launch (one at a
            // time while splits can grow the count)
            int run = 1;
            if (!h->cfg.use_split)
                while (run < nsteps - k && run < kPersistMaxSteps && !surface_due(h->step_index + run)) ++run;
            if (run > 1 && h->rb_pending[h->cur]) {   // it writes both state buffers
                cudaStreamWaitEvent(h->stream, h->rb_done[h->cur], 0);
                h->rb_pending[h->cur] = false;
            }
            rc = h->cfg.dim == 3 ? run_step_persistent<3>(h, run) : run_step_persistent<2>(h, run);
            k += run - 1;
        } else if (h->use_graph && !h->profiling && !surface_due(h->step_index)) {
            const int p = h->cur;
            if (!h->graph[p] || h->graph_grid[p] != launch_key(h)) {
                rc = capture_step(h);
                if (rc) return rc;
            }
            if (!hash_ready(h)) {   // the graph starts at the cell scan
                if (h->cfg.dim == 3) hash_prologue<3>(h);
                else hash_prologue<2>(h);
            }
            if (cudaGraphLaunch(h->graph[p], h->stream) != cudaSuccess) return cuda_check(h, "cudaGraphLaunch");
            // the bookkeeping run_step does on the host
            h->counts_zero = false;
            h->cur = p ^ 1;
            h->step_index++;
            h->counts_hashed = true;
            h->hashed_gen = h->state_gen;
            h->hashed_step = h->step_index;
            h->outputs_pending = defer_outputs(h);
            uint64_t ub = h->n_ub;
            if (h->cfg.use_split) ub *= (h->cfg.split_ways == 4 ? 4u : 2u);
            h->n_ub = (uint32_t)std::min<uint64_t>(ub, h->cap);
            h->last_launches += h->graph_launches[p];
            rc = SPH_OK;
        } else {
            rc = h->cfg.dim == 3 ? run_step<3>(h) : run_step<2>(h);
        }
        if (rc) return rc;
        h->have_step = true;
    }
    return SPH_OK;
}

int sph_set_persistent(sph_handle *h, int on, uint32_t spin_limit)
{
    if (!h) return SPH_ERR_INVALID;
    h->persistent = on != 0;
    h->spin_limit = spin_limit;
    // a wait limit other than the default asks for the polled barriers,
    // which are the ones a limit applies to
    h->persist_use_cluster = spin_limit == SPH_PERSISTENT_SPIN_DEFAULT;
    return SPH_OK;
}

int sph_set_graph(sph_handle *h, int on)
{
    if (!h) return SPH_ERR_INVALID;
    h->use_graph = on != 0;
    if (!h->use_graph) drop_graphs(h);
    return SPH_OK;
}

int sph_set_scenes(sph_handle *h, uint32_t nscenes, const sph_scene *scenes)
{
    if (!h || (nscenes && !scenes)) return SPH_ERR_INVALID;
    const sph_config &c = h->cfg;
    const uint32_t dim = c.dim;
    // boxes at whole-cell offsets exactly SPH_SCENE_GAP_CELLS apart pass
    // despite the FP32 rounding of lo and hi
    const float gap = (SPH_SCENE_GAP_CELLS - 0.01f) * c.cell_size;
    for (uint32_t s = 0; s < nscenes; ++s) {
        const sph_scene &a = scenes[s];
        if (!std::isfinite(a.viscosity) || !std::isfinite(a.gas_constant)) {
            h->err = "sph_set_scenes: non-finite scene constant";
            return SPH_ERR_INVALID;
        }
        for (uint32_t d = 0; d < dim; ++d)
            if (!(a.lo[d] >= 0.0f && a.hi[d] <= c.world[d] && a.hi[d] - a.lo[d] > 2.0f * c.radius[0])) {
                h->err = "sph_set_scenes: scene box outside the world or thinner than a particle";
                return SPH_ERR_INVALID;
            }
    }
    // any two boxes are separated along some axis by the gap
    for (uint32_t s = 0; s < nscenes; ++s)
        for (uint32_t t = s + 1; t < nscenes; ++t) {
            bool apart = false;
            for (uint32_t d = 0; d < dim && !apart; ++d)
                apart = scenes[t].lo[d] >= scenes[s].hi[d] + gap || scenes[s].lo[d] >= scenes[t].hi[d] + gap;
            if (!apart) {
                h->err = "sph_set_scenes: scene boxes " + std::to_string(s) + " and " + std::to_string(t) +
                         " are closer than SPH_SCENE_GAP_CELLS cells";
                return SPH_ERR_INVALID;
            }
        }
    sph_readback_wait(h);
    const uint32_t n = read_n(h);
    if (nscenes && n) {   // scene indices already held must name a scene
        std::vector<uint32_t> ids(n);
        cudaMemcpy(ids.data(), h->buf[h->cur].scene, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
        for (uint32_t i = 0; i < n; ++i)
            if (ids[i] >= nscenes) { h->err = "sph_set_scenes: a particle's scene index is out of range"; return SPH_ERR_RANGE; }
    }
    cudaStreamSynchronize(h->stream);
    if (nscenes > h->scene_tab_cap) {
        if (h->scene_tab) cudaFree(h->scene_tab);
        h->scene_tab = nullptr;
        h->scene_tab_cap = 0;
        if (cudaMalloc(&h->scene_tab, sizeof(float4) * 2 * nscenes) != cudaSuccess)
            return cuda_check(h, "sph_set_scenes");
        h->scene_tab_cap = nscenes;
    }
    if (nscenes) {
        std::vector<float4> tab(2 * (size_t)nscenes);
        for (uint32_t s = 0; s < nscenes; ++s) {
            const sph_scene &a = scenes[s];
            tab[2 * s] = make_float4(a.lo[0], a.lo[1], dim == 3 ? a.lo[2] : 0.0f, a.viscosity);
            tab[2 * s + 1] = make_float4(a.hi[0], a.hi[1], dim == 3 ? a.hi[2] : 0.0f, a.gas_constant);
        }
        cudaMemcpy(h->scene_tab, tab.data(), sizeof(float4) * tab.size(), cudaMemcpyHostToDevice);
    }
    h->w.scene_tab = nscenes ? h->scene_tab : nullptr;
    h->w.nscenes = nscenes;
    h->state_gen++;
    drop_graphs(h);   // captured steps hold the work pointers as arguments
    return cuda_check(h, "sph_set_scenes");
}

int sph_sync(sph_handle *h)
{
    if (!h) return SPH_ERR_INVALID;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { h->err = cudaGetErrorString(e); return SPH_ERR_CUDA; }
    Counters c0;
    cudaMemcpy(&c0, &h->cnt[h->cur], sizeof(Counters), cudaMemcpyDeviceToHost);
    if (c0.error) {
        uint32_t err = c0.error;
        c0.error = 0;
        cudaMemcpy(&h->cnt[h->cur], &c0, sizeof(Counters), cudaMemcpyHostToDevice);
        for (int code = 1; code < 32; ++code)
            if (err & (1u << code)) {
                h->err = code == SPH_ERR_CAPACITY    ? "particle capacity exceeded by a split (splits skipped)"
                         : code == SPH_ERR_NONFINITE ? "a particle's position or velocity became non-finite"
                         : code == SPH_ERR_TIMEOUT   ? "a barrier of the persistent step gave up waiting; "
                                                       "restore the state with sph_set_state"
                                                     : "device reported an error";
                return code;
            }
    }
    return SPH_OK;
}

int sph_conserved(sph_handle *h, double *out)
{
    if (!h || !out) return SPH_ERR_INVALID;
    const uint32_t G = grid_for(h, h->n_ub);
    if (!h->cons) {
        if (cudaMalloc(&h->cons, sizeof(double) * ((size_t)h->num_sms * 8u + 1) * kConservedTerms) != cudaSuccess) {
            cudaGetLastError();
            h->cons = nullptr;
            h->err = "sph_conserved: out of device memory";
            return SPH_ERR_CUDA;
        }
    }
    double *fin = h->cons + (size_t)h->num_sms * 8u * kConservedTerms;
    cudaStream_t s = h->stream;
    if (h->cfg.dim == 3) k_conserved<3><<<G, kThreads, 0, s>>>(h->cfg, h->cnt + h->cur, h->buf[h->cur], h->cons);
    else k_conserved<2><<<G, kThreads, 0, s>>>(h->cfg, h->cnt + h->cur, h->buf[h->cur], h->cons);
    k_conserved_final<<<1, 32, 0, s>>>(h->cons, G, fin);
    double v[kConservedTerms];
    cudaMemcpyAsync(v, fin, sizeof(v), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    for (int k = 0; k < kConservedTerms; ++k) out[k] = v[k];
    out[6] = v[4] + v[5];
    return cuda_check(h, "sph_conserved");
}

int sph_get_num_particles(sph_handle *h, uint32_t *n)
{
    if (!h || !n) return SPH_ERR_INVALID;
    *n = read_n(h);
    return cuda_check(h, "sph_get_num_particles");
}

int sph_get_state(sph_handle *h, sph_state_view *st)
{
    if (!h || !st) return SPH_ERR_INVALID;
    ensure_outputs(h);
    const uint32_t n = read_n(h);
    const uint32_t lim = st->n;   // caller's capacity; 0 = just report n
    st->n = n;
    if (lim == 0) return SPH_OK;
    if (lim < n) { h->err = "sph_get_state: host arrays too small"; return SPH_ERR_INVALID; }
    const int dim = (int)h->cfg.dim;
    const CanonPtrs &b = h->buf[h->cur];
    std::vector<float4> t(n);
    auto get4 = [&](const float4 *src, float *dst) {
        if (!dst) return;
        cudaMemcpy(t.data(), src, sizeof(float4) * n, cudaMemcpyDeviceToHost);
        unpack4(t, dim, n, dst);
    };
    get4(b.pos, st->pos);
    get4(b.vel, st->vel);
    get4(b.ev, st->ev);
    get4(b.acc, st->acc);
    if (st->level) {
        cudaMemcpy(t.data(), b.pos, sizeof(float4) * n, cudaMemcpyDeviceToHost);
        for (uint32_t i = 0; i < n; ++i) st->level[i] = (uint32_t)t[i].w;
    }
    if (st->dens) cudaMemcpy(st->dens, b.dens, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (st->press) cudaMemcpy(st->press, b.press, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (st->energy) cudaMemcpy(st->energy, b.energy, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (st->surface) cudaMemcpy(st->surface, b.surface, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (st->interior) cudaMemcpy(st->interior, b.interior, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    if (st->scene) cudaMemcpy(st->scene, b.scene, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    if (st->sibling) cudaMemcpy(st->sibling, b.sibling, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    return cuda_check(h, "sph_get_state");
}

int sph_get_debug(sph_handle *h, sph_debug_view *d)
{
    if (!h || !d) return SPH_ERR_INVALID;
    if (!h->have_step) { h->err = "no step run since the last state change"; return SPH_ERR_INVALID; }
    cudaStreamSynchronize(h->stream);
    Counters c0;
    cudaMemcpy(&c0, &h->cnt[h->cur ^ 1], sizeof(Counters), cudaMemcpyDeviceToHost);
    const uint32_t n = c0.n;   // count the last step started with
    d->n_sorted = n;
    d->total_cell = h->ncells;
    const WorkPtrs &w = h->w;
    const int dim = (int)h->cfg.dim;
    std::vector<uint32_t> sidx(n);
    cudaMemcpy(sidx.data(), w.sidx, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    if (d->hash) cudaMemcpy(d->hash, w.skey, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    if (d->index) std::memcpy(d->index, sidx.data(), sizeof(uint32_t) * n);
    if (d->cell_start || d->cell_end) {
        uint32_t *ds = nullptr, *de = nullptr;
        cudaMalloc(&ds, sizeof(uint32_t) * h->ncells);
        cudaMalloc(&de, sizeof(uint32_t) * h->ncells);
        k_cell_ranges<<<grid_for(h, h->ncells), kThreads, 0, h->stream>>>(w.cell_off, h->ncells, ds, de);
        cudaStreamSynchronize(h->stream);
        if (d->cell_start) cudaMemcpy(d->cell_start, ds, sizeof(uint32_t) * h->ncells, cudaMemcpyDeviceToHost);
        if (d->cell_end) cudaMemcpy(d->cell_end, de, sizeof(uint32_t) * h->ncells, cudaMemcpyDeviceToHost);
        cudaFree(ds);
        cudaFree(de);
    }
    if (d->trans_vel) {
        std::vector<float4> t(n);
        cudaMemcpy(t.data(), w.stv, sizeof(float4) * n, cudaMemcpyDeviceToHost);
        for (uint32_t s = 0; s < n; ++s) {
            float *o = d->trans_vel + (size_t)sidx[s] * dim;
            o[0] = t[s].x; o[1] = t[s].y;
            if (dim == 3) o[2] = t[s].z;
        }
    }
    if (d->nbr_count) {
        std::vector<uint32_t> t(n);
        cudaMemcpy(t.data(), w.snbr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
        for (uint32_t s = 0; s < n; ++s) d->nbr_count[sidx[s]] = t[s];
    }
    if (d->split_flag) {
        cudaMemcpy(d->split_flag, w.split_c, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
        if (c0.split_off) std::memset(d->split_flag, 0, sizeof(uint32_t) * n);
    }
    if (d->removed) cudaMemcpy(d->removed, w.removed_c, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    return cuda_check(h, "sph_get_debug");
}

uint32_t sph_particle_record_size(const sph_handle *h)
{
    if (!h) return 0;
    return h->cfg.dim == 3 ? 4u * AosLayout<3>::words : 4u * AosLayout<2>::words;
}

static int ensure_aos(sph_handle *h)
{
    if (h->aos) return SPH_OK;
    return dalloc(h, &h->aos, (size_t)h->cap * AosLayout<3>::words);
}

int sph_read_particles(sph_handle *h, void *host_dst, uint64_t capacity_bytes, uint32_t *n_out)
{
    if (!h || !n_out) return SPH_ERR_INVALID;
    if (int rc = ensure_aos(h)) return rc;
    ensure_outputs(h);
    const uint32_t n = read_n(h);
    const uint64_t rec = sph_particle_record_size(h);
    *n_out = n;
    if (!host_dst) return SPH_OK;
    if (capacity_bytes < rec * n) { h->err = "sph_read_particles: destination too small"; return SPH_ERR_INVALID; }
    const uint32_t G = grid_for(h, n);
    if (h->cfg.dim == 3) k_to_aos<3><<<G, kThreads, 0, h->stream>>>(h->cnt + h->cur, h->buf[h->cur], h->aos);
    else k_to_aos<2><<<G, kThreads, 0, h->stream>>>(h->cnt + h->cur, h->buf[h->cur], h->aos);
    cudaMemcpyAsync(host_dst, h->aos, rec * n, cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { h->err = cudaGetErrorString(e); return SPH_ERR_CUDA; }
    return cuda_check(h, "sph_read_particles");
}

int sph_write_particles(sph_handle *h, const void *host_src, uint32_t n)
{
    if (!h || (n && !host_src)) return SPH_ERR_INVALID;
    if (n > h->cap) { h->err = "sph_write_particles: capacity exceeded"; return SPH_ERR_CAPACITY; }
    if (h->w.nscenes) {
        h->err = "sph_write_particles: the record format carries no scene index (use sph_set_state)";
        return SPH_ERR_INVALID;
    }
    sph_readback_wait(h);
    if (int rc = ensure_aos(h)) return rc;
    const uint64_t rec = sph_particle_record_size(h);
    cudaMemcpyAsync(h->aos, host_src, rec * n, cudaMemcpyHostToDevice, h->stream);
    const uint32_t G = grid_for(h, n);
    if (h->cfg.dim == 3) k_from_aos<3><<<G, kThreads, 0, h->stream>>>(n, h->buf[h->cur], h->aos);
    else k_from_aos<2><<<G, kThreads, 0, h->stream>>>(n, h->buf[h->cur], h->aos);
    write_n(h, n);
    h->n_ub = n;
    h->have_step = false;
    h->state_gen++;
    return cuda_check(h, "sph_write_particles");
}

int sph_read_particles_async(sph_handle *h, void *mapped_dst, uint64_t capacity_bytes, uint32_t *mapped_count_dst)
{
    if (!h || !mapped_dst || !mapped_count_dst) return SPH_ERR_INVALID;
    void *dst_dev = nullptr, *cnt_dev = nullptr;
    if (cudaHostGetDevicePointer(&dst_dev, mapped_dst, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(&cnt_dev, mapped_count_dst, 0) != cudaSuccess) {
        cudaGetLastError();
        h->err = "sph_read_particles_async: destination is not mapped page-locked memory";
        return SPH_ERR_INVALID;
    }
    if (!h->rb_stream) {
        if (cudaStreamCreateWithFlags(&h->rb_stream, cudaStreamNonBlocking) != cudaSuccess)
            return cuda_check(h, "readback stream");
        cudaEventCreateWithFlags(&h->rb_ready, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&h->rb_done[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&h->rb_done[1], cudaEventDisableTiming);
    }
    if ((reinterpret_cast<uintptr_t>(dst_dev) | reinterpret_cast<uintptr_t>(cnt_dev)) & 3u) {
        h->err = "sph_read_particles_async: destination and count need 4-byte alignment";
        return SPH_ERR_INVALID;
    }
    const int p = h->cur;
    const uint64_t rec = sph_particle_record_size(h);
    const uint32_t max_rec = (uint32_t)std::min<uint64_t>(capacity_bytes / rec, h->cap);
    ensure_outputs(h);
    cudaEventRecord(h->rb_ready, h->stream);
    cudaStreamWaitEvent(h->rb_stream, h->rb_ready, 0);
    // a few blocks keep PCIe busy; the rest of the GPU stays with the next step
    const uint32_t G = std::min<uint32_t>(grid_for(h, h->n_ub), (uint32_t)std::max(1, h->num_sms / 4));
    if (h->cfg.dim == 3)
        k_to_aos_mapped<3><<<G, kThreads, 0, h->rb_stream>>>(h->cnt + p, h->buf[p], (float *)dst_dev, max_rec,
                                                             (uint32_t *)cnt_dev);
    else
        k_to_aos_mapped<2><<<G, kThreads, 0, h->rb_stream>>>(h->cnt + p, h->buf[p], (float *)dst_dev, max_rec,
                                                             (uint32_t *)cnt_dev);
    cudaEventRecord(h->rb_done[p], h->rb_stream);
    h->rb_pending[p] = true;
    return cuda_check(h, "sph_read_particles_async");
}

int sph_readback_wait(sph_handle *h)
{
    if (!h) return SPH_ERR_INVALID;
    if (h->rb_stream && cudaStreamSynchronize(h->rb_stream) != cudaSuccess) return cuda_check(h, "readback wait");
    return SPH_OK;
}

int sph_set_profiling(sph_handle *h, int on)
{
    if (!h) return SPH_ERR_INVALID;
    if (on && !h->ev[0])
        for (int k = 0; k <= sph_handle::kMaxStages; ++k) cudaEventCreate(&h->ev[k]);
    h->profiling = on != 0;
    return cuda_check(h, "sph_set_profiling");
}

int sph_stage_times(sph_handle *h, float *ms, const char **names, int max, int *count)
{
    if (!h || !count) return SPH_ERR_INVALID;
    if (!h->profiling) { h->err = "profiling is off"; return SPH_ERR_INVALID; }
    cudaStreamSynchronize(h->stream);
    *count = h->nstages;
    for (int k = 0; k < h->nstages && k < max; ++k) {
        float t = 0.f;
        cudaEventElapsedTime(&t, h->ev[k], h->ev[k + 1]);
        if (ms) ms[k] = t;
        if (names) names[k] = h->stage_name[k];
    }
    return cuda_check(h, "sph_stage_times");
}

void *sph_get_stream(sph_handle *h) { return h ? (void *)h->stream : nullptr; }

int sph_set_stream(sph_handle *h, void *stream)
{
    if (!h) return SPH_ERR_INVALID;
    sph_readback_wait(h);
    cudaStreamSynchronize(h->stream);   // the handle's work so far is done before the switch
    drop_graphs(h);                     // recaptured on the next graph step
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return cuda_check(h, "sph_set_stream");
}

int sph_last_launch_count(const sph_handle *h, uint32_t *launches)
{
    if (!h || !launches) return SPH_ERR_INVALID;
    *launches = h->last_launches;
    return SPH_OK;
}

int sph_last_step_stats(sph_handle *h, sph_step_stats *out)
{
    if (!h || !out) return SPH_ERR_INVALID;
    if (!h->have_step) { h->err = "no step run since the last state change"; return SPH_ERR_INVALID; }
    cudaStream_t s = h->stream;
    cudaMemsetAsync(h->stat_buf, 0, sizeof(uint32_t), s);
    k_count_level2<<<grid_for(h, h->n_ub), kThreads, 0, s>>>(h->cnt + h->cur, h->buf[h->cur].pos, h->stat_buf);
    Counters c[2];
    uint32_t level2 = 0;
    cudaMemcpyAsync(c, h->cnt, sizeof(c), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&level2, h->stat_buf, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { h->err = cudaGetErrorString(e); return SPH_ERR_CUDA; }
    const Counters &last = c[h->cur ^ 1], &now = c[h->cur];   // the last step's input, its output
    out->n_start = last.n;
    out->split_suppressed = last.split_off ? 1u : 0u;
    out->n_split = last.split_off ? 0u : last.n_split;
    out->n_removed = last.n_removed;
    out->n_end = now.n;
    out->n_level2 = level2;
    out->error = now.error;
    return cuda_check(h, "sph_last_step_stats");
}

int sph_set_debug(sph_handle *h, int on)
{
    if (!h) return SPH_ERR_INVALID;
    h->debug = on != 0;
    for (int p = 0; p < 2; ++p) {   // the flag is a captured kernel argument
        if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
        h->graph[p] = nullptr;
    }
    return SPH_OK;
}

const char *sph_last_error(const sph_handle *h) { return h ? h->err.c_str() : kNoHandle; }

}  // extern "C"

extern "C" {

int sph_density_grid(sph_handle *h, float *dens, float *normal)
{
    if (!h) return SPH_ERR_INVALID;
    if (!h->mc.nodes) { h->err = "no density grid (2D, or ndens unset)"; return SPH_ERR_INVALID; }
    if (!h->grid_valid) { h->err = "no grid yet: set grid_every and step"; return SPH_ERR_INVALID; }
    cudaStreamSynchronize(h->stream);
    const uint32_t G = h->mc.nodes;
    if (dens) cudaMemcpy(dens, h->mc.dens, sizeof(float) * G, cudaMemcpyDeviceToHost);
    if (normal) {
        std::vector<float4> t(G);
        cudaMemcpy(t.data(), h->mc.normal, sizeof(float4) * G, cudaMemcpyDeviceToHost);
        for (uint32_t g = 0; g < G; ++g) {
            normal[3 * (size_t)g] = t[g].x;
            normal[3 * (size_t)g + 1] = t[g].y;
            normal[3 * (size_t)g + 2] = t[g].z;
        }
    }
    return cuda_check(h, "sph_density_grid");
}

static int copy_mesh(sph_handle *h, sph_mesh_view *mesh)
{
    cudaStreamSynchronize(h->stream);
    uint32_t total = 0;
    cudaMemcpy(&total, h->mc.num_tri, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    mesh->num_triangles = total;
    const uint32_t on_dev = std::min(total, h->mc.max_tri);
    const uint32_t nt = std::min(on_dev, mesh->max_triangles);
    float *dst[6] = {mesh->v0, mesh->v1, mesh->v2, mesh->n0, mesh->n1, mesh->n2};
    for (int k = 0; k < 6; ++k)
        if (dst[k] && nt)
            cudaMemcpy(dst[k], h->mc.tri + 3ull * h->mc.max_tri * k, sizeof(float) * 3ull * nt,
                       cudaMemcpyDeviceToHost);
    if (int rc = cuda_check(h, "surface copy")) return rc;
    if (total > h->mc.max_tri || total > mesh->max_triangles) {
        h->err = "surface has more triangles than the mesh capacity (truncated)";
        return SPH_ERR_CAPACITY;
    }
    return SPH_OK;
}

int sph_extract_surface(sph_handle *h, sph_mesh_view *mesh)
{
    if (!h || !mesh) return SPH_ERR_INVALID;
    if (!h->mc.nodes) { h->err = "no density grid (2D, or ndens unset)"; return SPH_ERR_INVALID; }
    if (!h->grid_valid) { h->err = "no surface yet: set grid_every and step"; return SPH_ERR_INVALID; }
    return copy_mesh(h, mesh);
}

int sph_surface_from_grid(sph_handle *h, const float *dens, const float *normal, sph_mesh_view *mesh)
{
    if (!h || !dens || !normal || !mesh) return SPH_ERR_INVALID;
    if (!h->mc.nodes) { h->err = "no density grid (2D, or ndens unset)"; return SPH_ERR_INVALID; }
    const uint32_t G = h->mc.nodes;
    std::vector<float4> t(G);
    for (uint32_t g = 0; g < G; ++g)
        t[g] = make_float4(normal[3 * (size_t)g], normal[3 * (size_t)g + 1], normal[3 * (size_t)g + 2], 0.f);
    cudaMemcpyAsync(h->mc.dens, dens, sizeof(float) * G, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->mc.normal, t.data(), sizeof(float4) * G, cudaMemcpyHostToDevice, h->stream);
    run_mc(h);
    h->grid_valid = true;
    return copy_mesh(h, mesh);
}

}  // extern "C"

// ---------------------------------------------------------------- launch tuning
namespace {

bool tune_valid(int st, uint32_t bs, uint32_t bpsm, uint32_t cap)
{
    const bool listed = st == SPH_TUNE_FORCE || st == SPH_TUNE_ENERGY;   // kernels with shared-memory lists
    return (bs == 128 || bs == 256 || (bs == 512 && !listed)) && bpsm >= 1 && bpsm <= 64 && cap <= 1 &&
           (st == SPH_TUNE_FORCE || st == SPH_TUNE_ENERGY || cap == 0);
}

const char *const kTuneStageName[SPH_TUNE_STAGES] = {"hash", "scatter", "reorder", "density",
                                                     "force_integrate", "energy_split", "merge", "write"};

}  // namespace

int sph_set_tuning(sph_handle *h, const sph_tuning *t)
{
    if (!h || !t) return SPH_ERR_INVALID;
    for (int st = 0; st < SPH_TUNE_STAGES; ++st)
        if (!tune_valid(st, t->block[st], t->blocks_per_sm[st], t->reg_cap[st])) {
            h->err = std::string("sph_set_tuning: unsupported shape for stage ") + kTuneStageName[st];
            return SPH_ERR_INVALID;
        }
    for (int st = 0; st < SPH_TUNE_STAGES; ++st) {
        h->tune_bs[st] = t->block[st];
        h->tune_bpsm[st] = t->blocks_per_sm[st];
        h->tune_minb[st] = t->reg_cap[st];
    }
    drop_graphs(h);
    return SPH_OK;
}

int sph_get_tuning(const sph_handle *h, sph_tuning *t)
{
    if (!h || !t) return SPH_ERR_INVALID;
    for (int st = 0; st < SPH_TUNE_STAGES; ++st) {
        t->block[st] = h->tune_bs[st];
        t->blocks_per_sm[st] = h->tune_bpsm[st];
        t->reg_cap[st] = h->tune_minb[st];
    }
    t->step_ms_before = t->step_ms_after = 0.0f;
    return SPH_OK;
}

int sph_autotune(sph_handle *h, uint32_t reps, sph_tuning *out)
{
    if (!h || reps == 0) return SPH_ERR_INVALID;
    sph_readback_wait(h);
    const uint32_t n = read_n(h);
    if (n == 0) { h->err = "sph_autotune: no particles"; return SPH_ERR_INVALID; }
    // the state every trial starts from
    CanonPtrs save{};
    std::vector<void *> tmp;
    auto talloc = [&](auto **p, size_t count) {
        void *q = nullptr;
        if (cudaMalloc(&q, sizeof(**p) * count) != cudaSuccess) return 1;
        tmp.push_back(q);
        *p = (std::remove_reference_t<decltype(*p)>)q;
        return 0;
    };
    int bad = talloc(&save.pos, n) | talloc(&save.vel, n) | talloc(&save.ev, n) | talloc(&save.acc, n) |
              talloc(&save.dens, n) | talloc(&save.press, n) | talloc(&save.energy, n) |
              talloc(&save.surface, n) | talloc(&save.interior, n) | talloc(&save.scene, n) |
              talloc(&save.pos_lo, n) | talloc(&save.sibling, n);
    if (bad) {
        cudaGetLastError();
        for (void *p : tmp) cudaFree(p);
        h->err = "sph_autotune: out of device memory for the saved state";
        return SPH_ERR_CUDA;
    }
    auto copy = [&](const CanonPtrs &d, const CanonPtrs &src) {
        auto c1 = [&](void *dd, const void *ss, size_t bytes) {
            cudaMemcpyAsync(dd, ss, bytes, cudaMemcpyDeviceToDevice, h->stream);
        };
        c1(d.pos, src.pos, 16ull * n); c1(d.vel, src.vel, 16ull * n); c1(d.ev, src.ev, 16ull * n);
        c1(d.acc, src.acc, 16ull * n); c1(d.dens, src.dens, 4ull * n); c1(d.press, src.press, 4ull * n);
        c1(d.energy, src.energy, 4ull * n); c1(d.surface, src.surface, 4ull * n);
        c1(d.interior, src.interior, 4ull * n); c1(d.scene, src.scene, 4ull * n);
        c1(d.pos_lo, src.pos_lo, 16ull * n); c1(d.sibling, src.sibling, 4ull * n);
    };
    ensure_outputs(h);
    copy(save, h->buf[h->cur]);
    const int cur0 = h->cur;
    const uint64_t step0 = h->step_index;
    const bool prof0 = h->profiling;
    const bool graph0 = h->use_graph;
    h->use_graph = false;
    drop_graphs(h);
    sph_set_profiling(h, 1);
    auto restore = [&]() {
        h->counts_hashed = false;
        h->outputs_pending = false;   // the saved state has every output
        h->cur = cur0;
        copy(h->buf[h->cur], save);
        Counters c0;
        std::memset(&c0, 0, sizeof(c0));
        c0.n = n;
        cudaMemcpyAsync(&h->cnt[h->cur], &c0, sizeof(Counters), cudaMemcpyHostToDevice, h->stream);
        h->n_ub = n;
        h->step_index = step0;
    };
    // per-stage and whole-step device time over `reps` steps from the saved state
    std::vector<float> stage_ms(SPH_TUNE_STAGES);
    float step_ms = 0.0f;
    auto trial = [&]() -> int {
        restore();
        std::fill(stage_ms.begin(), stage_ms.end(), 0.0f);
        step_ms = 0.0f;
        for (uint32_t r = 0; r < reps; ++r) {
            int rc = h->cfg.dim == 3 ? run_step<3>(h) : run_step<2>(h);
            if (rc) return rc;
            float ms[sph_handle::kMaxStages];
            const char *names[sph_handle::kMaxStages];
            int cnt = 0;
            if ((rc = sph_stage_times(h, ms, names, sph_handle::kMaxStages, &cnt))) return rc;
            for (int q = 0; q < cnt; ++q) {
                step_ms += ms[q];
                for (int st = 0; st < SPH_TUNE_STAGES; ++st)
                    if (!std::strcmp(names[q], kTuneStageName[st])) stage_ms[st] += ms[q];
            }
        }
        return SPH_OK;
    };
    int rc = trial();
    const float before = step_ms / reps;
    static const uint32_t kBs[3] = {128, 256, 512};
    static const uint32_t kBpsm[6] = {2, 4, 8, 16, 32, 64};
    for (int st = 0; st < SPH_TUNE_STAGES && !rc; ++st) {
        if (st == SPH_TUNE_MERGE && !h->cfg.use_merge) continue;
        const uint32_t inc_bs = h->tune_bs[st], inc_bp = h->tune_bpsm[st], inc_cap = h->tune_minb[st];
        uint32_t best_bs = inc_bs, best_bp = inc_bp, best_cap = inc_cap;
        if ((rc = trial())) break;
        float best = stage_ms[st];
        for (uint32_t cap = 0; cap <= 1 && !rc; ++cap)
            for (uint32_t bs : kBs)
                for (uint32_t bp : kBpsm) {
                    if (!tune_valid(st, bs, bp, cap) || (bs == best_bs && bp == best_bp && cap == best_cap))
                        continue;
                    h->tune_bs[st] = bs;
                    h->tune_bpsm[st] = bp;
                    h->tune_minb[st] = cap;
                    if ((rc = trial())) break;
                    if (stage_ms[st] < best * 0.98f) {   // keep a change only for a clear gain
                        best = stage_ms[st];
                        best_bs = bs;
                        best_bp = bp;
                        best_cap = cap;
                    }
                }
        // a change must win a second, fresh comparison with the shape it replaces
        if (!rc && (best_bs != inc_bs || best_bp != inc_bp || best_cap != inc_cap)) {
            h->tune_bs[st] = best_bs;
            h->tune_bpsm[st] = best_bp;
            h->tune_minb[st] = best_cap;
            if (!(rc = trial())) {
                const float t_new = stage_ms[st];
                h->tune_bs[st] = inc_bs;
                h->tune_bpsm[st] = inc_bp;
                h->tune_minb[st] = inc_cap;
                if (!(rc = trial()) && !(t_new < stage_ms[st] * 0.98f)) {
                    best_bs = inc_bs;
                    best_bp = inc_bp;
                    best_cap = inc_cap;
                }
            }
        }
        h->tune_bs[st] = best_bs;
        h->tune_bpsm[st] = best_bp;
        h->tune_minb[st] = best_cap;
    }
    float after = before;
    if (!rc && !(rc = trial())) after = step_ms / reps;
    restore();
    cudaStreamSynchronize(h->stream);
    for (void *p : tmp) cudaFree(p);
    sph_set_profiling(h, prof0 ? 1 : 0);
    h->use_graph = graph0;
    h->have_step = false;
    if (rc) return rc;
    if (out) {
        sph_get_tuning(h, out);
        out->step_ms_before = before;
        out->step_ms_after = after;
    }
    return cuda_check(h, "sph_autotune");
}

#include "sph_rollout_impl.cuh"
