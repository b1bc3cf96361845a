// sph_persistent.cuh — the whole step in one cooperative launch.
//
// The reference launches every stage of a step separately
// (SPHSystem::animation, SPH-3D-2/sph_system.cpp:302-404; animate,
// SPH-2D/sph_system.cpp:190-264), and so does sph_step's ordinary path (13
// launches and a memset, or one replayed CUDA graph of them).  On small scenes the step
// is then bound by the launches and the drain between them, not by the work.
// k_step_persistent runs the same stage bodies (sph_kernels.cuh,
// sph_scan.cuh) in one launch whose blocks are all resident (a cooperative
// launch), separated by grid-wide barriers:
//
//   hash | scan cells (1 or 2 phases) | scatter (and clear the counts) | reorder |
//   density | force + integrate | energy + split decision |
//   [split scan (2 phases) + capacity guard | merge | removal scan (2 phases)] |
//   write-out
//
// (the bracketed stages only when split or merge is on).  The write-out also
// hashes the state it writes for the next step, so a step whose state was
// written by a step before starts at the cell scan: 12 barriers per step with
// adaptivity.  Without it the write-out runs in the energy stage
// (write_hash_by_slot_body), and a small cell grid is scanned in one phase:
// 5 barriers per step.  One launch runs several steps without splits, one
// more barrier between two of them.  Each scan's second phase has every block sum
// the block totals itself (scan_phase23_body) instead of one block scanning
// them between two barriers.  Every particle's
// arithmetic is the ordinary path's, in the same order, so the results are
// bit for bit those of sph_step's launches.
//
// A grid of at most 16 blocks runs as one thread-block cluster and meets at
// the hardware cluster barrier instead, which needs no polling.
// Barrier: each block's thread 0 adds its arrival to one counter with a
// release add (publishing the block's writes) and polls the counter with
// acquire loads until all blocks have arrived at this barrier.  Launches
// alternate between two counters; each launch clears the other one for the
// next launch, so no memset runs between steps (the host clears both after
// a timeout).  Every poll counts against a limit; a block whose
// wait runs out sets the launch's abort flag and SPH_ERR_TIMEOUT in the
// step's error bits, and every block returns at its next barrier, so the
// kernel always ends.  The input state buffer is never written, but the step
// that gave up writes no output: the state after a timeout must be restored
// (sph_set_state).  A step whose input carries the timeout bit does nothing.
// A launch of several steps alternates the two state buffers and counters
// as that many separate steps would (the grid is sized for the first step's
// count, so only steps that cannot split share a launch).
// No stage reads data through the non-coherent path (loads are NC = false),
// since a stage reads what an earlier stage of the same launch wrote.
#pragma once
#include <cstdint>
#include "../../include/sph/sph.h"
#include "sph_kernels.cuh"
#include "sph_scan.cuh"

namespace sph {

// Barrier state of one launch (zero when the launch starts).
struct GridSync {
    uint32_t arrived;   // arrivals of all blocks at all barriers of the launch
    uint32_t abort;     // 1 once a block gave up waiting
    uint32_t where;     // the barrier (1-based) at which the first block gave up
    uint32_t pad;
};

struct PersistArgs {
    GridSync *gs;            // this launch's barrier state
    GridSync *gs_next;       // the next launch's, cleared by this one
    uint32_t spin_limit;     // polls a block makes before giving up at a barrier
    uint32_t ncells, cap;
    uint32_t *scan_blocks;   // at least gridDim.x entries
    uint32_t *scan_grand;    // the cell scan's total
    int want_tv;             // keep the wavelet-transformed velocity (debug view)
    int ranks;               // split or merge on: run the split and removal scans
    int cluster;             // the grid is one thread-block cluster: hardware cluster barriers
    int hash_ready;          // the previous launch hashed this step's state already
    int parity;              // the state buffer (and counters) the first step reads
    int nsteps;              // steps this launch runs
};

// Without split and merge (ranks = 0) the write-out needs no global step:
// particle i = sidx[s] goes to index i, and every value it writes was made for
// slot s by the same thread (density, force and energy give slot s to the
// same thread, and so does this loop).  So the thread that finished slot s's
// energy writes the particle out right away, and hashes its new position for
// the next step (hash_one; the counts were cleared after this step's scan).
// Values are write_body's for a particle that neither splits nor merges.
template <int DIM, int BS>
__device__ __forceinline__ void write_hash_by_slot_body(const sph_config &c, const Counters *cnt, Counters *cnt_next,
                                                        const CanonPtrs &in, const CanonPtrs &out, const WorkPtrs &w)
{
    const uint32_t n = cnt->n;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cnt_next->n = n;
        cnt_next->error = cnt->error;
        cnt_next->n_split = 0;
        cnt_next->n_removed = 0;
        cnt_next->split_off = 0;
        cnt_next->split_flags = 0;
        cnt_next->removed_flags = 0;
        cnt_next->merge_candidates = 0;
    }
    const bool inter_rule = c.merge_rule == SPH_MERGE_INTERIOR || c.merge_rule == SPH_MERGE_SIBLING;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (uint32_t base = blockIdx.x * BS + wib * 32u; base < n; base += gridDim.x * BS) {
        const uint32_t s = base + lane;
        if (s >= n) continue;
        const uint32_t i = w.sidx[s];
        const float4 p = w.spos_n[s];
        const float4 aux = w.saux[s];
        out.pos[i] = p; out.vel[i] = w.svel_n[s]; out.ev[i] = w.sev_n[s]; out.acc[i] = w.sacc_n[s];
        out.dens[i] = aux.x; out.press[i] = aux.y; out.energy[i] = w.senergy[s]; out.surface[i] = w.ssurf[s];
        out.interior[i] = inter_rule ? w.sinter[s] : 0u;
        const uint32_t j = in.sibling[i];
        out.sibling[i] = j < n ? j : kEmpty;
        if (w.nscenes) out.scene[i] = w.sscene[s];
        if (w.pos_comp) out.pos_lo[i] = w.spos_lo_n[s];
        hash_one<DIM>(c, w, i, p);   // the next step's hash of particle i
    }
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Barrier number k (1, 2, ...) of the launch.  Returns false, for the whole
// block, once any block has given up.
__device__ __forceinline__ bool grid_barrier(const PersistArgs &a, uint32_t k, Counters *cin, Counters *cout)
{
    if (a.cluster) {
        // the whole grid is one cluster, co-scheduled by the hardware: its
        // barrier (release on arrive, acquire on wait, at cluster scope)
        // orders every thread's global writes before every later read, and
        // every thread of every block reaches it, so it needs no limit
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                         : "memory");
        return true;
    }
    __shared__ uint32_t s_ok;
    __syncthreads();   // the block's writes are ordered before thread 0's release
    if (threadIdx.x == 0) {
        GridSync *gs = a.gs;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&gs->arrived) : "memory");
        const uint32_t target = k * gridDim.x;
        uint32_t ok = 1;
        for (uint32_t it = 0;; ++it) {
            if (it >= a.spin_limit || ld_relaxed_gpu(&gs->abort)) {
                if (atomicExch(&gs->abort, 1u) == 0u) {
                    gs->where = k;
                    atomicOr(&cin->error, 1u << SPH_ERR_TIMEOUT);
                    atomicOr(&cout->error, 1u << SPH_ERR_TIMEOUT);
                }
                ok = 0;
                break;
            }
            if (ld_acquire_gpu(&gs->arrived) >= target) break;
        }
        s_ok = ok;
    }
    __syncthreads();   // the acquire is ordered before the block's later reads
    return s_ok != 0;
}

// The scan between barriers: exclusive scan of in[0, len) into out, block
// totals in a.scan_blocks, grand total to *grand.
template <typename T>
__device__ __forceinline__ bool grid_scan(const PersistArgs &a, uint32_t &k, Counters *cin, Counters *cout,
                                          const T *in, T *out, uint32_t len, T *grand, int total_at_len,
                                          uint32_t *list)
{
    scan_phase1_body<T>(in, len, a.scan_blocks);
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    scan_phase23_body<T>(in, out, len, a.scan_blocks, grand, total_at_len, list);
    return true;
}

// Cell scans of at most this many cells per thread of a block run in one
// phase (scan_onepass_body): each block reads every count before its chunk.
constexpr uint32_t kOnePassPerThread = 16;

// One step's stages, from the hash (or, when the previous step hashed this
// state already, from the cell scan) to the write-out.  Returns false, for
// the whole block, once any block has given up at a barrier.
template <int DIM, int BS>
__device__ __forceinline__ bool step_stages(const sph_config &c, Counters *cin, Counters *cout, const CanonPtrs &in,
                                            const CanonPtrs &out, const WorkPtrs &w, const PersistArgs &a,
                                            uint32_t &k, bool hashed, WarpPairSmem *pair, MergeSmem *merge)
{
    if (!a.ranks && blockIdx.x == 0 && threadIdx.x == 0) {
        cin->n_split = 0u;
        cin->n_removed = 0u;
        cin->split_off = 0u;
    }
    if (!hashed) {
        hash_body<DIM>(c, cin, in, w);
        if (!grid_barrier(a, ++k, cin, cout)) return false;
    }
    if (a.ncells <= kOnePassPerThread * blockDim.x) {   // few cells: one phase, one barrier fewer
        scan_onepass_body<uint32_t, kOnePassPerThread>(w.cell_count, w.cell_off, a.ncells, a.scan_grand, 1);
    } else if (!grid_scan<uint32_t>(a, k, cin, cout, w.cell_count, w.cell_off, a.ncells, a.scan_grand, 1,
                                    nullptr)) {
        return false;
    }
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    scatter_body<false>(cin, w);
    // no stage reads the counts after the scan: clear them for the next hash
    for (uint32_t q = grid_stride_start(); q < a.ncells; q += grid_stride()) w.cell_count[q] = 0u;
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    reorder_body<false>(cin, in, w);
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    density_body<DIM, false>(c, cin, w);
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    force_integrate_body<DIM, BS, false>(c, cin, w, pair);
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    energy_split_body<DIM, BS, false>(c, cin, in, w, a.want_tv, pair);
    if (!a.ranks) {
        write_hash_by_slot_body<DIM, BS>(c, cin, cout, in, out, w);
        return true;
    }
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    const uint32_t n = cin->n;
    // a scan of all-zero flags is all zeros: written directly, no barrier
    if (cin->split_flags) {
        if (!grid_scan<uint32_t>(a, k, cin, cout, w.split_c, w.split_rank, n, &cin->n_split, 0, w.split_list))
            return false;
    } else {
        for (uint32_t q = grid_stride_start(); q < n; q += grid_stride()) w.split_rank[q] = 0u;
        if (blockIdx.x == 0 && threadIdx.x == 0) cin->n_split = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) split_guard_body(c, cin, a.cap);
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    // no merge stage when the energy pass found no candidate (read after its barrier)
    if (c.use_merge && (c.merge_rule == SPH_MERGE_WAVELET_CELL || cin->merge_candidates)) {
        if (c.merge_rule == SPH_MERGE_SIBLING) merge_sibling_body<DIM>(c, cin, in, w);
        else merge_body<DIM>(c, cin, in, w, a.ncells, a.cap, merge);
        if (!grid_barrier(a, ++k, cin, cout)) return false;
    }
    if (cin->removed_flags) {
        if (!grid_scan<uint32_t>(a, k, cin, cout, w.removed_c, w.removed_rank, n, &cin->n_removed, 0, nullptr))
            return false;
    } else {
        for (uint32_t q = grid_stride_start(); q < n; q += grid_stride()) w.removed_rank[q] = 0u;
        if (blockIdx.x == 0 && threadIdx.x == 0) cin->n_removed = 0u;
    }
    if (!grid_barrier(a, ++k, cin, cout)) return false;
    write_body<DIM>(c, cin, cout, in, out, w, true, true);
    return true;
}

// a.nsteps steps from state buffer a.parity (buf.b[parity], cnt[parity]);
// step j reads buffer (parity + j) & 1 and writes the other, as that many
// separate steps would.  A barrier separates one step's write-out from the
// next step's first stage.
struct CanonPair {
    CanonPtrs b[2];
};

template <int DIM, int BS>
__global__ void __launch_bounds__(BS, 2) k_step_persistent(sph_config c, Counters *cnt,
                                                        const __grid_constant__ CanonPair buf, WorkPtrs w,
                                                        PersistArgs a)
{
    // one shared buffer for the stages that use shared memory
    __shared__ union {
        WarpPairSmem pair[BS / 32];
        MergeSmem merge[BS / 32];
    } sm;
    const int p = a.parity;
    if (cnt[p].error & (1u << SPH_ERR_TIMEOUT)) {   // a step before gave up: nothing to step from
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&cnt[p ^ 1].error, cnt[p].error);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.gs_next = GridSync{0u, 0u, 0u, 0u};
    uint32_t k = 0;
    for (int j = 0; j < a.nsteps; ++j) {
        const int q = (p + j) & 1;
        Counters *cin = cnt + q, *cout = cnt + (q ^ 1);
        if (j > 0 && !grid_barrier(a, ++k, cin, cout)) return;
        const bool hashed = j > 0 || a.hash_ready != 0;
        if (!step_stages<DIM, BS>(c, cin, cout, buf.b[q], buf.b[q ^ 1], w, a, k, hashed, sm.pair, sm.merge))
            return;
    }
}

}  // namespace sph
