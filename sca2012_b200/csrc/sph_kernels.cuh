// sph_kernels.cuh — sm_100a kernels of one adaptive-SPH step.
//
// Layout in HBM (all SoA, 16-byte aligned):
//   canonical state, two buffers swapped every step, in the reference's
//   particle-index order (the order split/merge/compaction and the readback
//   depend on): pos4 = (x, y, z, level), vel4, ev4, acc4, dens, press,
//   energy, surface, interior, and when in use scene (batched scenes) and
//   pos_lo (compensated positions);
//   sorted working copies, in cell-key order, that the neighbour loops read
//   contiguously: spos/svel/sev (gathered), saux = (rho, p, p/rho^2, m/rho),
//   and the post-integration spos_n/svel_n/sev_n/sacc_n, ssurf, senergy;
//   a force neighbour's values in two 16-byte records fnb_a = (x, y, z,
//   p/rho^2) and fnb_b = (m/rho signed by level, ev), written by density;
//   per-particle neighbour candidate lists (nlist, rows of four-entry
//   chunks), written by the density pass and read by the force and energy
//   passes.
// Cell key = z*R*C + y*R + x with x = floor(pos / cell) in FP32, exactly the
// reference's calc_grid_pos/calc_grid_hash (SPH-3D-2/sph_system.cu:18-32).
// Neighbour search visits the 3 (2D) or 9 (3D) rows of x-adjacent cells; in
// key order each row is one contiguous slot range.
//
// Every decision that is an integer outcome of float arithmetic (cell keys,
// r^2 < h^2, h - r > 0, the split/merge scores) is evaluated with explicit
// round-to-nearest intrinsics in a fixed order, so the CPU oracle's FP32
// replica reproduces it bit for bit.  Every sum with a product operand in the
// step's bodies is written as an explicit __fmaf_rn / __fadd_rn too: the
// compiler then has no multiply-add to contract, so a body compiled into a
// standalone kernel and into the persistent step kernel (sph_persistent.cuh)
// rounds the same way and the two give the same bits.
#pragma once
#include <cstdint>
#include "../../include/sph/sph.h"

namespace sph {

constexpr uint32_t kEmpty = 0xffffffffu;
constexpr int kThreads = 256;

// Device-side counters of one step parity.
struct Counters {
    uint32_t n;            // live particles at step start
    uint32_t n_split;      // split particles this step
    uint32_t n_removed;    // merged-away particles this step
    uint32_t error;        // SPH_ERR_* bit flags (1 << code)
    uint32_t split_off;    // 1: splits suppressed this step (capacity)
    uint32_t disp2_max;    // bits of the step's largest squared displacement (FP32 >= 0), by the force pass
    uint32_t split_flags;  // particles the energy pass flagged to split this step
    uint32_t removed_flags;  // particles the merge pass flagged as merged away this step
                           // (a rank scan whose flags are all zero writes zeros instead of scanning)
    uint32_t merge_candidates;  // particles that may be merge-eligible this step, by the energy
                           // pass (at 0 the merge pass has nothing to do and returns at once)
};

struct CanonPtrs {
    float4 *pos, *vel, *ev, *acc;
    float *dens, *press, *energy, *surface;
    uint32_t *interior;
    uint32_t *sibling;                   // next member of the particle's split group (kEmpty: none)
    uint32_t *scene;                     // scene index (batched scenes)
    float4 *pos_lo;                      // low part of the position (compensated positions)
};

struct WorkPtrs {
    uint32_t *key, *slot, *tmp;          // per canonical particle / slot
    uint32_t *cell_count, *cell_off;     // C, C+1
    uint32_t *sidx, *skey, *inv;         // sorted slot -> particle, key; particle -> slot
    float4 *spos, *svel, *sev, *saux;
    float4 *spos_n, *svel_n, *sev_n, *sacc_n;
    float *ssurf, *senergy;
    uint32_t *snbr, *sinter;
    float4 *stv;                         // debug: wavelet-transformed velocity
    uint32_t *split_c, *removed_c;       // per canonical particle
    uint32_t *split_rank, *removed_rank; // exclusive scans
    uint32_t *split_list;                // split rank -> particle
    uint32_t *leader;                    // per sorted slot: 1 if merge survivor
    float4 *mpos, *mvel, *mev, *macc;    // merged values at the leader's slot
    float *menergy;
    uint32_t *sscene;                    // scene index per sorted slot
    const float4 *scene_tab;             // per scene: (lo.xyz, viscosity), (hi.xyz, gas constant)
    uint32_t nscenes;                    // 0: one scene in [0, world]
    uint32_t *merge_to;                  // taped steps only: slot -> its merge leader's slot
    float *mvs;                          // taped steps only: leader slot -> summed member volume
    uint32_t *wall;                      // taped steps only: wall contacts per slot
    float4 *spos_lo, *spos_lo_n;         // low position parts per slot (compensated positions)
    uint32_t pos_comp;                   // the config's compensated_positions
    uint32_t *nlist, *ncnt;              // neighbour candidates (layout: nl_at), by the density pass
    uint32_t nl_stride;                  // slots per list chunk row (the capacity)
    float4 *fnb_a, *fnb_b;               // a force neighbour in two loads: (x, y, z, p/rho^2) and
                                         // (m/rho with the sign bit set for level 2, ev.xyz), by the density pass
    uint32_t *out_src;                   // deferred outputs: per output index its sorted slot and kOut* flags
                                         // (nullptr: the write-out writes acc, dens, press, energy, surface)
};

// Deferred outputs.  acc, dens, press, energy and surface are outputs only:
// no stage of the next step reads them.  With w.out_src set the write-out
// records, per output index, the sorted slot its values come from (and how:
// a split parent, a child, a merge leader), and k_materialize writes the five
// fields from the step's sorted arrays when something reads the state; the
// values are write_body's.
constexpr uint32_t kOutChild = 1u << 31, kOutSplit = 1u << 30, kOutLeader = 1u << 29;
constexpr uint32_t kOutSlot = (1u << 29) - 1u;

// Neighbour candidates the density pass records per particle: every stencil
// neighbour within (1 + kNbrListMargin) h_max of the start-of-step position,
// in stencil-walk order (more than kNbrListCap: the consumers walk).
//  - The force pass uses the same positions: filtering the list with its own
//    test (r^2 < max(h_i^2, h_j^2), r^2 >= close_r2) gives its walk's pairs
//    in its walk's order.
//  - The energy pass tests the particles' integrated positions against the
//    stale cell lists of the particle's NEW cell.  When that cell is the old
//    one and |d_i| + max_j |d_j| (d: the step's displacements) stays under
//    the margin, every pair it accepts has a start-of-step distance below
//    h + margin, so it is on the list: filtering the list gives the walk's
//    pairs in the walk's order.  Other particles walk the stencil.
// Either way the sums are those of the walk, bit for bit.
constexpr uint32_t kNbrListCap = 128;
constexpr float kNbrListMargin = 0.05f;

// Pulls a line into L2 ahead of its use (no register, no result).
__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Entry k of slot s's list.  Entries come in chunks of four (one 16-byte
// load); chunk j of every slot is one row, so the chunk-j loads of a warp's
// 32 consecutive slots read 512 contiguous bytes.
__device__ __forceinline__ size_t nl_at(const WorkPtrs &w, uint32_t s, uint32_t k)
{
    return (size_t)(k >> 2) * ((size_t)w.nl_stride * 4u) + (size_t)s * 4u + (k & 3u);
}

__device__ __forceinline__ float energy_list_r2(const sph_config &c)
{
    const float r = 1.0f + kNbrListMargin;
    return fmaxf(c.kernel2[0], c.kernel2[1]) * (r * r);
}

// the displacement budget the list covers: 1% under the margin, far above
// the FP32 rounding of the distances involved (~1e-7 relative)
__device__ __forceinline__ float energy_list_budget(const sph_config &c)
{
    return 0.99f * kNbrListMargin * sqrtf(fmaxf(c.kernel2[0], c.kernel2[1]));
}

// hi + lo += d with hi, lo FP32 (Fast2Sum; |hi| >= |d + lo| holds for a
// position and one step's displacement).
__device__ __forceinline__ void comp_add(float &hi, float &lo, float d)
{
    const float y = __fadd_rn(d, lo);
    const float t = __fadd_rn(hi, y);
    lo = __fadd_rn(__fsub_rn(hi, t), y);
    hi = t;
}

// ------------------------------------------------------------ helpers
__device__ __forceinline__ int lv(float w) { return w == 1.0f ? 0 : 1; }

__device__ __forceinline__ uint32_t cell_coord(float x, float cs, uint32_t n)
{
    float f = floorf(__fdiv_rn(x, cs));
    if (!(f >= 0.0f)) return 0u;
    if (f >= (float)n) return n - 1u;
    return (uint32_t)f;
}

template <int DIM>
__device__ __forceinline__ uint3 cell_of(const sph_config &c, float4 p)
{
    uint3 q;
    q.x = cell_coord(p.x, c.cell_size, c.ncell[0]);
    q.y = cell_coord(p.y, c.cell_size, c.ncell[1]);
    q.z = DIM == 3 ? cell_coord(p.z, c.cell_size, c.ncell[2]) : 0u;
    return q;
}

__device__ __forceinline__ uint32_t key_of(const sph_config &c, uint32_t x, uint32_t y, uint32_t z)
{
    return z * c.ncell[0] * c.ncell[1] + y * c.ncell[0] + x;
}

// fma(dz, dz, fma(dx, dx, dy*dy)) with d = a - b, all round-to-nearest.
template <int DIM>
__device__ __forceinline__ float r2_of(float4 a, float4 b, float &dx, float &dy, float &dz)
{
    dx = __fsub_rn(a.x, b.x);
    dy = __fsub_rn(a.y, b.y);
    float t = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    if (DIM == 3) {
        dz = __fsub_rn(a.z, b.z);
        t = __fmaf_rn(dz, dz, t);
    } else {
        dz = 0.0f;
    }
    return t;
}

__device__ __forceinline__ float split_score(const sph_config &c, float e, float s)
{
    return __fmaf_rn(s, c.co_surface, __fmul_rn(e, c.co_energy));
}

__device__ __forceinline__ uint32_t grid_stride_start() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t grid_stride() { return gridDim.x * blockDim.x; }

// A load of data the kernel does not write.  NC = true takes the read-only
// (non-coherent) data path; the persistent step kernel (sph_persistent.cuh)
// passes NC = false, because inside its single launch a later stage reads
// what an earlier stage wrote.
template <bool NC, class T> __device__ __forceinline__ T ldro(const T *p)
{
    if constexpr (NC) return __ldg(p);
    else return *p;
}

// Row ranges of the 3^DIM neighbourhood of cell q: rows (dy, dz); each row is
// the slot range [off[key(x0)], off[key(x1)+1]) of cells x0..x1.
template <int DIM, bool NC = true>
__device__ __forceinline__ int row_range(const sph_config &c, const uint32_t *__restrict__ off, uint3 q,
                                         int dy, int dz, uint32_t &b, uint32_t &e)
{
    int y = (int)q.y + dy, z = (int)q.z + dz;
    if (y < 0 || y >= (int)c.ncell[1]) return 0;
    if (DIM == 3 && (z < 0 || z >= (int)c.ncell[2])) return 0;
    uint32_t x0 = q.x > 0 ? q.x - 1 : 0;
    uint32_t x1 = q.x + 1 < c.ncell[0] ? q.x + 1 : q.x;
    uint32_t k0 = key_of(c, x0, (uint32_t)y, (uint32_t)z);
    uint32_t k1 = key_of(c, x1, (uint32_t)y, (uint32_t)z);
    b = ldro<NC>(off + k0);
    e = ldro<NC>(off + k1 + 1);
    return 1;
}

// ------------------------------------------------------------ 1. hash
// Particle i at p: its cell key, and a slot among its cell's members from
// the cell's counter (which must start the step at zero).  One atomic per
// group of lanes in the same cell (consecutive particles often share one);
// any distinct slots do, k_reorder restores the order.
template <int DIM>
__device__ __forceinline__ void hash_one(const sph_config &c, const WorkPtrs &w, uint32_t i, float4 p)
{
    const uint3 q = cell_of<DIM>(c, p);
    const uint32_t k = key_of(c, q.x, q.y, q.z);
    w.key[i] = k;
    const unsigned grp = __match_any_sync(__activemask(), k);
    const int lead = __ffs(grp) - 1, lane = threadIdx.x & 31;
    uint32_t first = 0;
    if (lane == lead) first = atomicAdd(w.cell_count + k, (uint32_t)__popc(grp));
    first = __shfl_sync(grp, first, lead);
    w.slot[i] = first + __popc(grp & ((1u << lane) - 1u));
}

template <int DIM>
__device__ __forceinline__ void hash_body(const sph_config &c, const Counters *cnt, const CanonPtrs &st,
                                          const WorkPtrs &w)
{
    const uint32_t n = cnt->n;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) hash_one<DIM>(c, w, i, st.pos[i]);
}

template <int DIM, int BS = kThreads>
__global__ void __launch_bounds__(BS) k_hash(sph_config c, const Counters *__restrict__ cnt,
                                                  CanonPtrs st, WorkPtrs w)
{
    hash_body<DIM>(c, cnt, st, w);
}

// ------------------------------------------------------------ 3. scatter
template <bool NC>
__device__ __forceinline__ void scatter_body(const Counters *cnt, const WorkPtrs &w)
{
    const uint32_t n = cnt->n;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        // always below n when the counts, keys and slots come from one hash;
        // the test keeps a state left inconsistent by an abandoned persistent
        // step (SPH_ERR_TIMEOUT, not yet replaced by sph_set_state) in bounds
        const uint32_t d = ldro<NC>(w.cell_off + w.key[i]) + w.slot[i];
        if (d < n) w.tmp[d] = i;
    }
}

template <int BS = kThreads>
__global__ void __launch_bounds__(BS) k_scatter(const Counters *__restrict__ cnt, WorkPtrs w)
{
    scatter_body<true>(cnt, w);
}

// ------------------------------------------------------------ 4. stable order + gather
// The atomic slot order inside a cell is arbitrary; the stable order (equal
// keys in ascending particle index, as thrust's radix sort_by_key leaves
// them, SPH-3D-2/sph_system.cu:119-129) is restored by ranking each particle
// among its cell's members.  Then the state is gathered into key order.
template <bool NC>
__device__ __forceinline__ void reorder_body(const Counters *cnt, const CanonPtrs &st, const WorkPtrs &w)
{
    const uint32_t n = cnt->n;
    for (uint32_t s = grid_stride_start(); s < n; s += grid_stride()) {
        uint32_t i = w.tmp[s];
        uint32_t k = w.key[i];
        uint32_t b = ldro<NC>(w.cell_off + k), e = ldro<NC>(w.cell_off + k + 1);
        uint32_t r = 0;
        for (uint32_t t = b; t < e; ++t) r += w.tmp[t] < i;
        uint32_t d = b + r;
        w.sidx[d] = i;
        w.skey[d] = k;
        w.inv[i] = d;
        w.spos[d] = st.pos[i];
        w.svel[d] = st.vel[i];
        w.sev[d] = st.ev[i];
        if (w.nscenes) w.sscene[d] = st.scene[i];
        if (w.pos_comp) w.spos_lo[d] = st.pos_lo[i];
    }
}

template <int BS = kThreads>
__global__ void __launch_bounds__(BS) k_reorder(const Counters *__restrict__ cnt, CanonPtrs st, WorkPtrs w)
{
    reorder_body<true>(cnt, st, w);
}

// ------------------------------------------------------------ warp-lockstep pair loop
// The force and energy loops walk each particle's 3^DIM-cell stencil with the
// particle's whole warp in lockstep (up to 4 candidates per lane per step,
// their loads in flight together).  A lane appends the candidates it accepts
// to its list in shared memory; as soon as any lane's list holds kWarpCap
// entries, the whole warp runs the pair math over the lists in rounds (round
// k: every lane's k-th entry), each lane adding into its own sums in list
// order.  Flushing together keeps the expensive pair math converged (lists
// fill at similar rates, so few lanes idle in a round), and every particle's
// sums take the same order whichever particles share its warp.
constexpr uint32_t kWarpCap = 40;             // list fill that triggers a warp flush (44 x 32 x 4 B per warp)
constexpr uint32_t kWarpSlot = kWarpCap + 4;  // a step can add 4 more before the check

struct NbrPV { float4 p, v; };       // position, velocity

// Bundles a fetch(t) and a use(fetched) callable for warp_pairs<.., AHEAD>.
template <class F, class U> struct FetchUse {
    F fetch;
    U use;
};
template <class F, class U> __device__ __forceinline__ FetchUse<F, U> fetch_use(F f, U u) { return {f, u}; }

struct WarpPairSmem {
    uint32_t lst[kWarpSlot][32];     // per-lane lists, entry-major (appends hit 32 banks)
};

// accept(t, pj): this lane's test of candidate slot t at position pj.
// pair(t): adds this lane's pair with neighbour slot t into its sums.
// AHEAD > 0: pair is instead a fetch(t) / use(fetched) pair of callables
// (FetchUse) and a flush fetches AHEAD pairs before their math (entries past
// the lane's list read slot `self`), for callers whose fetched data fits in
// registers.  Every lane of the warp must call it (active = false for a lane
// without a particle).
template <int DIM, int AHEAD = 0, bool NC = true, class Accept, class Pair>
__device__ __forceinline__ void warp_pairs(const sph_config &c, const uint32_t *__restrict__ off,
                                           const float4 *__restrict__ pos, bool active, uint3 q,
                                           WarpPairSmem &sm, Accept accept, Pair pair, uint32_t self = 0)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    constexpr int nrows = DIM == 3 ? 9 : 3;   // rows (dy, dz), dz outer as in the reference loops
    int row = -1;
    uint32_t t = 0, e = 0;
    auto next_row = [&]() -> bool {
        while (++row < nrows) {
            const int dy = row % 3 - 1, dz = DIM == 3 ? row / 3 - 1 : 0;
            uint32_t b, ee;
            if (row_range<DIM, NC>(c, off, q, dy, dz, b, ee) && ee > b) {
                t = b;
                e = ee;
                return true;
            }
        }
        return false;
    };
    uint32_t cnt = 0;
    auto flush = [&]() {
        const uint32_t m = __reduce_max_sync(full, cnt);
        if constexpr (AHEAD == 0) {
            for (uint32_t k = 0; k < m; ++k)
                if (k < cnt) pair(sm.lst[k][lane]);
        } else {
            uint32_t k = 0;
            for (; k + AHEAD <= m; k += AHEAD) {
                decltype(pair.fetch(self)) got[AHEAD];
#pragma unroll
                for (int u = 0; u < AHEAD; ++u) got[u] = pair.fetch(k + u < cnt ? sm.lst[k + u][lane] : self);
#pragma unroll
                for (int u = 0; u < AHEAD; ++u)
                    if (k + u < cnt) pair.use(got[u]);
            }
            for (; k < m; ++k)
                if (k < cnt) pair.use(pair.fetch(sm.lst[k][lane]));
        }
        cnt = 0;
        __syncwarp();
    };
    bool more = active && next_row();
    while (__any_sync(full, more)) {
        if (more) {
            const uint32_t t0 = t, last = e - 1u;
            float4 pj[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) pj[u] = pos[min(t0 + u, last)];   // independent loads in flight
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (t0 + u < e && accept(t0 + u, pj[u])) sm.lst[cnt++][lane] = t0 + u;
            t = t0 + 4u;
            if (t >= e) more = next_row();
        }
        if (__any_sync(full, cnt >= kWarpCap)) flush();
    }
    if (__any_sync(full, cnt > 0)) flush();
}

// ------------------------------------------------------------ 5. density
// rho_i = m_i poly6_i h_i^6 + sum_{j != i, skip <= r^2 < h_i^2} m_j poly6_i (h_i^2 - r^2)^3
// p_i = k ((rho_i / rho0)^3 - 1)         (SPH-3D-2/sph_system.cu:338-677)
// SKIP = false: the config skips no close pairs (density_skip_r2 == 0), so
// the test !(r^2 < skip) is true for every r^2 and is left out.
template <int DIM, bool NC, bool SKIP>
__device__ __forceinline__ void density_walk(const sph_config &c, Counters *cnt, const WorkPtrs &w)
{
    const uint32_t n = cnt->n;
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt->disp2_max = 0u;   // the force pass takes the max
    for (uint32_t s = grid_stride_start(); s < n; s += grid_stride()) {
        const float4 pi = w.spos[s];
        const int li = lv(pi.w);
        const float h2 = c.kernel2[li];
        const float poly6 = c.poly6[li];
        const uint32_t k = w.skey[s];
        uint3 q;
        q.x = k % c.ncell[0];
        q.y = (k / c.ncell[0]) % c.ncell[1];
        q.z = DIM == 3 ? k / (c.ncell[0] * c.ncell[1]) : 0u;
        float rho = 0.0f;
        uint32_t nb = 0, nl = 0;
        const float m0 = c.mass[0], m1 = c.mass[1], skip = c.density_skip_r2;
        // the force and energy passes' candidates on the way
        // (r^2 < (1 + margin)^2 h_max^2), in the order their walks find them
        const bool rec = w.nlist != nullptr;
        const float re2 = energy_list_r2(c);
        // (m_j * poly6) once per level: the same product the sum takes first
        const float mp0 = m0 * poly6, mp1 = m1 * poly6;
        // single pass: the kernel sum is cheap enough to run predicated
        // (:394-417, j != i with skip <= r^2 < h_i^2)
        // list entry k at lbase[(k >> 2) * row4 + (k & 3)] (nl_at; the offset
        // fits 32 bits under the lists' 12 GB allocation limit)
        uint32_t *const lbase = rec ? w.nlist + (size_t)s * 4u : nullptr;
        const uint32_t row4 = w.nl_stride * 4u;
        // dx, dy as one packed FP32 subtraction (sm_100 f32x2; each half is the
        // IEEE round-to-nearest x_j - x_i, so r^2 is r2_of's to the bit)
        const float2 npi = make_float2(-pi.x, -pi.y);
        auto add = [&](uint32_t t, float4 pj) {   // t != s (the walk skips s)
            const float2 dxy = __fadd2_rn(make_float2(pj.x, pj.y), npi);
            float r2 = __fmaf_rn(dxy.x, dxy.x, __fmul_rn(dxy.y, dxy.y));
            if (DIM == 3) {
                const float dzz = __fsub_rn(pj.z, pi.z);
                r2 = __fmaf_rn(dzz, dzz, r2);
            }
            if ((!SKIP || !(r2 < skip)) && r2 < h2) {
                const float x = h2 - r2;
                rho = __fmaf_rn(pj.w == 1.0f ? mp0 : mp1, x * x * x, rho);
                ++nb;
            }
            if (rec && r2 < re2) {
                if (nl < kNbrListCap) lbase[(nl >> 2) * row4 + (nl & 3u)] = t;
                ++nl;
            }
        };
        auto range = [&](uint32_t b, uint32_t e) {
            uint32_t t = b;
            for (; t + 4 <= e; t += 4) {
                const float4 p0 = ldro<NC>(w.spos + t), p1 = ldro<NC>(w.spos + t + 1),
                             p2 = ldro<NC>(w.spos + t + 2), p3 = ldro<NC>(w.spos + t + 3);
                add(t, p0);
                add(t + 1, p1);
                add(t + 2, p2);
                add(t + 3, p3);
            }
            for (; t < e; ++t) add(t, ldro<NC>(w.spos + t));
        };
#pragma unroll 1
        for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz)
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                uint32_t b, e;
                if (!row_range<DIM, NC>(c, w.cell_off, q, dy, dz, b, e)) continue;
                if (dy == 0 && dz == 0) {   // the particle's own row: around its slot
                    range(b, s);
                    range(s + 1u, e);
                } else {
                    range(b, e);
                }
            }
        rho = __fadd_rn(rho, c.mass[li] * poly6 * c.kernel6[li]);   // self term
        float r = rho / c.rest_density;
        const float gas = w.nscenes ? w.scene_tab[2 * min(w.sscene[s], w.nscenes - 1u) + 1].w : c.gas_constant;
        float p = __fsub_rn(r * r * r, 1.0f) * gas;
        const float pr2 = p / (rho * rho), mr = c.mass[li] / rho;
        w.saux[s] = make_float4(rho, p, pr2, mr);
        const float4 evs = w.sev[s];
        w.fnb_a[s] = make_float4(pi.x, pi.y, pi.z, pr2);
        w.fnb_b[s] = make_float4(li ? -mr : mr, evs.x, evs.y, evs.z);
        w.snbr[s] = nb;
        if (rec) w.ncnt[s] = nl;
    }
}

template <int DIM, bool NC>
__device__ __forceinline__ void density_body(const sph_config &c, Counters *cnt, const WorkPtrs &w)
{
    if (c.density_skip_r2 == 0.0f) density_walk<DIM, NC, false>(c, cnt, w);
    else density_walk<DIM, NC, true>(c, cnt, w);
}

// The standalone kernel is instantiated per SKIP (the host picks it): one
// walk per kernel keeps its registers at the walk's own need.
template <int DIM, int BS = kThreads, bool SKIP = true>
__global__ void __launch_bounds__(BS) k_density(sph_config c, Counters *__restrict__ cnt, WorkPtrs w)
{
    density_walk<DIM, true, SKIP>(c, cnt, w);
}

// ------------------------------------------------------------ 6. force + integrate
// Pressure, viscosity and colour-field terms (SPH-3D-2/sph_system.cu:679-1137,
// 2D SPH-2D/sph_system.cu:462-790), then the integrator and walls
// (SPH-3D-2/sph_system.cu:204-322, SPH-2D/sph_system.cu:198-252).  The
// integrated state goes to the *_n arrays so the loop never sees it.
template <int DIM, int BS, bool NC>
__device__ __forceinline__ void force_integrate_body(const sph_config &c, Counters *cnt, const WorkPtrs &w,
                                                     WarpPairSmem *smem)
{
    const uint32_t n = cnt->n;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    // warp-uniform grid-stride loop: a warp takes 32 consecutive slots
    for (uint32_t base = blockIdx.x * BS + wib * 32u; base < n; base += gridDim.x * BS) {
        const uint32_t s_raw = base + lane;
        const bool valid = s_raw < n;
        const uint32_t s = valid ? s_raw : n - 1u;
        const float4 pi = w.spos[s];
        const float4 evi = w.sev[s];
        const float4 ai = w.saux[s];   // rho, p, p/rho^2, m/rho
        const int li = lv(pi.w);
        const float hi = c.kernel[li], hi2 = c.kernel2[li];
        const float mi = c.mass[li];
        const float ispk = c.kernel_h6_twice ? c.spiky[li] / c.kernel6[li] : c.spiky[li];
        const float ivis = c.kernel_h6_twice ? c.visco[li] / c.kernel6[li] : c.visco[li];
        const float igrad = -c.grad_poly6[li];
        const float ilap = c.lapc_poly6[li];
        const uint32_t sid = w.nscenes ? min(w.sscene[s], w.nscenes - 1u) : 0u;
        const float visc = w.nscenes ? w.scene_tab[2 * sid].w : c.viscosity;
        const uint32_t k = w.skey[s];
        uint3 q;
        q.x = k % c.ncell[0];
        q.y = (k / c.ncell[0]) % c.ncell[1];
        q.z = DIM == 3 ? k / (c.ncell[0] * c.ncell[1]) : 0u;
        float fx = 0.f, fy = 0.f, fz = 0.f, gx = 0.f, gy = 0.f, gz = 0.f, lap = 0.f;
        if (DIM == 2)   // self term, SPH-2D/sph_system.cu:599-603 (0 with the integer 3/4)
            lap = __fmaf_rn(ilap * ai.w * hi2, __fsub_rn(0.0f, c.lapc_three_quarters * hi2), lap);
        // pairs with r^2 < max(h_i^2, h_j^2) and r^2 >= close_r2 (:797-804)
        const float cut0 = fmaxf(hi2, c.kernel2[0]), cut1 = fmaxf(hi2, c.kernel2[1]);
        const float close = c.close_r2;
        // neighbour-level constants, once per particle instead of per pair
        const float jspk0 = c.kernel_h6_twice ? c.spiky[0] / c.kernel6[0] : c.spiky[0];
        const float jspk1 = c.kernel_h6_twice ? c.spiky[1] / c.kernel6[1] : c.spiky[1];
        const float jvis0 = c.kernel_h6_twice ? c.visco[0] / c.kernel6[0] : c.visco[0];
        const float jvis1 = c.kernel_h6_twice ? c.visco[1] / c.kernel6[1] : c.visco[1];
        const float mimj0 = mi * c.mass[0], mimj1 = mi * c.mass[1];
        auto accept = [&](uint32_t t, const float4 &pj) {
            float rx, ry, rz;
            const float r2 = r2_of<DIM>(pi, pj, rx, ry, rz);
            const float cut = pj.w == 1.0f ? cut0 : cut1;
            return t != s && r2 < cut && !(r2 < close);
        };
        // pressure, viscosity and colour-field terms of one neighbour
        // (a, b: the neighbour's two records)
        auto pair_ab = [&](const float4 a, const float4 b) {
            float rx, ry, rz;
            const float r2 = r2_of<DIM>(pi, a, rx, ry, rz);
            const int lj = signbit(b.x) ? 1 : 0;
            const float mrj = fabsf(b.x);   // m_j/rho_j
            const float r = __fsqrt_rn(r2);
            float ipk = 0.f, ivk = 0.f, jpk = 0.f, jvk = 0.f;
            const float ikr = __fsub_rn(hi, r);
            if (ikr > 0.0f) {
                ipk = ispk * ikr * ikr;
                ivk = ivis * ikr;
                const float x = hi2 - r2;
                const float tg = igrad * mrj * x * x;   // -grad_poly6 * m_j/rho_j * (h^2-r^2)^2
                gx = __fmaf_rn(tg, rx, gx); gy = __fmaf_rn(tg, ry, gy); gz = __fmaf_rn(tg, rz, gz);
                lap = __fmaf_rn(ilap * mrj * x, __fsub_rn(r2, c.lapc_three_quarters * x), lap);
            }
            const float jkr = __fsub_rn(c.kernel[lj], r);
            if (jkr > 0.0f) {
                jpk = (lj ? jspk1 : jspk0) * jkr * jkr;
                jvk = (lj ? jvis1 : jvis0) * jkr;
            }
            // 1/r from the approximate reciprocal square root of r^2 (the h - r
            // decisions above keep the IEEE square root)
            const float tp = (lj ? mimj1 : mimj0) * __fadd_rn(ai.z, a.w) * __fadd_rn(ipk, jpk) * 0.5f * rsqrtf(r2);
            const float tv = (ai.w * mrj) * visc * __fadd_rn(ivk, jvk) * 0.5f;
            fx = __fmaf_rn(__fsub_rn(b.y, evi.x), tv, __fmaf_rn(-rx, tp, fx));
            fy = __fmaf_rn(__fsub_rn(b.z, evi.y), tv, __fmaf_rn(-ry, tp, fy));
            if (DIM == 3) fz = __fmaf_rn(__fsub_rn(b.w, evi.z), tv, __fmaf_rn(-rz, tp, fz));
        };
        // the walk's test for a list entry (a list never holds the particle itself)
        auto accept_ab = [&](const float4 &a, const float4 &b) {
            float rx, ry, rz;
            const float r2 = r2_of<DIM>(pi, a, rx, ry, rz);
            const float cut = signbit(b.x) ? cut1 : cut0;
            return r2 < cut && !(r2 < close);
        };
        auto pair = [&](uint32_t t) { pair_ab(w.fnb_a[t], w.fnb_b[t]); };
        const unsigned full = 0xffffffffu;
        const uint32_t nf = valid && w.nlist ? w.ncnt[s] : 0u;
        if (__all_sync(full, w.nlist != nullptr && nf <= kNbrListCap)) {
            // the density pass's candidates, filtered by the walk's test: same
            // neighbours, same order as the walk
            const uint32_t m = __reduce_max_sync(full, nf);
            uint32_t kk = 0;
            // four entries per 16-byte load, their neighbours' loads issued
            // before the math (entries past nf are replaced by the particle itself)
            if (4 < m) prefetch_l2(w.nlist + nl_at(w, s, 4));
            for (; kk + 4 <= m; kk += 4) {
                if (kk + 8 < m) prefetch_l2(w.nlist + nl_at(w, s, kk + 8));   // 2 rounds ahead
                const uint4 t4 = *reinterpret_cast<const uint4 *>(w.nlist + nl_at(w, s, kk));
                const uint32_t tt[4] = {kk < nf ? t4.x : s, kk + 1 < nf ? t4.y : s, kk + 2 < nf ? t4.z : s,
                                        kk + 3 < nf ? t4.w : s};
                float4 na[4], nb[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    na[u] = w.fnb_a[tt[u]];
                    nb[u] = w.fnb_b[tt[u]];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (kk + u < nf && accept_ab(na[u], nb[u])) pair_ab(na[u], nb[u]);
            }
            for (; kk < m; ++kk)
                if (kk < nf) {
                    const uint32_t t = w.nlist[nl_at(w, s, kk)];
                    const float4 a = w.fnb_a[t], b = w.fnb_b[t];
                    if (accept_ab(a, b)) pair_ab(a, b);
                }
        } else {
            warp_pairs<DIM, 0, NC>(c, w.cell_off, w.spos, valid, q, smem[wib], accept, pair);
        }
        if (!valid) continue;
        // surface tension switch (SPH-3D-2/sph_system.cu:1113-1136)
        const float nrm = sqrtf(__fmaf_rn(gz, gz, __fmaf_rn(gy, gy, __fmul_rn(gx, gx))));
        if (nrm > c.surface_threshold) {
            const float f = c.surface_coef * lap / nrm;
            fx = __fmaf_rn(f, gx, fx); fy = __fmaf_rn(f, gy, fy); fz = __fmaf_rn(f, gz, fz);
        }
        if (DIM == 2 && c.extern_force_on) {   // SPH-2D/sph_system.cu:781-789
            float xl = __fsub_rn(pi.x, c.extern_click[0]), yl = __fsub_rn(pi.y, c.extern_click[1]);
            if (__fmaf_rn(xl, xl, __fmul_rn(yl, yl)) <= __fmul_rn(c.extern_len, c.extern_len)) {
                fx = __fmaf_rn(c.extern_force[0], c.extern_coe, fx);
                fy = __fmaf_rn(c.extern_force[1], c.extern_coe, fy);
            }
        }
        w.ssurf[s] = nrm;

        // ---- integrate ----
        const float rho = ai.x, dt = c.time_step;
        float4 x = pi;
        float4 lo = make_float4(0.f, 0.f, 0.f, 0.f);   // low position part (compensated positions)
        float4 v = w.svel[s];
        float4 ev = evi;
        float4 a = make_float4(fx, fy, fz, 0.f);
        float rad;
        if (c.integrator == SPH_INTEGRATE_REF2D) {
            rad = c.radius[li] / 2.0f;
            a.x = __fmaf_rn(c.gravity[0], dt, a.x) / rho;
            a.y = __fmaf_rn(c.gravity[1], dt, a.y) / rho;
            v.x = __fmaf_rn(a.x, dt, v.x); v.y = __fmaf_rn(a.y, dt, v.y);
            ev.x = (ev.x + v.x) / 2.0f; ev.y = (ev.y + v.y) / 2.0f;
            x.x = __fmaf_rn(v.x, dt, x.x); x.y = __fmaf_rn(v.y, dt, x.y);
        } else {
            rad = c.radius[li];
            if (c.integrator == SPH_INTEGRATE_REF3D) {
                if (c.push_left && pi.x < __fdiv_rn(c.world[0], 3.0f) &&
                    pi.y > __fdiv_rn(c.world[1], (float)c.push_y_div))
                    a.x += 20.0f;
                if (c.push_right && pi.x > __fmul_rn(__fdiv_rn(c.world[0], 3.0f), 2.0f) &&
                    pi.y > __fdiv_rn(c.world[1], (float)c.push_y_div))
                    a.x -= 20.0f;
                v.x += a.x * dt / rho; v.y += a.y * dt / rho; v.z += a.z * dt / rho;
                v.x += c.gravity[0] * dt / rho; v.y += c.gravity[1] * dt / rho; v.z += c.gravity[2] * dt / rho;
            } else {
                const float im = 1.0f / mi;
                v.x = __fmaf_rn(__fmaf_rn(a.x, im, c.gravity[0]), dt, v.x);
                v.y = __fmaf_rn(__fmaf_rn(a.y, im, c.gravity[1]), dt, v.y);
                v.z = __fmaf_rn(__fmaf_rn(a.z, im, c.gravity[2]), dt, v.z);
            }
            if (w.pos_comp) {
                lo = w.spos_lo[s];
                comp_add(x.x, lo.x, __fmul_rn(v.x, dt));
                comp_add(x.y, lo.y, __fmul_rn(v.y, dt));
                if (DIM == 3) comp_add(x.z, lo.z, __fmul_rn(v.z, dt));
            } else {
                x.x = __fmaf_rn(v.x, dt, x.x); x.y = __fmaf_rn(v.y, dt, x.y); x.z = __fmaf_rn(v.z, dt, x.z);
            }
            if (DIM == 3 && c.use_cylinder) {   // SPH-3D-2/sph_system.cu:242-282
                for (int qq = 0; qq < 3; ++qq) {
                    const sph_sphere S = c.sphere[qq];
                    float dxs = x.x - S.pos[0], dys = x.y - S.pos[1], dzs = x.z - S.pos[2];
                    float dist = sqrtf(__fmaf_rn(dzs, dzs, __fmaf_rn(dys, dys, __fmul_rn(dxs, dxs))));
                    float R = S.radius + rad;
                    if (dist < R) {
                        float sx = dxs / dist * R, sy = dys / dist * R, sz = dzs / dist * R;
                        float il = rsqrtf(__fmaf_rn(sz, sz, __fmaf_rn(sy, sy, __fmul_rn(sx, sx))));
                        float nx = sx * il, ny = sy * il, nz = sz * il;
                        x.x = S.pos[0] + sx; x.y = S.pos[1] + sy; x.z = S.pos[2] + sz;
                        lo = make_float4(0.f, 0.f, 0.f, 0.f);
                        float vn = __fmaf_rn(v.z, nz, __fmaf_rn(v.y, ny, __fmul_rn(v.x, nx)));
                        const float dv = S.damping * vn;
                        v.x = __fmaf_rn(-dv, nx, v.x); v.y = __fmaf_rn(-dv, ny, v.y); v.z = __fmaf_rn(-dv, nz, v.z);
                    }
                }
            }
        }
        // walls x, y, z (SPH-3D-2/sph_system.cu:285-319); a batched scene
        // has its own box
        {
            const float4 blo = w.nscenes ? w.scene_tab[2 * sid] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 bhi = w.nscenes ? w.scene_tab[2 * sid + 1]
                                         : make_float4(c.world[0], c.world[1], c.world[2], 0.f);
            const float damp = c.wall_damping;
            uint32_t hit = 0;
            auto wall = [&](float &xd, float &vd, float &xl, float lo_b, float hi_b, int d) {
                const float hi_w = hi_b - rad, lo_w = lo_b + rad;
                if (xd >= hi_w) { vd *= damp; xd = hi_w; xl = 0.0f; hit |= 1u << (2 * d); }
                if (xd < lo_w) { vd *= damp; xd = lo_w; xl = 0.0f; hit |= 2u << (2 * d); }
            };
            wall(x.x, v.x, lo.x, blo.x, bhi.x, 0);
            wall(x.y, v.y, lo.y, blo.y, bhi.y, 1);
            if (DIM == 3) wall(x.z, v.z, lo.z, blo.z, bhi.z, 2);
            if (w.wall) w.wall[s] = hit;   // recorded for the adjoint
        }
        // a non-finite position is reported (the walls would hide +-inf); the
        // neighbour tests fail for it, so it interacts with nothing
        if (!(isfinite(x.x) && isfinite(x.y) && isfinite(x.z)) || !isfinite(v.x + v.y + v.z))
            atomicOr(&cnt->error, 1u << SPH_ERR_NONFINITE);
        if (c.integrator != SPH_INTEGRATE_REF2D) {
            ev.x = (ev.x + v.x) / 2.0f; ev.y = (ev.y + v.y) / 2.0f; ev.z = (ev.z + v.z) / 2.0f;
        }
        w.spos_n[s] = x;        // .w keeps the level
        if (w.pos_comp) w.spos_lo_n[s] = lo;
        w.svel_n[s] = v;
        w.sev_n[s] = ev;
        w.sacc_n[s] = a;
        if (w.nlist) {   // the step's largest squared displacement, one atomic per group of lanes
            float ddx, ddy, ddz;
            const float d2 = r2_of<DIM>(x, pi, ddx, ddy, ddz);
            // non-negative floats order as their bits; a NaN position (which
            // passes no neighbour test) is left out
            const uint32_t bits = d2 == d2 ? __float_as_uint(d2) : 0u;
            const unsigned am = __activemask();
            const uint32_t m = __reduce_max_sync(am, bits);
            if (lane == __ffs(am) - 1) atomicMax(&cnt->disp2_max, m);
        }
    }
}

template <int DIM, int BS = kThreads, int MINB = 3>
__global__ void __launch_bounds__(BS, MINB) k_force_integrate(sph_config c, Counters *__restrict__ cnt,
                                                              WorkPtrs w)
{
    __shared__ WarpPairSmem smem[BS / 32];
    force_integrate_body<DIM, BS, true>(c, cnt, w, smem);
}

// ------------------------------------------------------------ 7. energy + split decision
// Wavelet energy on the STALE cell lists (built at step start) with the NEW
// positions (SPH-3D-2/sph_system.cu:1169-1546), then the split decision
// (decide_adaptive_kernel, :1548-1574) written per particle index.
__device__ __forceinline__ float wavelet(float x, float amp)
{
    // psi(x) = amp * (x^2/4 - 1) * EXP^(-x^2/8), EXP = 2.718281f (sigma = 2)
    const float x2 = x * x;
    return amp * __fsub_rn(x2 * 0.25f, 1.0f) * exp2f(-x2 * 0.125f * 1.44269476f);
}

template <int DIM, int BS, bool NC>
__device__ __forceinline__ void energy_split_body(const sph_config &c, Counters *cnt, const CanonPtrs &st,
                                                  const WorkPtrs &w, int want_tv, WarpPairSmem *smem)
{
    const uint32_t n = cnt->n;
    // 2/(PI^0.25 * sqrt(3 sigma)) with PI = 3.141592f, sigma = 2
    const float amp = 2.0f / (powf(3.141592f, 0.25f) * sqrtf(6.0f));
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    // displacement budget left for this particle's own move (the list covers
    // |d_i| + max_j |d_j| up to energy_list_budget)
    const float own_budget = w.nlist ? energy_list_budget(c) - sqrtf(__uint_as_float(cnt->disp2_max)) : -1.0f;
    for (uint32_t base = blockIdx.x * BS + wib * 32u; base < n; base += gridDim.x * BS) {
        const uint32_t s_raw = base + lane;
        const bool valid = s_raw < n;
        const uint32_t s = valid ? s_raw : n - 1u;
        const float4 pi = w.spos_n[s];
        const int li = lv(pi.w);
        const int lk = c.energy_large_kernel ? 0 : li;
        const float h = c.kernel[lk], h2 = c.kernel2[lk];
        const float ih = 1.0f / h, isq = 1.0f / sqrtf(h);
        const uint3 q = cell_of<DIM>(c, pi);
        float tsx = 0.f, tsy = 0.f, tsz = 0.f, tvx = 0.f, tvy = 0.f, tvz = 0.f;
        const float skip = c.energy_skip_close ? c.close_r2 : 0.0f;   // :1229-1232 (2D keeps close pairs)
        // j != i with skip <= r^2 < h^2 (:1222-1233), on the stale lists
        auto accept = [&](uint32_t t, const float4 &pj) {
            float rx, ry, rz;
            const float r2 = r2_of<DIM>(pi, pj, rx, ry, rz);
            return t != s && r2 < h2 && !(r2 < skip);
        };
        // the wavelet transform of one neighbour (its loads fetched ahead)
        auto fetch = [&](uint32_t t) { return NbrPV{w.spos_n[t], w.svel_n[t]}; };
        auto use = [&](const NbrPV &g) {
            const float4 pj = g.p, vj = g.v;
            float rx, ry, rz;
            r2_of<DIM>(pi, pj, rx, ry, rz);
            const float wx = wavelet(rx * ih, amp), wy = wavelet(ry * ih, amp);
            tsx = __fadd_rn(tsx, wx); tsy = __fadd_rn(tsy, wy);
            tvx = __fmaf_rn(vj.x * wx, isq, tvx); tvy = __fmaf_rn(vj.y * wy, isq, tvy);
            if (DIM == 3) {
                const float wz = wavelet(rz * ih, amp);
                tsz = __fadd_rn(tsz, wz);
                tvz = __fmaf_rn(vj.z * wz, isq, tvz);
            }
        };
        // the density pass's candidates when the particle kept its cell and the
        // step's moves fit the margin; the stencil walk otherwise
        // (every test is false for a NaN distance or budget: such a lane walks)
        uint32_t ne = 0;
        bool walk = valid;
        if (valid && own_budget >= 0.0f) {
            float ddx, ddy, ddz;
            const float d2 = r2_of<DIM>(pi, w.spos[s], ddx, ddy, ddz);
            const uint32_t cand = w.ncnt[s];
            if (cand <= kNbrListCap && key_of(c, q.x, q.y, q.z) == w.skey[s] && sqrtf(d2) <= own_budget) {
                ne = cand;
                walk = false;
            }
        }
        const uint32_t m = __reduce_max_sync(0xffffffffu, ne);
        if (m) {
            // four entries per 16-byte load, their neighbours fetched before the
            // math (entries past ne are replaced by the particle itself)
            if (4 < m) prefetch_l2(w.nlist + nl_at(w, s, 4));
            for (uint32_t kk = 0; kk < m; kk += 4) {
                if (kk + 8 < m) prefetch_l2(w.nlist + nl_at(w, s, kk + 8));   // 2 rounds ahead
                const uint4 t4 = kk < ne ? *reinterpret_cast<const uint4 *>(w.nlist + nl_at(w, s, kk))
                                         : make_uint4(s, s, s, s);
                const uint32_t tt[4] = {kk < ne ? t4.x : s, kk + 1 < ne ? t4.y : s, kk + 2 < ne ? t4.z : s,
                                        kk + 3 < ne ? t4.w : s};
                NbrPV g[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) g[u] = fetch(tt[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (kk + u < ne && accept(tt[u], g[u].p)) use(g[u]);
            }
        }
        warp_pairs<DIM, 4, NC>(c, w.cell_off, w.spos_n, walk, q, smem[wib], accept, fetch_use(fetch, use), s);
        if (!valid) continue;
        tvx /= tsx; tvy /= tsy; tvz = DIM == 3 ? tvz / tsz : 0.f;
        float energy = 0.5f * __fmaf_rn(tvx, tvx, __fmul_rn(tvy, tvy));
        if (c.energy_mass_weight) energy *= c.mass[li];
        w.senergy[s] = energy;
        if (want_tv) w.stv[s] = make_float4(tvx, tvy, tvz, 0.f);

        const uint32_t i = w.sidx[s];
        const float surf = w.ssurf[s];
        const float dens = w.saux[s].x;
        const uint32_t nb = w.snbr[s];
        uint32_t split = 0;
        if (c.use_split && pi.w == 1.0f) {
            if (c.split_rule == SPH_SPLIT_DEFICIT)
                split = (nb < c.split_min_neighbors || dens < c.split_density_ratio * c.rest_density) ? 1u : 0u;
            else
                split = split_score(c, energy, surf) > c.split_criteria ? 1u : 0u;
        }
        w.split_c[i] = split;
        if (split) atomicAdd(&cnt->split_flags, 1u);
        w.removed_c[i] = 0u;
        uint32_t inter = 0;
        if (c.merge_rule == SPH_MERGE_INTERIOR || c.merge_rule == SPH_MERGE_SIBLING) {
            const int flagged = nb < c.split_min_neighbors || dens < c.split_density_ratio * c.rest_density;
            inter = (flagged || split) ? 0u : st.interior[i] + 1u;
            w.sinter[s] = inter;
        }
        // a superset of merge_eligible's particles, whichever way the capacity
        // guard decides this step's splits (a split particle becomes level 2)
        if (c.use_merge && c.merge_rule != SPH_MERGE_WAVELET_CELL) {
            const bool l2 = pi.w != 1.0f;
            bool may;
            if (c.merge_rule == SPH_MERGE_WAVELET)
                may = (l2 && split_score(c, energy, surf) < c.merge_criteria) ||
                      (split && split_score(c, c.split_ways == 4 ? energy / 4.0f : energy, surf) < c.merge_criteria);
            else
                may = (l2 || split) && inter >= c.merge_interior_steps;
            if (may) atomicAdd(&cnt->merge_candidates, 1u);
        }
    }
}

template <int DIM, int BS = kThreads, int MINB = 3>
__global__ void __launch_bounds__(BS, MINB) k_energy_split(sph_config c, Counters *__restrict__ cnt,
                                                           CanonPtrs st, WorkPtrs w, int want_tv)
{
    __shared__ WarpPairSmem smem[BS / 32];
    energy_split_body<DIM, BS, true>(c, cnt, st, w, want_tv, smem);
}

// Capacity guard after the split scan: if the children would not fit, this
// step runs without splits and reports SPH_ERR_CAPACITY (the reference writes
// past its buffer, SPH-3D-2/sph_system.cu:1645-1656).
__device__ __forceinline__ void split_guard_body(const sph_config &c, Counters *cnt, uint32_t cap)
{
    uint64_t extra = c.split_ways == 4 ? 3u : 1u;
    uint64_t after = (uint64_t)cnt->n + (uint64_t)cnt->n_split * extra;
    if (after > cap) {
        cnt->split_off = 1u;
        cnt->error |= 1u << SPH_ERR_CAPACITY;
    } else {
        cnt->split_off = 0u;
    }
}

__global__ void k_split_guard(const sph_config c, Counters *cnt, uint32_t cap) { split_guard_body(c, cnt, cap); }

// ------------------------------------------------------------ 8. merge
// One warp per cell over its sorted members (merge_kernel,
// SPH-3D-2/sph_system.cu:1661-1789; 3D-4 :1702-1888; 2D :1177-1270).
// Eligible members (evaluated on the post-split values) are ranked by warp
// ballots in slot order; groups of `ways` consecutive eligible members merge
// into the first, with V = m/rho weights (level already set to 1 for the
// survivor, :1742-1777) or the plain mean in 2D.
constexpr int kMergeListMax = 256;   // eligible members held per warp in shared memory

template <int DIM>
__device__ __forceinline__ int merge_eligible(const sph_config &c, const WorkPtrs &w, uint32_t t,
                                              uint32_t split_on, uint32_t ways, float cell_score)
{
    const uint32_t i = w.sidx[t];
    const uint32_t sp = split_on & w.split_c[i];
    const float lvl = sp ? 2.0f : w.spos_n[t].w;
    if (c.merge_rule == SPH_MERGE_WAVELET) {
        float en = w.senergy[t];
        if (sp && ways == 4) en = en / 4.0f;
        return lvl != 1.0f && split_score(c, en, w.ssurf[t]) < c.merge_criteria;
    }
    if (c.merge_rule == SPH_MERGE_WAVELET_CELL) return lvl == 2.0f && cell_score < c.merge_criteria;
    return lvl != 1.0f && w.sinter[t] >= c.merge_interior_steps;   // SPH_MERGE_INTERIOR, SPH_MERGE_SIBLING
}

// Merges the group g[0..ways) into g[0] (values on the post-split state).
template <int DIM>
__device__ __forceinline__ void merge_group(const sph_config &c, const WorkPtrs &w, const uint32_t *g,
                                            uint32_t ways, uint32_t split_on, float hs2, uint32_t *removed_flags)
{
    float V[4], Vs = 0.f;
    for (uint32_t k = 0; k < ways; ++k) {
        // eligible members are level 2; the survivor's level is set to 1
        // before its volume is taken (SPH-3D-2/sph_system.cu:1742-1756)
        V[k] = DIM == 2 ? 1.0f : (k == 0 ? c.mass[0] : c.mass[1]) / w.saux[g[k]].x;
        Vs += V[k];
    }
    float4 P = make_float4(0.f, 0.f, 0.f, 0.f), Vv = P, E = P, A = P;
    float en = 0.f;
    for (uint32_t k = 0; k < ways; ++k) {
        const uint32_t t = g[k];
        const uint32_t sp = split_on & w.split_c[w.sidx[t]];
        float4 p = w.spos_n[t];
        if (sp) p.x += hs2;
        const float4 vv = w.svel_n[t], ee = w.sev_n[t], aa = w.sacc_n[t];
        float ek = w.senergy[t];
        if (sp && ways == 4) ek = ek / 4.0f;
        P.x = __fmaf_rn(p.x, V[k], P.x); P.y = __fmaf_rn(p.y, V[k], P.y); P.z = __fmaf_rn(p.z, V[k], P.z);
        Vv.x = __fmaf_rn(vv.x, V[k], Vv.x); Vv.y = __fmaf_rn(vv.y, V[k], Vv.y); Vv.z = __fmaf_rn(vv.z, V[k], Vv.z);
        E.x = __fmaf_rn(ee.x, V[k], E.x); E.y = __fmaf_rn(ee.y, V[k], E.y); E.z = __fmaf_rn(ee.z, V[k], E.z);
        A.x = __fmaf_rn(aa.x, V[k], A.x); A.y = __fmaf_rn(aa.y, V[k], A.y); A.z = __fmaf_rn(aa.z, V[k], A.z);
        en += ek;
    }
    const uint32_t t1 = g[0];
    w.mpos[t1] = make_float4(P.x / Vs, P.y / Vs, P.z / Vs, 1.0f);
    w.mvel[t1] = make_float4(Vv.x / Vs, Vv.y / Vs, Vv.z / Vs, 0.f);
    w.mev[t1] = make_float4(E.x / Vs, E.y / Vs, E.z / Vs, 0.f);
    w.macc[t1] = make_float4(A.x / Vs, A.y / Vs, A.z / Vs, 0.f);
    w.menergy[t1] = en / (float)ways;
    w.leader[t1] = 1u;
    for (uint32_t k = 1; k < ways; ++k) w.removed_c[w.sidx[g[k]]] = 1u;
    atomicAdd(removed_flags, ways - 1u);
    if (w.merge_to) {   // recorded for the adjoint
        for (uint32_t k = 0; k < ways; ++k) w.merge_to[g[k]] = t1;
        w.mvs[t1] = Vs;
    }
}

// Shared memory of one warp of the merge pass.
struct MergeSmem {
    uint32_t list[kMergeListMax];    // eligible slots in slot order
    uint32_t lcell[kMergeListMax];   // their cells
    uint8_t lrank[kMergeListMax];    // their ranks among their cell's eligible members
};

template <int DIM>
__device__ __forceinline__ void merge_body(const sph_config &c, Counters *cnt, const CanonPtrs &st,
                                           const WorkPtrs &w, uint32_t ncells, uint32_t cap, MergeSmem *ms)
{
    // the energy pass found no candidate (the 2D cell rule is not counted there)
    if (c.merge_rule != SPH_MERGE_WAVELET_CELL && cnt->merge_candidates == 0u) return;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);
    const uint32_t n = cnt->n;
    const uint32_t split_on = cnt->split_off ? 0u : 1u;
    const uint32_t ways = c.split_ways == 4 ? 4u : 2u;
    const uint32_t extra = ways - 1u;
    const float hs2 = c.kernel[1] / 2.0f;
    // 2D rule: the criterion of the particle whose INDEX equals the cell
    // index, as memory holds it at merge time (SPH-2D/sph_system.cu:1207)
    auto cell_score_of = [&](uint32_t cell) -> float {
        if (c.merge_rule != SPH_MERGE_WAVELET_CELL) return 0.f;
        float eq, sq;
        const uint32_t n_after = n + (split_on ? cnt->n_split * extra : 0u);
        if (cell < n) {
            const uint32_t sl = w.inv[cell];
            eq = w.senergy[sl]; sq = w.ssurf[sl];
        } else if (cell < n_after) {
            const uint32_t sl = w.inv[w.split_list[(cell - n) / extra]];
            eq = w.senergy[sl]; sq = w.ssurf[sl];
        } else if (cell < cap) {
            eq = st.energy[cell]; sq = st.surface[cell];
        } else {
            eq = 0.f; sq = 0.f;   // beyond the allocation: treated as zeroed memory
        }
        return split_score(c, eq, sq);
    };
    // each warp takes 32 consecutive cells at a time; their members are one
    // contiguous slot range, tested 32 slots at a time
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + wib) * 32u; base < ncells; base += warps_total * 32u) {
        const uint32_t cend = min(base + 32u, ncells);
        const uint32_t sb = w.cell_off[base], se = w.cell_off[cend];
        // every eligible member is listed with its cell and its rank among
        // the cell's eligible members (cells are contiguous in slot order; the
        // count of the chunk's last cell carries into the next chunk)
        uint32_t len = 0, carry_cell = kEmpty, carry_cnt = 0;
        for (uint32_t t0 = sb; t0 < se; t0 += 32) {
            const uint32_t t = t0 + lane;
            const bool in = t < se;
            const uint32_t cell = in ? w.skey[t] : kEmpty;
            const int el = in ? merge_eligible<DIM>(c, w, t, split_on, ways, cell_score_of(cell)) : 0;
            const unsigned same = __match_any_sync(full, cell);
            const unsigned eb = __ballot_sync(full, el);
            const uint32_t rank = __popc(eb & same & lt) + (cell == carry_cell ? carry_cnt : 0u);
            const uint32_t pos = len + __popc(eb & lt);
            if (el && pos < (uint32_t)kMergeListMax) {
                ms[wib].list[pos] = t;
                ms[wib].lcell[pos] = cell;
                ms[wib].lrank[pos] = (uint8_t)min(rank, 255u);   // a rank inside the list is below its length
            }
            len += __popc(eb);
            const int last = __popc(__ballot_sync(full, in)) - 1;
            const uint32_t lc = __shfl_sync(full, cell, last);
            const unsigned lsame = __shfl_sync(full, same, last);
            carry_cnt = (lc == carry_cell ? carry_cnt : 0u) + __popc(eb & lsame);
            carry_cell = lc;
        }
        __syncwarp();
        if (len <= (uint32_t)kMergeListMax) {
            // a group = `ways` consecutive eligible members of one cell, from
            // rank 0 on; its first member is the survivor
            for (uint32_t k = lane; k < len; k += 32)
                if (ms[wib].lrank[k] % ways == 0 && k + ways - 1 < len &&
                    ms[wib].lcell[k + ways - 1] == ms[wib].lcell[k])
                    merge_group<DIM>(c, w, &ms[wib].list[k], ways, split_on, hs2, &cnt->removed_flags);
            __syncwarp();
            continue;
        }
        // more eligible members than the list holds: the cells one at a time
        const uint32_t mine = base + lane;
        const uint32_t members = mine < cend ? w.cell_off[mine + 1] - w.cell_off[mine] : 0u;
        uint32_t todo = __ballot_sync(full, members >= ways);
        while (todo) {
            const uint32_t cell = base + (__ffs(todo) - 1);
            todo &= todo - 1;
            const uint32_t b = w.cell_off[cell], e = w.cell_off[cell + 1];
            const float cell_score = cell_score_of(cell);
            uint32_t count = 0;
            for (uint32_t t0 = b; t0 < e; t0 += 32) {
                const uint32_t t = t0 + lane;
                const int el = t < e ? merge_eligible<DIM>(c, w, t, split_on, ways, cell_score) : 0;
                const unsigned m = __ballot_sync(full, el);
                const uint32_t r = count + __popc(m & lt);
                if (el && r < (uint32_t)kMergeListMax) ms[wib].list[r] = t;
                count += __popc(m);
            }
            __syncwarp();
            const uint32_t groups = count / ways;
            if (count <= (uint32_t)kMergeListMax) {
                for (uint32_t g = lane; g < groups; g += 32)
                    merge_group<DIM>(c, w, &ms[wib].list[g * ways], ways, split_on, hs2, &cnt->removed_flags);
            } else if (lane == 0) {
                // more eligible members than the list holds: walk the cell
                // serially with the same group arithmetic
                uint32_t grp[4], got = 0, done = 0;
                for (uint32_t t = b; t < e && done < groups; ++t) {
                    if (!merge_eligible<DIM>(c, w, t, split_on, ways, cell_score)) continue;
                    grp[got++] = t;
                    if (got == ways) {
                        merge_group<DIM>(c, w, grp, ways, split_on, hs2, &cnt->removed_flags);
                        got = 0;
                        ++done;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// SPH_MERGE_SIBLING: a split group (the parent and its children, linked in a
// ring by `sibling`) merges back into one particle when all its `ways`
// members are level 2 and have been interior for merge_interior_steps
// steps.  The member with the smallest particle index survives; the group
// is averaged in ring order from it, with merge_group's weights.  One thread
// per particle; only the survivor-to-be writes, so no group is merged twice.
template <int DIM>
__device__ __forceinline__ void merge_sibling_body(const sph_config &c, Counters *cnt, const CanonPtrs &st,
                                                   const WorkPtrs &w)
{
    if (cnt->merge_candidates == 0u) return;   // the energy pass found no candidate
    const uint32_t n = cnt->n;
    const uint32_t split_on = cnt->split_off ? 0u : 1u;
    const uint32_t ways = c.split_ways == 4 ? 4u : 2u;
    const float hs2 = c.kernel[1] / 2.0f;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const uint32_t si = w.inv[i];
        if (!merge_eligible<DIM>(c, w, si, split_on, ways, 0.f)) continue;
        uint32_t g[4];
        g[0] = si;
        uint32_t j = st.sibling[i];
        bool ok = true;
        for (uint32_t k = 1; k < ways && ok; ++k) {
            // a ring member of smaller index is the survivor-to-be; it merges
            ok = j < n && j > i;
            if (ok) {
                g[k] = w.inv[j];
                ok = merge_eligible<DIM>(c, w, g[k], split_on, ways, 0.f);
                j = st.sibling[j];
            }
        }
        if (ok && j == i) merge_group<DIM>(c, w, g, ways, split_on, hs2, &cnt->removed_flags);
    }
}

template <int DIM, int BS = kThreads>
__global__ void __launch_bounds__(BS) k_merge(sph_config c, Counters *__restrict__ cnt,
                                                   CanonPtrs st, WorkPtrs w, uint32_t ncells, uint32_t cap)
{
    __shared__ MergeSmem ms[BS / 32];
    if (c.merge_rule == SPH_MERGE_SIBLING) merge_sibling_body<DIM>(c, cnt, st, w);
    else merge_body<DIM>(c, cnt, st, w, ncells, cap, ms);
}

// ------------------------------------------------------------ 10. write-out
// Stable partition by status (rearrange, SPH-3D-2/sph_system.cu:1818-1840):
// [surviving particles in index order][children in split order][removed].
// Children follow adaptive_particle_kernel (:1576-1615; 3D-4 :1583-1656;
// 2D :1133-1160).  Writes the other canonical buffer.
// ranks = false: the step ran no split and removal scans (split and merge
// both off), so there are no children and nothing is removed.
// hash_next: also hash every particle it writes for the next step (hash_one
// at its new index; the cell counts were cleared after this step's scan), so
// the next step starts at the cell scan.
// Split groups: a parent and its children form a ring through `sibling`
// (parent -> child 0 -> ... -> last child -> parent); a surviving member's
// link follows the compaction; a merged survivor and everything else has none.
template <int DIM>
__device__ __forceinline__ void write_body(const sph_config &c, const Counters *cnt, Counters *cnt_next,
                                           const CanonPtrs &in, const CanonPtrs &out, const WorkPtrs &w,
                                           bool ranks = true, bool hash_next = false)
{
    const uint32_t n = cnt->n;
    const uint32_t split_on = ranks && !cnt->split_off ? 1u : 0u;
    const uint32_t ways = c.split_ways == 4 ? 4u : 2u;
    const uint32_t extra = ways - 1u;
    const uint32_t n_split = split_on ? cnt->n_split : 0u;
    const uint32_t n_removed = ranks ? cnt->n_removed : 0u;
    const uint32_t n_after = n + n_split * extra;
    const uint32_t n_live = n_after - n_removed;
    const float hs2 = c.kernel[1] / 2.0f;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cnt_next->n = n_live;
        cnt_next->error = cnt->error;
        cnt_next->n_split = 0;
        cnt_next->n_removed = 0;
        cnt_next->split_off = 0;
        cnt_next->split_flags = 0;
        cnt_next->removed_flags = 0;
        cnt_next->merge_candidates = 0;
    }
    // one thread per particle index: reads gather from the sorted slot, the
    // writes (survivors keep their order) stay coalesced
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const uint32_t s = w.inv[i];
        const uint32_t sp = split_on & w.split_c[i];
        const uint32_t rm = ranks ? w.removed_c[i] : 0u;
        const uint32_t rr = ranks ? w.removed_rank[i] : 0u;
        const uint32_t dst = rm ? n_live + rr : i - rr;
        float4 p = w.spos_n[s], v = w.svel_n[s], e = w.sev_n[s];
        uint32_t inter = (c.merge_rule == SPH_MERGE_INTERIOR || c.merge_rule == SPH_MERGE_SIBLING) ? w.sinter[s] : 0u;
        const float4 p_pre = p;
        if (sp) {
            p.x += hs2;
            p.w = 2.0f;
            inter = 0u;
        }
        float4 plo = w.pos_comp ? w.spos_lo_n[s] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 plo_pre = plo;
        uint32_t sib = kEmpty;
        if (!rm && !w.leader[s]) {
            const uint32_t j = in.sibling[i];
            if (j < n) sib = j - (ranks ? w.removed_rank[j] : 0u);
        }
        if (sp) sib = n - n_removed + w.split_rank[i] * extra;   // the first child
        const uint32_t leader = w.leader[s];
        if (leader) {
            plo = make_float4(0.f, 0.f, 0.f, 0.f);   // a merged position is a fresh FP32 mean
            p = w.mpos[s]; v = w.mvel[s]; e = w.mev[s];
            inter = 0u;
            w.leader[s] = 0u;   // reset for the next step
        }
        out.pos[dst] = p; out.vel[dst] = v; out.ev[dst] = e;
        if (w.out_src) {
            if (!rm) w.out_src[dst] = s | (sp ? kOutSplit : 0u) | (leader ? kOutLeader : 0u);
        } else {
            const float4 aux = w.saux[s];
            float en = w.senergy[s];
            if (sp && ways == 4) en = en / 4.0f;
            float4 a = w.sacc_n[s];
            if (leader) {
                a = w.macc[s];
                if (DIM == 2) en = w.menergy[s];
            }
            out.acc[dst] = a; out.dens[dst] = aux.x; out.press[dst] = aux.y; out.energy[dst] = en;
            out.surface[dst] = w.ssurf[s];
        }
        out.interior[dst] = inter;
        out.sibling[dst] = sib;
        const uint32_t sid = w.nscenes ? w.sscene[s] : 0u;   // a merge group never spans scenes
        if (w.nscenes) out.scene[dst] = sid;
        if (w.pos_comp) out.pos_lo[dst] = plo;
        if (hash_next && !rm) hash_one<DIM>(c, w, dst, p);
        if (sp) {
            const uint32_t base = n - n_removed + w.split_rank[i] * extra;
            const float4 v0 = w.svel_n[s], e0 = w.sev_n[s];
            for (uint32_t k = 0; k < extra; ++k) {
                float4 pc = p_pre;
                pc.w = 2.0f;
                if (k == 0) pc.x = p_pre.x - hs2;
                else if (k == 1) pc.z = p_pre.z - hs2;
                else pc.z = p_pre.z + hs2;
                const uint32_t cd = base + k;
                out.pos[cd] = pc; out.vel[cd] = v0; out.ev[cd] = e0;
                if (w.out_src) {
                    w.out_src[cd] = s | kOutChild;
                } else {
                    const float4 aux = w.saux[s];
                    out.acc[cd] = w.sacc_n[s]; out.dens[cd] = aux.x; out.press[cd] = aux.y;
                    out.energy[cd] = ways == 4 ? w.senergy[s] / 4.0f : w.senergy[s]; out.surface[cd] = w.ssurf[s];
                }
                out.interior[cd] = 0u;
                out.sibling[cd] = k + 1 < extra ? cd + 1 : dst;
                if (w.nscenes) out.scene[cd] = sid;
                if (w.pos_comp) out.pos_lo[cd] = plo_pre;
                if (hash_next) hash_one<DIM>(c, w, cd, pc);
            }
        }
    }
}

// The deferred outputs of the state st (count cnt->n) from the sorted arrays
// of the step that wrote it, as write_body writes them.
template <int DIM>
__global__ void __launch_bounds__(kThreads) k_materialize(sph_config c, const Counters *__restrict__ cnt,
                                                         CanonPtrs st, WorkPtrs w)
{
    const uint32_t n = cnt->n;
    const uint32_t ways = c.split_ways == 4 ? 4u : 2u;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const uint32_t code = w.out_src[i], s = code & kOutSlot;
        const float4 aux = w.saux[s];
        float en = w.senergy[s];
        float4 a = w.sacc_n[s];
        if (code & kOutChild) {
            en = ways == 4 ? en / 4.0f : en;
        } else {
            if ((code & kOutSplit) && ways == 4) en = en / 4.0f;
            if (code & kOutLeader) {
                a = w.macc[s];
                if (DIM == 2) en = w.menergy[s];
            }
        }
        st.acc[i] = a; st.dens[i] = aux.x; st.press[i] = aux.y; st.energy[i] = en; st.surface[i] = w.ssurf[s];
    }
}

template <int DIM, int BS = kThreads>
__global__ void __launch_bounds__(BS) k_write(sph_config c, const Counters *__restrict__ cnt,
                                                   Counters *__restrict__ cnt_next, CanonPtrs in, CanonPtrs out,
                                                   WorkPtrs w, int hash_next)
{
    write_body<DIM>(c, cnt, cnt_next, in, out, w, true, hash_next != 0);
}

// ------------------------------------------------------------ reference-layout records
// 3D Particle (SPH-3D-2/sph_system.h:8-24), 18 words:
//   pos3 vel3 ev3 acc3 dens press energy surface tension level(u32)
// 2D Particle (SPH-2D/sph_system.h:7-22), 14 words (56 B, 8-byte aligned):
//   pos2 vel2 ev2 acc2 dens pres energy level(u32) surface_normal pad
template <int DIM> struct AosLayout;
template <> struct AosLayout<3> { static constexpr int words = 18; };
template <> struct AosLayout<2> { static constexpr int words = 14; };

template <int DIM>
__global__ void __launch_bounds__(kThreads) k_to_aos(const Counters *__restrict__ cnt, CanonPtrs st, float *aos)
{
    const uint32_t n = cnt->n;
    constexpr int W = AosLayout<DIM>::words;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const float4 p = st.pos[i], v = st.vel[i], e = st.ev[i], a = st.acc[i];
        float *o = aos + (size_t)i * W;
        if (DIM == 3) {
            o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = v.x; o[4] = v.y; o[5] = v.z;
            o[6] = e.x; o[7] = e.y; o[8] = e.z; o[9] = a.x; o[10] = a.y; o[11] = a.z;
            o[12] = st.dens[i]; o[13] = st.press[i]; o[14] = st.energy[i]; o[15] = st.surface[i];
            o[16] = 0.0f; o[17] = __uint_as_float((uint32_t)p.w);
        } else {
            o[0] = p.x; o[1] = p.y; o[2] = v.x; o[3] = v.y; o[4] = e.x; o[5] = e.y; o[6] = a.x; o[7] = a.y;
            o[8] = st.dens[i]; o[9] = st.press[i]; o[10] = st.energy[i];
            o[11] = __uint_as_float((uint32_t)p.w); o[12] = st.surface[i]; o[13] = 0.0f;
        }
    }
}

// Same records written straight into mapped page-locked host memory (at most
// max_rec of them) plus the live count.  Each block builds 256 records in
// shared memory and then stores them as one contiguous run, a warp writing
// 128 consecutive bytes per store, so the writes cross PCIe as full lines
// (a thread storing its own record would scatter 4-byte writes 72 bytes
// apart).  dst needs 4-byte alignment only.
template <int DIM>
__global__ void __launch_bounds__(kThreads) k_to_aos_mapped(const Counters *__restrict__ cnt, CanonPtrs st,
                                                           float *dst, uint32_t max_rec, uint32_t *count_dst)
{
    constexpr int W = AosLayout<DIM>::words;
    __shared__ float stage[kThreads * W];
    const uint32_t n = cnt->n;
    const uint32_t m = min(n, max_rec);
    if (blockIdx.x == 0 && threadIdx.x == 0) *count_dst = n;
    for (uint32_t base = blockIdx.x * kThreads; base < m; base += gridDim.x * kThreads) {
        const uint32_t i = base + threadIdx.x;
        if (i < m) {
            const float4 p = st.pos[i], v = st.vel[i], e = st.ev[i], a = st.acc[i];
            float *o = stage + threadIdx.x * W;
            if (DIM == 3) {
                o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = v.x; o[4] = v.y; o[5] = v.z;
                o[6] = e.x; o[7] = e.y; o[8] = e.z; o[9] = a.x; o[10] = a.y; o[11] = a.z;
                o[12] = st.dens[i]; o[13] = st.press[i]; o[14] = st.energy[i]; o[15] = st.surface[i];
                o[16] = 0.0f; o[17] = __uint_as_float((uint32_t)p.w);
            } else {
                o[0] = p.x; o[1] = p.y; o[2] = v.x; o[3] = v.y; o[4] = e.x; o[5] = e.y; o[6] = a.x; o[7] = a.y;
                o[8] = st.dens[i]; o[9] = st.press[i]; o[10] = st.energy[i];
                o[11] = __uint_as_float((uint32_t)p.w); o[12] = st.surface[i]; o[13] = 0.0f;
            }
        }
        __syncthreads();
        const uint32_t words = min((uint32_t)kThreads, m - base) * W;
        float *out = dst + (size_t)base * W;
        for (uint32_t q = threadIdx.x; q < words; q += kThreads) out[q] = stage[q];
        __syncthreads();   // the stage is refilled next round
    }
}

template <int DIM>
__global__ void __launch_bounds__(kThreads) k_from_aos(uint32_t n, CanonPtrs st, const float *aos)
{
    constexpr int W = AosLayout<DIM>::words;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const float *o = aos + (size_t)i * W;
        if (DIM == 3) {
            st.pos[i] = make_float4(o[0], o[1], o[2], (float)__float_as_uint(o[17]));
            st.vel[i] = make_float4(o[3], o[4], o[5], 0.f);
            st.ev[i] = make_float4(o[6], o[7], o[8], 0.f);
            st.acc[i] = make_float4(o[9], o[10], o[11], 0.f);
            st.dens[i] = o[12]; st.press[i] = o[13]; st.energy[i] = o[14]; st.surface[i] = o[15];
        } else {
            st.pos[i] = make_float4(o[0], o[1], 0.f, (float)__float_as_uint(o[11]));
            st.vel[i] = make_float4(o[2], o[3], 0.f, 0.f);
            st.ev[i] = make_float4(o[4], o[5], 0.f, 0.f);
            st.acc[i] = make_float4(o[6], o[7], 0.f, 0.f);
            st.dens[i] = o[8]; st.press[i] = o[9]; st.energy[i] = o[10]; st.surface[i] = o[12];
        }
        st.interior[i] = 0u;
        st.sibling[i] = kEmpty;   // nor split groups
        st.scene[i] = 0u;    // the record format carries no scene index
        st.pos_lo[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// ------------------------------------------------------------ conserved quantities
// Per-block FP64 partial sums of mass, momentum (3), kinetic energy and
// gravitational potential energy (-m g.x) over the canonical state; a second
// single-block pass adds the partials in block order (deterministic).
constexpr int kConservedTerms = 6;

template <int DIM>
__global__ void __launch_bounds__(kThreads) k_conserved(sph_config c, const Counters *__restrict__ cnt, CanonPtrs st,
                                                        double *partial)
{
    const uint32_t n = cnt->n;
    double acc[kConservedTerms] = {0, 0, 0, 0, 0, 0};
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const float4 p = st.pos[i], v = st.vel[i];
        const double m = c.mass[lv(p.w)];
        const double vx = v.x, vy = v.y, vz = DIM == 3 ? v.z : 0.0;
        acc[0] += m;
        acc[1] += m * vx; acc[2] += m * vy; acc[3] += m * vz;
        acc[4] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        acc[5] -= m * ((double)c.gravity[0] * p.x + (double)c.gravity[1] * p.y +
                       (DIM == 3 ? (double)c.gravity[2] * p.z : 0.0));
    }
    __shared__ double red[kThreads / 32][kConservedTerms];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < kConservedTerms; ++k) {
        double x = acc[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[wid][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < kConservedTerms) {
        double x = 0.0;
        for (int q = 0; q < kThreads / 32; ++q) x += red[q][threadIdx.x];
        partial[(size_t)blockIdx.x * kConservedTerms + threadIdx.x] = x;
    }
}

// Level-2 particles of the state (sph_last_step_stats): *out += the count.
__global__ void __launch_bounds__(kThreads) k_count_level2(const Counters *__restrict__ cnt,
                                                          const float4 *__restrict__ pos, uint32_t *out)
{
    const uint32_t n = cnt->n;
    uint32_t k = 0;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) k += pos[i].w != 1.0f ? 1u : 0u;
    k = __reduce_add_sync(0xffffffffu, k);
    if ((threadIdx.x & 31) == 0 && k) atomicAdd(out, k);
}

__global__ void k_conserved_final(const double *partial, uint32_t blocks, double *out)
{
    if (threadIdx.x < kConservedTerms) {
        double x = 0.0;
        for (uint32_t b = 0; b < blocks; ++b) x += partial[(size_t)b * kConservedTerms + threadIdx.x];
        out[threadIdx.x] = x;
    }
}

// ------------------------------------------------------------ debug helpers
__global__ void k_cell_ranges(const uint32_t *__restrict__ off, uint32_t ncells, uint32_t *start, uint32_t *end)
{
    for (uint32_t q = grid_stride_start(); q < ncells; q += grid_stride()) {
        uint32_t b = off[q], e = off[q + 1];
        start[q] = e > b ? b : kEmpty;
        end[q] = e > b ? e : 0u;
    }
}

}  // namespace sph
