// sph_rollout_impl.cuh — differentiable rollout on a handle: checkpoints,
// taped replay of a checkpoint interval, the adjoint sweep, the density-grid
// loss and the topology export.  Included at the end of sph_api.cu, whose
// handle, launch helpers and run_step it uses.
//
// Memory: checkpoints hold the full canonical state (what split and merge
// decisions read too: energy, interior counters), so a replay from one is
// bit-identical to the forward; the tape holds one interval's sorted-order
// arrays (about 220 bytes per particle of capacity per step).
#include "sph_adjoint.cuh"

struct Rollout {
    uint32_t cap = 0, ncells = 0, tape_slots = 0;
    std::vector<CanonPtrs> ckpt;       // k: state at step k * every; back(): final state
    std::vector<uint32_t> ckpt_n;
    uint32_t nsteps = 0, every = 0;
    uint64_t gen = 0, end_step = 0;
    bool valid = false;
    std::vector<TapeStep> tape;
    std::vector<StepCounts> counts;    // of the taped interval
    StepCounts *dcounts = nullptr;     // the same, written on the device as each step is taped
    int taped_seg = -1;
    float4 *gx[2] = {}, *gv[2] = {}, *gev[2] = {};
    float4 *gx2 = nullptr, *gv2 = nullptr, *gev2 = nullptr, *gxd = nullptr, *gf = nullptr, *gevd = nullptr;
    float *grho = nullptr;
    double *param = nullptr;
    uint32_t param_cap = 0;
    LossGrid grid{};
    uint32_t nodes = 0, node_cap = 0;
    float *target = nullptr, *gridv = nullptr, *resid = nullptr;
    double *lsum = nullptr;
    bool have_loss = false;
    uint64_t loss_gen = 0, loss_step = 0;
    uint32_t *tcount[2] = {}, *toff[2] = {}, *tnbr[2] = {};
    uint64_t tnbr_cap[2] = {0, 0};
    std::vector<void *> allocs;
};

namespace {

template <typename T> int ralloc(sph_handle *h, Rollout *r, T **p, size_t count)
{
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        h->err = "rollout: out of device memory";
        return SPH_ERR_CUDA;
    }
    r->allocs.push_back(q);
    *p = (T *)q;
    return SPH_OK;
}

void rollout_free(Rollout *r)
{
    if (!r) return;
    for (void *p : r->allocs) cudaFree(p);
    delete r;
}

int alloc_canon(sph_handle *h, Rollout *r, CanonPtrs &q)
{
    const size_t n = r->cap;
    int rc = ralloc(h, r, &q.pos, n);
    rc |= ralloc(h, r, &q.vel, n); rc |= ralloc(h, r, &q.ev, n); rc |= ralloc(h, r, &q.acc, n);
    rc |= ralloc(h, r, &q.dens, n); rc |= ralloc(h, r, &q.press, n); rc |= ralloc(h, r, &q.energy, n);
    rc |= ralloc(h, r, &q.surface, n); rc |= ralloc(h, r, &q.interior, n); rc |= ralloc(h, r, &q.scene, n);
    rc |= ralloc(h, r, &q.pos_lo, n); rc |= ralloc(h, r, &q.sibling, n);
    return rc ? SPH_ERR_CUDA : SPH_OK;
}

int alloc_tape(sph_handle *h, Rollout *r, TapeStep &t)
{
    const size_t n = r->cap;
    int rc = ralloc(h, r, &t.sidx, n);
    rc |= ralloc(h, r, &t.inv, n); rc |= ralloc(h, r, &t.skey, n); rc |= ralloc(h, r, &t.cell_off, r->ncells + 1);
    rc |= ralloc(h, r, &t.spos, n); rc |= ralloc(h, r, &t.svel, n); rc |= ralloc(h, r, &t.sev, n);
    rc |= ralloc(h, r, &t.saux, n); rc |= ralloc(h, r, &t.sacc, n);
    rc |= ralloc(h, r, &t.spos_n, n); rc |= ralloc(h, r, &t.svel_n, n); rc |= ralloc(h, r, &t.sev_n, n);
    rc |= ralloc(h, r, &t.split_c, n); rc |= ralloc(h, r, &t.split_rank, n);
    rc |= ralloc(h, r, &t.removed_c, n); rc |= ralloc(h, r, &t.removed_rank, n);
    rc |= ralloc(h, r, &t.merge_to, n);
    rc |= ralloc(h, r, &t.mpos, n); rc |= ralloc(h, r, &t.mvel, n); rc |= ralloc(h, r, &t.mev, n);
    rc |= ralloc(h, r, &t.mvs, n); rc |= ralloc(h, r, &t.wall, n); rc |= ralloc(h, r, &t.sscene, n);
    return rc ? SPH_ERR_CUDA : SPH_OK;
}

template <typename T> void d2d(T *dst, const T *src, size_t count, cudaStream_t s)
{
    if (count) cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToDevice, s);
}

void copy_canon(const CanonPtrs &dst, const CanonPtrs &src, uint32_t n, cudaStream_t s)
{
    d2d(dst.pos, src.pos, n, s); d2d(dst.vel, src.vel, n, s); d2d(dst.ev, src.ev, n, s);
    d2d(dst.acc, src.acc, n, s); d2d(dst.dens, src.dens, n, s); d2d(dst.press, src.press, n, s);
    d2d(dst.energy, src.energy, n, s); d2d(dst.surface, src.surface, n, s);
    d2d(dst.interior, src.interior, n, s); d2d(dst.scene, src.scene, n, s);
    d2d(dst.pos_lo, src.pos_lo, n, s); d2d(dst.sibling, src.sibling, n, s);
}

// Makes checkpoint k the handle's current state (all counters reset).
int restore_ckpt(sph_handle *h, Rollout *r, size_t k)
{
    const uint32_t n = r->ckpt_n[k];
    copy_canon(h->buf[h->cur], r->ckpt[k], n, h->stream);
    Counters c0;
    std::memset(&c0, 0, sizeof(c0));
    c0.n = n;
    cudaMemcpyAsync(&h->cnt[h->cur], &c0, sizeof(Counters), cudaMemcpyHostToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
    h->n_ub = n;
    h->counts_hashed = false;   // the hash a persistent step left is not this state's
    h->outputs_pending = false;
    return cuda_check(h, "rollout: restore checkpoint");
}

int save_ckpt(sph_handle *h, Rollout *r, size_t k)
{
    ensure_outputs(h);
    const uint32_t n = read_n(h);
    copy_canon(r->ckpt[k], h->buf[h->cur], n, h->stream);
    r->ckpt_n[k] = n;
    return cuda_check(h, "rollout: save checkpoint");
}

const char *rollout_unsupported(const sph_config &c)
{
    if (c.integrator != SPH_INTEGRATE_PHYS) return "the adjoint covers SPH_INTEGRATE_PHYS only";
    if (c.surface_coef != 0.0f) return "the adjoint does not cover surface tension (surface_coef != 0)";
    if (c.use_cylinder || c.extern_force_on || c.push_left || c.push_right)
        return "the adjoint does not cover obstacles or interactive forces";
    return nullptr;
}

// One forward step with its topology written into tape slot l.
// Copies a finished step's sorted-order arrays into tape slot t and its
// counters into *counts, over the live count the device holds (no host
// round trip per step).
__global__ void __launch_bounds__(kThreads) k_tape_record(const Counters *__restrict__ cnt, WorkPtrs w, TapeStep t,
                                                        uint32_t ncells, StepCounts *counts)
{
    const uint32_t n = cnt->n;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *counts = StepCounts{cnt->n, cnt->n_split, cnt->n_removed, cnt->split_off ? 0u : 1u};
    for (uint32_t s = grid_stride_start(); s < n; s += grid_stride()) {
        t.sidx[s] = w.sidx[s]; t.inv[s] = w.inv[s]; t.skey[s] = w.skey[s];
        t.spos[s] = w.spos[s]; t.svel[s] = w.svel[s]; t.sev[s] = w.sev[s];
        t.saux[s] = w.saux[s]; t.sacc[s] = w.sacc_n[s];
        t.spos_n[s] = w.spos_n[s]; t.svel_n[s] = w.svel_n[s]; t.sev_n[s] = w.sev_n[s];
        t.split_c[s] = w.split_c[s]; t.split_rank[s] = w.split_rank[s];
        t.removed_c[s] = w.removed_c[s]; t.removed_rank[s] = w.removed_rank[s];
        t.mpos[s] = w.mpos[s]; t.mvel[s] = w.mvel[s]; t.mev[s] = w.mev[s];
        if (w.nscenes) t.sscene[s] = w.sscene[s];
    }
    for (uint32_t k = grid_stride_start(); k <= ncells; k += grid_stride()) t.cell_off[k] = w.cell_off[k];
}

template <int DIM> int taped_step(sph_handle *h, Rollout *r, uint32_t l)
{
    TapeStep &t = r->tape[l];
    cudaStream_t s = h->stream;
    // merge leaders fill merge_to; n_ub bounds the live count
    cudaMemsetAsync(t.merge_to, 0xff, sizeof(uint32_t) * (h->n_ub ? h->n_ub : 1), s);
    const WorkPtrs saved = h->w;
    h->w.merge_to = t.merge_to;
    h->w.mvs = t.mvs;
    h->w.wall = t.wall;
    const int p = h->cur;
    const uint32_t nub = h->n_ub;
    const int rc = run_step<DIM>(h);
    h->w = saved;
    if (rc) return rc;
    k_tape_record<<<grid_for(h, std::max(nub, h->ncells + 1)), kThreads, 0, s>>>(h->cnt + p, h->w, t, h->ncells,
                                                                                r->dcounts + l);
    return cuda_check(h, "rollout: taped step");
}

uint32_t seg_len(const Rollout *r, uint32_t seg)
{
    return std::min(r->every, r->nsteps - seg * r->every);
}

// Replays checkpoint interval `seg` with every step taped.
template <int DIM> int tape_segment(sph_handle *h, Rollout *r, uint32_t seg)
{
    if (r->taped_seg == (int)seg) return SPH_OK;
    r->taped_seg = -1;
    if (int rc = restore_ckpt(h, r, seg)) return rc;
    const uint32_t len = seg_len(r, seg);
    for (uint32_t l = 0; l < len; ++l)
        if (int rc = taped_step<DIM>(h, r, l)) return rc;
    // the interval's step counters, read once
    cudaMemcpyAsync(r->counts.data(), r->dcounts, sizeof(StepCounts) * len, cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    if (int rc = cuda_check(h, "rollout: taped interval")) return rc;
    r->taped_seg = (int)seg;
    return SPH_OK;
}

// Leaves the handle as the forward left it.
int restore_final(sph_handle *h, Rollout *r)
{
    int rc = restore_ckpt(h, r, r->ckpt.size() - 1);
    h->step_index = r->end_step;
    h->have_step = false;
    return rc;
}

// Hash, counting sort and reorder of the current state (the first stages of
// a step), so the sorted arrays and cell lists describe it.
template <int DIM> void sort_only(sph_handle *h)
{
    const sph_config &c = h->cfg;
    Counters *cin = h->cnt + h->cur;
    const CanonPtrs in = h->buf[h->cur];
    h->w.pos_comp = c.compensated_positions ? 1u : 0u;
    const WorkPtrs w = h->w;
    const uint32_t G = grid_for(h, h->n_ub);
    cudaStream_t s = h->stream;
    cudaMemsetAsync(w.cell_count, 0, sizeof(uint32_t) * h->ncells, s);
    h->counts_zero = false;
    h->counts_hashed = false;
    k_hash<DIM><<<G, kThreads, 0, s>>>(c, cin, in, w);
    scan_u32(h, w.cell_count, w.cell_off, nullptr, h->ncells, h->scan_grand, 1, nullptr);
    k_scatter<<<G, kThreads, 0, s>>>(cin, w);
    k_reorder<<<G, kThreads, 0, s>>>(cin, in, w);
}

bool rollout_current(const sph_handle *h, const Rollout *r)
{
    return r && r->valid && r->gen == h->state_gen && r->end_step == h->step_index;
}

template <int DIM> int backward_impl(sph_handle *h, Rollout *r, float *d_vel0, float *d_pos0, double *d_params,
                                     uint32_t nparams)
{
    const sph_config &c = h->cfg;
    cudaStream_t s = h->stream;
    const uint32_t nscn = std::max(1u, h->w.nscenes);
    if (d_params && nparams < 2 * nscn) { h->err = "sph_rollout_backward: d_params too short"; return SPH_ERR_INVALID; }
    if (int rc = restore_final(h, r)) return rc;
    // seed: adjoint of the loss with respect to the final positions
    const uint32_t nT = r->ckpt_n.back();
    int p = 0;
    k_loss_grad<DIM><<<grid_for(h, nT), kThreads, 0, s>>>(c, h->cnt + h->cur, h->buf[h->cur], r->grid, r->resid,
                                                         2.0f / (float)r->nodes, r->gx[p]);
    cudaMemsetAsync(r->gv[p], 0, sizeof(float4) * (nT ? nT : 1), s);
    cudaMemsetAsync(r->gev[p], 0, sizeof(float4) * (nT ? nT : 1), s);
    cudaMemsetAsync(r->param, 0, sizeof(double) * 2 * nscn, s);
    const uint32_t nseg = (r->nsteps + r->every - 1) / r->every;
    WorkPtrs w = h->w;
    if (c.walk_only) {   // the same pairs found by the stencil walks
        w.nlist = w.ncnt = nullptr;
    }
    for (uint32_t seg = nseg; seg-- > 0;) {
        if (int rc = tape_segment<DIM>(h, r, seg)) return rc;
        for (uint32_t l = seg_len(r, seg); l-- > 0;) {
            const StepCounts k = r->counts[l];
            AdjPtrs a;
            a.gx_out = r->gx[p]; a.gv_out = r->gv[p]; a.gev_out = r->gev[p];
            a.gx_in = r->gx[p ^ 1]; a.gv_in = r->gv[p ^ 1]; a.gev_in = r->gev[p ^ 1];
            a.gx2 = r->gx2; a.gv2 = r->gv2; a.gev2 = r->gev2;
            a.gxd = r->gxd; a.gf = r->gf; a.gevd = r->gevd;
            a.grho = r->grho;
            a.param = r->param;
            const uint32_t G = grid_for(h, k.n);
            adj_write<DIM><<<G, kThreads, 0, s>>>(c, k, r->tape[l], a);
            adj_integrate<DIM><<<G, kThreads, 0, s>>>(c, k, r->tape[l], a);
            // the step's candidate lists, rebuilt from its tape (the working
            // lists are free during the backward pass)
            if (w.nlist) adj_lists<DIM><<<G, kThreads, 0, s>>>(c, k, r->tape[l], w);
            adj_force<DIM><<<G, kThreads, 0, s>>>(c, k, r->tape[l], w, a);
            adj_density<DIM><<<G, kThreads, 0, s>>>(c, k, r->tape[l], w, a);
            p ^= 1;
        }
    }
    if (int rc = cuda_check(h, "sph_rollout_backward launch")) return rc;
    const uint32_t n0 = r->ckpt_n[0];
    const int dim = (int)c.dim;
    std::vector<float4> t(n0);
    if (d_vel0) {
        cudaMemcpyAsync(t.data(), r->gv[p], sizeof(float4) * n0, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        unpack4(t, dim, n0, d_vel0);
    }
    if (d_pos0) {
        cudaMemcpyAsync(t.data(), r->gx[p], sizeof(float4) * n0, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        unpack4(t, dim, n0, d_pos0);
    }
    if (d_params) {
        cudaMemcpyAsync(d_params, r->param, sizeof(double) * 2 * nscn, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
    }
    int rc = cuda_check(h, "sph_rollout_backward");
    int rc2 = restore_final(h, r);
    return rc ? rc : rc2;
}

template <int DIM> int topology_impl(sph_handle *h, Rollout *r, uint32_t step, sph_topology_view *v)
{
    const uint32_t seg = step / r->every, l = step % r->every;
    if (int rc = tape_segment<DIM>(h, r, seg)) return rc;
    const StepCounts k = r->counts[l];
    const TapeStep &t = r->tape[l];
    const sph_config &c = h->cfg;
    cudaStream_t s = h->stream;
    const uint32_t n = k.n;
    const uint32_t extra = c.split_ways == 4 ? 3u : 1u;
    v->n = n;
    v->n_split = k.n_split;
    v->n_removed = k.n_removed;
    v->split_on = k.split_on;
    v->n_next = n + (k.split_on ? k.n_split * extra : 0u) - k.n_removed;
    const uint32_t G = grid_for(h, n);
    k_topo_pairs<DIM, false><<<G, kThreads, 0, s>>>(c, k, t, r->tcount[0], r->tcount[1], nullptr, nullptr, nullptr,
                                                     nullptr);
    for (int q = 0; q < 2; ++q)
        scan_u32(h, r->tcount[q], r->toff[q], nullptr, n, h->scan_grand, 1, nullptr);
    uint32_t tot[2];
    for (int q = 0; q < 2; ++q)
        cudaMemcpyAsync(&tot[q], r->toff[q] + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    v->n_dens_pairs = tot[0];
    v->n_force_pairs = tot[1];
    const bool fill_d = v->dens_nbr && v->dens_cap >= tot[0];
    const bool fill_f = v->force_nbr && v->force_cap >= tot[1];
    if (fill_d || fill_f) {
        for (int q = 0; q < 2; ++q)
            if (r->tnbr_cap[q] < tot[q]) {
                if (r->tnbr[q]) cudaFree(r->tnbr[q]);
                r->tnbr[q] = nullptr;
                r->tnbr_cap[q] = 0;
                if (cudaMalloc(&r->tnbr[q], sizeof(uint32_t) * tot[q]) != cudaSuccess) {
                    cudaGetLastError();
                    h->err = "sph_rollout_topology: out of device memory";
                    return SPH_ERR_CUDA;
                }
                r->tnbr_cap[q] = tot[q];
            }
        k_topo_pairs<DIM, true><<<G, kThreads, 0, s>>>(c, k, t, nullptr, nullptr, r->toff[0], r->toff[1],
                                                        r->tnbr[0], r->tnbr[1]);
        if (fill_d) cudaMemcpyAsync(v->dens_nbr, r->tnbr[0], sizeof(uint32_t) * tot[0], cudaMemcpyDeviceToHost, s);
        if (fill_f) cudaMemcpyAsync(v->force_nbr, r->tnbr[1], sizeof(uint32_t) * tot[1], cudaMemcpyDeviceToHost, s);
    }
    if (v->dens_off) cudaMemcpyAsync(v->dens_off, r->toff[0], sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost, s);
    if (v->force_off) cudaMemcpyAsync(v->force_off, r->toff[1], sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost, s);
    std::vector<uint32_t> inv(n), sidx(n), wall(n), split_c(n), removed_c(n), removed_rank(n), split_rank(n), mt(n);
    std::vector<float4> spos(n), svel, sev;
    auto get = [&](void *dst, const void *src, size_t bytes) {
        if (bytes) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    };
    get(inv.data(), t.inv, 4ull * n); get(sidx.data(), t.sidx, 4ull * n); get(wall.data(), t.wall, 4ull * n);
    get(split_c.data(), t.split_c, 4ull * n); get(removed_c.data(), t.removed_c, 4ull * n);
    get(removed_rank.data(), t.removed_rank, 4ull * n); get(split_rank.data(), t.split_rank, 4ull * n);
    get(mt.data(), t.merge_to, 4ull * n); get(spos.data(), t.spos, 16ull * n);
    if (v->vel) { svel.resize(n); get(svel.data(), t.svel, 16ull * n); }
    if (v->ev) { sev.resize(n); get(sev.data(), t.sev, 16ull * n); }
    cudaStreamSynchronize(s);
    const int dim = (int)c.dim;
    auto put = [&](float *dst, const std::vector<float4> &src) {
        if (!dst) return;
        for (uint32_t i = 0; i < n; ++i) {
            const float4 q = src[inv[i]];
            dst[(size_t)i * dim] = q.x;
            dst[(size_t)i * dim + 1] = q.y;
            if (dim == 3) dst[(size_t)i * dim + 2] = q.z;
        }
    };
    put(v->pos, spos);
    put(v->vel, svel);
    put(v->ev, sev);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t sl = inv[i];
        if (v->level) v->level[i] = (uint32_t)spos[sl].w;
        if (v->wall) v->wall[i] = wall[sl];
        if (v->split) v->split[i] = k.split_on & split_c[i];
        if (v->dst) v->dst[i] = removed_c[i] ? kEmpty : i - removed_rank[i];
        if (v->child) v->child[i] = n - k.n_removed + split_rank[i] * extra;
        if (v->merge_leader) v->merge_leader[i] = mt[sl] == kEmpty ? kEmpty : sidx[mt[sl]];
    }
    int rc = cuda_check(h, "sph_rollout_topology");
    int rc2 = restore_final(h, r);
    return rc ? rc : rc2;
}

}  // namespace

int sph_rollout_forward(sph_handle *h, uint32_t nsteps, uint32_t every)
{
    if (!h) return SPH_ERR_INVALID;
    if (nsteps == 0 || every == 0) { h->err = "sph_rollout_forward: nsteps and checkpoint_every must be > 0"; return SPH_ERR_INVALID; }
    if (const char *why = rollout_unsupported(h->cfg)) { h->err = why; return SPH_ERR_INVALID; }
    sph_readback_wait(h);
    Rollout *r = h->ro;
    const uint32_t nck = (nsteps + every - 1) / every + 1;
    const uint32_t slots = std::min(every, nsteps);
    if (r && (r->ckpt.size() < nck || r->tape_slots < slots)) {
        rollout_free(r);
        r = h->ro = nullptr;
    }
    if (!r) {
        r = h->ro = new Rollout();
        r->cap = h->cap;
        r->ncells = h->ncells;
        r->ckpt.resize(nck);
        int rc = SPH_OK;
        for (auto &q : r->ckpt) rc |= alloc_canon(h, r, q);
        r->tape.resize(slots);
        r->tape_slots = slots;
        for (auto &t : r->tape) rc |= alloc_tape(h, r, t);
        rc |= ralloc(h, r, &r->dcounts, slots);
        for (int q = 0; q < 2; ++q) {
            rc |= ralloc(h, r, &r->gx[q], r->cap); rc |= ralloc(h, r, &r->gv[q], r->cap);
            rc |= ralloc(h, r, &r->gev[q], r->cap);
            rc |= ralloc(h, r, &r->tcount[q], r->cap); rc |= ralloc(h, r, &r->toff[q], (size_t)r->cap + 1);
        }
        rc |= ralloc(h, r, &r->gx2, r->cap); rc |= ralloc(h, r, &r->gv2, r->cap); rc |= ralloc(h, r, &r->gev2, r->cap);
        rc |= ralloc(h, r, &r->gxd, r->cap); rc |= ralloc(h, r, &r->gf, r->cap); rc |= ralloc(h, r, &r->gevd, r->cap);
        rc |= ralloc(h, r, &r->grho, r->cap);
        rc |= ralloc(h, r, &r->lsum, 2 + kLossPartials);
        if (rc) {
            rollout_free(r);
            h->ro = nullptr;
            return SPH_ERR_CUDA;
        }
    }
    r->ckpt.resize(nck);
    r->ckpt_n.assign(nck, 0);
    r->counts.assign(r->tape_slots, StepCounts{0, 0, 0, 0});
    r->valid = false;
    r->have_loss = false;
    r->taped_seg = -1;
    r->nsteps = nsteps;
    r->every = every;
    const uint32_t nseg = nck - 1;
    for (uint32_t seg = 0; seg < nseg; ++seg) {
        if (int rc = save_ckpt(h, r, seg)) return rc;
        if (int rc = sph_step(h, (int)seg_len(r, seg))) return rc;
    }
    if (int rc = save_ckpt(h, r, nseg)) return rc;
    if (int rc = sph_sync(h)) return rc;
    r->gen = h->state_gen;
    r->end_step = h->step_index;
    r->valid = true;
    return SPH_OK;
}

int sph_splat_loss(sph_handle *h, const sph_loss_grid *g, const float *target, float *grid_out, double *loss)
{
    if (!h || !g || !target || !loss) return SPH_ERR_INVALID;
    const uint32_t dim = h->cfg.dim;
    if (!g->n[0] || !g->n[1] || (dim == 3 && !g->n[2]) || !(g->spacing > 0.0f)) {
        h->err = "sph_splat_loss: empty grid or non-positive spacing";
        return SPH_ERR_INVALID;
    }
    const uint64_t N = (uint64_t)g->n[0] * g->n[1] * (dim == 3 ? g->n[2] : 1u);
    if (N >= (1ull << 31)) { h->err = "sph_splat_loss: grid too large"; return SPH_ERR_INVALID; }
    sph_readback_wait(h);
    if (!h->ro) {   // a loss without a rollout: only the buffers it needs
        Rollout *r = h->ro = new Rollout();
        r->cap = h->cap;
        r->ncells = h->ncells;
        if (ralloc(h, r, &r->lsum, 2 + kLossPartials)) { rollout_free(r); h->ro = nullptr; return SPH_ERR_CUDA; }
    }
    Rollout *r = h->ro;
    if (N > r->node_cap) {
        int rc = ralloc(h, r, &r->target, N);
        rc |= ralloc(h, r, &r->gridv, N);
        rc |= ralloc(h, r, &r->resid, N);
        if (rc) return SPH_ERR_CUDA;
        r->node_cap = (uint32_t)N;
    }
    r->nodes = (uint32_t)N;
    for (int d = 0; d < 3; ++d) {
        r->grid.n[d] = d < (int)dim ? g->n[d] : 1u;
        r->grid.origin[d] = d < (int)dim ? g->origin[d] : 0.0f;
    }
    r->grid.spacing = g->spacing;
    cudaStream_t s = h->stream;
    cudaMemcpyAsync(r->target, target, sizeof(float) * N, cudaMemcpyHostToDevice, s);
    const uint32_t G = grid_for(h, (uint32_t)N);
    if (dim == 3) {
        sort_only<3>(h);
        k_loss_grid<3><<<G, kThreads, 0, s>>>(h->cfg, h->w, r->grid, r->target, r->gridv, r->resid);
    } else {
        sort_only<2>(h);
        k_loss_grid<2><<<G, kThreads, 0, s>>>(h->cfg, h->w, r->grid, r->target, r->gridv, r->resid);
    }
    const uint32_t GL = std::min<uint32_t>(G, kLossPartials);
    k_sumsq_blocks<<<GL, kThreads, 0, s>>>(r->resid, (uint32_t)N, r->lsum + 2);
    k_sum_blocks<<<1, 1, 0, s>>>(r->lsum + 2, GL, r->lsum);
    double sum = 0.0;
    cudaMemcpyAsync(&sum, r->lsum, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (grid_out) cudaMemcpyAsync(grid_out, r->gridv, sizeof(float) * N, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    *loss = sum / (double)N;
    h->have_step = false;   // the sorted arrays now describe this state
    r->have_loss = true;
    r->loss_gen = h->state_gen;
    r->loss_step = h->step_index;
    return cuda_check(h, "sph_splat_loss");
}

int sph_rollout_backward(sph_handle *h, float *d_vel0, float *d_pos0, double *d_params, uint32_t nparams)
{
    if (!h) return SPH_ERR_INVALID;
    Rollout *r = h->ro;
    if (!rollout_current(h, r)) { h->err = "sph_rollout_backward: no rollout ends at the current state"; return SPH_ERR_INVALID; }
    if (!r->have_loss || r->loss_gen != h->state_gen || r->loss_step != h->step_index) {
        h->err = "sph_rollout_backward: call sph_splat_loss on the rollout's final state first";
        return SPH_ERR_INVALID;
    }
    if (const char *why = rollout_unsupported(h->cfg)) { h->err = why; return SPH_ERR_INVALID; }
    const uint32_t nscn = std::max(1u, h->w.nscenes);
    if (r->param_cap < 2 * nscn) {
        if (ralloc(h, r, &r->param, 2 * nscn)) return SPH_ERR_CUDA;
        r->param_cap = 2 * nscn;
    }
    sph_readback_wait(h);
    return h->cfg.dim == 3 ? backward_impl<3>(h, r, d_vel0, d_pos0, d_params, nparams)
                           : backward_impl<2>(h, r, d_vel0, d_pos0, d_params, nparams);
}

int sph_rollout_topology(sph_handle *h, uint32_t step, sph_topology_view *v)
{
    if (!h || !v) return SPH_ERR_INVALID;
    Rollout *r = h->ro;
    if (!rollout_current(h, r)) { h->err = "sph_rollout_topology: no rollout ends at the current state"; return SPH_ERR_INVALID; }
    if (step >= r->nsteps) { h->err = "sph_rollout_topology: step out of range"; return SPH_ERR_RANGE; }
    sph_readback_wait(h);
    return h->cfg.dim == 3 ? topology_impl<3>(h, r, step, v) : topology_impl<2>(h, r, step, v);
}
