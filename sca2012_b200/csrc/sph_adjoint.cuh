// sph_adjoint.cuh — reverse-mode kernels of one SI step (PHYS integrator)
// with the step's topology held fixed.
//
// A forward step run in taping mode leaves its sorted-order arrays in a
// TapeStep: the cell lists, the start-of-step state, the densities and
// forces, the wall contacts, the split flags and the merge groups.  The
// backward of that step maps the adjoint of the next canonical state
// (x', v', ev') to the adjoint of this step's canonical state in four
// gathers over sorted slots, each owning its slot's outputs (no atomics but
// the per-scene parameter sums):
//   adj_write      write-out: survivors, split children (copies) and merge
//                  groups (volume-weighted means, whose weights m/rho also
//                  send an adjoint into rho)
//   adj_integrate  walls (clamped axes pass no position adjoint, velocity
//                  scaled by the damping), ev' = (ev + v)/2, x' = x + v dt,
//                  v' = v + (f/m + g) dt
//   adj_force      the pressure and viscosity pair terms; a pair's term
//                  enters f_i and, negated, f_j, so each slot sums the
//                  derivative of (fbar_i - fbar_j) . F_ij over its own
//                  variables; rho gets the adjoint of p/rho^2 and m/rho
//   adj_density    rho_i = sum_j m_j W_i(r_ij): each slot gathers the terms
//                  of its own density and of its neighbours' densities
// Neighbour pairs are re-derived from the taped FP32 positions with the
// forward's own predicates (r^2 < max(h_i^2, h_j^2), r^2 >= close_r2 for forces;
// r^2 < h_i^2 for densities; h - r > 0 for each kernel's term), so the pair
// sets are exactly the forward's.
#pragma once
#include "sph_kernels.cuh"

namespace sph {

// One recorded step (sorted-slot arrays unless marked canonical).
struct TapeStep {
    uint32_t *sidx, *inv, *skey, *cell_off;   // inv: canonical -> slot
    float4 *spos, *svel, *sev, *saux, *sacc;  // start of step; saux = (rho, p, p/rho^2, m/rho); sacc = force
    float4 *spos_n, *svel_n, *sev_n;          // after integration and walls
    uint32_t *split_c, *split_rank;           // canonical
    uint32_t *removed_c, *removed_rank;       // canonical
    uint32_t *merge_to;                       // slot -> leader slot, kEmpty if not merged
    float4 *mpos, *mvel, *mev;                // merged values at leader slots
    float *mvs;                               // summed member volume at leader slots
    uint32_t *wall;                           // bit 2d: high wall of axis d clamped, 2d+1: low wall
    uint32_t *sscene;                         // scene per slot (batched scenes)
};

struct StepCounts {
    uint32_t n, n_split, n_removed, split_on;
};

struct AdjPtrs {
    const float4 *gx_out, *gv_out, *gev_out;  // canonical, the next step's count
    float4 *gx_in, *gv_in, *gev_in;           // canonical, this step's count
    float4 *gx2, *gv2, *gev2;                 // per slot: adjoint of the post-wall state
    float4 *gxd, *gf, *gevd;                  // per slot: position adjoint so far, force adjoint, ev adjoint
    float *grho;                              // per slot
    double *param;                            // per scene: [2s] viscosity, [2s+1] gas constant
};

__device__ __forceinline__ float dot3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ void axpy3(float4 &y, float a, float4 x)
{
    y.x += a * x.x; y.y += a * x.y; y.z += a * x.z;
}
__device__ __forceinline__ float4 sub3(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, 0.f); }

// Lanes with the same scene add their values with one FP64 atomic.
__device__ __forceinline__ void add_param(double *dst, uint32_t sid, double a, double b)
{
    const unsigned act = __activemask();
    const unsigned grp = __match_any_sync(act, sid);
    const int lane = threadIdx.x & 31;
    double sa = 0.0, sb = 0.0;
    for (unsigned m = grp; m; m &= m - 1) {
        const int l = __ffs(m) - 1;
        sa += __shfl_sync(grp, a, l);
        sb += __shfl_sync(grp, b, l);
    }
    if (lane == __ffs(grp) - 1) {
        atomicAdd(dst + 2 * sid, sa);
        atomicAdd(dst + 2 * sid + 1, sb);
    }
}

// Scene constants of a slot (single scene: the config's).
__device__ __forceinline__ uint32_t scene_of(const WorkPtrs &w, const TapeStep &t, uint32_t s)
{
    return w.nscenes ? min(t.sscene[s], w.nscenes - 1u) : 0u;
}

// ---------------------------------------------------------------- write-out
template <int DIM>
__global__ void __launch_bounds__(kThreads) adj_write(sph_config c, StepCounts k, TapeStep t, AdjPtrs a)
{
    const uint32_t ways = c.split_ways == 4 ? 4u : 2u, extra = ways - 1u;
    const float hs2 = c.kernel[1] / 2.0f;
    for (uint32_t i = grid_stride_start(); i < k.n; i += grid_stride()) {
        const uint32_t s = t.inv[i];
        const uint32_t sp = k.split_on & t.split_c[i];
        const uint32_t rm = t.removed_c[i];
        const uint32_t L = t.merge_to[s];
        float4 gx = make_float4(0.f, 0.f, 0.f, 0.f), gv = gx, ge = gx;
        float gr = 0.0f;
        if (!rm && L == kEmpty) {   // own record: the value itself (+ a constant shift when split)
            const uint32_t o = i - t.removed_rank[i];
            axpy3(gx, 1.0f, a.gx_out[o]); axpy3(gv, 1.0f, a.gv_out[o]); axpy3(ge, 1.0f, a.gev_out[o]);
        }
        if (sp) {                   // children copy the pre-split values
            const uint32_t base = k.n - k.n_removed + t.split_rank[i] * extra;
            for (uint32_t q = 0; q < extra; ++q) {
                axpy3(gx, 1.0f, a.gx_out[base + q]); axpy3(gv, 1.0f, a.gv_out[base + q]);
                axpy3(ge, 1.0f, a.gev_out[base + q]);
            }
        }
        if (L != kEmpty) {          // member of a merge group led by slot L
            const uint32_t iL = t.sidx[L];
            const uint32_t o = iL - t.removed_rank[iL];
            const float rho = t.saux[s].x;
            const float V = DIM == 2 ? 1.0f : (s == L ? c.mass[0] : c.mass[1]) / rho;
            const float Vs = t.mvs[L];
            const float wgt = V / Vs;
            const float4 gxo = a.gx_out[o], gvo = a.gv_out[o], geo = a.gev_out[o];
            axpy3(gx, wgt, gxo); axpy3(gv, wgt, gvo); axpy3(ge, wgt, geo);
            if (DIM == 3) {         // d mean / d V_k = (value_k - mean) / Vs, dV/drho = -V/rho
                float4 p = t.spos_n[s];
                if (sp) p.x += hs2;
                const float d = dot3(sub3(p, t.mpos[L]), gxo) + dot3(sub3(t.svel_n[s], t.mvel[L]), gvo) +
                                dot3(sub3(t.sev_n[s], t.mev[L]), geo);
                gr = -(V / rho) / Vs * d;
            }
        }
        a.gx2[s] = gx; a.gv2[s] = gv; a.gev2[s] = ge;
        a.grho[s] = gr;
    }
}

// ---------------------------------------------------------------- integrate + walls
template <int DIM>
__global__ void __launch_bounds__(kThreads) adj_integrate(sph_config c, StepCounts k, TapeStep t, AdjPtrs a)
{
    const float dt = c.time_step, damp = c.wall_damping;
    for (uint32_t s = grid_stride_start(); s < k.n; s += grid_stride()) {
        const float mi = c.mass[lv(t.spos[s].w)];
        const float im = 1.0f / mi;
        const uint32_t flags = t.wall[s];
        const float4 gx2 = a.gx2[s], ge2 = a.gev2[s];
        float4 gv2 = a.gv2[s];
        axpy3(gv2, 0.5f, ge2);                       // ev' = (ev + v')/2
        float g2[3] = {gx2.x, gx2.y, gx2.z}, w2[3] = {gv2.x, gv2.y, gv2.z};
        float gx1[3], gv1[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const uint32_t b = d < DIM ? (flags >> (2 * d) & 3u) : 0u;   // both bits: damped twice
            gx1[d] = b ? 0.0f : g2[d];
            gv1[d] = b == 0u ? w2[d] : (b == 3u ? damp * damp * w2[d] : damp * w2[d]);
            gv1[d] += gx1[d] * dt;                   // x' = x + v' dt
        }
        if (DIM == 2) { gx1[2] = 0.f; gv1[2] = 0.f; }
        a.gv_in[t.sidx[s]] = make_float4(gv1[0], gv1[1], gv1[2], 0.f);
        a.gxd[s] = make_float4(gx1[0], gx1[1], gx1[2], 0.f);
        a.gf[s] = make_float4(gv1[0] * dt * im, gv1[1] * dt * im, gv1[2] * dt * im, 0.f);
        a.gevd[s] = make_float4(0.5f * ge2.x, 0.5f * ge2.y, 0.5f * ge2.z, 0.f);
    }
}

// ---------------------------------------------------------------- force pairs
// ---------------------------------------------------------------- candidate lists
// The neighbour candidate list of a taped step, rebuilt from the tape: the
// step's start-of-step positions and cell ranges give the same stencil walk,
// and so the same entries in the same order, as the forward density pass
// recorded (every neighbour within (1 + margin) h_max).
template <int DIM>
__global__ void __launch_bounds__(kThreads) adj_lists(sph_config c, StepCounts k, TapeStep t, WorkPtrs w)
{
    const float re2 = energy_list_r2(c);
    for (uint32_t s = grid_stride_start(); s < k.n; s += grid_stride()) {
        const float4 pi = t.spos[s];
        const uint32_t key = t.skey[s];
        uint3 q;
        q.x = key % c.ncell[0];
        q.y = (key / c.ncell[0]) % c.ncell[1];
        q.z = DIM == 3 ? key / (c.ncell[0] * c.ncell[1]) : 0u;
        uint32_t nl = 0;
        auto add = [&](uint32_t j, float4 pj) {   // j != s
            float dx, dyy, dzz;
            if (r2_of<DIM>(pj, pi, dx, dyy, dzz) < re2) {
                if (nl < kNbrListCap) w.nlist[nl_at(w, s, nl)] = j;
                ++nl;
            }
        };
        auto range = [&](uint32_t b, uint32_t e) {
            uint32_t j = b;
            for (; j + 4 <= e; j += 4) {
                const float4 p0 = t.spos[j], p1 = t.spos[j + 1], p2 = t.spos[j + 2], p3 = t.spos[j + 3];
                add(j, p0);
                add(j + 1, p1);
                add(j + 2, p2);
                add(j + 3, p3);
            }
            for (; j < e; ++j) add(j, t.spos[j]);
        };
#pragma unroll 1
        for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz)
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                uint32_t b, e;
                if (!row_range<DIM>(c, t.cell_off, q, dy, dz, b, e)) continue;
                if (dy == 0 && dz == 0) {
                    range(b, s);
                    range(s + 1u, e);
                } else {
                    range(b, e);
                }
            }
        w.ncnt[s] = nl;
    }
}

// The pairs come from the step's candidate list, filtered by the forward
// pass's test, or, when a lane's list overflowed, from the warp-lockstep
// stencil walk (warp_pairs).  Either way each lane adds its pairs in walk
// order, so the sums do not depend on the path or on which particles share
// its warp.
template <int DIM>
__global__ void __launch_bounds__(kThreads) adj_force(sph_config c, StepCounts k, TapeStep t, WorkPtrs w, AdjPtrs a)
{
    __shared__ WarpPairSmem smem[kThreads / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t n = k.n;
    for (uint32_t base = blockIdx.x * kThreads + wib * 32u; base < n; base += gridDim.x * kThreads) {
        const uint32_t s_raw = base + lane;
        const bool valid = s_raw < n;
        const uint32_t s = valid ? s_raw : n - 1u;
        const float4 pi = t.spos[s], evi = t.sev[s], ai = t.saux[s], gfi = a.gf[s];
        const int li = lv(pi.w);
        const float hi = c.kernel[li], hi2 = c.kernel2[li], mi = c.mass[li];
        const float ispk = c.kernel_h6_twice ? c.spiky[li] / c.kernel6[li] : c.spiky[li];
        const float ivis = c.kernel_h6_twice ? c.visco[li] / c.kernel6[li] : c.visco[li];
        const uint32_t sid = scene_of(w, t, s);
        const float visc = w.nscenes ? w.scene_tab[2 * sid].w : c.viscosity;
        const float gas = w.nscenes ? w.scene_tab[2 * sid + 1].w : c.gas_constant;
        const uint32_t key = t.skey[s];
        uint3 q;
        q.x = key % c.ncell[0];
        q.y = (key / c.ncell[0]) % c.ncell[1];
        q.z = DIM == 3 ? key / (c.ncell[0] * c.ncell[1]) : 0u;
        const float cut0 = fmaxf(hi2, c.kernel2[0]), cut1 = fmaxf(hi2, c.kernel2[1]);
        float4 gx = make_float4(0.f, 0.f, 0.f, 0.f), ge = gx;
        float gA = 0.f, gV = 0.f, gmu = 0.f;
        // the forward pass's pairs: j != i, r^2 < max(h_i^2, h_j^2), r^2 >= close_r2
        auto accept = [&](uint32_t j, const float4 &pj) {
            float rx, ry, rz;
            const float r2 = r2_of<DIM>(pi, pj, rx, ry, rz);
            const float cut = pj.w == 1.0f ? cut0 : cut1;
            return j != s && r2 < cut && !(r2 < c.close_r2);
        };
        auto pair = [&](uint32_t j) {
            const float4 pj = t.spos[j];
            float rx, ry, rz;
            const float r2 = r2_of<DIM>(pi, pj, rx, ry, rz);
            const int lj = lv(pj.w);
            const float r = __fsqrt_rn(r2);
            const float ikr = __fsub_rn(hi, r), jkr = __fsub_rn(c.kernel[lj], r);
            float S = 0.f, dS = 0.f, T = 0.f, dT = 0.f;
            if (ikr > 0.0f) { S += ispk * ikr * ikr; dS -= 2.0f * ispk * ikr; T += ivis * ikr; dT -= ivis; }
            if (jkr > 0.0f) {
                const float jspk = c.kernel_h6_twice ? c.spiky[lj] / c.kernel6[lj] : c.spiky[lj];
                const float jvis = c.kernel_h6_twice ? c.visco[lj] / c.kernel6[lj] : c.visco[lj];
                S += jspk * jkr * jkr; dS -= 2.0f * jspk * jkr; T += jvis * jkr; dT -= jvis;
            }
            const float4 aj = t.saux[j], evj = t.sev[j], gfj = a.gf[j];
            const float mm = mi * c.mass[lj];
            const float Cp = mm * (ai.z + aj.z) * 0.5f;
            const float ir = rsqrtf(r2);   // 1/r as the forward pass takes it
            const float tp = Cp * S * ir, dtp = Cp * (dS - S * ir) * ir;
            const float VV = ai.w * aj.w;
            const float tv = VV * visc * 0.5f * T, dtv = VV * visc * 0.5f * dT;
            const float4 D = sub3(gfi, gfj);
            const float4 rv = make_float4(rx, ry, rz, 0.f);
            const float4 dv = sub3(evj, evi);
            const float Dr = dot3(D, rv), Ddv = dot3(D, dv);
            const float coef = (Ddv * dtv - Dr * dtp) * ir;
            axpy3(gx, -tp, D);
            axpy3(gx, coef, rv);
            axpy3(ge, -tv, D);
            gA -= Dr * mm * 0.5f * S * ir;
            gV += Ddv * aj.w * visc * 0.5f * T;
            gmu += 0.25f * Ddv * VV * T;     // each unordered pair is visited from both ends
        };
        const unsigned full = 0xffffffffu;
        const uint32_t nf = valid && w.nlist ? w.ncnt[s] : 0u;
        if (__all_sync(full, w.nlist != nullptr && nf <= kNbrListCap)) {
            const uint32_t m = __reduce_max_sync(full, nf);
            if (4 < m) prefetch_l2(w.nlist + nl_at(w, s, 4));
            for (uint32_t kk = 0; kk < m; kk += 4) {
                if (kk + 8 < m) prefetch_l2(w.nlist + nl_at(w, s, kk + 8));   // two rounds ahead
                const uint4 t4 = *reinterpret_cast<const uint4 *>(w.nlist + nl_at(w, s, kk));
                const uint32_t tt[4] = {kk < nf ? t4.x : s, kk + 1 < nf ? t4.y : s, kk + 2 < nf ? t4.z : s,
                                        kk + 3 < nf ? t4.w : s};
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (kk + u < nf && accept(tt[u], t.spos[tt[u]])) pair(tt[u]);
            }
        } else {
            warp_pairs<DIM>(c, t.cell_off, t.spos, valid, q, smem[wib], accept, pair);
        }
        if (!valid) continue;
        // p = gas ((rho/rho0)^3 - 1); A = p / rho^2; V = m / rho
        const float rho = ai.x, p = ai.y;
        const float rr = rho / c.rest_density;
        const float dp = 3.0f * gas * rr * rr / c.rest_density;
        const float irho = 1.0f / rho;
        const float dA = (dp - 2.0f * p * irho) * irho * irho;
        const float dV = -mi * irho * irho;
        a.grho[s] += gA * dA + gV * dV;
        const float4 gxd = a.gxd[s], ged = a.gevd[s];
        a.gxd[s] = make_float4(gxd.x + gx.x, gxd.y + gx.y, gxd.z + gx.z, 0.f);
        a.gevd[s] = make_float4(ged.x + ge.x, ged.y + ge.y, ged.z + ge.z, 0.f);
        add_param(a.param, sid, (double)gmu, (double)(gA * (rr * rr * rr - 1.0f) * irho * irho));
    }
}

// ---------------------------------------------------------------- density pairs
template <int DIM>
__global__ void __launch_bounds__(kThreads) adj_density(sph_config c, StepCounts k, TapeStep t, WorkPtrs w,
                                                        AdjPtrs a)
{
    const float skip = c.density_skip_r2;
    for (uint32_t s = grid_stride_start(); s < k.n; s += grid_stride()) {
        const float4 pi = t.spos[s];
        const int li = lv(pi.w);
        const float h2 = c.kernel2[li], w6 = c.poly6[li], mi = c.mass[li];
        const float gri = a.grho[s];
        const uint32_t key = t.skey[s];
        uint3 q;
        q.x = key % c.ncell[0];
        q.y = (key / c.ncell[0]) % c.ncell[1];
        q.z = DIM == 3 ? key / (c.ncell[0] * c.ncell[1]) : 0u;
        float4 gx = a.gxd[s];
        auto visit = [&](uint32_t j, float4 pj) {   // j != s
            float dx, dy_, dz_;
            const float r2 = r2_of<DIM>(pj, pi, dx, dy_, dz_);   // d = x_j - x_i
            if (r2 < skip) return;
            const int lj = lv(pj.w);
            float acc = 0.0f;
            if (r2 < h2) {          // term of rho_i
                const float x = h2 - r2;
                acc += gri * c.mass[lj] * w6 * x * x;
            }
            const float hj2 = c.kernel2[lj];
            if (r2 < hj2) {         // term of rho_j
                const float x = hj2 - r2;
                acc += a.grho[j] * mi * c.poly6[lj] * x * x;
            }
            // d/dx_i (h^2 - r^2)^3 = -6 (h^2 - r^2)^2 (x_i - x_j) = +6 (...)^2 d
            gx.x += 6.0f * acc * dx; gx.y += 6.0f * acc * dy_; gx.z += 6.0f * acc * dz_;
        };
        // slot order, four candidates' loads in flight; the own row around s
        auto range = [&](uint32_t b, uint32_t e) {
            uint32_t j = b;
            for (; j + 4 <= e; j += 4) {
                const float4 p0 = t.spos[j], p1 = t.spos[j + 1], p2 = t.spos[j + 2], p3 = t.spos[j + 3];
                visit(j, p0);
                visit(j + 1, p1);
                visit(j + 2, p2);
                visit(j + 3, p3);
            }
            for (; j < e; ++j) visit(j, t.spos[j]);
        };
        // the step's candidate list holds every pair with a term (r^2 below
        // h_i^2 or h_j^2), in walk order; an overflowed list walks
        const uint32_t nl = w.nlist ? w.ncnt[s] : kEmpty;
        if (nl <= kNbrListCap) {
            uint32_t kk = 0;
            for (; kk + 4 <= nl; kk += 4) {
                const uint4 t4 = *reinterpret_cast<const uint4 *>(w.nlist + nl_at(w, s, kk));
                const float4 p0 = t.spos[t4.x], p1 = t.spos[t4.y], p2 = t.spos[t4.z], p3 = t.spos[t4.w];
                visit(t4.x, p0);
                visit(t4.y, p1);
                visit(t4.z, p2);
                visit(t4.w, p3);
            }
            for (; kk < nl; ++kk) {
                const uint32_t j = w.nlist[nl_at(w, s, kk)];
                visit(j, t.spos[j]);
            }
        } else {
#pragma unroll 1
            for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz)
#pragma unroll 1
                for (int dy = -1; dy <= 1; ++dy) {
                    uint32_t b, e;
                    if (!row_range<DIM>(c, t.cell_off, q, dy, dz, b, e)) continue;
                    if (dy == 0 && dz == 0) {
                        range(b, s);
                        range(s + 1u, e);
                    } else {
                        range(b, e);
                    }
                }
        }
        const uint32_t i = t.sidx[s];
        a.gx_in[i] = make_float4(gx.x, gx.y, DIM == 3 ? gx.z : 0.f, 0.f);
        a.gev_in[i] = a.gevd[s];
    }
}

// ---------------------------------------------------------------- density-grid loss
struct LossGrid {
    uint32_t n[3];
    float origin[3];
    float spacing;
};

__device__ __forceinline__ float4 node_pos(const LossGrid &g, uint32_t a, uint32_t b, uint32_t cc)
{
    return make_float4(g.origin[0] + (float)a * g.spacing, g.origin[1] + (float)b * g.spacing,
                       g.origin[2] + (float)cc * g.spacing, 0.f);
}

// G_g = sum_i m_i W_i(|x_g - x_i|) over the sorted state (cell lists fresh),
// residual G - target, and sum of squared residuals (FP64).
template <int DIM>
__global__ void __launch_bounds__(kThreads) k_loss_grid(sph_config c, WorkPtrs w, LossGrid g, const float *target,
                                                        float *grid, float *resid)
{
    const uint32_t N = g.n[0] * g.n[1] * (DIM == 3 ? g.n[2] : 1u);
    for (uint32_t id = grid_stride_start(); id < N; id += grid_stride()) {
        const uint32_t a0 = id % g.n[0], a1 = (id / g.n[0]) % g.n[1], a2 = DIM == 3 ? id / (g.n[0] * g.n[1]) : 0u;
        const float4 x = node_pos(g, a0, a1, a2);
        const uint3 q = cell_of<DIM>(c, x);
        float G = 0.0f;
#pragma unroll 1
        for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz)
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                uint32_t b, e;
                if (!row_range<DIM>(c, w.cell_off, q, dy, dz, b, e)) continue;
                for (uint32_t j = b; j < e; ++j) {
                    const float4 pj = w.spos[j];
                    float dx, dy_, dz_;
                    const float r2 = r2_of<DIM>(pj, x, dx, dy_, dz_);
                    const int lj = lv(pj.w);
                    const float h2 = c.kernel2[lj];
                    if (r2 < h2) {
                        const float u = h2 - r2;
                        G += c.mass[lj] * c.poly6[lj] * u * u * u;
                    }
                }
            }
        grid[id] = G;
        resid[id] = G - target[id];
    }
}

// The loss's FP64 sum of squares of the residuals x[0, n), the same bits on
// every run: each block sums its grid-stride share and tree-reduces it in a
// fixed order into part[block]; k_sum_blocks adds the partials in block order.
// (Atomic adds would sum in arrival order, which varies between runs.)
constexpr uint32_t kLossPartials = 4096;

__global__ void __launch_bounds__(kThreads) k_sumsq_blocks(const float *__restrict__ x, uint32_t n, double *part)
{
    __shared__ double sh[kThreads];
    double acc = 0.0;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const double v = (double)x[i];
        acc += v * v;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t off = kThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_blocks(const double *__restrict__ part, uint32_t nb, double *out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double t = 0.0;
    for (uint32_t b = 0; b < nb; ++b) t += part[b];
    *out = t;
}

// Adjoint of mean((G - target)^2) with respect to the canonical positions.
template <int DIM>
__global__ void __launch_bounds__(kThreads) k_loss_grad(sph_config c, const Counters *__restrict__ cnt, CanonPtrs st,
                                                        LossGrid g, const float *resid, float scale, float4 *gx)
{
    const uint32_t n = cnt->n;
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const float4 p = st.pos[i];
        const int li = lv(p.w);
        const float h = c.kernel[li], h2 = c.kernel2[li], mw = c.mass[li] * c.poly6[li];
        int lo[3], hi[3];
        const float pc[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d >= DIM) { lo[d] = 0; hi[d] = 0; continue; }
            lo[d] = max(0, (int)floorf((pc[d] - h - g.origin[d]) / g.spacing) - 1);
            hi[d] = min((int)g.n[d] - 1, (int)floorf((pc[d] + h - g.origin[d]) / g.spacing) + 1);
        }
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int a2 = lo[2]; a2 <= hi[2]; ++a2)
            for (int a1 = lo[1]; a1 <= hi[1]; ++a1)
                for (int a0 = lo[0]; a0 <= hi[0]; ++a0) {
                    const float4 x = node_pos(g, (uint32_t)a0, (uint32_t)a1, (uint32_t)a2);
                    float dx, dy, dz;
                    const float r2 = r2_of<DIM>(p, x, dx, dy, dz);   // d = x_i - x_g
                    if (!(r2 < h2)) continue;
                    const float u = h2 - r2;
                    const uint32_t id = (uint32_t)a0 + g.n[0] * ((uint32_t)a1 + g.n[1] * (uint32_t)a2);
                    const float f = scale * resid[id] * mw * -6.0f * u * u;
                    acc.x += f * dx; acc.y += f * dy; acc.z += f * dz;
                }
        if (DIM == 2) acc.z = 0.f;
        gx[i] = acc;
    }
}

// ---------------------------------------------------------------- topology export
// Density and force neighbour lists of one taped step in canonical indices
// (for the FP64 host replay); force entries carry bit 30 (i-kernel term
// active) and bit 31 (j-kernel term active).
template <int DIM, bool FILL>
__global__ void __launch_bounds__(kThreads) k_topo_pairs(sph_config c, StepCounts k, TapeStep t, uint32_t *dcount,
                                                         uint32_t *fcount, const uint32_t *doff, const uint32_t *foff,
                                                         uint32_t *dnbr, uint32_t *fnbr)
{
    const float skip = c.density_skip_r2;
    for (uint32_t s = grid_stride_start(); s < k.n; s += grid_stride()) {
        const float4 pi = t.spos[s];
        const int li = lv(pi.w);
        const float hi = c.kernel[li], hi2 = c.kernel2[li];
        const float cut0 = fmaxf(hi2, c.kernel2[0]), cut1 = fmaxf(hi2, c.kernel2[1]);
        const uint32_t key = t.skey[s];
        uint3 q;
        q.x = key % c.ncell[0];
        q.y = (key / c.ncell[0]) % c.ncell[1];
        q.z = DIM == 3 ? key / (c.ncell[0] * c.ncell[1]) : 0u;
        const uint32_t i = t.sidx[s];
        uint32_t nd = 0, nf = 0;
        const uint32_t d0 = FILL ? doff[i] : 0u, f0 = FILL ? foff[i] : 0u;
        for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy) {
                uint32_t b, e;
                if (!row_range<DIM>(c, t.cell_off, q, dy, dz, b, e)) continue;
                for (uint32_t j = b; j < e; ++j) {
                    if (j == s) continue;
                    const float4 pj = t.spos[j];
                    float dx, dy_, dz_;
                    const float r2d = r2_of<DIM>(pj, pi, dx, dy_, dz_);
                    if (!(r2d < skip) && r2d < hi2) {
                        if (FILL) dnbr[d0 + nd] = t.sidx[j];
                        ++nd;
                    }
                    const float r2 = r2_of<DIM>(pi, pj, dx, dy_, dz_);
                    const float cut = pj.w == 1.0f ? cut0 : cut1;
                    if (r2 < cut && !(r2 < c.close_r2)) {
                        if (FILL) {
                            const float r = __fsqrt_rn(r2);
                            const uint32_t fi = __fsub_rn(hi, r) > 0.0f ? 1u << 30 : 0u;
                            const uint32_t fj = __fsub_rn(c.kernel[lv(pj.w)], r) > 0.0f ? 1u << 31 : 0u;
                            fnbr[f0 + nf] = t.sidx[j] | fi | fj;
                        }
                        ++nf;
                    }
                }
            }
        if (!FILL) { dcount[i] = nd; fcount[i] = nf; }
    }
}

}  // namespace sph
