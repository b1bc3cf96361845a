/*
 * sph_rollout_ref.c — FP64 host replay of a recorded rollout and its adjoint.
 * TEST INFRASTRUCTURE: the checker of the GPU adjoint (tests/ only).
 *
 * The GPU forward of each step records its topology (sph_rollout_topology):
 * density and force neighbour lists, which kernel terms are active per force
 * pair, wall contacts, splits and merge groups.  This file replays the SI
 * step (SPH_INTEGRATE_PHYS, no surface tension) with that topology held
 * fixed, entirely in FP64:
 *   rho_i = sum_{j in D(i)} m_j W6_i (h_i^2 - r^2)^3 + m_i W6_i h_i^6
 *   p_i   = k ((rho_i / rho0)^3 - 1),  A_i = p_i / rho_i^2,  V_i = m_i / rho_i
 *   f_i   = sum_{j in F(i)} -r_ij m_i m_j (A_i + A_j) S_ij / (2 r)
 *                          + (ev_j - ev_i) V_i V_j mu T_ij / 2
 *           S = [h_i>r] spk_i (h_i - r)^2 + [h_j>r] spk_j (h_j - r)^2,
 *           T = [h_i>r] vis_i (h_i - r)   + [h_j>r] vis_j (h_j - r)
 *   v' = v + (f/m + g) dt,  x' = x + v' dt,  clamped axes: x' = wall,
 *   v' *= damping,  ev' = (ev + v')/2
 * (the equations of SPH-3D-2/sph_system.cu:338-677 density, :679-1137
 * force, with SI constants and the PHYS integrator), then the write-out:
 * survivors, split children at -hs2 offsets (parent +hs2), merge groups as
 * volume-weighted means (3D; plain means in 2D).  The loss splats the final
 * state onto the node grid, G_g = sum_i m_i W6_i (h_i^2 - r^2)^3 over
 * r^2 < h_i^2, and returns mean (G - target)^2.
 *
 * ref_rollout_grad runs the same forward keeping every step, then the
 * adjoint in scatter form over the directed pair lists (each f_i term
 * differentiated on its own), an independent formulation of the GPU's
 * gather kernels.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/sph/sph.h"

#define EMPTY 0xffffffffu
#define IDX_MASK 0x3fffffffu

typedef struct ref_topo {
    uint32_t n, n_next, split_on;
    const uint32_t *level, *dens_off, *dens_nbr, *force_off, *force_nbr, *wall, *split, *dst, *child, *merge_leader;
    const float *x_rec, *v_rec, *ev_rec;   /* optional: the recorded FP32 state the step started from */
} ref_topo;

typedef struct {
    uint32_t n;
    double *x, *v, *ev;          /* 3 per particle (z = 0 in 2D) */
    /* intermediates of the step that starts from this state */
    double *rho, *p, *A, *V, *f, *x2, *v2, *ev2;
} step_rec;

static int lvi(uint32_t level) { return level == 1u ? 0 : 1; }

static double spk_of(const sph_config *c, int l)
{
    return c->kernel_h6_twice ? (double)c->spiky[l] / (double)c->kernel6[l] : (double)c->spiky[l];
}
static double vis_of(const sph_config *c, int l)
{
    return c->kernel_h6_twice ? (double)c->visco[l] / (double)c->kernel6[l] : (double)c->visco[l];
}

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

static void rec_alloc(step_rec *s, uint32_t n, int full)
{
    s->n = n;
    s->x = dalloc(3 * (size_t)n); s->v = dalloc(3 * (size_t)n); s->ev = dalloc(3 * (size_t)n);
    if (full) {
        s->rho = dalloc(n); s->p = dalloc(n); s->A = dalloc(n); s->V = dalloc(n);
        s->f = dalloc(3 * (size_t)n); s->x2 = dalloc(3 * (size_t)n); s->v2 = dalloc(3 * (size_t)n);
        s->ev2 = dalloc(3 * (size_t)n);
    } else {
        s->rho = s->p = s->A = s->V = s->f = s->x2 = s->v2 = s->ev2 = NULL;
    }
}

static void rec_free(step_rec *s)
{
    free(s->x); free(s->v); free(s->ev);
    free(s->rho); free(s->p); free(s->A); free(s->V); free(s->f); free(s->x2); free(s->v2); free(s->ev2);
}

/* One step from s (intermediates into s) to the next state nx. */
static void step_forward(const sph_config *c, const ref_topo *t, step_rec *s, step_rec *nx, double mu, double kgas)
{
    const uint32_t n = t->n;
    const int dim = (int)c->dim;
    const double rho0 = c->rest_density, dt = c->time_step, damp = c->wall_damping;
    #pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < n; ++i) {
        const int li = lvi(t->level[i]);
        const double h2 = (double)c->kernel2[li], w6 = c->poly6[li];
        double rho = (double)c->mass[li] * w6 * (double)c->kernel6[li];
        for (uint32_t q = t->dens_off[i]; q < t->dens_off[i + 1]; ++q) {
            const uint32_t j = t->dens_nbr[q];
            double r2 = 0.0;
            for (int d = 0; d < 3; ++d) { const double e = s->x[3 * j + d] - s->x[3 * i + d]; r2 += e * e; }
            const double u = h2 - r2;
            rho += (double)c->mass[lvi(t->level[j])] * w6 * u * u * u;
        }
        const double rr = rho / rho0;
        const double p = kgas * (rr * rr * rr - 1.0);
        s->rho[i] = rho; s->p[i] = p; s->A[i] = p / (rho * rho); s->V[i] = (double)c->mass[li] / rho;
    }
    #pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < n; ++i) {
        const int li = lvi(t->level[i]);
        const double hi = c->kernel[li], mi = c->mass[li];
        double f[3] = {0, 0, 0};
        for (uint32_t q = t->force_off[i]; q < t->force_off[i + 1]; ++q) {
            const uint32_t e = t->force_nbr[q], j = e & IDX_MASK;
            const int lj = lvi(t->level[j]);
            double rv[3], r2 = 0.0;
            for (int d = 0; d < 3; ++d) { rv[d] = s->x[3 * i + d] - s->x[3 * j + d]; r2 += rv[d] * rv[d]; }
            const double r = sqrt(r2), hj = c->kernel[lj];
            double S = 0.0, T = 0.0;
            if (e >> 30 & 1u) { S += spk_of(c, li) * (hi - r) * (hi - r); T += vis_of(c, li) * (hi - r); }
            if (e >> 31 & 1u) { S += spk_of(c, lj) * (hj - r) * (hj - r); T += vis_of(c, lj) * (hj - r); }
            const double tp = mi * (double)c->mass[lj] * (s->A[i] + s->A[j]) * 0.5 * S / r;
            const double tv = s->V[i] * s->V[j] * mu * 0.5 * T;
            for (int d = 0; d < 3; ++d) f[d] += -rv[d] * tp + (s->ev[3 * j + d] - s->ev[3 * i + d]) * tv;
        }
        const double rad = c->radius[li];
        for (int d = 0; d < 3; ++d) {
            s->f[3 * i + d] = f[d];
            double v1 = s->v[3 * i + d], x1 = s->x[3 * i + d];
            if (d < dim) {
                v1 += (f[d] / mi + (double)c->gravity[d]) * dt;
                x1 += v1 * dt;
                const uint32_t b = t->wall[i] >> (2 * d) & 3u;
                if (b & 1u) { v1 *= damp; x1 = (double)c->world[d] - rad; }
                if (b & 2u) { v1 *= damp; x1 = rad; }
            } else {
                v1 = 0.0; x1 = 0.0;
            }
            s->x2[3 * i + d] = x1;
            s->v2[3 * i + d] = v1;
            s->ev2[3 * i + d] = d < dim ? 0.5 * (s->ev[3 * i + d] + v1) : 0.0;
        }
    }
    /* write-out */
    const uint32_t ways = c->split_ways == 4 ? 4u : 2u, extra = ways - 1u;
    const double hs2 = (double)c->kernel[1] / 2.0;
    double *Vs = dalloc(n), *acc = dalloc(9 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t sp = t->split[i];
        double xs[3] = {s->x2[3 * i], s->x2[3 * i + 1], s->x2[3 * i + 2]};
        if (sp) xs[0] += hs2;
        const uint32_t L = t->merge_leader[i];
        if (L != EMPTY) {
            const double V = dim == 2 ? 1.0 : (i == L ? (double)c->mass[0] : (double)c->mass[1]) / s->rho[i];
            Vs[L] += V;
            for (int d = 0; d < 3; ++d) {
                acc[9 * L + d] += V * xs[d];
                acc[9 * L + 3 + d] += V * s->v2[3 * i + d];
                acc[9 * L + 6 + d] += V * s->ev2[3 * i + d];
            }
        } else if (t->dst[i] != EMPTY) {
            const uint32_t o = t->dst[i];
            for (int d = 0; d < 3; ++d) {
                nx->x[3 * o + d] = xs[d]; nx->v[3 * o + d] = s->v2[3 * i + d]; nx->ev[3 * o + d] = s->ev2[3 * i + d];
            }
        }
        if (sp)
            for (uint32_t k = 0; k < extra; ++k) {
                const uint32_t o = t->child[i] + k;
                double pc[3] = {s->x2[3 * i], s->x2[3 * i + 1], s->x2[3 * i + 2]};
                if (k == 0) pc[0] -= hs2;
                else if (k == 1) pc[2] -= hs2;
                else pc[2] += hs2;
                for (int d = 0; d < 3; ++d) {
                    nx->x[3 * o + d] = pc[d]; nx->v[3 * o + d] = s->v2[3 * i + d]; nx->ev[3 * o + d] = s->ev2[3 * i + d];
                }
            }
    }
    for (uint32_t L = 0; L < n; ++L)
        if (Vs[L] > 0.0) {
            const uint32_t o = t->dst[L];
            for (int d = 0; d < 3; ++d) {
                nx->x[3 * o + d] = acc[9 * L + d] / Vs[L];
                nx->v[3 * o + d] = acc[9 * L + 3 + d] / Vs[L];
                nx->ev[3 * o + d] = acc[9 * L + 6 + d] / Vs[L];
            }
        }
    free(Vs);
    free(acc);
}

/* Node range of particle x on axis d that can lie within h. */
static void node_range(const sph_loss_grid *g, double x, double h, int d, int *lo, int *hi)
{
    int a = (int)floor((x - h - g->origin[d]) / g->spacing) - 1;
    int b = (int)floor((x + h - g->origin[d]) / g->spacing) + 1;
    *lo = a < 0 ? 0 : a;
    *hi = b > (int)g->n[d] - 1 ? (int)g->n[d] - 1 : b;
}

static double loss_of(const sph_config *c, const step_rec *s, const uint32_t *level, const sph_loss_grid *g,
                      const double *target, double *grid, double *resid)
{
    const int dim = (int)c->dim;
    const size_t N = (size_t)g->n[0] * g->n[1] * (dim == 3 ? g->n[2] : 1u);
    memset(grid, 0, N * sizeof(double));
    for (uint32_t i = 0; i < s->n; ++i) {
        const int li = lvi(level[i]);
        const double h = c->kernel[li], h2 = c->kernel2[li], mw = (double)c->mass[li] * c->poly6[li];
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) node_range(g, s->x[3 * i + d], h, d, &lo[d], &hi[d]);
        for (int a2 = lo[2]; a2 <= hi[2]; ++a2)
            for (int a1 = lo[1]; a1 <= hi[1]; ++a1)
                for (int a0 = lo[0]; a0 <= hi[0]; ++a0) {
                    const int ax[3] = {a0, a1, a2};
                    double r2 = 0.0;
                    for (int d = 0; d < dim; ++d) {
                        const double e = s->x[3 * i + d] - (g->origin[d] + ax[d] * (double)g->spacing);
                        r2 += e * e;
                    }
                    if (!(r2 < h2)) continue;
                    const double u = h2 - r2;
                    grid[a0 + (size_t)g->n[0] * (a1 + (size_t)g->n[1] * a2)] += mw * u * u * u;
                }
    }
    double L = 0.0;
    for (size_t q = 0; q < N; ++q) {
        const double R = grid[q] - target[q];
        if (resid) resid[q] = R;
        L += R * R;
    }
    return L / (double)N;
}

static void init_state(const sph_config *c, step_rec *s, uint32_t n0, const double *x0, const double *v0)
{
    const int dim = (int)c->dim;
    for (uint32_t i = 0; i < n0; ++i)
        for (int d = 0; d < dim; ++d) {
            s->x[3 * i + d] = x0[(size_t)i * dim + d];
            s->v[3 * i + d] = v0[(size_t)i * dim + d];
        }
}

/* Levels of the state after the last step (needed by the loss). */
static void final_levels(const sph_config *c, const ref_topo *t, uint32_t *lf)
{
    const uint32_t extra = c->split_ways == 4 ? 3u : 1u;
    for (uint32_t i = 0; i < t->n; ++i) {
        if (t->dst[i] != EMPTY) lf[t->dst[i]] = t->merge_leader[i] == i ? 1u : (t->split[i] ? 2u : t->level[i]);
        if (t->split[i])
            for (uint32_t k = 0; k < extra; ++k) lf[t->child[i] + k] = 2u;
    }
}

double ref_rollout_forward(const sph_config *c, const ref_topo *steps, uint32_t T, uint32_t n0, const double *x0,
                           const double *v0, double mu, double kgas, const sph_loss_grid *g, const double *target,
                           double *grid_out)
{
    step_rec cur, nx;
    rec_alloc(&cur, n0, 1);
    init_state(c, &cur, n0, x0, v0);
    for (uint32_t t = 0; t < T; ++t) {
        rec_alloc(&nx, steps[t].n_next, 1);
        step_forward(c, &steps[t], &cur, &nx, mu, kgas);
        rec_free(&cur);
        cur = nx;
    }
    const size_t N = (size_t)g->n[0] * g->n[1] * (c->dim == 3 ? g->n[2] : 1u);
    double *grid = grid_out ? grid_out : dalloc(N);
    uint32_t *lf = (uint32_t *)calloc(cur.n ? cur.n : 1, sizeof(uint32_t));
    if (T) final_levels(c, &steps[T - 1], lf);
    const double L = loss_of(c, &cur, lf, g, target, grid, NULL);
    if (!grid_out) free(grid);
    free(lf);
    rec_free(&cur);
    return L;
}

/* Overwrites a state with recorded FP32 values (dim per particle). */
static void load_rec(const sph_config *c, step_rec *s, const float *x, const float *v, const float *ev)
{
    const int dim = (int)c->dim;
    for (uint32_t i = 0; i < s->n; ++i)
        for (int d = 0; d < dim; ++d) {
            if (x) s->x[3 * i + d] = x[(size_t)i * dim + d];
            if (v) s->v[3 * i + d] = v[(size_t)i * dim + d];
            if (ev) s->ev[3 * i + d] = ev[(size_t)i * dim + d];
        }
}

/* follow != 0: every step starts from its recorded FP32 state (x_rec, ...)
 * and the loss is taken at x_final, so the FP64 adjoint is linearised about
 * the GPU's own trajectory. */
static double grad_impl(const sph_config *c, const ref_topo *steps, uint32_t T, uint32_t n0, const double *x0,
                        const double *v0, double mu, double kgas, const sph_loss_grid *g, const double *target,
                        double *g_x0, double *g_v0, double *g_mu, double *g_k, int follow, const float *x_final)
{
    if (T == 0) return 0.0;
    const int dim = (int)c->dim;
    step_rec *rec = (step_rec *)calloc(T + 1, sizeof(step_rec));
    rec_alloc(&rec[0], n0, 1);
    init_state(c, &rec[0], n0, x0, v0);
    for (uint32_t t = 0; t < T; ++t) {
        if (follow) load_rec(c, &rec[t], steps[t].x_rec, steps[t].v_rec, steps[t].ev_rec);
        rec_alloc(&rec[t + 1], steps[t].n_next, t + 1 < T);
        step_forward(c, &steps[t], &rec[t], &rec[t + 1], mu, kgas);
    }
    if (follow && x_final) load_rec(c, &rec[T], x_final, NULL, NULL);
    const size_t N = (size_t)g->n[0] * g->n[1] * (dim == 3 ? g->n[2] : 1u);
    double *grid = dalloc(N), *resid = dalloc(N);
    uint32_t *lf = (uint32_t *)calloc(rec[T].n ? rec[T].n : 1, sizeof(uint32_t));
    final_levels(c, &steps[T - 1], lf);
    const double L = loss_of(c, &rec[T], lf, g, target, grid, resid);
    /* seed: dL/dx_T */
    const uint32_t nT = rec[T].n;
    double *gx = dalloc(3 * (size_t)nT), *gv = dalloc(3 * (size_t)nT), *gev = dalloc(3 * (size_t)nT);
    for (uint32_t i = 0; i < nT; ++i) {
        const int li = lvi(lf[i]);
        const double h = c->kernel[li], h2 = c->kernel2[li], mw = (double)c->mass[li] * c->poly6[li];
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) node_range(g, rec[T].x[3 * i + d], h, d, &lo[d], &hi[d]);
        for (int a2 = lo[2]; a2 <= hi[2]; ++a2)
            for (int a1 = lo[1]; a1 <= hi[1]; ++a1)
                for (int a0 = lo[0]; a0 <= hi[0]; ++a0) {
                    const int ax[3] = {a0, a1, a2};
                    double e[3] = {0, 0, 0}, r2 = 0.0;
                    for (int d = 0; d < dim; ++d) {
                        e[d] = rec[T].x[3 * i + d] - (g->origin[d] + ax[d] * (double)g->spacing);
                        r2 += e[d] * e[d];
                    }
                    if (!(r2 < h2)) continue;
                    const double u = h2 - r2;
                    const double R = resid[a0 + (size_t)g->n[0] * (a1 + (size_t)g->n[1] * a2)];
                    const double f = 2.0 * R / (double)N * mw * -6.0 * u * u;
                    for (int d = 0; d < dim; ++d) gx[3 * i + d] += f * e[d];
                }
    }
    free(lf);
    double gmu = 0.0, gk = 0.0;
    const double dt = c->time_step, damp = c->wall_damping, rho0 = c->rest_density;
    const uint32_t ways = c->split_ways == 4 ? 4u : 2u, extra = ways - 1u;
    const double hs2 = (double)c->kernel[1] / 2.0;
    for (uint32_t t = T; t-- > 0;) {
        const ref_topo *tp = &steps[t];
        step_rec *s = &rec[t];
        const uint32_t n = tp->n;
        double *gx2 = dalloc(3 * (size_t)n), *gv2 = dalloc(3 * (size_t)n), *ge2 = dalloc(3 * (size_t)n);
        double *grho = dalloc(n), *gA = dalloc(n), *gV = dalloc(n);
        double *gxi = dalloc(3 * (size_t)n), *gvi = dalloc(3 * (size_t)n), *gei = dalloc(3 * (size_t)n);
        double *gf = dalloc(3 * (size_t)n);
        /* merge groups: sums and means */
        double *Vs = dalloc(n);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t Lk = tp->merge_leader[i];
            if (Lk == EMPTY) continue;
            Vs[Lk] += dim == 2 ? 1.0 : (i == Lk ? (double)c->mass[0] : (double)c->mass[1]) / s->rho[i];
        }
        /* write-out adjoint */
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t sp = tp->split[i];
            const uint32_t Lk = tp->merge_leader[i];
            if (Lk == EMPTY && tp->dst[i] != EMPTY) {
                const uint32_t o = tp->dst[i];
                for (int d = 0; d < 3; ++d) {
                    gx2[3 * i + d] += gx[3 * o + d]; gv2[3 * i + d] += gv[3 * o + d]; ge2[3 * i + d] += gev[3 * o + d];
                }
            }
            if (sp)
                for (uint32_t k = 0; k < extra; ++k) {
                    const uint32_t o = tp->child[i] + k;
                    for (int d = 0; d < 3; ++d) {
                        gx2[3 * i + d] += gx[3 * o + d]; gv2[3 * i + d] += gv[3 * o + d];
                        ge2[3 * i + d] += gev[3 * o + d];
                    }
                }
            if (Lk != EMPTY) {
                const uint32_t o = tp->dst[Lk];
                const double V = dim == 2 ? 1.0 : (i == Lk ? (double)c->mass[0] : (double)c->mass[1]) / s->rho[i];
                const double w = V / Vs[Lk];
                for (int d = 0; d < 3; ++d) {
                    gx2[3 * i + d] += w * gx[3 * o + d]; gv2[3 * i + d] += w * gv[3 * o + d];
                    ge2[3 * i + d] += w * gev[3 * o + d];
                }
                if (dim == 3) {
                    /* mean of the group = next state's record o */
                    const step_rec *nx = &rec[t + 1];
                    double dsum = 0.0;
                    for (int d = 0; d < 3; ++d) {
                        const double xs = s->x2[3 * i + d] + (sp && d == 0 ? hs2 : 0.0);
                        dsum += (xs - nx->x[3 * o + d]) * gx[3 * o + d] +
                                (s->v2[3 * i + d] - nx->v[3 * o + d]) * gv[3 * o + d] +
                                (s->ev2[3 * i + d] - nx->ev[3 * o + d]) * gev[3 * o + d];
                    }
                    grho[i] += -(V / s->rho[i]) / Vs[Lk] * dsum;
                }
            }
        }
        free(Vs);
        /* integrate + walls adjoint */
        for (uint32_t i = 0; i < n; ++i) {
            const double mi = c->mass[lvi(tp->level[i])];
            for (int d = 0; d < dim; ++d) {
                double gvv = gv2[3 * i + d] + 0.5 * ge2[3 * i + d];
                gei[3 * i + d] = 0.5 * ge2[3 * i + d];
                const uint32_t b = tp->wall[i] >> (2 * d) & 3u;
                double gx1 = b ? 0.0 : gx2[3 * i + d];
                double gv1 = b == 0 ? gvv : (b == 3 ? damp * damp * gvv : damp * gvv);
                gv1 += gx1 * dt;
                gxi[3 * i + d] = gx1;
                gvi[3 * i + d] = gv1;
                gf[3 * i + d] = gv1 * dt / mi;
            }
        }
        /* force adjoint, one directed pair term at a time */
        for (uint32_t i = 0; i < n; ++i) {
            const int li = lvi(tp->level[i]);
            const double hi = c->kernel[li], mi = c->mass[li];
            for (uint32_t q = tp->force_off[i]; q < tp->force_off[i + 1]; ++q) {
                const uint32_t e = tp->force_nbr[q], j = e & IDX_MASK;
                const int lj = lvi(tp->level[j]);
                double rv[3], dv[3], r2 = 0.0;
                for (int d = 0; d < 3; ++d) {
                    rv[d] = s->x[3 * i + d] - s->x[3 * j + d];
                    dv[d] = s->ev[3 * j + d] - s->ev[3 * i + d];
                    r2 += rv[d] * rv[d];
                }
                const double r = sqrt(r2), hj = c->kernel[lj];
                double S = 0, dS = 0, Tt = 0, dT = 0;
                if (e >> 30 & 1u) {
                    const double a = hi - r;
                    S += spk_of(c, li) * a * a; dS -= 2.0 * spk_of(c, li) * a; Tt += vis_of(c, li) * a; dT -= vis_of(c, li);
                }
                if (e >> 31 & 1u) {
                    const double a = hj - r;
                    S += spk_of(c, lj) * a * a; dS -= 2.0 * spk_of(c, lj) * a; Tt += vis_of(c, lj) * a; dT -= vis_of(c, lj);
                }
                const double mm = mi * (double)c->mass[lj];
                const double Cp = mm * (s->A[i] + s->A[j]) * 0.5;
                const double tpv = Cp * S / r, dtp = Cp * (dS / r - S / (r * r));
                const double VV = s->V[i] * s->V[j];
                const double tv = VV * mu * 0.5 * Tt, dtv = VV * mu * 0.5 * dT;
                const double *fb = &gf[3 * i];
                double Fr = 0.0, Fdv = 0.0;
                for (int d = 0; d < 3; ++d) { Fr += fb[d] * rv[d]; Fdv += fb[d] * dv[d]; }
                const double coef = (Fdv * dtv - Fr * dtp) / r;
                for (int d = 0; d < 3; ++d) {
                    const double gxd = -fb[d] * tpv + coef * rv[d];
                    gxi[3 * i + d] += gxd;
                    gxi[3 * j + d] -= gxd;
                    gei[3 * i + d] -= fb[d] * tv;
                    gei[3 * j + d] += fb[d] * tv;
                }
                const double dA = -Fr * mm * 0.5 * S / r;
                gA[i] += dA;
                gA[j] += dA;
                gV[i] += Fdv * s->V[j] * mu * 0.5 * Tt;
                gV[j] += Fdv * s->V[i] * mu * 0.5 * Tt;
                gmu += Fdv * VV * 0.5 * Tt;
            }
        }
        for (uint32_t i = 0; i < n; ++i) {
            const double mi = c->mass[lvi(tp->level[i])];
            const double rho = s->rho[i], p = s->p[i], rr = rho / rho0;
            const double dp = 3.0 * kgas * rr * rr / rho0;
            grho[i] += gA[i] * (dp / (rho * rho) - 2.0 * p / (rho * rho * rho)) + gV[i] * (-mi / (rho * rho));
            gk += gA[i] * (rr * rr * rr - 1.0) / (rho * rho);
        }
        /* density adjoint */
        for (uint32_t i = 0; i < n; ++i) {
            const int li = lvi(tp->level[i]);
            const double h2 = c->kernel2[li], w6 = c->poly6[li];
            for (uint32_t q = tp->dens_off[i]; q < tp->dens_off[i + 1]; ++q) {
                const uint32_t j = tp->dens_nbr[q];
                double e[3], r2 = 0.0;
                for (int d = 0; d < 3; ++d) { e[d] = s->x[3 * i + d] - s->x[3 * j + d]; r2 += e[d] * e[d]; }
                const double u = h2 - r2;
                const double f = grho[i] * (double)c->mass[lvi(tp->level[j])] * w6 * -6.0 * u * u;
                for (int d = 0; d < 3; ++d) {
                    gxi[3 * i + d] += f * e[d];
                    gxi[3 * j + d] -= f * e[d];
                }
            }
        }
        free(gx); free(gv); free(gev);
        gx = gxi; gv = gvi; gev = gei;
        free(gx2); free(gv2); free(ge2); free(grho); free(gA); free(gV); free(gf);
    }
    for (uint32_t i = 0; i < n0; ++i)
        for (int d = 0; d < dim; ++d) {
            if (g_x0) g_x0[(size_t)i * dim + d] = gx[3 * i + d];
            if (g_v0) g_v0[(size_t)i * dim + d] = gv[3 * i + d];
        }
    if (g_mu) *g_mu = gmu;
    if (g_k) *g_k = gk;
    free(gx); free(gv); free(gev);
    free(grid); free(resid);
    for (uint32_t t = 0; t <= T; ++t) rec_free(&rec[t]);
    free(rec);
    return L;
}

double ref_rollout_grad(const sph_config *c, const ref_topo *steps, uint32_t T, uint32_t n0, const double *x0,
                        const double *v0, double mu, double kgas, const sph_loss_grid *g, const double *target,
                        double *g_x0, double *g_v0, double *g_mu, double *g_k)
{
    return grad_impl(c, steps, T, n0, x0, v0, mu, kgas, g, target, g_x0, g_v0, g_mu, g_k, 0, NULL);
}

double ref_rollout_grad_along(const sph_config *c, const ref_topo *steps, uint32_t T, uint32_t n0, const double *x0,
                              const double *v0, double mu, double kgas, const sph_loss_grid *g, const double *target,
                              const float *x_final, double *g_x0, double *g_v0, double *g_mu, double *g_k)
{
    return grad_impl(c, steps, T, n0, x0, v0, mu, kgas, g, target, g_x0, g_v0, g_mu, g_k, 1, x_final);
}
