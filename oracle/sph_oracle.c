/*
 * sph_oracle.c — CPU oracle for the adaptive SPH step.  TEST INFRASTRUCTURE
 * (see sph_oracle.h): it is the checker for the CUDA path and the timed CPU
 * port, never part of the product.
 *
 * FP64 restatement of the reference pipeline with the integer-deciding
 * arithmetic replicated in FP32.  Reference citations are file:line in the
 * reference tree (SPH-3D-2 unless stated; SPH-2D and SPH-3D-4 differences are
 * selected by fields of sph_config, each documented where it is read).
 *
 * Parity pinned by tests/test_oracle_golden.py against outputs of the
 * unmodified reference compiled for sm_100a and run on a B200
 * (fixtures under tests/golden, produced by tests/golden/make_golden.py).
 */
#include "sph_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EMPTY_CELL 0xffffffffu
#define NO_SIBLING 0xffffffffu   /* a particle outside any split group */

static int g_threads = 0;

void oracle_set_threads(int n) { g_threads = n; }

int oracle_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

#ifdef _OPENMP
#define OMP_THREADS num_threads(oracle_get_threads())
#endif

/* level 1 -> slot 0 ("large"), anything else -> slot 1 ("small") */
static inline int lv(uint32_t level) { return level == 1u ? 0 : 1; }

/* (uint)floor(x / cell) as the reference computes it in FP32
 * (sph_system.cu:18-27), with the device conversion's behaviour for NaN and
 * negative values (0) and a clamp to the grid (the reference would index out
 * of bounds; positions are clamped to the box so this never triggers in a
 * valid state). */
static inline uint32_t cell_coord(float x, float cs, uint32_t ncell)
{
    float q = x / cs;
    float f = floorf(q);
    if (!(f >= 0.0f)) return 0u;
    if (f >= (float)ncell) return ncell - 1u;
    return (uint32_t)f;
}

static inline void cell_of(const sph_config *c, const float *p, uint32_t *cx)
{
    cx[0] = cell_coord(p[0], c->cell_size, c->ncell[0]);
    cx[1] = cell_coord(p[1], c->cell_size, c->ncell[1]);
    cx[2] = c->dim == 3 ? cell_coord(p[2], c->cell_size, c->ncell[2]) : 0u;
}

static inline uint32_t cell_key(const sph_config *c, const uint32_t *cx)
{
    /* z*row*col + y*row + x (sph_system.cu:29-32; 2D :23-26) */
    return cx[2] * c->ncell[0] * c->ncell[1] + cx[1] * c->ncell[0] + cx[0];
}

static inline uint32_t total_cells(const sph_config *c)
{
    return c->ncell[0] * c->ncell[1] * (c->dim == 3 ? c->ncell[2] : 1u);
}

/* Squared distance in FP32 exactly as the CUDA kernels evaluate it:
 * fma(dz, dz, fma(dx, dx, dy*dy)) with d = a - b per axis. */
static inline float r2_f32(const sph_config *c, const float *a, const float *b)
{
    float dx = a[0] - b[0], dy = a[1] - b[1];
    float t = fmaf(dx, dx, dy * dy);
    if (c->dim == 3) {
        float dz = a[2] - b[2];
        t = fmaf(dz, dz, t);
    }
    return t;
}

/* Iterates the (up to) 3^dim neighbour cells of cell cx that exist inside
 * the grid (the reference's neighbor_status border rules,
 * sph_system.cu:564-652, are exactly "skip offsets that leave the grid"). */
#define FOR_NEIGHBOUR_CELLS(c, cx, key_var)                                          \
    for (int dz_ = ((c)->dim == 3 ? -1 : 0); dz_ <= ((c)->dim == 3 ? 1 : 0); ++dz_) \
        for (int dy_ = -1; dy_ <= 1; ++dy_)                                          \
            for (int dx_ = -1; dx_ <= 1; ++dx_)                                      \
                for (uint32_t key_var = 0, ok_ = neighbour_key(c, cx, dx_, dy_, dz_, &key_var); ok_; ok_ = 0)

static inline uint32_t neighbour_key(const sph_config *c, const uint32_t *cx, int dx, int dy,
                                     int dz, uint32_t *key)
{
    long x = (long)cx[0] + dx, y = (long)cx[1] + dy, z = (long)cx[2] + dz;
    if (x < 0 || y < 0 || z < 0) return 0;
    if (x >= (long)c->ncell[0] || y >= (long)c->ncell[1]) return 0;
    if (c->dim == 3 && z >= (long)c->ncell[2]) return 0;
    uint32_t q[3] = {(uint32_t)x, (uint32_t)y, (uint32_t)z};
    *key = cell_key(c, q);
    return 1;
}

/* ------------------------------------------------------------------ sort */
void oracle_sort(const sph_config *c, uint32_t n, const float *pos, uint32_t *key,
                 uint32_t *index, uint32_t *cs_out, uint32_t *ce_out)
{
    const int d = (int)c->dim;
    const uint32_t C = total_cells(c);
    uint32_t *count = (uint32_t *)calloc((size_t)C + 1, sizeof(uint32_t));
    uint32_t *k = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t cx[3];
        cell_of(c, pos + (size_t)i * d, cx);
        k[i] = cell_key(c, cx);
        count[k[i] + 1]++;
    }
    for (uint32_t q = 0; q < C; ++q) count[q + 1] += count[q];
    /* stable counting sort == thrust::sort_by_key on u32 keys (stable radix,
     * sph_system.cu:119-129): equal keys keep ascending particle index */
    for (uint32_t q = 0; q < C; ++q) { cs_out[q] = EMPTY_CELL; ce_out[q] = 0u; }
    uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)C);
    memcpy(fill, count, sizeof(uint32_t) * (size_t)C);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t s = fill[k[i]]++;
        key[s] = k[i];
        index[s] = i;
    }
    /* cell_start / cell_end (find_start_end, sph_system.cu:131-202) */
    for (uint32_t q = 0; q < C; ++q)
        if (count[q + 1] > count[q]) { cs_out[q] = count[q]; ce_out[q] = count[q + 1]; }
    free(fill);
    free(k);
    free(count);
}

/* --------------------------------------------------------------- density */
void oracle_density(const sph_config *c, uint32_t n, const float *pos, const uint32_t *level,
                    const uint32_t *index, const uint32_t *cs, const uint32_t *ce,
                    double *dens, double *press, uint32_t *nbr)
{
    const int d = (int)c->dim;
#pragma omp parallel for schedule(dynamic, 256) OMP_THREADS
    for (long ii = 0; ii < (long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const float *pi = pos + (size_t)i * d;
        const int li = lv(level[i]);
        const float h2 = c->kernel2[li];
        const double poly6 = c->poly6[li];
        uint32_t cx[3];
        cell_of(c, pi, cx);
        double rho = 0.0;
        uint32_t count = 0;
        FOR_NEIGHBOUR_CELLS(c, cx, key) {
            uint32_t s0 = cs[key];
            if (s0 == EMPTY_CELL) continue;
            for (uint32_t s = s0; s < ce[key]; ++s) {
                uint32_t j = index[s];
                if (j == i) {
                    /* self term m_i*poly6_i*h_i^6 (sph_system.cu:419-422) */
                    rho += (double)c->mass[li] * poly6 * (double)c->kernel6[li];
                    continue;
                }
                const float *pj = pos + (size_t)j * d;
                float r2f = r2_f32(c, pj, pi);
                if (r2f < c->density_skip_r2) continue;   /* :399-402 (2D 1e-12, :396) */
                if (r2f < h2) {
                    double r2 = 0.0;
                    for (int a = 0; a < d; ++a) {
                        double q = (double)pj[a] - (double)pi[a];
                        r2 += q * q;
                    }
                    double t = (double)h2 - r2;
                    /* j's mass, i's kernel (:404-417) */
                    rho += (double)c->mass[lv(level[j])] * poly6 * t * t * t;
                    count++;
                }
            }
        }
        dens[i] = rho;
        double q = rho / (double)c->rest_density;
        press[i] = (q * q * q - 1.0) * (double)c->gas_constant;   /* :674-675 */
        if (nbr) nbr[i] = count;
    }
}

/* ----------------------------------------------------------------- force */
void oracle_force(const sph_config *c, uint32_t n, const float *pos, const float *ev,
                  const uint32_t *level, const double *dens, const double *press,
                  const uint32_t *index, const uint32_t *cs, const uint32_t *ce, double *acc,
                  double *surface, uint8_t *amb)
{
    const int d = (int)c->dim;
#pragma omp parallel for schedule(dynamic, 256) OMP_THREADS
    for (long ii = 0; ii < (long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const float *pi = pos + (size_t)i * d;
        const int li = lv(level[i]);
        const double hi = c->kernel[li], hi2 = c->kernel2[li], hi6 = c->kernel6[li];
        const double mi = c->mass[li];
        const double rhoi = dens[i], pri = press[i];
        uint32_t cx[3];
        cell_of(c, pi, cx);
        double F[3] = {0, 0, 0}, grad[3] = {0, 0, 0}, lapc = 0.0;
        FOR_NEIGHBOUR_CELLS(c, cx, key) {
            uint32_t s0 = cs[key];
            if (s0 == EMPTY_CELL) continue;
            for (uint32_t s = s0; s < ce[key]; ++s) {
                uint32_t j = index[s];
                if (j == i) {
                    /* 2D only: colour Laplacian self term
                     * lapc_i*m/rho*h^2*(0 - 3/4*h^2) (SPH-2D/sph_system.cu:599-603);
                     * the reference multiplies by the integer 3/4 == 0 and reads
                     * an unset j_mass, here m_i. */
                    if (d == 2)
                        lapc += (double)c->lapc_poly6[li] * mi / rhoi * hi2 *
                                (0.0 - (double)c->lapc_three_quarters * hi2);
                    continue;
                }
                const float *pj = pos + (size_t)j * d;
                const int lj = lv(level[j]);
                float r2f = r2_f32(c, pi, pj);
                float maxh2 = c->kernel2[li] > c->kernel2[lj] ? c->kernel2[li] : c->kernel2[lj];
                if (!(r2f < maxh2)) continue;             /* :797-799 */
                if (r2f < c->close_r2) continue;          /* :801-804 (1e-4 in the reference) */
                float rf = sqrtf(r2f);
                double rel[3] = {0, 0, 0}, r2 = 0.0;
                for (int a = 0; a < d; ++a) {
                    rel[a] = (double)pi[a] - (double)pj[a];
                    r2 += rel[a] * rel[a];
                }
                double r = sqrt(r2);
                const double hj = c->kernel[lj], hj6 = c->kernel6[lj], mj = c->mass[lj];
                const double rhoj = dens[j], prj = press[j];
                double ipk = 0, ivk = 0, jpk = 0, jvk = 0;
                /* h - r > 0 decided in FP32 (:813-816) */
                if (c->kernel[li] - rf > 0.0f) {
                    double kr = hi - r;
                    if (c->kernel_h6_twice) {             /* :818-819 */
                        ipk = (double)c->spiky[li] * kr * kr / hi6;
                        ivk = (double)c->visco[li] / hi6 * kr;
                    } else {
                        ipk = (double)c->spiky[li] * kr * kr;
                        ivk = (double)c->visco[li] * kr;
                    }
                    /* colour field gradient / Laplacian (:821-828) */
                    double w = hi2 - r2;
                    double t = -(double)c->grad_poly6[li] * mj / rhoj * w * w;
                    for (int a = 0; a < d; ++a) grad[a] += t * rel[a];
                    lapc += (double)c->lapc_poly6[li] * mj / rhoj * w *
                            (r2 - (double)c->lapc_three_quarters * w);
                }
                if (c->kernel[lj] - rf > 0.0f) {
                    double kr = hj - r;
                    if (c->kernel_h6_twice) {             /* :838-839 */
                        jpk = (double)c->spiky[lj] * kr * kr / hj6;
                        jvk = (double)c->visco[lj] / hj6 * kr;
                    } else {
                        jpk = (double)c->spiky[lj] * kr * kr;
                        jvk = (double)c->visco[lj] * kr;
                    }
                }
                /* pressure (:847-848) and viscosity (:850-853) */
                double tp = mi * mj * (pri / (rhoi * rhoi) + prj / (rhoj * rhoj)) * (ipk + jpk) / 2.0;
                double iV = mi / rhoi, jV = mj / rhoj;
                double tv = (iV * jV) * (double)c->viscosity * (ivk + jvk) / 2.0;
                const float *evi = ev + (size_t)i * d, *evj = ev + (size_t)j * d;
                for (int a = 0; a < d; ++a) {
                    F[a] -= rel[a] * tp / r;
                    F[a] += ((double)evj[a] - (double)evi[a]) * tv;
                }
            }
        }
        /* surface tension switch (:1113-1136; 2D :737-766) */
        double nrm = 0.0;
        for (int a = 0; a < d; ++a) nrm += grad[a] * grad[a];
        nrm = sqrt(nrm);
        surface[i] = nrm;
        const double thr = c->surface_threshold;
        if (amb) amb[i] = fabs(nrm - thr) <= 1e-5 * (thr > 1e-30 ? thr : 1e-30) ? 1 : 0;
        if (nrm > thr)
            for (int a = 0; a < d; ++a) F[a] += (double)c->surface_coef * lapc * grad[a] / nrm;
        /* 2D mouse force (SPH-2D/sph_system.cu:781-789) */
        if (d == 2 && c->extern_force_on) {
            float xl = pi[0] - c->extern_click[0], yl = pi[1] - c->extern_click[1];
            if (fmaf(xl, xl, yl * yl) <= c->extern_len * c->extern_len)
                for (int a = 0; a < 2; ++a)
                    F[a] += (double)c->extern_force[a] * (double)c->extern_coe;
        }
        for (int a = 0; a < d; ++a) acc[(size_t)i * d + a] = F[a];
    }
}

/* ------------------------------------------------------------- integrate */
static inline int near_wall(double x, double w) { return fabs(x - w) <= 1e-6 * (fabs(w) + 1.0); }

void oracle_integrate(const sph_config *c, uint32_t n, const float *pos, const float *vel,
                      const float *ev, const uint32_t *level, const double *acc,
                      const double *dens, double *pos_out, double *vel_out, double *ev_out,
                      double *acc_out, uint8_t *amb)
{
    const int d = (int)c->dim;
    const double dt = c->time_step;
#pragma omp parallel for schedule(static) OMP_THREADS
    for (long ii = 0; ii < (long)n; ++ii) {
        const size_t i = (size_t)ii;
        const int li = lv(level[i]);
        double x[3] = {0, 0, 0}, v[3] = {0, 0, 0}, e[3] = {0, 0, 0}, a[3] = {0, 0, 0};
        for (int k = 0; k < d; ++k) {
            x[k] = pos[i * d + k];
            v[k] = vel[i * d + k];
            e[k] = ev[i * d + k];
            a[k] = acc[i * d + k];
        }
        const double rho = dens[i];
        uint8_t ambig = 0;
        double r;
        if (c->integrator == SPH_INTEGRATE_REF2D) {
            /* SPH-2D/sph_system.cu:219-251: wall at radius/2 */
            r = (double)(c->radius[li] / 2.0f);
            for (int k = 0; k < d; ++k) {
                a[k] = (a[k] + (double)c->gravity[k] * dt) / rho;
                v[k] += a[k] * dt;
                e[k] = (e[k] + v[k]) / 2.0;
                x[k] += v[k] * dt;
            }
        } else {
            r = c->radius[li];
            if (c->integrator == SPH_INTEGRATE_REF3D) {
                /* push forces (SPH-3D-2/sph_system.cu:228-235, SPH-3D-4 :229-242) */
                const float *p32 = pos + i * d;
                if (c->push_left && p32[0] < c->world[0] / 3 && p32[1] > c->world[1] / (float)c->push_y_div)
                    a[0] += 20.0;
                if (c->push_right && p32[0] > c->world[0] / 3 * 2 && p32[1] > c->world[1] / (float)c->push_y_div)
                    a[0] -= 20.0;
                for (int k = 0; k < d; ++k) {      /* :237-240 */
                    v[k] += a[k] * dt / rho;
                    v[k] += (double)c->gravity[k] * dt / rho;
                    x[k] += v[k] * dt;
                }
            } else {                                /* SPH_INTEGRATE_PHYS */
                const double m = c->mass[li];
                for (int k = 0; k < d; ++k) {
                    v[k] += (a[k] / m + (double)c->gravity[k]) * dt;
                    x[k] += v[k] * dt;
                }
            }
            if (c->use_cylinder && d == 3) {        /* :242-282 */
                for (int q = 0; q < 3; ++q) {
                    const sph_sphere *S = &c->sphere[q];
                    double dv[3], dist = 0.0;
                    for (int k = 0; k < 3; ++k) { dv[k] = x[k] - (double)S->pos[k]; dist += dv[k] * dv[k]; }
                    dist = sqrt(dist);
                    double R = (double)S->radius + r;
                    if (fabs(dist - R) <= 1e-6 * R) ambig = 1;
                    if (dist < R) {
                        double nn[3], nl = 0.0;
                        for (int k = 0; k < 3; ++k) { nn[k] = dv[k] / dist * R; nl += nn[k] * nn[k]; }
                        nl = sqrt(nl);
                        double vn = 0.0;
                        for (int k = 0; k < 3; ++k) { x[k] = (double)S->pos[k] + nn[k]; nn[k] /= nl; vn += v[k] * nn[k]; }
                        for (int k = 0; k < 3; ++k) v[k] -= (double)S->damping * vn * nn[k];
                    }
                }
            }
        }
        /* walls, x then y then z (:285-319; 2D :226-250) */
        for (int k = 0; k < d; ++k) {
            double hi = (double)c->world[k] - r;
            if (near_wall(x[k], hi) || near_wall(x[k], r)) ambig = 1;
            if (x[k] >= hi) { v[k] *= (double)c->wall_damping; x[k] = hi; }
            if (x[k] < r) { v[k] *= (double)c->wall_damping; x[k] = r; }
        }
        if (c->integrator != SPH_INTEGRATE_REF2D)
            for (int k = 0; k < d; ++k) e[k] = (e[k] + v[k]) / 2.0;   /* :321 */
        for (int k = 0; k < d; ++k) {
            pos_out[i * d + k] = x[k];
            vel_out[i * d + k] = v[k];
            ev_out[i * d + k] = e[k];
            acc_out[i * d + k] = a[k];
        }
        if (amb) amb[i] = ambig;
    }
}

/* ---------------------------------------------------------------- energy */
/* psi(x) = 2/(pi^0.25*sqrt(3*sigma)) * (x^2/sigma^2 - 1) * EXP^(-x^2/(2 sigma^2)),
 * sigma = 2, with the reference's truncated PI = 3.141592f and
 * EXP = 2.718281f (sph_system.cu:7,11-16; sph_header.h:22). */
static inline double wavelet(double x)
{
    const double sigma = 2.0;
    const double PI_ = (double)3.141592f, EXP_ = (double)2.718281f;
    return 2.0 / (pow(PI_, 0.25) * sqrt(3.0 * sigma)) * ((x * x) / (sigma * sigma) - 1.0) *
           pow(EXP_, -(x * x) / (2.0 * sigma * sigma));
}

void oracle_energy(const sph_config *c, uint32_t n, const float *pos, const float *vel,
                   const uint32_t *level, const uint32_t *index, const uint32_t *cs,
                   const uint32_t *ce, double *energy, double *trans_vel)
{
    const int d = (int)c->dim;
#pragma omp parallel for schedule(dynamic, 256) OMP_THREADS
    for (long ii = 0; ii < (long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const float *pi = pos + (size_t)i * d;
        const int li = lv(level[i]);
        /* 3D: large kernel for both levels (:1199-1209); 2D: own level */
        const int lk = c->energy_large_kernel ? 0 : li;
        const double h = c->kernel[lk];
        const float h2 = c->kernel2[lk];
        uint32_t cx[3];
        cell_of(c, pi, cx);
        double tsum[3] = {0, 0, 0}, tv[3] = {0, 0, 0};
        FOR_NEIGHBOUR_CELLS(c, cx, key) {
            uint32_t s0 = cs[key];
            if (s0 == EMPTY_CELL) continue;
            for (uint32_t s = s0; s < ce[key]; ++s) {
                uint32_t j = index[s];
                if (j == i) continue;
                const float *pj = pos + (size_t)j * d;
                float r2f = r2_f32(c, pi, pj);
                if (!(r2f < h2)) continue;                        /* :1227 */
                if (c->energy_skip_close && r2f < c->close_r2) continue;  /* :1229-1232 */
                for (int a = 0; a < d; ++a) {
                    double t = wavelet(((double)pi[a] - (double)pj[a]) / h);   /* :1238-1240 */
                    tsum[a] += t;
                    tv[a] += (double)vel[(size_t)j * d + a] * t / sqrt(h);    /* :1244-1246 */
                }
            }
        }
        for (int a = 0; a < d; ++a) tv[a] /= tsum[a];          /* :1520 (0/0 -> NaN) */
        double e = 0.5 * (tv[0] * tv[0] + tv[1] * tv[1]);      /* :1521, z omitted */
        if (c->energy_mass_weight) e *= (double)c->mass[li];   /* SPH-3D-4 :1528 */
        energy[i] = e;
        if (trans_vel)
            for (int a = 0; a < d; ++a) trans_vel[(size_t)i * d + a] = tv[a];
    }
}

/* ----------------------------------------------------------------- adapt */
static inline float split_score(const sph_config *c, float energy, float surface)
{
    /* energy*co_energy + surface*co_surface, in FP32 as the kernels do it
     * (sph_system.cu:1564): fma(surface, co_surface, energy*co_energy) */
    return fmaf(surface, c->co_surface, energy * c->co_energy);
}

static inline int split_decision(const sph_config *c, uint32_t level, float energy, float surface,
                                 float dens, uint32_t nbr)
{
    if (level != 1u) return 0;
    if (c->split_rule == SPH_SPLIT_DEFICIT)
        return nbr < c->split_min_neighbors || dens < c->split_density_ratio * c->rest_density;
    return split_score(c, energy, surface) > c->split_criteria;
}

int64_t oracle_adapt(const sph_config *c, uint32_t n, uint32_t cap, const sph_state_view *in,
                     const uint32_t *nbr, const uint32_t *index, const uint32_t *cs,
                     const uint32_t *ce, sph_state_view *out, uint32_t *split_flag,
                     uint32_t *removed)
{
    const int d = (int)c->dim;
    const uint32_t C = total_cells(c);
    const uint32_t ways = c->split_ways == 4 ? 4u : 2u;
    const uint32_t extra = ways - 1u;     /* children per split */
    const float hs2 = c->kernel[1] / 2.0f;

    /* ---- split decision + rank (decide_adaptive_kernel :1548-1574; the
     * stable sort by flag :1641 == ascending particle index) ---- */
    uint32_t *rank = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t n_split = 0;
    for (uint32_t i = 0; i < n; ++i) {
        int s = c->use_split && split_decision(c, in->level[i], in->energy[i], in->surface[i],
                                               in->dens[i], nbr ? nbr[i] : 0u);
        split_flag[i] = (uint32_t)s;
        rank[i] = n_split;
        n_split += (uint32_t)s;
    }
    uint64_t n_after = (uint64_t)n + (uint64_t)n_split * extra;
    if (n_after > cap) { free(rank); return -1; }

    /* post-split per-particle values the merge pass reads
     * (adaptive_particle_kernel :1576-1615; 3D-4 :1583-1656) */
    float *px = (float *)malloc(sizeof(float) * (n ? n : 1));
    float *en = (float *)malloc(sizeof(float) * (n ? n : 1));
    uint32_t *lev = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) {
        px[i] = in->pos[(size_t)i * d];
        en[i] = in->energy[i];
        lev[i] = in->level[i];
        if (split_flag[i]) {
            px[i] = in->pos[(size_t)i * d] + hs2;
            lev[i] = 2u;
            if (ways == 4) en[i] = in->energy[i] / 4.0f;   /* 3D-4 :1653 */
        }
    }
    /* interior counter (SPH_MERGE_INTERIOR) after this step's decision */
    uint32_t *inter = NULL;
    if (c->merge_rule == SPH_MERGE_INTERIOR || c->merge_rule == SPH_MERGE_SIBLING) {
        inter = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
        for (uint32_t i = 0; i < n; ++i) {
            int flagged = (nbr ? nbr[i] : 0u) < c->split_min_neighbors ||
                          in->dens[i] < c->split_density_ratio * c->rest_density;
            uint32_t prev = in->interior ? in->interior[i] : 0u;
            inter[i] = (flagged || split_flag[i]) ? 0u : prev + 1u;
        }
    }

    /* ---- merge (merge_kernel :1661-1789, 3D-4 :1702-1888, 2D :1177-1270) ----
     * one cell at a time over its sorted members; eligible members are taken
     * in groups of `ways` in sorted order; the first member of a group
     * survives with the V-weighted average (V = m/rho, its level already set
     * to 1, :1742-1777) or, in 2D, the plain average (:1242-1246). */
    double *mx = (double *)calloc((size_t)(n ? n : 1) * 4 * d, sizeof(double));  /* merged pos/vel/ev/acc */
    double *men = (double *)calloc((size_t)(n ? n : 1), sizeof(double));
    uint8_t *leader = (uint8_t *)calloc((size_t)(n ? n : 1), 1);
    for (uint32_t i = 0; i < n; ++i) removed[i] = 0u;
    /* one group's merge: V-weighted average into grp[0] (merge_kernel :1742-1777) */
#define MERGE_GROUP(grp)                                                                            \
    do {                                                                                            \
        uint32_t p1 = (grp)[0];                                                                     \
        double V[4], Vs = 0.0;                                                                      \
        for (uint32_t k = 0; k < ways; ++k) {                                                       \
            uint32_t p = (grp)[k];                                                                  \
            uint32_t l = k == 0 ? 1u : lev[p];                                                      \
            V[k] = d == 2 ? 1.0 : (double)c->mass[lv(l)] / (double)in->dens[p];                    \
            Vs += V[k];                                                                             \
        }                                                                                           \
        for (int f = 0; f < 4; ++f)                                                                 \
            for (int a = 0; a < d; ++a) {                                                           \
                double acc_ = 0.0;                                                                  \
                for (uint32_t k = 0; k < ways; ++k) {                                               \
                    uint32_t p = (grp)[k];                                                          \
                    double val;                                                                     \
                    if (f == 0) val = a == 0 ? (double)px[p] : (double)in->pos[(size_t)p * d + a];  \
                    else if (f == 1) val = in->vel[(size_t)p * d + a];                              \
                    else if (f == 2) val = in->ev[(size_t)p * d + a];                               \
                    else val = in->acc[(size_t)p * d + a];                                          \
                    acc_ += val * V[k];                                                             \
                }                                                                                   \
                mx[((size_t)p1 * 4 + f) * d + a] = acc_ / Vs;                                       \
            }                                                                                       \
        double es = 0.0;                                                                            \
        for (uint32_t k = 0; k < ways; ++k) es += en[(grp)[k]];                                     \
        men[p1] = es / (double)ways;                                                                \
        leader[p1] = 1;                                                                             \
        for (uint32_t k = 1; k < ways; ++k) removed[(grp)[k]] = 1u;                                 \
    } while (0)
    if (c->use_merge && c->merge_rule == SPH_MERGE_SIBLING) {
        /* a split group (ring through `sibling`) merges back into its member
         * of smallest index when every one of its `ways` members is level 2
         * and interior for merge_interior_steps steps; averaged in ring order */
        for (uint32_t i = 0; i < n; ++i) {
            if (!(lev[i] != 1u && inter[i] >= c->merge_interior_steps) || !in->sibling) continue;
            uint32_t grp[4] = {i, 0, 0, 0}, j = in->sibling[i];
            int ok = 1;
            for (uint32_t k = 1; k < ways && ok; ++k) {
                ok = j < n && j > i && lev[j] != 1u && inter[j] >= c->merge_interior_steps;
                if (ok) {
                    grp[k] = j;
                    j = in->sibling[j];
                }
            }
            if (ok && j == i) MERGE_GROUP(grp);
        }
    } else if (c->use_merge) {
#pragma omp parallel for schedule(dynamic, 64) OMP_THREADS
        for (long qq = 0; qq < (long)C; ++qq) {
            const uint32_t q = (uint32_t)qq;
            if (cs[q] == EMPTY_CELL) continue;
            uint32_t mem[64], *members = mem, cnt = 0;
            uint32_t len = ce[q] - cs[q];
            if (len > 64) members = (uint32_t *)malloc(sizeof(uint32_t) * len);
            /* criterion value of the particle whose INDEX is q (2D rule);
             * children and stale slots resolved as the reference memory
             * holds them at merge time */
            float cell_score = 0.0f;
            if (c->merge_rule == SPH_MERGE_WAVELET_CELL) {
                float e_q, s_q;
                if (q < n) { e_q = en[q]; s_q = in->surface[q]; }
                else if (q < n_after) {
                    uint32_t k = (q - n) / extra, parent = 0;
                    for (uint32_t i = 0; i < n; ++i) if (split_flag[i] && rank[i] == k) { parent = i; break; }
                    e_q = in->energy[parent] / (ways == 4 ? 4.0f : 1.0f);
                    s_q = in->surface[parent];
                } else { e_q = in->energy[q]; s_q = in->surface[q]; }
                cell_score = split_score(c, e_q, s_q);
            }
            for (uint32_t s = cs[q]; s < ce[q]; ++s) {
                uint32_t p = index[s];
                int el;
                if (c->merge_rule == SPH_MERGE_WAVELET)
                    el = lev[p] != 1u && split_score(c, en[p], in->surface[p]) < c->merge_criteria;
                else if (c->merge_rule == SPH_MERGE_WAVELET_CELL)
                    el = lev[p] == 2u && cell_score < c->merge_criteria;
                else
                    el = lev[p] != 1u && inter[p] >= c->merge_interior_steps;
                if (el) members[cnt++] = p;
            }
            uint32_t groups = cnt / ways;
            for (uint32_t g = 0; g < groups; ++g) MERGE_GROUP(members + g * ways);
            if (members != mem) free(members);
        }
    }

#undef MERGE_GROUP
    /* ---- compaction: stable partition by status (rearrange :1818-1840) ----
     * [surviving old particles][children in split order][removed old ones];
     * split-group links follow their members (removed_before = new index
     * offset of a survivor) */
    uint32_t n_removed = 0;
    uint32_t *removed_before = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) {
        removed_before[i] = n_removed;
        n_removed += removed[i];
    }
    uint32_t n_live = (uint32_t)n_after - n_removed;
    uint32_t surv = 0, gone = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t dst = removed[i] ? n_live + gone++ : surv++;
        /* base values: post-split */
        for (int a = 0; a < d; ++a) {
            float pv = a == 0 ? px[i] : in->pos[(size_t)i * d + a];
            out->pos[(size_t)dst * d + a] = pv;
            out->vel[(size_t)dst * d + a] = in->vel[(size_t)i * d + a];
            out->ev[(size_t)dst * d + a] = in->ev[(size_t)i * d + a];
            out->acc[(size_t)dst * d + a] = in->acc[(size_t)i * d + a];
        }
        out->dens[dst] = in->dens[i];
        out->press[dst] = in->press[i];
        out->energy[dst] = en[i];
        out->surface[dst] = in->surface[i];
        out->level[dst] = lev[i];
        if (out->interior) out->interior[dst] = inter ? inter[i] : 0u;
        if (out->sibling) {
            uint32_t sib = NO_SIBLING;
            if (!removed[i] && !leader[i] && in->sibling && in->sibling[i] < n)
                sib = in->sibling[i] - removed_before[in->sibling[i]];
            if (split_flag[i]) sib = n - n_removed + rank[i] * extra;   /* the first child */
            out->sibling[dst] = sib;
        }
        if (leader[i]) {
            for (int a = 0; a < d; ++a) {
                out->pos[(size_t)dst * d + a] = (float)mx[((size_t)i * 4 + 0) * d + a];
                out->vel[(size_t)dst * d + a] = (float)mx[((size_t)i * 4 + 1) * d + a];
                out->ev[(size_t)dst * d + a] = (float)mx[((size_t)i * 4 + 2) * d + a];
                out->acc[(size_t)dst * d + a] = (float)mx[((size_t)i * 4 + 3) * d + a];
            }
            if (d == 2) out->energy[dst] = (float)men[i];   /* 2D averages energy (:1246) */
            out->level[dst] = 1u;
            if (out->interior) out->interior[dst] = 0u;
        }
        /* children (:1594-1607; 3D-4 :1599-1648; 2D copies dens/pres/surface :1152-1158) */
        if (split_flag[i]) {
            for (uint32_t k = 0; k < extra; ++k) {
                uint32_t cdst = n - n_removed + rank[i] * extra + k;
                const float *pp = in->pos + (size_t)i * d;
                for (int a = 0; a < d; ++a) {
                    out->pos[(size_t)cdst * d + a] = pp[a];
                    out->vel[(size_t)cdst * d + a] = in->vel[(size_t)i * d + a];
                    out->ev[(size_t)cdst * d + a] = in->ev[(size_t)i * d + a];
                    out->acc[(size_t)cdst * d + a] = in->acc[(size_t)i * d + a];
                }
                if (k == 0) out->pos[(size_t)cdst * d + 0] = pp[0] - hs2;
                else if (k == 1) out->pos[(size_t)cdst * d + 2] = pp[2] - hs2;
                else out->pos[(size_t)cdst * d + 2] = pp[2] + hs2;
                out->energy[cdst] = ways == 4 ? in->energy[i] / 4.0f : in->energy[i];
                /* the 3D reference leaves dens/press/surface of a child
                 * unwritten; here they copy the parent in every mode */
                out->dens[cdst] = in->dens[i];
                out->press[cdst] = in->press[i];
                out->surface[cdst] = in->surface[i];
                out->level[cdst] = 2u;
                if (out->interior) out->interior[cdst] = 0u;
                if (out->sibling) out->sibling[cdst] = k + 1 < extra ? cdst + 1 : dst;
            }
        }
    }
    free(rank); free(px); free(en); free(lev); free(inter); free(removed_before);
    free(mx); free(men); free(leader);
    return (int64_t)n_live;
}

/* ------------------------------------------------------------------ step */
int64_t oracle_step(const sph_config *c, uint32_t n, uint32_t cap, const sph_state_view *in,
                    sph_state_view *out, sph_debug_view *dbg)
{
    const int d = (int)c->dim;
    const uint32_t C = total_cells(c);
    const size_t nn = n ? n : 1;
    uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    uint32_t *index = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    uint32_t *cs = (uint32_t *)malloc(sizeof(uint32_t) * C);
    uint32_t *ce = (uint32_t *)malloc(sizeof(uint32_t) * C);
    uint32_t *nbr = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    double *dens = (double *)malloc(sizeof(double) * nn), *press = (double *)malloc(sizeof(double) * nn);
    double *acc = (double *)malloc(sizeof(double) * nn * d), *surf = (double *)malloc(sizeof(double) * nn);
    double *p64 = (double *)malloc(sizeof(double) * nn * d), *v64 = (double *)malloc(sizeof(double) * nn * d);
    double *e64 = (double *)malloc(sizeof(double) * nn * d), *a64 = (double *)malloc(sizeof(double) * nn * d);
    double *en = (double *)malloc(sizeof(double) * nn), *tv = (double *)malloc(sizeof(double) * nn * d);
    float *mid = (float *)malloc(sizeof(float) * (size_t)cap * (4 * d + 5));

    oracle_sort(c, n, in->pos, key, index, cs, ce);
    oracle_density(c, n, in->pos, in->level, index, cs, ce, dens, press, nbr);
    oracle_force(c, n, in->pos, in->ev, in->level, dens, press, index, cs, ce, acc, surf, NULL);
    oracle_integrate(c, n, in->pos, in->vel, in->ev, in->level, acc, dens, p64, v64, e64, a64, NULL);

    /* post-integration FP32 state (the GPU stores floats between kernels) */
    sph_state_view m;
    memset(&m, 0, sizeof(m));
    m.n = n;
    m.pos = mid; m.vel = mid + (size_t)cap * d; m.ev = mid + (size_t)cap * 2 * d;
    m.acc = mid + (size_t)cap * 3 * d; m.dens = mid + (size_t)cap * 4 * d;
    m.press = m.dens + cap; m.energy = m.press + cap; m.surface = m.energy + cap;
    m.level = in->level; m.interior = in->interior; m.sibling = in->sibling;
    float *lvl_f = m.surface + cap;   /* unused slot kept for layout */
    (void)lvl_f;
    for (size_t i = 0; i < (size_t)n * d; ++i) {
        m.pos[i] = (float)p64[i]; m.vel[i] = (float)v64[i];
        m.ev[i] = (float)e64[i]; m.acc[i] = (float)a64[i];
    }
    /* slots beyond n: carry the caller's stale contents (2D merge rule) */
    for (size_t i = n; i < cap; ++i) {
        m.energy[i] = in->energy ? in->energy[i] : 0.0f;
        m.surface[i] = in->surface ? in->surface[i] : 0.0f;
    }
    for (uint32_t i = 0; i < n; ++i) {
        m.dens[i] = (float)dens[i]; m.press[i] = (float)press[i]; m.surface[i] = (float)surf[i];
    }
    oracle_energy(c, n, m.pos, m.vel, in->level, index, cs, ce, en, tv);
    for (uint32_t i = 0; i < n; ++i) m.energy[i] = (float)en[i];

    uint32_t *split = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    uint32_t *rem = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    int64_t n_out = oracle_adapt(c, n, cap, &m, nbr, index, cs, ce, out, split, rem);
    if (n_out >= 0) out->n = (uint32_t)n_out;

    if (dbg) {
        dbg->n_sorted = n;
        dbg->total_cell = C;
        if (dbg->hash) memcpy(dbg->hash, key, sizeof(uint32_t) * n);
        if (dbg->index) memcpy(dbg->index, index, sizeof(uint32_t) * n);
        if (dbg->cell_start) memcpy(dbg->cell_start, cs, sizeof(uint32_t) * C);
        if (dbg->cell_end) memcpy(dbg->cell_end, ce, sizeof(uint32_t) * C);
        if (dbg->trans_vel) for (size_t i = 0; i < (size_t)n * d; ++i) dbg->trans_vel[i] = (float)tv[i];
        if (dbg->nbr_count) memcpy(dbg->nbr_count, nbr, sizeof(uint32_t) * n);
        if (dbg->split_flag) memcpy(dbg->split_flag, split, sizeof(uint32_t) * n);
        if (dbg->removed) memcpy(dbg->removed, rem, sizeof(uint32_t) * n);
    }
    free(key); free(index); free(cs); free(ce); free(nbr); free(dens); free(press);
    free(acc); free(surf); free(p64); free(v64); free(e64); free(a64); free(en); free(tv);
    free(mid); free(split); free(rem);
    return n_out;
}

/* ----------------------------------------------------------- density grid */
void oracle_density_grid(const sph_config *c, uint32_t n, const float *pos, const uint32_t *level,
                         const uint32_t *index, const uint32_t *cs, const uint32_t *ce,
                         double *dens, double *normal)
{
    (void)n;
    const uint32_t R = c->ndens[0], Cc = c->ndens[1], L = c->ndens[2];
    const size_t G = (size_t)R * Cc * L;
    /* integrate_dens_kernel (:1905-2183): nodes on the lower faces stay 0
     * (the upper-face test compares with row_dens itself and never fires) */
#pragma omp parallel for schedule(dynamic, 1024) OMP_THREADS
    for (long gg = 0; gg < (long)G; ++gg) {
        const size_t g = (size_t)gg;
        uint32_t vx = (uint32_t)(g % ((size_t)R * Cc) % R);
        uint32_t vy = (uint32_t)(g % ((size_t)R * Cc) / R);
        uint32_t vz = (uint32_t)(g / ((size_t)R * Cc));
        dens[g] = 0.0;
        if (vx == 0 || vy == 0 || vz == 0) continue;
        /* node position = index * den_size (SPH-3D-2/sph_system.cpp:214-226) */
        float np[3] = {(float)vx * c->den_size, (float)vy * c->den_size, (float)vz * c->den_size};
        /* cell = floor(vox / n_dens * n_cell) in FP32 (:1942-1944) */
        uint32_t cx[3];
        cx[0] = (uint32_t)floorf((float)vx / (float)R * (float)c->ncell[0]);
        cx[1] = (uint32_t)floorf((float)vy / (float)Cc * (float)c->ncell[1]);
        cx[2] = (uint32_t)floorf((float)vz / (float)L * (float)c->ncell[2]);
        double acc_ = 0.0;
        FOR_NEIGHBOUR_CELLS(c, cx, key) {
            uint32_t s0 = cs[key];
            if (s0 == EMPTY_CELL) continue;
            for (uint32_t s = s0; s < ce[key]; ++s) {
                uint32_t j = index[s];
                const int lj = lv(level[j]);
                const float *pj = pos + (size_t)j * 3;
                /* particle radius (reference) or kernel length (splat_with_kernel) */
                float rad = c->splat_with_kernel ? c->kernel[lj] : c->radius[lj];
                float rad2 = rad * rad;
                float r2f = r2_f32(c, pj, np);
                if (r2f < rad2) {                        /* :1894-1900 */
                    double r2 = 0.0;
                    for (int a = 0; a < 3; ++a) { double q = (double)pj[a] - (double)np[a]; r2 += q * q; }
                    double t = (double)rad2 - r2;
                    double w = c->splat_with_kernel ? (double)c->poly6[lj] : (double)c->poly6_radius[lj];
                    acc_ += (double)c->mass[lj] * w * t * t * t;
                }
            }
        }
        dens[g] = acc_;
    }
    /* integrate_normall (:2221-2335): central differences, one-sided with 0
     * outside the grid, divided by den_size, normalised (0 if zero) */
#pragma omp parallel for schedule(static) OMP_THREADS
    for (long gg = 0; gg < (long)G; ++gg) {
        const size_t g = (size_t)gg;
        uint32_t v[3] = {(uint32_t)(g % ((size_t)R * Cc) % R), (uint32_t)(g % ((size_t)R * Cc) / R),
                         (uint32_t)(g / ((size_t)R * Cc))};
        const uint32_t dims[3] = {R, Cc, L};
        const size_t stride[3] = {1, R, (size_t)R * Cc};
        double nv[3], len = 0.0;
        for (int a = 0; a < 3; ++a) {
            double lo = v[a] == 0 ? 0.0 : dens[g - stride[a]];
            double hi = v[a] == dims[a] - 1 ? 0.0 : dens[g + stride[a]];
            nv[a] = (lo - hi) / (double)c->den_size;
            len += nv[a] * nv[a];
        }
        len = sqrt(len);
        for (int a = 0; a < 3; ++a) normal[g * 3 + a] = len == 0.0 ? 0.0 : nv[a] / len;
    }
}
