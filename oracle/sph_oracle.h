/*
 * sph_oracle.h — CPU oracle for the adaptive SPH step.  TEST INFRASTRUCTURE:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * always as the checker / the timed CPU port, never as the product path.
 *
 * A restatement of the reference's per-step pipeline (SPH-2D, SPH-3D-2,
 * SPH-3D-4 sph_system.cu) in FP64, with the integer-deciding arithmetic
 * (cell keys, neighbour cut-offs r^2 < h^2, h - r > 0) replicated in FP32 so
 * keys, sort order, cell ranges and neighbour sets are bit-exact.  Each stage
 * is a separate function so a test can feed every stage the same FP32 inputs
 * the GPU saw.  Vectors are `dim` values per particle.  Loops over particles
 * are OpenMP-parallel; each particle's sums run in one thread in a fixed
 * order, so results do not depend on the thread count.
 */
#ifndef SPH_ORACLE_H
#define SPH_ORACLE_H
#include <stdint.h>
#include "../include/sph/sph.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Set OpenMP threads for subsequent calls (<=0: library default). */
void oracle_set_threads(int n);
int oracle_get_threads(void);

/* Hash + stable sort + cell ranges (SPH-3D-2/sph_system.cu:18-32,78-202). */
void oracle_sort(const sph_config *c, uint32_t n, const float *pos,
                 uint32_t *key, uint32_t *index, uint32_t *cell_start, uint32_t *cell_end);

/* Density + pressure (SPH-3D-2/sph_system.cu:338-677; 2D :268-460).
 * dens/press out in FP64; nbr = neighbours with skip <= r^2 < h_i^2. */
void oracle_density(const sph_config *c, uint32_t n, const float *pos, const uint32_t *level,
                    const uint32_t *index, const uint32_t *cs, const uint32_t *ce,
                    double *dens, double *press, uint32_t *nbr);

/* Forces (SPH-3D-2/sph_system.cu:679-1137; 2D :462-790).  acc/surface in
 * FP64; amb[i] = 1 when |grad c| lies within 1e-5 (relative) of the surface
 * threshold, i.e. the tension switch is numerically ambiguous. */
void oracle_force(const sph_config *c, uint32_t n, const float *pos, const float *ev,
                  const uint32_t *level, const double *dens, const double *press,
                  const uint32_t *index, const uint32_t *cs, const uint32_t *ce,
                  double *acc, double *surface, uint8_t *amb);

/* Integration + boundaries (SPH-3D-2/sph_system.cu:204-322; 2D :198-252).
 * Inputs FP32 state + FP64 acc/dens; outputs FP64.  acc_out is the stored
 * acceleration after the integrator (push force / 2D rescale applied). */
void oracle_integrate(const sph_config *c, uint32_t n, const float *pos, const float *vel,
                      const float *ev, const uint32_t *level, const double *acc,
                      const double *dens, double *pos_out, double *vel_out, double *ev_out,
                      double *acc_out, uint8_t *amb);

/* Wavelet energy on the STALE cell lists with the NEW positions
 * (SPH-3D-2/sph_system.cu:11-16,1169-1546; 2D :827-1065). */
void oracle_energy(const sph_config *c, uint32_t n, const float *pos_new, const float *vel_new,
                   const uint32_t *level, const uint32_t *index, const uint32_t *cs,
                   const uint32_t *ce, double *energy, double *trans_vel);

/* Split + merge + compaction (SPH-3D-2/sph_system.cu:1548-1840,
 * 3D-4 :1555-1915, 2D :1067-1296) on a post-energy FP32 state of n
 * particles held in arrays of capacity `cap` (slots >= n hold whatever the
 * previous step left there, read only by the 2D cell-index merge rule).
 * nbr (per particle) feeds the deficit split rule.  Writes the new state
 * (capacity-sized outputs; slots beyond the live count carry the removed
 * particles, as the reference's stable sort by status leaves them) and
 * returns the new particle count, or -1 on capacity overflow.
 * split_flag / removed are per input particle. */
int64_t oracle_adapt(const sph_config *c, uint32_t n, uint32_t cap, const sph_state_view *in,
                     const uint32_t *nbr, const uint32_t *index, const uint32_t *cs,
                     const uint32_t *ce, sph_state_view *out, uint32_t *split_flag,
                     uint32_t *removed);

/* Whole step: composition of the stages above (FP64 between stages, FP32 at
 * the state boundary).  dbg may be NULL.  Returns the new count or -1. */
int64_t oracle_step(const sph_config *c, uint32_t n, uint32_t cap, const sph_state_view *in,
                    sph_state_view *out, sph_debug_view *dbg);

/* Density grid splat + normals (SPH-3D-2/sph_system.cu:1842-2351), on the
 * stale cell lists with the given positions.  dens: G floats, normal: 3G. */
void oracle_density_grid(const sph_config *c, uint32_t n, const float *pos, const uint32_t *level,
                         const uint32_t *index, const uint32_t *cs, const uint32_t *ce,
                         double *dens, double *normal);

#ifdef __cplusplus
}
#endif
#endif
