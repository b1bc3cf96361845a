/*
 * CPU-only build of the reference's OWN marching cubes (test infrastructure).
 *
 * The reference extracts its surface on the host: SPHSystem::marching_cube()
 * and marching_cube_cell() with the 256-entry edge/triangle tables, all in
 * SPH-3D-2/sph_system.cpp:406-821 (SPH-3D-4/sph_system.cpp:455-870).  That
 * file is compiled unmodified from the reference tree by oracle/build_ref.sh
 * and linked with this driver into oracle/_ref/libref_<variant>_mc.so.  The
 * device-side wrappers it references (SPH-3D-2/sph_system.cuh) are stubbed
 * here with host memory so the object links and runs without a GPU: only the
 * constructor's buffer allocation and the grid-position upload are exercised.
 *
 * Used only by tests as the marching-cubes oracle.
 */
#include "sph_system.h"
#include "sph_system.cuh"
#include <stdlib.h>
#include <string.h>

/* ---- host stand-ins for the reference's launch wrappers (never timed) ---- */
void set_parameters(SysParam *) {}
void alloc_array(void **dev_ptr, size_t size) { *dev_ptr = calloc(1, size); }
void free_array(void *dev_ptr) { free(dev_ptr); }
void copy_array(void *a, void *b, size_t size, int) { memcpy(a, b, size); }
void compute_grid_size(uint, uint, uint &nb, uint &nt) { nb = nt = 0; }
void calc_hash(uint *, uint *, Particle *, uint) {}
void sort_particles(uint *, uint *, uint) {}
void find_start_end(uint *, uint *, uint *, uint *, uint, uint) {}
void integrate_velocity(Particle *, uint) {}
void compute(Particle *, uint *, uint *, uint *, uint *, uint, uint) {}
void compute_energy(Particle *, uint *, uint *, uint *, uint *, uint, uint, float3 *) {}
uint adaptive_particle(Particle *, uint *, uint *, uint *, uint *, uint n, uint, uint *, uint *) { return n; }
void merge(Particle *, uint *, uint *, uint *, uint *, uint, uint, uint *, uint *) {}
uint rearrange(Particle *, uint *, uint n) { return n; }
void integrate_dens(Particle *, uint *, uint *, uint *, uint *, uint, uint, uint, uint, uint, uint,
                    float, float *, float3 *) {}
void integrate_normal(float *, float3 *, float3 *, uint) {}

extern "C" {

void *mc_create(void) { return new SPHSystem(); }

void mc_grid_dims(void *h, unsigned *dims)
{
    SPHSystem *s = (SPHSystem *)h;
    dims[0] = s->m_row_dens; dims[1] = s->m_col_dens; dims[2] = s->m_len_dens;
}

float mc_den_size(void *h) { return ((SPHSystem *)h)->m_den_size; }

/* Runs the reference's marching_cube() on the given node densities and
 * normals (node index = z*row*col + y*row + x) and returns the triangle
 * count; vertex and normal arrays receive 3 floats per triangle corner. */
unsigned mc_run(void *h, const float *dens, const float *normal,
                float *t0, float *t1, float *t2, float *n0, float *n1, float *n2,
                unsigned max_tri)
{
    SPHSystem *s = (SPHSystem *)h;
    memcpy(s->m_host_dens, dens, sizeof(float) * s->m_tot_dens);
    memcpy(s->m_host_dens_normal, normal, sizeof(float3) * s->m_tot_dens);
    s->marching_cube();
    unsigned nt = s->m_num_triangle;
    if (nt > max_tri) nt = max_tri;
    memcpy(t0, s->m_host_triangle0, sizeof(float3) * nt);
    memcpy(t1, s->m_host_triangle1, sizeof(float3) * nt);
    memcpy(t2, s->m_host_triangle2, sizeof(float3) * nt);
    memcpy(n0, s->m_host_triangle_normal0, sizeof(float3) * nt);
    memcpy(n1, s->m_host_triangle_normal1, sizeof(float3) * nt);
    memcpy(n2, s->m_host_triangle_normal2, sizeof(float3) * nt);
    return s->m_num_triangle;
}

/* The reference's case tables, exposed so a test can check the project's
 * independently generated tables against them. */
extern int aiCubeEdgeFlags[256];
extern int a2iTriangleConnectionTable[256][16];
void mc_tables(int *edge_flags, int *tri_table)
{
    memcpy(edge_flags, aiCubeEdgeFlags, sizeof(int) * 256);
    memcpy(tri_table, a2iTriangleConnectionTable, sizeof(int) * 256 * 16);
}

} /* extern "C" */
