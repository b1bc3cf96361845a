/*
 * Headless driver for the UNMODIFIED reference solver (test infrastructure).
 *
 * Compiled together with the reference's own SPH-2D / SPH-3D-2 / SPH-3D-4
 * sources (sph_system.cu + sph_system.cpp, read in place from the reference
 * tree by oracle/build_ref.sh) into oracle/_ref/libref_<variant>_gpu.so.  It
 * replaces the GLUT application (SPH-3D-2/sph_main.cpp:278-323 init,
 * :613-733 display loop) with plain C entry points so a script can construct
 * the reference SPHSystem, load a particle state, run animation()/animate()
 * and read back the state plus the step's intermediate device buffers
 * (hash keys, sorted index, cell ranges, wavelet-transformed velocity).
 *
 * Used only to generate golden fixtures that pin the CPU oracle; nothing in
 * the product links it.
 */
#include "sph_system.h"
#include "sph_system.cuh"
#include <cuda_runtime.h>
#include <string.h>

#ifndef REF_DIM
#error "REF_DIM must be 2 or 3"
#endif

extern "C" {

void *ref_create(void)
{
    cudaSetDevice(0);
    cudaFree(0);   /* create the context before the constructor's allocations */
    return new SPHSystem();
}

int ref_dim(void) { return REF_DIM; }

int ref_particle_size(void) { return (int)sizeof(Particle); }

unsigned ref_total_cell(void *h) { return ((SPHSystem *)h)->m_total_cell; }

unsigned ref_num_particles(void *h) { return ((SPHSystem *)h)->m_num_particle; }

/* which = 0: initial fluid block (add_box_particle / add_init_particle);
 * which = 1: add_new_particle (3D only). */
void ref_add_default_scene(void *h, int which)
{
    SPHSystem *s = (SPHSystem *)h;
#if REF_DIM == 2
    (void)which;
    s->add_init_particle();
#else
    if (which == 0) s->add_box_particle();
    else s->add_new_particle();
#endif
}

/* Replace the particle state with n raw reference-layout Particle records. */
void ref_set_state(void *h, const void *particles, unsigned n)
{
    SPHSystem *s = (SPHSystem *)h;
    memcpy(s->m_host_mem, particles, sizeof(Particle) * (size_t)n);
    s->m_num_particle = n;
    copy_array(s->m_dev_mem, s->m_host_mem, sizeof(Particle) * (size_t)n, CUDA_HOST_TO_DEV);
}

/* The constants the reference constructor computed, in a fixed order:
 * mass L/S, kernel L/S, kernel^2 L/S, kernel^6 L/S, radius L/S,
 * poly6 L/S, spiky L/S, visco L/S, grad_poly6 L/S, lapc_poly6 L/S,
 * poly6_radius L/S (3D) / 0 (2D), cell_size, world x, y, (z), rest_density,
 * gas_constant, time_step, viscosity, surface threshold, co_surface,
 * co_energy, split threshold, merge threshold, gravity x, y, (z),
 * wall_damping, den_size (3D).  Returns the count written. */
int ref_param_floats(void *h, float *o)
{
    SPHSystem *s = (SPHSystem *)h;
    int k = 0;
#if REF_DIM == 2
    float v[] = {s->m_large_mass, s->m_small_mass, s->m_large_kernel, s->m_small_kernel,
                 s->m_large_kernel2, s->m_small_kernel2, s->m_large_kernel6, s->m_small_kernel6,
                 s->m_large_radius, s->m_small_radius, s->m_large_poly6, s->m_small_poly6,
                 s->m_large_spiky, s->m_small_spiky, s->m_large_visco, s->m_small_visco,
                 s->m_large_grad_poly6, s->m_small_grad_poly6, s->m_large_lapc_poly6, s->m_small_lapc_poly6,
                 0.0f, 0.0f, s->m_cell_size, s->m_world_width, s->m_world_depth, s->m_rest_density,
                 s->m_gas_constant, s->m_time_step, s->m_viscosity, s->m_surface_normal, s->m_co_surface,
                 s->m_co_energy, s->m_thresh_split, s->m_thresh_merge, s->m_gravity.x, s->m_gravity.y,
                 s->m_wall_damping};
#else
    float v[] = {s->m_large_mass, s->m_small_mass, s->m_large_kernel, s->m_small_kernel,
                 s->m_large_kernel_2, s->m_small_kernel_2, s->m_large_kernel_6, s->m_small_kernel_6,
                 s->m_large_radius, s->m_small_radius, s->m_large_poly6, s->m_small_poly6,
                 s->m_large_spiky, s->m_small_spiky, s->m_large_visco, s->m_small_visco,
                 s->m_large_grad_poly6, s->m_small_grad_poly6, s->m_large_lapc_poly6, s->m_small_lapc_poly6,
                 s->m_large_poly6_radius, s->m_small_poly6_radius, s->m_cell_size, s->m_world_width,
                 s->m_world_height, s->m_world_length, s->m_rest_density, s->m_gas_constant, s->m_time_step,
                 s->m_viscosity, s->m_surface_tension, s->m_co_surface, s->m_co_energy, s->m_split_criteria,
                 s->m_merge_criteria, s->m_gravity.x, s->m_gravity.y, s->m_gravity.z, s->m_wall_damping,
                 s->m_den_size};
#endif
    for (unsigned q = 0; q < sizeof(v) / sizeof(v[0]); ++q) o[k++] = v[q];
    return k;
}

void ref_set_flags(void *h, int use_split, int use_merge, int disp_mode)
{
    SPHSystem *s = (SPHSystem *)h;
#if REF_DIM == 2
    (void)disp_mode;
    s->m_enable_split = (uint)use_split;
    s->m_enable_merge = (uint)use_merge;
#else
    s->m_use_split = (uint)use_split;
    s->m_use_merge = (uint)use_merge;
    s->m_disp_mode = (uint)disp_mode;
#endif
}

void ref_set_time_step(void *h, float dt)
{
    SPHSystem *s = (SPHSystem *)h;
    s->m_time_step = dt;
    s->m_host_param->time_step = dt;
}

#if REF_DIM == 3
void ref_set_use_cylinder(void *h, int on)
{
    ((SPHSystem *)h)->m_host_param->use_cylinder = on ? true : false;
}
#endif

/* One reference step, then a device synchronise so errors surface here.
 * Before stepping, the reference's own set_parameters() is called once and
 * its status checked: if the parameter block does not reach the device
 * (see ref_shim/cutil_math.h), the step would hash every particle to an
 * out-of-range cell, so the driver refuses to run it and returns -1. */
int ref_step(void *h)
{
    SPHSystem *s = (SPHSystem *)h;
    /* every particle inside the box: its hash indexes the cell arrays */
    for (uint i = 0; i < s->m_num_particle; ++i) {
        const Particle &p = s->m_host_mem[i];
#if REF_DIM == 2
        if (!(p.pos.x >= 0.0f && p.pos.x < s->m_world_width && p.pos.y >= 0.0f && p.pos.y < s->m_world_depth))
            return -2;
#else
        if (!(p.pos.x >= 0.0f && p.pos.x < s->m_world_width && p.pos.y >= 0.0f && p.pos.y < s->m_world_height &&
              p.pos.z >= 0.0f && p.pos.z < s->m_world_length))
            return -2;
#endif
        if (p.level != 1 && p.level != 2) return -3;
    }
    cudaGetLastError();
    s->m_host_param->num_particle = s->m_num_particle;
    set_parameters(s->m_host_param);
    if (cudaGetLastError() != cudaSuccess) return -1;
    s->m_sys_running = 1;
#if REF_DIM == 2
    s->animate();
#else
    s->animation();
#endif
    cudaError_t e = cudaDeviceSynchronize();
    return (int)e;
}

void ref_read_particles(void *h, void *out)
{
    SPHSystem *s = (SPHSystem *)h;
    memcpy(out, s->m_host_mem, sizeof(Particle) * (size_t)s->m_num_particle);
}

/* Intermediate buffers of the LAST step.  n_sorted is the particle count the
 * step started with (the caller knows it).  trans_vel has REF_DIM floats per
 * particle. */
void ref_read_debug(void *h, unsigned n_sorted, unsigned *hash, unsigned *index,
                    unsigned *cell_start, unsigned *cell_end, float *trans_vel)
{
    SPHSystem *s = (SPHSystem *)h;
    cudaMemcpy(hash, s->m_dev_hash, sizeof(uint) * n_sorted, cudaMemcpyDeviceToHost);
    cudaMemcpy(index, s->m_dev_index, sizeof(uint) * n_sorted, cudaMemcpyDeviceToHost);
    cudaMemcpy(cell_start, s->m_cell_start, sizeof(uint) * s->m_total_cell, cudaMemcpyDeviceToHost);
    cudaMemcpy(cell_end, s->m_cell_end, sizeof(uint) * s->m_total_cell, cudaMemcpyDeviceToHost);
    cudaMemcpy(trans_vel, s->m_trans_vel, sizeof(float) * REF_DIM * n_sorted, cudaMemcpyDeviceToHost);
}

#if REF_DIM == 3
unsigned ref_grid_nodes(void *h) { return ((SPHSystem *)h)->m_tot_dens; }

void ref_grid_dims(void *h, unsigned *dims)
{
    SPHSystem *s = (SPHSystem *)h;
    dims[0] = s->m_row_dens; dims[1] = s->m_col_dens; dims[2] = s->m_len_dens;
}

/* Density grid and normals of the last disp_mode==2 step (host copies the
 * reference made for its CPU marching cubes). */
void ref_read_grid(void *h, float *dens, float *normal)
{
    SPHSystem *s = (SPHSystem *)h;
    memcpy(dens, s->m_host_dens, sizeof(float) * s->m_tot_dens);
    memcpy(normal, s->m_host_dens_normal, sizeof(float3) * s->m_tot_dens);
}

unsigned ref_read_mesh(void *h, float *t0, float *t1, float *t2, float *n0, float *n1, float *n2)
{
    SPHSystem *s = (SPHSystem *)h;
    unsigned nt = s->m_num_triangle;
    memcpy(t0, s->m_host_triangle0, sizeof(float3) * nt);
    memcpy(t1, s->m_host_triangle1, sizeof(float3) * nt);
    memcpy(t2, s->m_host_triangle2, sizeof(float3) * nt);
    memcpy(n0, s->m_host_triangle_normal0, sizeof(float3) * nt);
    memcpy(n1, s->m_host_triangle_normal1, sizeof(float3) * nt);
    memcpy(n2, s->m_host_triangle_normal2, sizeof(float3) * nt);
    return nt;
}
#endif

} /* extern "C" */
