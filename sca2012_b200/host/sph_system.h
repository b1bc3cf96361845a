// sph_system.h — drop-in SPHSystem for the reference's applications.
//
// The reference builds three programs, each with its own host class
// SPHSystem (SPH-2D/sph_system.h:24-108, SPH-3D-2/sph_system.h:26-154,
// SPH-3D-4/sph_system.h).  This header provides a class of the same name,
// public fields and methods for one of them, selected at compile time:
//
//     -DSCA2012_VARIANT=2   SPH-2D        (animate, add_init_particle, add_extern_force)
//     -DSCA2012_VARIANT=32  SPH-3D-2      (default; animation, add_box_particle, ...)
//     -DSCA2012_VARIANT=34  SPH-3D-4
//
// The fields the applications read (m_host_mem with the reference's Particle
// record, m_num_particle, the world/cell/grid sizes, the mesh arrays, the
// toggles m_use_split / m_use_merge / m_disp_mode / m_sys_running, the
// m_host_param switches) keep their names, types and meaning.  The step runs
// on the B200 through the C-ABI (include/sph/sph.h); the per-step readback
// into m_host_mem, and in display mode 2 the density grid and the mesh, are
// refreshed after every animation() like the reference does.
#ifndef SCA2012_B200_SPH_SYSTEM_H
#define SCA2012_B200_SPH_SYSTEM_H

#include <vector_functions.h>
#include <vector_types.h>

#include "../../include/sph/sph.h"

#ifndef SCA2012_VARIANT
#define SCA2012_VARIANT 32
#endif

typedef unsigned int uint;

#if SCA2012_VARIANT == 2
// SPH-2D/sph_system.h:7-22 (56 bytes)
class Particle {
public:
    float2 pos, vel, ev, acc;
    float dens, pres, energy;
    uint level;
    float surface_normal;
};

// the switches of SysParam the 2D application writes (SPH-2D/sph_param.h:6-70)
class SysParam {
public:
    bool force_waiting;
    float2 extern_force, extern_click;
    uint2 extern_pos;
    float extern_len, extern_coe;
    float time_step, viscosity, gas_constant, rest_density, wall_damping;
    float2 gravity;
};

class SPHSystem {
public:
    uint m_num_particle, m_max_particle;
    float m_world_width, m_world_depth;
    float m_large_mass, m_small_mass, m_large_kernel, m_small_kernel, m_large_kernel2, m_small_kernel2;
    float m_large_kernel6, m_small_kernel6, m_large_radius, m_small_radius;
    float m_large_poly6, m_small_poly6, m_large_spiky, m_small_spiky, m_large_visco, m_small_visco;
    float m_large_grad_poly6, m_small_grad_poly6, m_large_lapc_poly6, m_small_lapc_poly6;
    float2 m_gravity;
    float m_wall_damping, m_rest_density, m_gas_constant, m_viscosity, m_time_step, m_surface_normal;
    uint m_sys_running;
    float m_cell_size;
    uint m_row_cell, m_col_cell, m_total_cell;
    float m_co_surface, m_co_energy, m_thresh_split, m_thresh_merge;
    Particle *m_host_mem;
    uint m_enable_split, m_enable_merge;
    SysParam *m_host_param;

    SPHSystem();
    ~SPHSystem();
    void add_init_particle();
    void add_particle(float2 pos, float2 vel, uint level);
    void animate();
    void add_extern_force(float2 pos, float2 force);

    // status of the last C-ABI call (SPH_OK == 0); not in the reference
    int last_status() const { return m_status; }

private:
    sph_handle *m_h;
    sph_config m_cfg;
    uint m_uploaded;
    int m_status;
    void upload_if_needed();
};

#else
// SPH-3D-2/sph_object.h:4-9
class Sphere {
public:
    float3 pos;
    float radius;
    float damping;
};

// SPH-3D-2/sph_system.h:8-24 (72 bytes)
class Particle {
public:
    float3 pos, vel, ev, acc;
    float dens, press, energy, surface, tension;
    uint level;
};

// the fields of SysParam the 3D applications and the step read
// (SPH-3D-2/sph_param.h:8-87); applied at every animation() like the
// reference's set_parameters upload
class SysParam {
public:
    float3 gravity;
    float wall_damping, rest_density, gas_constant, time_step, viscosity, surface_tension;
    float co_surface, co_energy, split_criteria, merge_criteria;
    Sphere sphere1, sphere2, sphere3, sphere4;
    float split_energy, merge_energy;
#if SCA2012_VARIANT == 34
    bool force_waiting_left, force_waiting_right;
#else
    bool force_waiting;
#endif
    bool use_cylinder;
};

class SPHSystem {
public:
    Particle *m_host_mem;
    uint m_num_particle, m_max_particle;
    float m_world_width, m_world_height, m_world_length;
    float m_large_radius, m_small_radius, m_large_kernel, m_small_kernel, m_large_mass, m_small_mass;
    float m_cell_size;
    uint m_row_cell, m_col_cell, m_len_cell, m_total_cell;
    float3 m_gravity;
    float m_wall_damping, m_rest_density, m_gas_constant, m_time_step, m_viscosity, m_surface_tension;
    float m_co_surface, m_co_energy, m_split_criteria, m_merge_criteria;
    float m_large_poly6, m_large_spiky, m_large_visco, m_large_grad_poly6, m_large_lapc_poly6;
    float m_small_poly6, m_small_spiky, m_small_visco, m_small_grad_poly6, m_small_lapc_poly6;
    float m_large_kernel_2, m_large_kernel_6, m_small_kernel_2, m_small_kernel_6;
    float m_large_poly6_radius, m_small_poly6_radius;
    uint m_dens_mul;
    float m_den_size;
    uint m_row_dens, m_col_dens, m_len_dens, m_tot_dens;
    float *m_host_dens;
    float3 *m_host_dens_pos, *m_host_dens_normal;
    uint m_num_lines;
    float3 *m_host_line0, *m_host_line1;
    uint m_num_triangle;
    float3 *m_host_triangle0, *m_host_triangle1, *m_host_triangle2;
    float3 *m_host_triangle_normal0, *m_host_triangle_normal1, *m_host_triangle_normal2;
    Sphere m_sphere1, m_sphere2, m_sphere3, m_sphere4;
    SysParam *m_host_param;
    uint m_sys_running, m_trans_once, m_use_split, m_use_merge, m_disp_mode;

    SPHSystem();
    ~SPHSystem();
    void add_box_particle();
    void add_new_particle();
    void animation();
    void add_particle(float3 pos, float3 vel, uint level);
    void marching_cube();

    int last_status() const { return m_status; }

private:
    sph_handle *m_h;
    sph_config m_cfg;
    uint m_uploaded;
    uint m_max_triangle;
    int m_status;
    void upload_if_needed();
    void apply_params();
};
#endif

#endif
