// sph_system.cpp — drop-in SPHSystem over the C-ABI (see sph_system.h).
//
// Scene builders replicate the reference's lattice loops with the same FP32
// loop arithmetic (SPH-3D-2/sph_system.cpp:247-283, SPH-3D-4/sph_system.cpp:248-332,
// SPH-2D/sph_system.cpp:148-162) so a drop-in run starts from the same
// particles.  The SPH-3D-4 sphere scene is built without the reference's
// double increment of m_num_particle (its sph_system.cpp:324), which leaves
// every other record uninitialised there.
#include "sph_system.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace {

int preset_of_variant()
{
#if SCA2012_VARIANT == 2
    return SPH_PRESET_REF_2D;
#elif SCA2012_VARIANT == 34
    return SPH_PRESET_REF_3D4;
#else
    return SPH_PRESET_REF_3D2;
#endif
}

void report(int rc, const char *what, sph_handle *h)
{
    if (rc != SPH_OK) fprintf(stderr, "SPHSystem: %s failed (%d): %s\n", what, rc, h ? sph_last_error(h) : "");
}

}  // namespace

#if SCA2012_VARIANT == 2
// ============================================================== SPH-2D
SPHSystem::SPHSystem() : m_h(nullptr), m_uploaded(0), m_status(SPH_OK)
{
    sph_config_preset(preset_of_variant(), &m_cfg);
    m_num_particle = 0;
    m_max_particle = m_cfg.max_particle;
    m_world_width = m_cfg.world[0];
    m_world_depth = m_cfg.world[1];
    m_large_mass = m_cfg.mass[0]; m_small_mass = m_cfg.mass[1];
    m_large_kernel = m_cfg.kernel[0]; m_small_kernel = m_cfg.kernel[1];
    m_large_kernel2 = m_cfg.kernel2[0]; m_small_kernel2 = m_cfg.kernel2[1];
    m_large_kernel6 = m_cfg.kernel6[0]; m_small_kernel6 = m_cfg.kernel6[1];
    m_large_radius = m_cfg.radius[0]; m_small_radius = m_cfg.radius[1];
    m_large_poly6 = m_cfg.poly6[0]; m_small_poly6 = m_cfg.poly6[1];
    m_large_spiky = m_cfg.spiky[0]; m_small_spiky = m_cfg.spiky[1];
    m_large_visco = m_cfg.visco[0]; m_small_visco = m_cfg.visco[1];
    m_large_grad_poly6 = m_cfg.grad_poly6[0]; m_small_grad_poly6 = m_cfg.grad_poly6[1];
    m_large_lapc_poly6 = m_cfg.lapc_poly6[0]; m_small_lapc_poly6 = m_cfg.lapc_poly6[1];
    m_gravity = make_float2(m_cfg.gravity[0], m_cfg.gravity[1]);
    m_wall_damping = m_cfg.wall_damping;
    m_rest_density = m_cfg.rest_density;
    m_gas_constant = m_cfg.gas_constant;
    m_viscosity = m_cfg.viscosity;
    m_time_step = m_cfg.time_step;
    m_surface_normal = m_cfg.surface_threshold;
    m_sys_running = 0;
    m_cell_size = m_cfg.cell_size;
    m_row_cell = m_cfg.ncell[0];
    m_col_cell = m_cfg.ncell[1];
    m_total_cell = m_row_cell * m_col_cell;
    m_co_surface = m_cfg.co_surface;
    m_co_energy = m_cfg.co_energy;
    m_thresh_split = m_cfg.split_criteria;
    m_thresh_merge = m_cfg.merge_criteria;
    m_host_mem = new Particle[m_max_particle]();
    m_enable_split = 0;
    m_enable_merge = 0;
    m_host_param = new SysParam();
    m_host_param->force_waiting = false;
    m_host_param->extern_force = make_float2(0.0f, 0.0f);
    m_host_param->extern_click = make_float2(0.0f, 0.0f);
    m_host_param->extern_pos = make_uint2(0, 0);
    m_host_param->extern_len = m_cfg.extern_len;
    m_host_param->extern_coe = m_cfg.extern_coe;
    m_host_param->time_step = m_cfg.time_step;
    m_host_param->viscosity = m_cfg.viscosity;
    m_host_param->gas_constant = m_cfg.gas_constant;
    m_host_param->rest_density = m_cfg.rest_density;
    m_host_param->wall_damping = m_cfg.wall_damping;
    m_host_param->gravity = m_gravity;
    m_status = sph_create(&m_cfg, &m_h);
    report(m_status, "sph_create", m_h);
}

SPHSystem::~SPHSystem()
{
    if (m_h) sph_destroy(m_h);
    delete[] m_host_mem;
    delete m_host_param;
}

void SPHSystem::add_particle(float2 pos, float2 vel, uint level)
{
    Particle *p = &m_host_mem[m_num_particle];
    p->pos = pos;
    p->vel = vel;
    p->ev = make_float2(0.0f, 0.0f);
    p->acc = make_float2(0.0f, 0.0f);
    p->dens = 0.0f;
    p->pres = 0.0f;
    p->energy = 0.0f;
    p->level = level;
    p->surface_normal = 0.0f;
    m_num_particle++;
}

void SPHSystem::add_init_particle()
{
    // SPH-2D/sph_system.cpp:148-162
    float2 pos;
    const float2 vel = make_float2(0.0f, 0.0f);
    for (pos.x = m_large_radius / 2.0f; pos.x < m_world_width / 2; pos.x += m_large_kernel * 0.5f)
        for (pos.y = m_large_radius / 2.0f; m_world_depth - pos.y >= m_large_radius / 2.0f;
             pos.y += m_large_kernel * 0.5f)
            add_particle(pos, vel, 1);
    upload_if_needed();
}

void SPHSystem::add_extern_force(float2 pos, float2 force)
{
    // SPH-2D/sph_system.cpp:179-188: pos in [0,1]^2 window coordinates
    m_host_param->extern_click = make_float2(pos.x * m_world_width, pos.y * m_world_depth);
    m_host_param->extern_pos = make_uint2((uint)floor(pos.x * m_row_cell), (uint)floor(pos.y * m_col_cell));
    m_host_param->extern_force = force;
    m_host_param->force_waiting = true;
}

void SPHSystem::upload_if_needed()
{
    if (!m_h || m_uploaded == m_num_particle) return;
    m_status = sph_write_particles(m_h, m_host_mem, m_num_particle);
    report(m_status, "sph_write_particles", m_h);
    m_uploaded = m_num_particle;
}

void SPHSystem::animate()
{
    // SPH-2D/sph_system.cpp:190-264
    if (m_sys_running == 0 || !m_h) return;
    m_cfg.use_split = m_enable_split;
    m_cfg.use_merge = m_enable_merge;
    m_cfg.time_step = m_host_param->time_step;
    m_cfg.viscosity = m_host_param->viscosity;
    m_cfg.gas_constant = m_host_param->gas_constant;
    m_cfg.rest_density = m_host_param->rest_density;
    m_cfg.wall_damping = m_host_param->wall_damping;
    m_cfg.gravity[0] = m_host_param->gravity.x;
    m_cfg.gravity[1] = m_host_param->gravity.y;
    m_cfg.extern_force_on = m_host_param->force_waiting ? 1u : 0u;
    m_cfg.extern_click[0] = m_host_param->extern_click.x;
    m_cfg.extern_click[1] = m_host_param->extern_click.y;
    m_cfg.extern_force[0] = m_host_param->extern_force.x;
    m_cfg.extern_force[1] = m_host_param->extern_force.y;
    m_cfg.extern_len = m_host_param->extern_len;
    m_cfg.extern_coe = m_host_param->extern_coe;
    m_status = sph_set_config(m_h, &m_cfg);
    if (m_status) return report(m_status, "sph_set_config", m_h);
    upload_if_needed();
    m_status = sph_step(m_h, 1);
    if (m_status) return report(m_status, "sph_step", m_h);
    m_status = sph_read_particles(m_h, m_host_mem, (uint64_t)sizeof(Particle) * m_max_particle, &m_num_particle);
    report(m_status, "sph_read_particles", m_h);
    m_uploaded = m_num_particle;
    m_host_param->force_waiting = false;
}

#else
// ============================================================== SPH-3D-2 / SPH-3D-4
SPHSystem::SPHSystem() : m_h(nullptr), m_uploaded(0), m_status(SPH_OK)
{
    sph_config_preset(preset_of_variant(), &m_cfg);
    m_num_particle = 0;
    m_max_particle = m_cfg.max_particle;
    m_world_width = m_cfg.world[0];
    m_world_height = m_cfg.world[1];
    m_world_length = m_cfg.world[2];
    m_large_radius = m_cfg.radius[0]; m_small_radius = m_cfg.radius[1];
    m_large_kernel = m_cfg.kernel[0]; m_small_kernel = m_cfg.kernel[1];
    m_large_mass = m_cfg.mass[0]; m_small_mass = m_cfg.mass[1];
    m_cell_size = m_cfg.cell_size;
    m_row_cell = m_cfg.ncell[0];
    m_col_cell = m_cfg.ncell[1];
    m_len_cell = m_cfg.ncell[2];
    m_total_cell = m_row_cell * m_col_cell * m_len_cell;
    m_gravity = make_float3(m_cfg.gravity[0], m_cfg.gravity[1], m_cfg.gravity[2]);
    m_wall_damping = m_cfg.wall_damping;
    m_rest_density = m_cfg.rest_density;
    m_gas_constant = m_cfg.gas_constant;
    m_time_step = m_cfg.time_step;
    m_viscosity = m_cfg.viscosity;
    m_surface_tension = m_cfg.surface_threshold;
    m_co_surface = m_cfg.co_surface;
    m_co_energy = m_cfg.co_energy;
    m_split_criteria = m_cfg.split_criteria;
    m_merge_criteria = m_cfg.merge_criteria;
    m_large_poly6 = m_cfg.poly6[0]; m_large_spiky = m_cfg.spiky[0]; m_large_visco = m_cfg.visco[0];
    m_large_grad_poly6 = m_cfg.grad_poly6[0]; m_large_lapc_poly6 = m_cfg.lapc_poly6[0];
    m_small_poly6 = m_cfg.poly6[1]; m_small_spiky = m_cfg.spiky[1]; m_small_visco = m_cfg.visco[1];
    m_small_grad_poly6 = m_cfg.grad_poly6[1]; m_small_lapc_poly6 = m_cfg.lapc_poly6[1];
    m_large_kernel_2 = m_cfg.kernel2[0]; m_large_kernel_6 = m_cfg.kernel6[0];
    m_small_kernel_2 = m_cfg.kernel2[1]; m_small_kernel_6 = m_cfg.kernel6[1];
    m_large_poly6_radius = m_cfg.poly6_radius[0]; m_small_poly6_radius = m_cfg.poly6_radius[1];
    m_dens_mul = m_cfg.dens_mul;
    m_den_size = m_cfg.den_size;
    m_row_dens = m_cfg.ndens[0];
    m_col_dens = m_cfg.ndens[1];
    m_len_dens = m_cfg.ndens[2];
    m_tot_dens = m_row_dens * m_col_dens * m_len_dens;

    m_host_mem = new Particle[m_max_particle]();
    m_host_dens = new float[m_tot_dens]();
    m_host_dens_pos = new float3[m_tot_dens];
    m_host_dens_normal = new float3[m_tot_dens]();
    m_num_lines = 0;
    m_host_line0 = new float3[2 * (size_t)m_tot_dens]();
    m_host_line1 = new float3[2 * (size_t)m_tot_dens]();
    m_num_triangle = 0;
    // 3D-2 keeps one triangle slot per grid node, 3D-4 three
    // (SPH-3D-2/sph_system.cpp:108-114, SPH-3D-4/sph_system.cpp:108-114)
    m_max_triangle = SCA2012_VARIANT == 34 ? 3 * m_tot_dens : m_tot_dens;
    m_host_triangle0 = new float3[m_max_triangle]();
    m_host_triangle1 = new float3[m_max_triangle]();
    m_host_triangle2 = new float3[m_max_triangle]();
    m_host_triangle_normal0 = new float3[m_max_triangle]();
    m_host_triangle_normal1 = new float3[m_max_triangle]();
    m_host_triangle_normal2 = new float3[m_max_triangle]();
    for (uint x = 0; x < m_row_dens; x++)
        for (uint y = 0; y < m_col_dens; y++)
            for (uint z = 0; z < m_len_dens; z++) {
                const uint g = z * m_row_dens * m_col_dens + y * m_row_dens + x;
                m_host_dens_pos[g] = make_float3((float)x * m_den_size, (float)y * m_den_size, (float)z * m_den_size);
            }
    Sphere *sp[4] = {&m_sphere1, &m_sphere2, &m_sphere3, &m_sphere4};
    for (int q = 0; q < 4; ++q) {
        const int k = q < 3 ? q : 2;
        sp[q]->pos = make_float3(m_cfg.sphere[k].pos[0], m_cfg.sphere[k].pos[1], m_cfg.sphere[k].pos[2]);
        sp[q]->radius = q < 3 ? m_cfg.sphere[k].radius : 0.0f;
        sp[q]->damping = m_cfg.sphere[k].damping;
    }
    m_host_param = new SysParam();
    m_host_param->gravity = m_gravity;
    m_host_param->wall_damping = m_wall_damping;
    m_host_param->rest_density = m_rest_density;
    m_host_param->gas_constant = m_gas_constant;
    m_host_param->time_step = m_time_step;
    m_host_param->viscosity = m_viscosity;
    m_host_param->surface_tension = m_surface_tension;
    m_host_param->co_surface = m_co_surface;
    m_host_param->co_energy = m_co_energy;
    m_host_param->split_criteria = m_split_criteria;
    m_host_param->merge_criteria = m_merge_criteria;
    m_host_param->sphere1 = m_sphere1;
    m_host_param->sphere2 = m_sphere2;
    m_host_param->sphere3 = m_sphere3;
    m_host_param->sphere4 = m_sphere4;
    m_host_param->split_energy = 0.8f;   // SPH-3D-2/sph_system.cpp:198-199
    m_host_param->merge_energy = 0.02f;
#if SCA2012_VARIANT == 34
    m_host_param->force_waiting_left = false;
    m_host_param->force_waiting_right = false;
#else
    m_host_param->force_waiting = false;
#endif
    m_host_param->use_cylinder = false;
    m_sys_running = 0;
    m_trans_once = 0;
    m_use_split = 0;
    m_use_merge = 0;
    m_disp_mode = 1;
    m_status = sph_create(&m_cfg, &m_h);
    report(m_status, "sph_create", m_h);
}

SPHSystem::~SPHSystem()
{
    if (m_h) sph_destroy(m_h);
    delete[] m_host_mem;
    delete[] m_host_dens;
    delete[] m_host_dens_pos;
    delete[] m_host_dens_normal;
    delete[] m_host_line0;
    delete[] m_host_line1;
    delete[] m_host_triangle0;
    delete[] m_host_triangle1;
    delete[] m_host_triangle2;
    delete[] m_host_triangle_normal0;
    delete[] m_host_triangle_normal1;
    delete[] m_host_triangle_normal2;
    delete m_host_param;
}

void SPHSystem::add_particle(float3 pos, float3 vel, uint level)
{
    // SPH-3D-2/sph_system.cpp:285-300
    Particle *p = &m_host_mem[m_num_particle];
    p->pos = pos;
    p->vel = vel;
    p->ev = make_float3(0.0f, 0.0f, 0.0f);
    p->acc = make_float3(0.0f, 0.0f, 0.0f);
    p->dens = 0.0f;
    p->press = 0.0f;
    p->energy = 0.0f;
    p->surface = 0.0f;
    p->tension = 0.0f;
    p->level = level;
    m_num_particle++;
}

void SPHSystem::add_box_particle()
{
    float3 pos;
    const float3 vel = make_float3(0.0f, 0.0f, 0.0f);
#if SCA2012_VARIANT == 34
    // SPH-3D-4/sph_system.cpp:270-289: level-2 slab of height H/4
    const float space = m_small_kernel;
    for (pos.x = space; m_world_width - pos.x >= space; pos.x += space * 0.5f)
        for (pos.y = space; pos.y < m_world_height / 4; pos.y += space * 0.5f)
            for (pos.z = space; m_world_length - pos.z >= space; pos.z += space * 0.5f)
                add_particle(pos, vel, 2);
#else
    // SPH-3D-2/sph_system.cpp:247-264: level-1 block in the left half
    for (pos.x = m_large_kernel / 2.0f; pos.x <= m_world_width / 2; pos.x += m_large_kernel * 0.8f)
        for (pos.y = m_large_kernel / 2.0f; m_world_height - pos.y >= m_large_kernel / 2.0f;
             pos.y += m_large_kernel * 0.8f)
            for (pos.z = m_large_kernel / 2.0f; m_world_length - pos.z >= m_large_kernel / 2.0f;
                 pos.z += m_large_kernel * 0.8f)
                add_particle(pos, vel, 1);
#endif
    upload_if_needed();
}

void SPHSystem::add_new_particle()
{
#if SCA2012_VARIANT == 34
    // SPH-3D-4/sph_system.cpp:291-332: sphere of radius 5 at (24, 18, 12), v = (0, -10, 0)
    const float r = 10.0f, spacing = m_small_kernel * 0.5f;
    const float3 vel = make_float3(0.0f, -10.0f, 0.0f);
    for (float z = -r; z <= r; z += spacing)
        for (float y = -r; y <= r; y += spacing)
            for (float x = -r; x <= r; x += spacing)
                if (sqrtf(x * x + y * y + z * z) <= 5.0f)
                    add_particle(make_float3(24.0f + x, 18.0f + y, 12.0f + z), vel, 2);
#else
    // SPH-3D-2/sph_system.cpp:266-283: level-2 block 4 units in from the walls
    float3 pos;
    const float3 vel = make_float3(0.0f, 0.0f, 0.0f);
    for (pos.x = m_large_kernel / 2.0f + 4; m_world_width - 4 - pos.x >= m_large_kernel / 2.0f;
         pos.x += m_small_kernel * 0.4f)
        for (pos.y = m_large_kernel / 2.0f + 4; m_world_height - 4 - pos.y >= m_large_kernel / 2.0f;
             pos.y += m_small_kernel * 0.4f)
            for (pos.z = m_large_kernel / 2.0f + 4; m_world_length - 4 - pos.z >= m_large_kernel / 2.0f;
                 pos.z += m_small_kernel * 0.4f)
                add_particle(pos, vel, 2);
#endif
    upload_if_needed();
}

void SPHSystem::upload_if_needed()
{
    if (!m_h || m_uploaded == m_num_particle) return;
    m_status = sph_write_particles(m_h, m_host_mem, m_num_particle);
    report(m_status, "sph_write_particles", m_h);
    m_uploaded = m_num_particle;
}

void SPHSystem::apply_params()
{
    const SysParam &p = *m_host_param;
    m_cfg.use_split = m_use_split;
    m_cfg.use_merge = m_use_merge;
    m_cfg.grid_every = m_disp_mode == 2 ? 1u : 0u;
    m_cfg.gravity[0] = p.gravity.x;
    m_cfg.gravity[1] = p.gravity.y;
    m_cfg.gravity[2] = p.gravity.z;
    m_cfg.wall_damping = p.wall_damping;
    m_cfg.rest_density = p.rest_density;
    m_cfg.gas_constant = p.gas_constant;
    m_cfg.time_step = p.time_step;
    m_cfg.viscosity = p.viscosity;
    m_cfg.surface_threshold = p.surface_tension;
    m_cfg.co_surface = p.co_surface;
    m_cfg.co_energy = p.co_energy;
    m_cfg.split_criteria = p.split_criteria;
    m_cfg.merge_criteria = p.merge_criteria;
    const Sphere *sp[3] = {&p.sphere1, &p.sphere2, &p.sphere3};
    for (int q = 0; q < 3; ++q) {
        m_cfg.sphere[q].pos[0] = sp[q]->pos.x;
        m_cfg.sphere[q].pos[1] = sp[q]->pos.y;
        m_cfg.sphere[q].pos[2] = sp[q]->pos.z;
        m_cfg.sphere[q].radius = sp[q]->radius;
        m_cfg.sphere[q].damping = sp[q]->damping;
    }
    m_cfg.use_cylinder = p.use_cylinder ? 1u : 0u;
#if SCA2012_VARIANT == 34
    m_cfg.push_left = p.force_waiting_left ? 1u : 0u;
    m_cfg.push_right = p.force_waiting_right ? 1u : 0u;
#else
    m_cfg.push_left = p.force_waiting ? 1u : 0u;
    m_cfg.push_right = 0u;
#endif
}

void SPHSystem::animation()
{
    // SPH-3D-2/sph_system.cpp:302-404
    if (m_sys_running == 0 || !m_h) return;
    apply_params();
    m_status = sph_set_config(m_h, &m_cfg);
    if (m_status) return report(m_status, "sph_set_config", m_h);
    upload_if_needed();
    m_status = sph_step(m_h, 1);
    if (m_status) return report(m_status, "sph_step", m_h);
    m_status = sph_read_particles(m_h, m_host_mem, (uint64_t)sizeof(Particle) * m_max_particle, &m_num_particle);
    report(m_status, "sph_read_particles", m_h);
    m_uploaded = m_num_particle;
    if (m_disp_mode == 2) {
        m_status = sph_density_grid(m_h, m_host_dens, &m_host_dens_normal[0].x);
        report(m_status, "sph_density_grid", m_h);
        sph_mesh_view mesh = {m_max_triangle, 0, &m_host_triangle0[0].x, &m_host_triangle1[0].x,
                              &m_host_triangle2[0].x, &m_host_triangle_normal0[0].x,
                              &m_host_triangle_normal1[0].x, &m_host_triangle_normal2[0].x};
        m_status = sph_extract_surface(m_h, &mesh);
        m_num_triangle = mesh.num_triangles < m_max_triangle ? mesh.num_triangles : m_max_triangle;
    }
#if SCA2012_VARIANT == 34
    m_host_param->force_waiting_left = false;
    m_host_param->force_waiting_right = false;
#else
    m_host_param->force_waiting = false;
#endif
}

void SPHSystem::marching_cube()
{
    // SPH-3D-2/sph_system.cpp:517-542, on the device from the host grid
    if (!m_h) return;
    sph_mesh_view mesh = {m_max_triangle, 0, &m_host_triangle0[0].x, &m_host_triangle1[0].x,
                          &m_host_triangle2[0].x, &m_host_triangle_normal0[0].x,
                          &m_host_triangle_normal1[0].x, &m_host_triangle_normal2[0].x};
    m_status = sph_surface_from_grid(m_h, m_host_dens, &m_host_dens_normal[0].x, &mesh);
    m_num_triangle = mesh.num_triangles < m_max_triangle ? mesh.num_triangles : m_max_triangle;
    m_num_lines = 0;
}
#endif
