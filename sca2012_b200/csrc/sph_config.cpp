// sph_config.cpp — parameter presets for the C-ABI (host code).
//
// The three reference presets reproduce the constants the reference
// constructors compute (SPH-2D/sph_system.cpp:5-146, SPH-3D-2/sph_system.cpp:6-229,
// SPH-3D-4/sph_system.cpp:6-229) with the same host arithmetic: PI is the
// truncated float 3.141592f (sph_header.h:21-22), 64.0f*PI is a float product,
// pow() runs in double and the result is stored to float.  The SI presets are
// the synthetic dam-break workloads (2D plain, 3D two-way, 3D four-way at 1.1M
// particles, 32^3 rollout); their choices are listed next to each value.
#include "../../include/sph/sph.h"

#include <cmath>
#include <cstring>

namespace {

constexpr float kPI = 3.141592f;  // reference PI (sph_header.h)

// Coefficients exactly as the reference computes them (float(PI) products,
// double pow, assignment to float).
struct RefCoef {
    float poly6, spiky, visco, grad, lapc, k2, k6;
};

RefCoef ref_coef(float h)
{
    RefCoef c;
    c.poly6 = (float)(315.0f / ((double)(64.0f * kPI) * std::pow((double)h, 9)));
    c.spiky = (float)(-45.0f / ((double)kPI * std::pow((double)h, 6)));
    c.visco = (float)(45.0f / ((double)kPI * std::pow((double)h, 6)));
    c.grad = (float)(-945.0f / ((double)(32.0f * kPI) * std::pow((double)h, 9)));
    c.lapc = (float)(-945.0f / ((double)(8.0f * kPI) * std::pow((double)h, 9)));
    c.k2 = h * h;
    c.k6 = (float)std::pow((double)h, 6);
    return c;
}

float ref_poly6_radius(float r) { return (float)(315.0f / ((double)(64.0f * kPI) * std::pow((double)r, 9))); }

void set_level(sph_config *c, int l, float mass, float h, float radius)
{
    RefCoef k = ref_coef(h);
    c->mass[l] = mass;
    c->kernel[l] = h;
    c->kernel2[l] = k.k2;
    c->kernel6[l] = k.k6;
    c->radius[l] = radius;
    c->poly6[l] = k.poly6;
    c->spiky[l] = k.spiky;
    c->visco[l] = k.visco;
    c->grad_poly6[l] = k.grad;
    c->lapc_poly6[l] = k.lapc;
    c->poly6_radius[l] = ref_poly6_radius(radius);
}

// Grid from a world size and cell edge: ncell = ceil(W / cell), then the
// world is snapped to ncell*cell (SPH-3D-2/sph_system.cpp:24-32).
void set_grid(sph_config *c, float wx, float wy, float wz, float cell)
{
    c->cell_size = cell;
    c->ncell[0] = (uint32_t)std::ceil(wx / cell);
    c->ncell[1] = (uint32_t)std::ceil(wy / cell);
    c->ncell[2] = c->dim == 3 ? (uint32_t)std::ceil(wz / cell) : 1u;
    c->world[0] = c->ncell[0] * cell;
    c->world[1] = c->ncell[1] * cell;
    c->world[2] = c->dim == 3 ? c->ncell[2] * cell : 0.0f;
}

void set_mc_grid(sph_config *c, uint32_t mul)
{
    c->dens_mul = mul;
    c->den_size = c->cell_size / mul;   // SPH-3D-2/sph_system.cpp:86-92
    c->ndens[0] = c->ncell[0] * mul + 1;
    c->ndens[1] = c->ncell[1] * mul + 1;
    c->ndens[2] = c->dim == 3 ? c->ncell[2] * mul + 1 : 1u;
}

void ref_spheres(sph_config *c)
{
    // SPH-3D-2/sph_system.cpp:116-126
    const float p[3][3] = {{11.0f, 3.0f, 4.0f}, {11.0f, 3.0f, 12.0f}, {18.0f, 3.0f, 8.0f}};
    for (int q = 0; q < 3; ++q) {
        for (int a = 0; a < 3; ++a) c->sphere[q].pos[a] = p[q][a];
        c->sphere[q].radius = 2.0f;
        c->sphere[q].damping = 1.0f;
    }
}

void preset_ref_3d(sph_config *c, bool four_way)
{
    c->dim = 3;
    c->max_particle = 1000000;
    if (!four_way) {
        set_grid(c, 32, 16, 16, 1.0f);
        set_level(c, 0, 1.0f, 1.0f, 1.0f);
        set_level(c, 1, 0.5f, 0.9f, 0.8f);
        c->gravity[1] = -5.0f;
        c->rest_density = 1.0f;
        c->viscosity = 3.0f;
        c->co_surface = 1.0f;
        c->split_criteria = 1.2f;
        c->merge_criteria = 0.4f;
        c->surface_coef = 0.1f;     // SPH-3D-2/sph_system.cu:1129
        c->split_ways = 2;
        c->push_y_div = 5;          // SPH-3D-2/sph_system.cu:231
    } else {
        set_grid(c, 48, 24, 24, 1.2f);
        set_level(c, 0, 1.0f, 1.2f, 1.2f);
        set_level(c, 1, 0.25f, 1.0f, 0.8f);
        c->gravity[1] = -4.0f;
        c->rest_density = 0.5f;
        c->viscosity = 1.0f;
        c->co_surface = 1.5f;
        c->split_criteria = 1.0f;
        c->merge_criteria = 0.6f;
        c->surface_coef = 0.02f;    // SPH-3D-4/sph_system.cu:1136
        c->split_ways = 4;
        c->energy_mass_weight = 1;  // SPH-3D-4/sph_system.cu:1528
        c->push_y_div = 10;         // SPH-3D-4/sph_system.cu:231,238
    }
    c->wall_damping = -0.6f;
    c->gas_constant = 1.0f;
    c->time_step = 0.1f;
    c->surface_threshold = 0.8f;
    c->co_energy = 1.0f;
    c->density_skip_r2 = 0.0001f;
    c->close_r2 = 0.0001f;          // sph_system.cu:801-804, :1229-1232
    c->lapc_three_quarters = 0.0f;  // integer 3/4 (sph_system.cu:828)
    c->integrator = SPH_INTEGRATE_REF3D;
    c->kernel_h6_twice = 1;
    c->energy_large_kernel = 1;
    c->energy_skip_close = 1;
    c->split_rule = SPH_SPLIT_WAVELET;
    c->merge_rule = SPH_MERGE_WAVELET;
    c->split_copies_fields = 0;
    ref_spheres(c);
    set_mc_grid(c, 4);
    c->iso_value = 0.5f;            // ISOVALUE (sph_header.h:24)
    c->mc_interpolate = 0;
}

void preset_ref_2d(sph_config *c)
{
    // SPH-2D/sph_system.cpp:5-146
    c->dim = 2;
    c->max_particle = 100000;
    set_grid(c, 32.0f, 32.0f, 0.0f, 1.0f);
    set_level(c, 0, 1.0f, 1.0f, 1.0f);
    set_level(c, 1, 0.5f, 0.9f, 0.8f);
    c->gravity[1] = -4.5f;
    c->wall_damping = -0.6f;
    c->rest_density = 2.0f;
    c->gas_constant = 1.0f;
    c->viscosity = 2.0f;
    c->time_step = 0.1f;
    c->surface_threshold = 0.5f;    // m_surface_normal
    c->surface_coef = 0.04f;        // SPH-2D/sph_system.cu:770
    c->co_surface = 0.8f;
    c->co_energy = 1.0f;
    c->split_criteria = 0.7f;       // m_thresh_split
    c->merge_criteria = 0.04f;      // m_thresh_merge
    c->density_skip_r2 = 1e-12f;    // EXT2 (SPH-2D/sph_system.cu:8,396)
    c->close_r2 = 0.0001f;          // force loop (SPH-2D/sph_system.cu:584)
    c->lapc_three_quarters = 0.0f;
    c->split_ways = 2;
    c->integrator = SPH_INTEGRATE_REF2D;
    c->kernel_h6_twice = 1;
    c->energy_large_kernel = 0;     // own level (SPH-2D/sph_system.cu:867-877)
    c->energy_skip_close = 0;       // clamps r2 instead (SPH-2D/sph_system.cu:895-898)
    c->split_rule = SPH_SPLIT_WAVELET;
    c->merge_rule = SPH_MERGE_WAVELET_CELL;
    c->split_copies_fields = 1;
    c->extern_len = 2.0f;
    c->extern_coe = 1.0f;
}

// ---- SI-unit synthetic workloads -------------------------------------------
// rho0 = 1000, h = 2s, cell = h, k = 3, mu = 0.1, walls reflect with 0.5.
// Kernels carry their physical normalisation and are not divided by h^6 a
// second time; the integrator divides forces by mass; surface tension is off
// (the workloads name none).  Level 2 has mass m/w and h/w^(1/d) for a w-way
// split, radius (the wall margin) is s/2 scaled the same way.
void set_level_si(sph_config *c, int l, float mass, float h, float radius)
{
    c->mass[l] = mass;
    c->kernel[l] = h;
    c->kernel2[l] = h * h;
    c->kernel6[l] = (float)std::pow((double)h, 6);
    c->radius[l] = radius;
    const double pi = 3.14159265358979323846, hd = h;
    if (c->dim == 3) {
        c->poly6[l] = (float)(315.0 / (64.0 * pi * std::pow(hd, 9)));
        c->spiky[l] = (float)(-45.0 / (pi * std::pow(hd, 6)));
        c->visco[l] = (float)(45.0 / (pi * std::pow(hd, 6)));
        c->grad_poly6[l] = (float)(-945.0 / (32.0 * pi * std::pow(hd, 9)));
        c->lapc_poly6[l] = (float)(-945.0 / (8.0 * pi * std::pow(hd, 9)));
    } else {
        c->poly6[l] = (float)(4.0 / (pi * std::pow(hd, 8)));
        c->spiky[l] = (float)(-30.0 / (pi * std::pow(hd, 5)));
        c->visco[l] = (float)(40.0 / (pi * std::pow(hd, 5)));
        c->grad_poly6[l] = (float)(-24.0 / (pi * std::pow(hd, 8)));
        c->lapc_poly6[l] = (float)(-48.0 / (pi * std::pow(hd, 8)));
    }
    double rr = radius;
    c->poly6_radius[l] = c->dim == 3 ? (float)(315.0 / (64.0 * pi * std::pow(rr, 9)))
                                     : (float)(4.0 / (pi * std::pow(rr, 8)));
}

void preset_si(sph_config *c, int dim, float s, uint32_t ways, float dt)
{
    c->dim = (uint32_t)dim;
    const float h = 2.0f * s;
    const float m = dim == 3 ? 1000.0f * s * s * s : 1000.0f * s * s;
    const float shrink = (float)std::pow((double)ways, -1.0 / dim);
    set_level_si(c, 0, m, h, 0.5f * s);
    set_level_si(c, 1, m / ways, h * shrink, 0.5f * s * shrink);
    c->gravity[0] = 0.0f;
    c->gravity[1] = -9.8f;
    c->gravity[2] = 0.0f;
    c->wall_damping = -0.5f;
    c->rest_density = 1000.0f;
    c->gas_constant = 3.0f;
    c->time_step = dt;
    c->viscosity = 0.1f;
    c->surface_threshold = 0.0f;
    c->surface_coef = 0.0f;
    c->co_surface = 0.0f;
    c->co_energy = 0.0f;
    c->density_skip_r2 = 0.0f;
    // the reference's 1e-4 is a length of its own units (h ~ 1); at h = 2s
    // in metres it would drop every pair inside 0.01 m.  Only (nearly)
    // coincident pairs are skipped here.
    c->close_r2 = (1e-3f * h) * (1e-3f * h);
    c->lapc_three_quarters = 0.75f;
    c->split_ways = ways;
    c->integrator = SPH_INTEGRATE_PHYS;
    c->kernel_h6_twice = 0;
    c->energy_large_kernel = 1;
    c->energy_skip_close = 1;
    c->split_rule = SPH_SPLIT_DEFICIT;
    // a split group merges back when all its members have been interior for
    // merge_interior_steps steps (the configs' "children merge back")
    c->merge_rule = SPH_MERGE_SIBLING;
    // A particle on the simple-cubic lattice at spacing s has 26 neighbours
    // with r < 2s (|d|^2 in {1,2,3}); a free-surface particle keeps at most 17.
    // Fewer than 20 flags a deficit (2D: 12 interior, <= 8 at a face -> < 9).
    c->split_min_neighbors = dim == 3 ? 20u : 9u;
    c->split_density_ratio = 0.9f;
    c->merge_interior_steps = 50;
    c->split_copies_fields = 1;
    c->iso_value = 0.5f * 1000.0f;   // iso-level 0.5 * rest density
    c->mc_interpolate = 1;
    c->splat_with_kernel = 1;        // grid density ~ SPH density, so the iso value means 0.5 rho0
    c->max_triangles = 2000000;
}

}  // namespace

extern "C" size_t sph_config_size(void) { return sizeof(sph_config); }

extern "C" int sph_config_preset(int preset, sph_config *c)
{
    if (!c) return SPH_ERR_INVALID;
    std::memset(c, 0, sizeof(*c));
    switch (preset) {
    case SPH_PRESET_REF_2D: preset_ref_2d(c); return SPH_OK;
    case SPH_PRESET_REF_3D2: preset_ref_3d(c, false); return SPH_OK;
    case SPH_PRESET_REF_3D4: preset_ref_3d(c, true); return SPH_OK;
    case SPH_PRESET_DAM_2D:
        // 64x64 block at s = 0.01 in a 1.28 x 1.28 box, dt = 1e-4, no adaptivity
        preset_si(c, 2, 0.01f, 2, 1e-4f);
        set_grid(c, 1.28f, 1.28f, 0.0f, c->kernel[0]);
        c->max_particle = 4096;
        c->use_split = 0;
        c->use_merge = 0;
        return SPH_OK;
    case SPH_PRESET_DAM_3D2:
        // 64x64x32 block at s = 0.01 in 1.28 x 0.64 x 0.64, dt = 5e-5, two-way
        preset_si(c, 3, 0.01f, 2, 5e-5f);
        set_grid(c, 1.28f, 0.64f, 0.64f, c->kernel[0]);
        c->max_particle = 131072 * 4;
        c->use_split = 1;
        c->use_merge = 1;
        set_mc_grid(c, 2);
        return SPH_OK;
    case SPH_PRESET_DAM_3D4:
        // 128x128x64 block at s = 0.005 + a 65536-particle sphere in
        // 1.28 x 1.28 x 0.64 (128 x 128 x 64 cells of h = 0.01), dt = 2.5e-5,
        // four-way.  Capacity 4 x the initial count.
        preset_si(c, 3, 0.005f, 4, 2.5e-5f);
        set_grid(c, 1.28f, 1.28f, 0.64f, c->kernel[0]);
        c->max_particle = 1114112u * 4u;
        c->use_split = 1;
        c->use_merge = 1;
        set_mc_grid(c, 2);   // 257 x 257 x 129 nodes at 0.005
        c->grid_every = 10;  // marching cubes every 10 steps
        return SPH_OK;
    case SPH_PRESET_ROLLOUT_3D:
        // 32^3 block at s = 0.01 in 0.64^3, two-way; compensated positions
        // keep the FP32 trajectory within the rounding of a few steps
        preset_si(c, 3, 0.01f, 2, 5e-5f);
        set_grid(c, 0.64f, 0.64f, 0.64f, c->kernel[0]);
        c->max_particle = 32768 * 4;
        c->use_split = 1;
        c->use_merge = 1;
        c->compensated_positions = 1;
        set_mc_grid(c, 1);
        return SPH_OK;
    default:
        return SPH_ERR_INVALID;
    }
}
