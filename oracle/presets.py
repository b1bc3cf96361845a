"""Parameter presets restated for the oracle side (TEST INFRASTRUCTURE).

The CPU reference arm of the benchmark and the tests build their sph_config
from here, so that timing the oracle never loads the CUDA library.  Every
value is computed the way the reference constructors compute it, in float32
where they use float and in double where they call pow():

  REF_2D   SPH-2D/sph_system.cpp:5-146
  REF_3D2  SPH-3D-2/sph_system.cpp:6-229   (coefficients :63-84, PI = 3.141592f,
                                            SPH-3D-2/sph_header.h:22)
  REF_3D4  SPH-3D-4/sph_system.cpp:6-229

and the SI dam-break workloads (2D plain, 3D two-way, 3D four-way at 1.1M
particles, 32^3 rollout) with the choices of the library's presets.
tests/test_presets.py checks every preset byte for byte against the
library's sph_config_preset.
"""
import ctypes as C
import math

import numpy as np

from . import oracle as _O

f32 = np.float32
PI_REF = f32(3.141592)   # the reference's truncated PI

PRESET_REF_2D, PRESET_REF_3D2, PRESET_REF_3D4 = 0, 1, 2
PRESET_DAM_2D, PRESET_DAM_3D2, PRESET_DAM_3D4, PRESET_ROLLOUT_3D = 3, 4, 5, 6


def _f(x):
    return float(f32(x))


def _ref_coef(h):
    """Kernel coefficients as the reference constructor forms them: a float
    product n*PI, a double pow, the quotient in double, stored to float."""
    h = float(f32(h))
    pi64 = float(f32(64.0) * PI_REF)
    pi32 = float(f32(32.0) * PI_REF)
    pi8 = float(f32(8.0) * PI_REF)
    pi = float(PI_REF)
    return dict(poly6=_f(315.0 / (pi64 * math.pow(h, 9))), spiky=_f(-45.0 / (pi * math.pow(h, 6))),
                visco=_f(45.0 / (pi * math.pow(h, 6))), grad=_f(-945.0 / (pi32 * math.pow(h, 9))),
                lapc=_f(-945.0 / (pi8 * math.pow(h, 9))), k2=_f(f32(h) * f32(h)), k6=_f(math.pow(h, 6)))


def _set_level_ref(c, lvl, mass, h, radius):
    k = _ref_coef(h)
    c.mass[lvl], c.kernel[lvl], c.radius[lvl] = _f(mass), _f(h), _f(radius)
    c.kernel2[lvl], c.kernel6[lvl] = k["k2"], k["k6"]
    c.poly6[lvl], c.spiky[lvl], c.visco[lvl] = k["poly6"], k["spiky"], k["visco"]
    c.grad_poly6[lvl], c.lapc_poly6[lvl] = k["grad"], k["lapc"]
    c.poly6_radius[lvl] = _ref_coef(radius)["poly6"]


def _set_grid(c, w, cell):
    """ncell = ceil(W / cell) per axis in float, world = ncell * cell
    (SPH-3D-2/sph_system.cpp:24-32)."""
    cell = f32(cell)
    c.cell_size = float(cell)
    for a in range(3):
        if a == 2 and c.dim != 3:
            c.ncell[2], c.world[2] = 1, 0.0
            continue
        n = int(math.ceil(float(f32(w[a]) / cell)))
        c.ncell[a] = n
        c.world[a] = _f(f32(n) * cell)


def _set_mc_grid(c, mul):
    c.dens_mul = mul
    c.den_size = _f(f32(c.cell_size) / f32(mul))   # SPH-3D-2/sph_system.cpp:86-92
    c.ndens[0] = c.ncell[0] * mul + 1
    c.ndens[1] = c.ncell[1] * mul + 1
    c.ndens[2] = c.ncell[2] * mul + 1 if c.dim == 3 else 1


def _ref_3d(c, four_way):
    c.dim = 3
    c.max_particle = 1000000
    if not four_way:   # SPH-3D-2/sph_system.cpp:6-229
        _set_grid(c, (32, 16, 16), 1.0)
        _set_level_ref(c, 0, 1.0, 1.0, 1.0)
        _set_level_ref(c, 1, 0.5, 0.9, 0.8)
        c.gravity[1] = -5.0
        c.rest_density, c.viscosity, c.co_surface = 1.0, 3.0, 1.0
        c.split_criteria, c.merge_criteria = _f(1.2), _f(0.4)
        c.surface_coef = _f(0.1)           # SPH-3D-2/sph_system.cu:1129
        c.split_ways, c.push_y_div = 2, 5  # SPH-3D-2/sph_system.cu:231
    else:              # SPH-3D-4/sph_system.cpp:6-229
        _set_grid(c, (48, 24, 24), 1.2)
        _set_level_ref(c, 0, 1.0, 1.2, 1.2)
        _set_level_ref(c, 1, 0.25, 1.0, 0.8)
        c.gravity[1] = -4.0
        c.rest_density, c.viscosity, c.co_surface = 0.5, 1.0, 1.5
        c.split_criteria, c.merge_criteria = 1.0, _f(0.6)
        c.surface_coef = _f(0.02)          # SPH-3D-4/sph_system.cu:1136
        c.split_ways, c.energy_mass_weight, c.push_y_div = 4, 1, 10
    c.wall_damping, c.gas_constant, c.time_step = _f(-0.6), 1.0, _f(0.1)
    c.surface_threshold, c.co_energy = _f(0.8), 1.0
    c.density_skip_r2 = c.close_r2 = _f(0.0001)   # sph_system.cu:801-804, :1229-1232
    c.lapc_three_quarters = 0.0                    # integer 3/4 (sph_system.cu:828)
    c.integrator = 0          # SPH_INTEGRATE_REF3D
    c.kernel_h6_twice = c.energy_large_kernel = c.energy_skip_close = 1
    c.split_rule = c.merge_rule = 0
    c.split_copies_fields = 0
    for q, p in enumerate(((11.0, 3.0, 4.0), (11.0, 3.0, 12.0), (18.0, 3.0, 8.0))):   # :116-126
        for a in range(3):
            c.sphere[q].pos[a] = p[a]
        c.sphere[q].radius, c.sphere[q].damping = 2.0, 1.0
    _set_mc_grid(c, 4)
    c.iso_value = 0.5          # ISOVALUE (sph_header.h:24)
    c.mc_interpolate = 0


def _ref_2d(c):
    # SPH-2D/sph_system.cpp:5-146
    c.dim = 2
    c.max_particle = 100000
    _set_grid(c, (32.0, 32.0, 0.0), 1.0)
    _set_level_ref(c, 0, 1.0, 1.0, 1.0)
    _set_level_ref(c, 1, 0.5, 0.9, 0.8)
    c.gravity[1] = -4.5
    c.wall_damping, c.rest_density, c.gas_constant, c.viscosity = _f(-0.6), 2.0, 1.0, 2.0
    c.time_step, c.surface_threshold, c.surface_coef = _f(0.1), 0.5, _f(0.04)   # :770
    c.co_surface, c.co_energy = _f(0.8), 1.0
    c.split_criteria, c.merge_criteria = _f(0.7), _f(0.04)
    c.density_skip_r2 = _f(1e-12)   # EXT2 (SPH-2D/sph_system.cu:8,396)
    c.close_r2 = _f(0.0001)         # SPH-2D/sph_system.cu:584
    c.lapc_three_quarters = 0.0
    c.split_ways = 2
    c.integrator = 1                # SPH_INTEGRATE_REF2D
    c.kernel_h6_twice = 1
    c.energy_large_kernel = c.energy_skip_close = 0
    c.split_rule, c.merge_rule = 0, 1   # SPH_MERGE_WAVELET_CELL
    c.split_copies_fields = 1
    c.extern_len, c.extern_coe = 2.0, 1.0


def _set_level_si(c, lvl, mass, h, radius):
    """Physically normalised kernels at kernel length h (double arithmetic,
    stored to float): 3D poly6 315/(64 pi h^9), spiky -45/(pi h^6), viscosity
    45/(pi h^6); 2D poly6 4/(pi h^8), spiky -30/(pi h^5), viscosity 40/(pi h^5)."""
    h, radius = float(f32(h)), float(f32(radius))
    c.mass[lvl], c.kernel[lvl], c.radius[lvl] = _f(mass), h, radius
    c.kernel2[lvl] = _f(f32(h) * f32(h))
    c.kernel6[lvl] = _f(math.pow(h, 6))
    pi = math.pi
    if c.dim == 3:
        c.poly6[lvl] = _f(315.0 / (64.0 * pi * math.pow(h, 9)))
        c.spiky[lvl] = _f(-45.0 / (pi * math.pow(h, 6)))
        c.visco[lvl] = _f(45.0 / (pi * math.pow(h, 6)))
        c.grad_poly6[lvl] = _f(-945.0 / (32.0 * pi * math.pow(h, 9)))
        c.lapc_poly6[lvl] = _f(-945.0 / (8.0 * pi * math.pow(h, 9)))
        c.poly6_radius[lvl] = _f(315.0 / (64.0 * pi * math.pow(radius, 9)))
    else:
        c.poly6[lvl] = _f(4.0 / (pi * math.pow(h, 8)))
        c.spiky[lvl] = _f(-30.0 / (pi * math.pow(h, 5)))
        c.visco[lvl] = _f(40.0 / (pi * math.pow(h, 5)))
        c.grad_poly6[lvl] = _f(-24.0 / (pi * math.pow(h, 8)))
        c.lapc_poly6[lvl] = _f(-48.0 / (pi * math.pow(h, 8)))
        c.poly6_radius[lvl] = _f(4.0 / (pi * math.pow(radius, 8)))


def _si(c, dim, s, ways, dt):
    """rho0 = 1000, h = 2s, k = 3, mu = 0.1, walls reflecting with 0.5; level 2
    has mass m/w and h, wall margin scaled by w^(-1/dim) for a w-way split."""
    c.dim = dim
    s = f32(s)
    h = f32(2.0) * s
    m = f32(1000.0) * s * s * s if dim == 3 else f32(1000.0) * s * s
    shrink = f32(math.pow(float(ways), -1.0 / dim))
    half_s = f32(0.5) * s
    _set_level_si(c, 0, m, h, half_s)
    _set_level_si(c, 1, m / f32(ways), h * shrink, half_s * shrink)
    c.gravity[0], c.gravity[1], c.gravity[2] = 0.0, _f(-9.8), 0.0
    c.wall_damping, c.rest_density, c.gas_constant = -0.5, 1000.0, 3.0
    c.time_step, c.viscosity = _f(dt), _f(0.1)
    c.surface_threshold = c.surface_coef = c.co_surface = c.co_energy = 0.0
    c.density_skip_r2 = 0.0
    c.close_r2 = _f((f32(1e-3) * h) * (f32(1e-3) * h))
    c.lapc_three_quarters = 0.75
    c.split_ways = ways
    c.integrator = 2                 # SPH_INTEGRATE_PHYS
    c.kernel_h6_twice = 0
    c.energy_large_kernel = c.energy_skip_close = 1
    c.split_rule, c.merge_rule = 1, 3   # SPH_SPLIT_DEFICIT, SPH_MERGE_SIBLING
    c.split_min_neighbors = 20 if dim == 3 else 9
    c.split_density_ratio = _f(0.9)
    c.merge_interior_steps = 50
    c.split_copies_fields = 1
    c.iso_value = 500.0              # 0.5 * rest density
    c.mc_interpolate = c.splat_with_kernel = 1
    c.max_triangles = 2000000


def preset(which):
    """sph_config of preset `which`, as a ctypes struct of sph.h's layout."""
    c = _O.abi().Config()
    C.memset(C.byref(c), 0, C.sizeof(c))
    if which == PRESET_REF_2D:
        _ref_2d(c)
    elif which == PRESET_REF_3D2:
        _ref_3d(c, False)
    elif which == PRESET_REF_3D4:
        _ref_3d(c, True)
    elif which == PRESET_DAM_2D:
        _si(c, 2, 0.01, 2, 1e-4)
        _set_grid(c, (1.28, 1.28, 0.0), c.kernel[0])
        c.max_particle = 4096
        c.use_split = c.use_merge = 0
    elif which == PRESET_DAM_3D2:
        _si(c, 3, 0.01, 2, 5e-5)
        _set_grid(c, (1.28, 0.64, 0.64), c.kernel[0])
        c.max_particle = 131072 * 4
        c.use_split = c.use_merge = 1
        _set_mc_grid(c, 2)
    elif which == PRESET_DAM_3D4:
        _si(c, 3, 0.005, 4, 2.5e-5)
        _set_grid(c, (1.28, 1.28, 0.64), c.kernel[0])
        c.max_particle = 1114112 * 4
        c.use_split = c.use_merge = 1
        _set_mc_grid(c, 2)
        c.grid_every = 10
    elif which == PRESET_ROLLOUT_3D:
        _si(c, 3, 0.01, 2, 5e-5)
        _set_grid(c, (0.64, 0.64, 0.64), c.kernel[0])
        c.max_particle = 32768 * 4
        c.use_split = c.use_merge = 1
        c.compensated_positions = 1
        _set_mc_grid(c, 1)
    else:
        raise ValueError(f"unknown preset {which}")
    return c
