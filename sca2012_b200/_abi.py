"""ctypes mirror of include/sph/sph.h (the C-ABI of the adaptive SPH step).

Field order and types follow the C structs exactly; `load()` checks
sizeof(sph_config) against the library so a layout drift fails loudly.
"""
import ctypes as C
import os

SPH_OK = 0
SPH_ERR_INVALID = 1
SPH_ERR_CAPACITY = 2
SPH_ERR_CUDA = 3
SPH_ERR_NO_DEVICE = 4
SPH_ERR_NONFINITE = 5
SPH_ERR_RANGE = 6
SPH_ERR_TIMEOUT = 7
PERSISTENT_SPIN_DEFAULT = 1 << 22

PRESET_REF_2D = 0
PRESET_REF_3D2 = 1
PRESET_REF_3D4 = 2
PRESET_DAM_2D = 3
PRESET_DAM_3D2 = 4
PRESET_DAM_3D4 = 5
PRESET_ROLLOUT_3D = 6

INTEGRATE_REF3D = 0
INTEGRATE_REF2D = 1
INTEGRATE_PHYS = 2
SPLIT_WAVELET = 0
SPLIT_DEFICIT = 1
MERGE_WAVELET = 0
MERGE_WAVELET_CELL = 1
MERGE_INTERIOR = 2
MERGE_SIBLING = 3

F2 = C.c_float * 2
F3 = C.c_float * 3
U3 = C.c_uint32 * 3


class Sphere(C.Structure):
    _fields_ = [("pos", F3), ("radius", C.c_float), ("damping", C.c_float)]


class Config(C.Structure):
    _fields_ = [
        ("dim", C.c_uint32), ("max_particle", C.c_uint32), ("world", F3), ("cell_size", C.c_float),
        ("ncell", U3),
        ("mass", F2), ("kernel", F2), ("kernel2", F2), ("kernel6", F2), ("radius", F2),
        ("poly6", F2), ("spiky", F2), ("visco", F2), ("grad_poly6", F2), ("lapc_poly6", F2),
        ("poly6_radius", F2),
        ("gravity", F3), ("wall_damping", C.c_float), ("rest_density", C.c_float),
        ("gas_constant", C.c_float), ("time_step", C.c_float), ("viscosity", C.c_float),
        ("surface_threshold", C.c_float), ("surface_coef", C.c_float), ("co_surface", C.c_float),
        ("co_energy", C.c_float), ("split_criteria", C.c_float), ("merge_criteria", C.c_float),
        ("density_skip_r2", C.c_float), ("lapc_three_quarters", C.c_float),
        ("split_ways", C.c_uint32), ("use_split", C.c_uint32), ("use_merge", C.c_uint32),
        ("integrator", C.c_uint32), ("kernel_h6_twice", C.c_uint32), ("energy_large_kernel", C.c_uint32),
        ("energy_mass_weight", C.c_uint32), ("energy_skip_close", C.c_uint32), ("split_rule", C.c_uint32),
        ("merge_rule", C.c_uint32), ("split_min_neighbors", C.c_uint32), ("split_density_ratio", C.c_float),
        ("merge_interior_steps", C.c_uint32), ("split_copies_fields", C.c_uint32),
        ("use_cylinder", C.c_uint32), ("sphere", Sphere * 3),
        ("push_left", C.c_uint32), ("push_right", C.c_uint32), ("push_y_div", C.c_uint32),
        ("extern_force_on", C.c_uint32), ("extern_click", F2), ("extern_force", F2),
        ("extern_len", C.c_float), ("extern_coe", C.c_float),
        ("dens_mul", C.c_uint32), ("den_size", C.c_float), ("ndens", U3), ("iso_value", C.c_float),
        ("mc_interpolate", C.c_uint32), ("splat_with_kernel", C.c_uint32), ("grid_every", C.c_uint32),
        ("max_triangles", C.c_uint32), ("compensated_positions", C.c_uint32), ("close_r2", C.c_float),
        ("walk_only", C.c_uint32),
    ]

    def copy(self):
        c = Config()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(Config))
        return c


FP = C.POINTER(C.c_float)
UP = C.POINTER(C.c_uint32)


class StateView(C.Structure):
    _fields_ = [("n", C.c_uint32), ("pos", FP), ("vel", FP), ("ev", FP), ("acc", FP),
                ("dens", FP), ("press", FP), ("energy", FP), ("surface", FP),
                ("level", UP), ("interior", UP), ("scene", UP), ("sibling", UP)]


class Scene(C.Structure):
    _fields_ = [("lo", F3), ("hi", F3), ("viscosity", C.c_float), ("gas_constant", C.c_float)]


SCENE_GAP_CELLS = 2


class DebugView(C.Structure):
    _fields_ = [("n_sorted", C.c_uint32), ("total_cell", C.c_uint32), ("hash", UP), ("index", UP),
                ("cell_start", UP), ("cell_end", UP), ("trans_vel", FP), ("nbr_count", UP),
                ("split_flag", UP), ("removed", UP)]


class MeshView(C.Structure):
    _fields_ = [("max_triangles", C.c_uint32), ("num_triangles", C.c_uint32),
                ("v0", FP), ("v1", FP), ("v2", FP), ("n0", FP), ("n1", FP), ("n2", FP)]


class LossGrid(C.Structure):
    _fields_ = [("n", U3), ("origin", F3), ("spacing", C.c_float)]


class TopologyView(C.Structure):
    _fields_ = [("n", C.c_uint32), ("n_next", C.c_uint32), ("n_split", C.c_uint32), ("n_removed", C.c_uint32),
                ("split_on", C.c_uint32), ("n_dens_pairs", C.c_uint32), ("n_force_pairs", C.c_uint32),
                ("dens_cap", C.c_uint32), ("force_cap", C.c_uint32),
                ("level", UP), ("dens_off", UP), ("dens_nbr", UP), ("force_off", UP), ("force_nbr", UP),
                ("wall", UP), ("split", UP), ("dst", UP), ("child", UP), ("merge_leader", UP),
                ("pos", FP), ("vel", FP), ("ev", FP)]


TUNE_STAGES = 8
TUNE_STAGE_NAMES = ("hash", "scatter", "reorder", "density", "force_integrate", "energy_split", "merge", "write")


class Tuning(C.Structure):
    _fields_ = [("block", C.c_uint32 * TUNE_STAGES), ("blocks_per_sm", C.c_uint32 * TUNE_STAGES),
                ("reg_cap", C.c_uint32 * TUNE_STAGES), ("step_ms_before", C.c_float), ("step_ms_after", C.c_float)]


class StepStats(C.Structure):
    _fields_ = [(k, C.c_uint32) for k in ("n_start", "n_split", "n_removed", "n_end", "n_level2",
                                           "split_suppressed", "error")]


H = C.c_void_p
DP = C.POINTER(C.c_double)

# (name, restype, argtypes) of every entry point declared in include/sph/sph.h
SIGNATURES = [
    ("sph_config_size", C.c_size_t, []),
    ("sph_config_preset", C.c_int, [C.c_int, C.POINTER(Config)]),
    ("sph_create", C.c_int, [C.POINTER(Config), C.POINTER(H)]),
    ("sph_destroy", C.c_int, [H]),
    ("sph_set_config", C.c_int, [H, C.POINTER(Config)]),
    ("sph_get_config", C.c_int, [H, C.POINTER(Config)]),
    ("sph_add_particles", C.c_int, [H, C.c_uint32, FP, FP, UP]),
    ("sph_set_state", C.c_int, [H, C.POINTER(StateView)]),
    ("sph_step", C.c_int, [H, C.c_int]),
    ("sph_set_scenes", C.c_int, [H, C.c_uint32, C.POINTER(Scene)]),
    ("sph_set_graph", C.c_int, [H, C.c_int]),
    ("sph_set_persistent", C.c_int, [H, C.c_int, C.c_uint32]),
    ("sph_sync", C.c_int, [H]),
    ("sph_get_num_particles", C.c_int, [H, UP]),
    ("sph_get_state", C.c_int, [H, C.POINTER(StateView)]),
    ("sph_get_debug", C.c_int, [H, C.POINTER(DebugView)]),
    ("sph_particle_record_size", C.c_uint32, [H]),
    ("sph_read_particles", C.c_int, [H, C.c_void_p, C.c_uint64, UP]),
    ("sph_write_particles", C.c_int, [H, C.c_void_p, C.c_uint32]),
    ("sph_set_profiling", C.c_int, [H, C.c_int]),
    ("sph_stage_times", C.c_int, [H, FP, C.POINTER(C.c_char_p), C.c_int, C.POINTER(C.c_int)]),
    ("sph_get_stream", C.c_void_p, [H]),
    ("sph_set_stream", C.c_int, [H, C.c_void_p]),
    ("sph_set_debug", C.c_int, [H, C.c_int]),
    ("sph_last_launch_count", C.c_int, [H, UP]),
    ("sph_last_step_stats", C.c_int, [H, C.c_void_p]),
    ("sph_density_grid", C.c_int, [H, FP, FP]),
    ("sph_extract_surface", C.c_int, [H, C.POINTER(MeshView)]),
    ("sph_surface_from_grid", C.c_int, [H, FP, FP, C.POINTER(MeshView)]),
    ("sph_write_pov_mesh", C.c_int, [C.POINTER(MeshView), FP, FP, C.c_char_p]),
    ("sph_write_pov_particles", C.c_int, [FP, UP, C.c_uint32, C.c_uint32, FP, FP, C.c_char_p]),
    ("sph_read_particles_async", C.c_int, [H, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("sph_readback_wait", C.c_int, [H]),
    ("sph_rollout_forward", C.c_int, [H, C.c_uint32, C.c_uint32]),
    ("sph_splat_loss", C.c_int, [H, C.POINTER(LossGrid), FP, FP, DP]),
    ("sph_rollout_backward", C.c_int, [H, FP, FP, DP, C.c_uint32]),
    ("sph_rollout_topology", C.c_int, [H, C.c_uint32, C.POINTER(TopologyView)]),
    ("sph_conserved", C.c_int, [H, DP]),
    ("sph_set_tuning", C.c_int, [H, C.POINTER(Tuning)]),
    ("sph_get_tuning", C.c_int, [H, C.POINTER(Tuning)]),
    ("sph_autotune", C.c_int, [H, C.c_uint32, C.POINTER(Tuning)]),
    ("sph_last_error", C.c_char_p, [H]),
    ("sph_sort_cells_noalloc", C.c_int, [C.POINTER(Config), C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
]

NOALLOC_MAX_PARTICLES = 1 << 18
NOALLOC_MAX_CELLS = 1 << 16

LIB_NAME = "libsca2012_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

_lib = None


def load():
    """Loads the in-tree CUDA library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_NAME} not built (run __graft_entry__.build() or python -m sca2012_b200.build)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    size = lib.sph_config_size()
    if size != C.sizeof(Config):
        raise RuntimeError(f"sph_config layout mismatch: C {size} bytes, ctypes {C.sizeof(Config)}")
    _lib = lib
    return lib
