"""Speed against the reference itself, on the reference's own scenes.

The unmodified reference (oracle/_ref/libref_<v>_gpu.so, compiled from its
sources for sm_100a) steps the scene its app starts with, split and merge
on, in each of its three solvers:
  2d   SPH-2D add_init_particle   (SPH-2D/sph_system.cpp:148-162, sph_main.cpp:45)
  3d2  SPH-3D-2 add_box_particle  (SPH-3D-2/sph_system.cpp:247-264)
  3d4  SPH-3D-4 add_box_particle  (SPH-3D-4/sph_system.cpp:248-289, sph_main.cpp:341)
Each animation()/animate() ends with the synchronous readback of every
particle.  The same scene and constants through this library's C-ABI, with
the same per-step readback into page-locked host memory, must be faster.
Both times are host wall-clock per step (the reference is synchronous by
construction).  Prints one JSON line per solver with the numbers and this
library's stage times.
"""
import ctypes as C
import json
import os
import time

import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 40


VARIANTS = {"2d": (sph.PRESET_REF_2D, scenes.ref_init_2d, "SPH-2D add_init_particle"),
            "3d2": (sph.PRESET_REF_3D2, scenes.ref_box_3d2, "SPH-3D-2 add_box_particle"),
            "3d4": (sph.PRESET_REF_3D4, scenes.ref_box_3d4, "SPH-3D-4 add_box_particle")}


def _reference_ms_per_step(v):
    path = os.path.join(ROOT, "oracle", "_ref", f"libref_{v}_gpu.so")
    if not os.path.exists(path):
        return None, None
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.ref_create.restype = vp
    lib.ref_add_default_scene.argtypes = [vp, C.c_int]
    lib.ref_set_flags.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.ref_step.argtypes = [vp]
    lib.ref_step.restype = C.c_int
    lib.ref_num_particles.argtypes = [vp]
    lib.ref_num_particles.restype = C.c_uint
    h = C.c_void_p(lib.ref_create())
    lib.ref_add_default_scene(h, 0)
    lib.ref_set_flags(h, 1, 1, 1)
    for _ in range(3):
        assert lib.ref_step(h) == 0
    t0 = time.perf_counter()
    for _ in range(STEPS):
        assert lib.ref_step(h) == 0
    dt = (time.perf_counter() - t0) / STEPS
    return dt * 1e3, int(lib.ref_num_particles(h))


def _ours_ms_per_step(v, graph, persistent=False):
    import torch
    preset, scene, _ = VARIANTS[v]
    cfg = sph.preset(preset)
    cfg.use_split = cfg.use_merge = 1
    pos, vel, lvl = scene(cfg)
    s = sph.Solver(cfg)
    s.set_graph(graph)
    s.set_persistent(persistent)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    host = torch.empty(cfg.max_particle * s.record_size, dtype=torch.uint8, pin_memory=True)
    for _ in range(3):
        s.step(1)
        s.read_particles_into(host.data_ptr(), host.numel())
    t0 = time.perf_counter()
    for _ in range(STEPS):
        s.step(1)
        n = s.read_particles_into(host.data_ptr(), host.numel())
    dt = (time.perf_counter() - t0) / STEPS
    s.set_profiling(True)
    s.step(1)
    stages = s.stage_times()
    s.close()
    return dt * 1e3, n, stages


@pytest.mark.parametrize("v", list(VARIANTS))
def test_faster_than_reference_on_its_own_scene(v, gpu):
    ref_ms, ref_n = _reference_ms_per_step(v)
    ours_ms, n, stages = _ours_ms_per_step(v, False)
    graph_ms, _, _ = _ours_ms_per_step(v, True)
    persistent_ms, _, _ = _ours_ms_per_step(v, False, True)
    print(json.dumps({"scene": f"{VARIANTS[v][2]}, split+merge, readback every step", "steps": STEPS,
                      "reference_ms_per_step": ref_ms, "reference_particles": ref_n,
                      "ours_ms_per_step": ours_ms, "ours_graph_ms_per_step": graph_ms,
                      "ours_persistent_ms_per_step": persistent_ms, "ours_particles": n,
                      "ours_stages_ms": {k: round(v, 4) for k, v in stages}}))
    if ref_ms is None:
        pytest.skip("oracle/_ref not built")
    assert max(ours_ms, graph_ms, persistent_ms) < ref_ms
