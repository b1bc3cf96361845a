"""Speed against the reference itself, on the reference's own scene.

The unmodified reference (oracle/_ref/libref_3d2_gpu.so, compiled from its
sources for sm_100a) steps its default SPH-3D-2 scene with split and merge
on: each animation() ends with the synchronous readback of every particle.
The same scene and constants through this library's C-ABI, with the same
per-step readback into page-locked host memory, must be faster.  Both times
are host wall-clock per step (the reference is synchronous by construction).
Prints one JSON line with the numbers and this library's stage times.
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


def _reference_ms_per_step():
    path = os.path.join(ROOT, "oracle", "_ref", "libref_3d2_gpu.so")
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


def _ours_ms_per_step(graph):
    import torch
    cfg = sph.preset(sph.PRESET_REF_3D2)
    cfg.use_split = cfg.use_merge = 1
    pos, vel, lvl = scenes.ref_box_3d2(cfg)
    s = sph.Solver(cfg)
    s.set_graph(graph)
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


def test_faster_than_reference_on_its_own_scene(gpu):
    ref_ms, ref_n = _reference_ms_per_step()
    ours_ms, n, stages = _ours_ms_per_step(False)
    graph_ms, _, _ = _ours_ms_per_step(True)
    print(json.dumps({"scene": "SPH-3D-2 default, split+merge, readback every step", "steps": STEPS,
                      "reference_ms_per_step": ref_ms, "reference_particles": ref_n,
                      "ours_ms_per_step": ours_ms, "ours_graph_ms_per_step": graph_ms, "ours_particles": n,
                      "ours_stages_ms": {k: round(v, 4) for k, v in stages}}))
    if ref_ms is None:
        pytest.skip("oracle/_ref not built")
    assert ours_ms < ref_ms
