"""The drop-in C++ SPHSystem (sca2012_b200/host/sph_system.h) driven like the
reference's application, against the same scene stepped through the
Python/C-ABI path: identical particle records (bit for bit: same kernels,
same inputs) and, in display mode 2, the same mesh."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = {2: (sph.PRESET_REF_2D, scenes.ref_init_2d),
         32: (sph.PRESET_REF_3D2, scenes.ref_box_3d2),
         34: (sph.PRESET_REF_3D4, scenes.ref_box_3d4)}


def build_driver(variant, tmp):
    exe = os.path.join(tmp, f"dropin_{variant}")
    libdir = os.path.join(ROOT, "sca2012_b200")
    cmd = ["g++", "-std=c++17", "-O2", f"-DSCA2012_VARIANT={variant}",
           "-I", os.path.join(ROOT, "sca2012_b200", "host"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "sca2012_b200", "host", "sph_system.cpp"),
           os.path.join(ROOT, "tests", "cpp", "dropin_driver.cpp"),
           "-L", libdir, "-lsca2012_b200", f"-Wl,-rpath,{libdir}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


@pytest.mark.parametrize("variant", [2, 32, 34])
def test_dropin_matches_c_abi_path(variant, tmp_path, gpu):
    steps = 3
    exe = build_driver(variant, str(tmp_path))
    out = os.path.join(str(tmp_path), "out.bin")
    subprocess.run([exe, str(steps), out], check=True)
    raw = open(out, "rb").read()
    n, rec = np.frombuffer(raw[:8], np.uint32)
    recs = np.frombuffer(raw[8:8 + n * rec], sph.particle_dtype(2 if variant == 2 else 3))

    preset, scene = CASES[variant]
    cfg = sph.preset(preset)
    cfg.use_split = cfg.use_merge = 1
    pos, vel, lvl = scene(cfg)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(steps - 1)
    if variant != 2:
        cfg.grid_every = 1
        s.set_config(cfg)
    s.step(1)
    assert s.sync_status() == 0
    ref = s.read_particles()
    assert len(ref) == n
    assert ref.tobytes() == recs.tobytes(), "drop-in records differ from the C-ABI path"
    if variant != 2:
        nt = int(np.frombuffer(raw[8 + n * rec:12 + n * rec], np.uint32)[0])
        G = int(np.prod([cfg.ndens[a] for a in range(3)]))
        mv = sph.MeshView()
        mv.max_triangles = 3 * G
        bufs = [np.zeros((3 * G, 3), np.float32) for _ in range(6)]
        for k, b in zip(("v0", "v1", "v2", "n0", "n1", "n2"), bufs):
            setattr(mv, k, b.ctypes.data_as(C.POINTER(C.c_float)))
        assert s._lib.sph_extract_surface(s._h, C.byref(mv)) == 0
        assert nt == min(mv.num_triangles, G if variant == 32 else 3 * G)
        tri0 = np.frombuffer(raw[12 + n * rec:12 + n * rec + nt * 12], np.float32).reshape(-1, 3)
        assert np.array_equal(tri0, bufs[0][:nt])
    s.close()
