"""Headless POV-Ray writers (sph_write_pov_mesh / sph_write_pov_particles):
the object lines follow the reference app's make_mesh / make_particle
formats (SPH-3D-2/sph_main.cpp:114-220) with the display scale and offset
applied."""
import ctypes as C
import re

import numpy as np

import sca2012_b200 as sph
from sca2012_b200 import _abi

F = r"(-?\d+\.\d{6})"


def test_mesh_file(tmp_path):
    rng = np.random.default_rng(1)
    nt = 5
    arrs = [rng.standard_normal((nt, 3)).astype(np.float32) for _ in range(6)]
    mv = _abi.MeshView()
    mv.max_triangles = nt
    mv.num_triangles = nt
    for k, a in zip(("v0", "v1", "v2", "n0", "n1", "n2"), arrs):
        setattr(mv, k, a.ctypes.data_as(_abi.FP))
    scale = np.array([2.0, 3.0, 4.0], np.float32)
    off = np.array([-1.0, 0.5, 0.0], np.float32)
    path = str(tmp_path / "mesh.pov")
    assert sph.lib().sph_write_pov_mesh(C.byref(mv), scale.ctypes.data_as(_abi.FP),
                                        off.ctypes.data_as(_abi.FP), path.encode()) == 0
    txt = open(path).read()
    lines = [l for l in txt.splitlines() if l.startswith("smooth_triangle")]
    assert len(lines) == nt
    pat = re.compile(r"smooth_triangle \{ " + ", ".join([rf"<{F}, {F}, {F}>"] * 6) + r" \}")
    for t, line in enumerate(lines):
        m = pat.match(line)
        assert m, line
        vals = np.array([float(x) for x in m.groups()]).reshape(6, 3)
        for k in range(3):
            np.testing.assert_allclose(vals[2 * k], arrs[k][t] * scale + off, atol=1e-5)
            np.testing.assert_allclose(vals[2 * k + 1], arrs[3 + k][t], atol=1e-5)
    assert txt.startswith("#include \"colors.inc\"") and "mesh {" in txt


def test_particle_file(tmp_path):
    pos = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]], np.float32)
    lvl = np.array([1, 2], np.uint32)
    path = str(tmp_path / "p.pov")
    assert sph.lib().sph_write_pov_particles(pos.ctypes.data_as(_abi.FP), lvl.ctypes.data_as(_abi.UP), 2, 3,
                                             None, None, path.encode()) == 0
    lines = [l for l in open(path).read().splitlines() if l.startswith("sphere")]
    assert lines[0] == "sphere { <1.000000, 2.000000, 3.000000>, 0.300000 texture { pigment { color Red } } }"
    assert lines[1] == "sphere { <4.000000, 5.000000, 6.000000>, 0.240000 texture { pigment { color Yellow } } }"
