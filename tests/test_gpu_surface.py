"""Density grid, grid normals and marching cubes on the GPU, through the C-ABI.

* The grid the step builds (grid_every = 1, the reference's display mode 2)
  from the reference's own state S0 is compared with the reference's grid
  (tests/golden) and with the FP64 oracle.
* The config-mode surface the SI presets build (kernel-length splat,
  vertices interpolated at the iso value 0.5 rho0) is compared with the FP64
  oracle: the grid with the oracle's splat, and the mesh with the oracle's
  marching cubes (oracle/mc.py) on the same FP32 grid (cube cases and
  triangle counts bit-exact, vertices and normals within 1e-5), on an SI
  block and on a crop of the 1.1M-particle benchmark workload.
* Marching cubes on the reference's exact grid (sph_surface_from_grid) is
  compared with the reference's own CPU marching cubes on the same grid:
  same triangle count, same triangles per cube in the same cube order, the
  same vertices and normals bit for bit, and the same polygon loops per cube
  (a loop of 4+ vertices may be split along another diagonal; see
  sca2012_b200/csrc/gen_mc_tables.py).
"""
import ctypes as C
import os

import numpy as np
import pytest

import sca2012_b200 as sph
from oracle import oracle as O
from tests._parity import check_close
from tests._mc_ref import ref_mc
from tests.test_oracle_golden import load, state, grid_of, VARIANTS

pytestmark = pytest.mark.gpu


def _cfg(v, grid):
    c = sph.preset(VARIANTS[v])
    c.use_split = 0
    c.use_merge = 0
    c.grid_every = 1 if grid else 0
    c.max_particle = 200000
    return c


def _mesh(solver, fn, *args):
    G = int(np.prod([solver.cfg.ndens[a] for a in range(3)]))
    mx = min(3 * G, int(solver.cfg.max_triangles)) if solver.cfg.max_triangles else 3 * G
    bufs = [np.zeros((mx, 3), np.float32) for _ in range(6)]
    mv = sph.MeshView()
    mv.max_triangles = mx
    for k, b in zip(("v0", "v1", "v2", "n0", "n1", "n2"), bufs):
        setattr(mv, k, b.ctypes.data_as(C.POINTER(C.c_float)))
    rc = fn(solver._h, *args, C.byref(mv))
    assert rc == 0, solver._lib.sph_last_error(solver._h)
    nt = int(mv.num_triangles)
    return np.stack([b[:nt] for b in bufs], 1)


@pytest.mark.parametrize("v", ["3d2", "3d4"])
def test_step_density_grid_matches_reference_and_oracle(v, gpu):
    g = load(v)
    cfg = _cfg(v, True)
    s0 = state(g["s0"])
    s = sph.Solver(cfg)
    s.set_state(s0)
    s.step(1)
    assert s.sync_status() == 0
    G = int(np.prod([cfg.ndens[a] for a in range(3)]))
    dens = np.zeros(G, np.float32)
    nrm = np.zeros((G, 3), np.float32)
    assert s._lib.sph_density_grid(s._h, dens.ctypes.data_as(C.POINTER(C.c_float)),
                                   nrm.ctypes.data_as(C.POINTER(C.c_float))) == 0
    st = s.get_state()
    s.close()
    gd, gn = grid_of(g)
    check_close("grid density vs reference", dens, gd)
    key, idx, cs, ce = O.sort(cfg, s0["pos"])
    d64, n64 = O.density_grid(cfg, st["pos"], s0["level"], idx, cs, ce)
    check_close("grid density vs oracle", dens, d64)
    # normals: unit vectors of the FP32 grid's gradient; compared where the
    # gradient is not a cancellation (|grad| above 1e-3 of its maximum)
    gx = np.zeros((G, 3))
    R, Cn, L = (int(cfg.ndens[a]) for a in range(3))
    d3 = d64.reshape(L, Cn, R)
    for a, ax in enumerate((2, 1, 0)):
        lo = np.roll(d3, 1, ax)
        hi = np.roll(d3, -1, ax)
        sl = [slice(None)] * 3
        sl[ax] = 0
        lo[tuple(sl)] = 0
        sl[ax] = -1
        hi[tuple(sl)] = 0
        gx[:, a] = ((lo - hi) / float(cfg.den_size)).reshape(-1)
    mag = np.sqrt((gx ** 2).sum(1))
    ok = mag > 1e-3 * mag.max()
    check_close("grid normals", nrm[ok], n64[ok], rtol=1e-4)


def _cube_counts(cfg, dens):
    """Triangles per cube (x outer, z inner) from the iso flags."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "sca2012_b200", "csrc"))
    import gen_mc_tables as G
    counts = np.array([len(G.triangles(c)) for c in range(256)])
    R, Cn, L = (int(cfg.ndens[a]) for a in range(3))
    above = (dens.reshape(L, Cn, R) > np.float32(cfg.iso_value)).transpose(2, 1, 0)  # [x, y, z]
    flags = np.zeros((R - 1, Cn - 1, L - 1), np.int64)
    for vtx, (ox, oy, oz) in enumerate(G.CORNERS):
        flags |= above[ox:R - 1 + ox, oy:Cn - 1 + oy, oz:L - 1 + oz].astype(np.int64) << vtx
    return counts[flags.reshape(-1)]


def _loops(tris):
    de = set()
    for t in tris:
        a, b, c = (tuple(x) for x in t[:3])
        de |= {(a, b), (b, c), (c, a)}
    return {e for e in de if (e[1], e[0]) not in de}


@pytest.mark.parametrize("v", ["3d2", "3d4"])
def test_marching_cubes_matches_reference_cpu(v, gpu):
    g = load(v)
    gd, gn = grid_of(g)
    ref = ref_mc(v, gd, gn)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    cfg = _cfg(v, False)
    s = sph.Solver(cfg)
    ours = _mesh(s, s._lib.sph_surface_from_grid, gd.ctypes.data_as(C.POINTER(C.c_float)),
                 gn.ctypes.data_as(C.POINTER(C.c_float)))
    s.close()
    assert len(ours) == len(ref) == int(g["mesh_triangles"])
    counts = _cube_counts(cfg, gd)
    assert counts.sum() == len(ref)
    ends = np.cumsum(counts[counts > 0])
    starts = ends - counts[counts > 0]
    exact_cubes = 0
    for b, e in zip(starts, ends):
        o, r = ours[b:e], ref[b:e]
        # same vertices (and their normals), bit for bit
        ov = {tuple(np.concatenate([o[i, j], o[i, 3 + j]])) for i in range(len(o)) for j in range(3)}
        rv = {tuple(np.concatenate([r[i, j], r[i, 3 + j]])) for i in range(len(r)) for j in range(3)}
        assert ov == rv, f"cube at triangles {b}:{e}: vertices differ"
        assert _loops(o) == _loops(r), f"cube at triangles {b}:{e}: polygon loops differ"
        exact_cubes += np.array_equal(o, r)
    assert exact_cubes > 0


def test_in_step_surface_on_si_block(gpu):
    from sca2012_b200 import scenes
    cfg = sph.preset(sph.PRESET_DAM_3D2)
    pos, vel, lvl = scenes.block_3d(cfg, (24, 24, 12), 0.01, seed=1)
    cfg.grid_every = 1
    cfg.max_particle = 4 * len(pos)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(1)
    assert s.sync_status() == 0
    mesh = _mesh(s, s._lib.sph_extract_surface)
    s.close()
    assert len(mesh) > 1000
    v = mesh[:, :3].reshape(-1, 3)
    assert np.isfinite(v).all()
    assert (v >= 0).all() and (v <= np.array(list(cfg.world))).all()


def _crop_x(scene, xmax):
    pos, vel, lvl = scene
    m = pos[:, 0] < xmax
    return pos[m], vel[m], lvl[m]


SI_SURFACES = {
    # 24 x 24 x 12 block at s = 0.01 (two-way preset, 257 x 129 x 129 nodes)
    "dam_3d2_block": (sph.PRESET_DAM_3D2, lambda c: scenes_mod().block_3d(c, (24, 24, 12), 0.01, seed=1)),
    # the 1.1M-particle workload cut at x < 0.16 (262,144 particles; the full
    # 257 x 257 x 129 node grid of the benchmark)
    "dam_3d4_crop": (sph.PRESET_DAM_3D4, lambda c: _crop_x(scenes_mod().dam_3d4(c, seed=0), 0.16)),
}


def scenes_mod():
    from sca2012_b200 import scenes
    return scenes


@pytest.mark.parametrize("name", list(SI_SURFACES))
def test_si_surface_matches_oracle(name, gpu):
    from oracle import mc as M
    preset, scene = SI_SURFACES[name]
    cfg = sph.preset(preset)
    pos, vel, lvl = scene(cfg)
    cfg.use_split = cfg.use_merge = 0
    cfg.grid_every = 1
    cfg.max_particle = 2 * len(pos)
    assert cfg.mc_interpolate == 1 and cfg.splat_with_kernel == 1
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(2)
    assert s.sync_status() == 0
    s0 = s.get_state()
    s.set_state(s0)
    s.step(1)
    assert s.sync_status() == 0
    G = int(np.prod([cfg.ndens[a] for a in range(3)]))
    dens = np.zeros(G, np.float32)
    nrm = np.zeros((G, 3), np.float32)
    assert s._lib.sph_density_grid(s._h, dens.ctypes.data_as(C.POINTER(C.c_float)),
                                   nrm.ctypes.data_as(C.POINTER(C.c_float))) == 0
    mesh = _mesh(s, s._lib.sph_extract_surface)
    st = s.get_state()
    s.close()

    # (1) the kernel-length splat on the stale cells with the new positions
    key, idx, cs, ce = O.sort(cfg, s0["pos"])
    d64, n64 = O.density_grid(cfg, st["pos"], s0["level"], idx, cs, ce)
    check_close(f"{name}/grid density vs oracle", dens, d64)

    # (2) marching cubes on the GPU's own grid: same cases, same triangles in
    # the same order, vertices interpolated at the iso value within 1e-5
    tris, per_cube = M.marching_cubes(cfg, dens, nrm)
    assert len(mesh) == len(tris), (len(mesh), len(tris))
    assert len(mesh) > 1000
    check_close(f"{name}/mesh vertices", mesh[:, :3].reshape(-1, 3), tris[:, :3].reshape(-1, 3))
    np.testing.assert_allclose(mesh[:, 3:].reshape(-1, 3), tris[:, 3:].reshape(-1, 3), rtol=0, atol=1e-6)

    # (3) cube cases from the FP32 grid against those of the FP64 grid: every
    # cube that differs has a corner node within 1e-5 of the iso value
    c32 = M.cube_cases(cfg, dens)
    c64 = M.cube_cases(cfg, d64)
    diff = np.flatnonzero(c32 != c64)
    if len(diff):
        R, Cn, L = (int(cfg.ndens[a]) for a in range(3))
        near = np.abs(d64 - float(cfg.iso_value)) <= 1e-5 * float(cfg.iso_value)
        near3 = near.reshape(L, Cn, R).transpose(2, 1, 0)
        qx = diff // ((Cn - 1) * (L - 1))
        qy = (diff // (L - 1)) % (Cn - 1)
        qz = diff % (L - 1)
        amb = np.zeros(len(diff), bool)
        for ox in (0, 1):
            for oy in (0, 1):
                for oz in (0, 1):
                    amb |= near3[qx + ox, qy + oy, qz + oz]
        assert amb.all(), f"{int((~amb).sum())} cubes differ away from the iso value"
    print(f"{name}: {len(mesh)} triangles, {len(diff)} of {len(c32)} cube cases at an ambiguous node")
