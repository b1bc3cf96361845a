"""Pins the oracle's marching cubes (oracle/mc.py) against the reference's own
CPU marching cubes (SPHSystem::marching_cube, SPH-3D-2/sph_system.cpp:406-542,
compiled from the reference's sources into oracle/_ref) on the reference's
own density grids (tests/golden): the same triangle count, the same cubes in
the same order, and per cube the same edge-midpoint vertices and the same
polygon loops (a loop of 4+ vertices may be split along another diagonal,
see sca2012_b200/csrc/gen_mc_tables.py).  The interpolated mode the SI
presets use differs only in where a vertex sits on its edge; it is checked
here on a grid with known crossings."""
import numpy as np
import pytest

from oracle import mc as M
from tests._mc_ref import ref_mc
from tests.test_oracle_golden import load, grid_of, cfg_of


def _half_node(v, h):
    """Vertex on the lattice of half node spacings (exact for midpoints)."""
    return tuple(np.rint(np.asarray(v, np.float64) / (0.5 * h)).astype(np.int64))


def _loops(tris):
    de = set()
    for t in tris:
        a, b, c = t
        de |= {(a, b), (b, c), (c, a)}
    return {e for e in de if (e[1], e[0]) not in de}


@pytest.mark.parametrize("v", ["3d2", "3d4"])
def test_oracle_mc_matches_reference_cpu(v):
    g = load(v)
    gd, gn = grid_of(g)
    ref = ref_mc(v, gd, gn)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    cfg = cfg_of(v)
    assert cfg.mc_interpolate == 0
    ours, per_cube = M.marching_cubes(cfg, gd, gn)
    assert len(ours) == len(ref) == int(g["mesh_triangles"])
    h = float(cfg.den_size)
    ends = np.cumsum(per_cube[per_cube > 0])
    starts = ends - per_cube[per_cube > 0]
    worst = 0.0
    for b, e in zip(starts, ends):
        o = [tuple(_half_node(ours[i, j], h) for j in range(3)) for i in range(b, e)]
        r = [tuple(_half_node(ref[i, j], h) for j in range(3)) for i in range(b, e)]
        assert {x for t in o for x in t} == {x for t in r for x in t}, f"cube at triangles {b}:{e}"
        assert _loops(o) == _loops(r), f"cube at triangles {b}:{e}"
        # each vertex: position (the FP32 midpoint) and normal (mean of the node normals)
        on = {o[i - b][j]: (ours[i, j], ours[i, 3 + j]) for i in range(b, e) for j in range(3)}
        rn = {r[i - b][j]: (ref[i, j], ref[i, 3 + j]) for i in range(b, e) for j in range(3)}
        for key, (pv, nv) in on.items():
            worst = max(worst, np.abs(pv - rn[key][0]).max(), np.abs(nv - rn[key][1]).max())
    assert worst <= 1e-6 * max(cfg.world)


def test_oracle_mc_interpolates_at_the_iso_value():
    # one cube per axis direction: density rises linearly along x, so every
    # vertex must sit where the linear field crosses the iso value
    cfg = cfg_of("3d2")
    cfg.mc_interpolate = 1
    cfg.iso_value = 0.5
    R, Cn, L = (int(cfg.ndens[a]) for a in range(3))
    x = np.arange(R, dtype=np.float64) * float(cfg.den_size)
    field = np.broadcast_to(0.3 * x[None, None, :] / x[-1] * 3.0, (L, Cn, R)).astype(np.float32).reshape(-1)
    tris, per_cube = M.marching_cubes(cfg, field, np.zeros((len(field), 3), np.float32))
    assert len(tris) > 0
    slope = 0.9 / x[-1]
    xs = tris[:, :3, 0].reshape(-1)
    f32x = (np.rint(xs / float(cfg.den_size))).astype(np.int64)   # the crossing's lower node
    lo = field.reshape(L, Cn, R)[0, 0, :].astype(np.float64)
    # exact crossing of the FP32 node values along the edge
    expect = []
    for xv in xs:
        i = int(np.floor(xv / float(cfg.den_size)))
        da, db = lo[i], lo[i + 1]
        expect.append(x[i] + (0.5 - da) / (db - da) * (x[i + 1] - x[i]))
    assert np.abs(xs - np.array(expect)).max() < 1e-9 and slope > 0 and f32x.min() >= 0
