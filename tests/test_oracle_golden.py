"""Pins the CPU oracle against the UNMODIFIED reference.

tests/golden/ref_<variant>.npz hold states and intermediates produced by the
reference solver itself (compiled from its sources for sm_100a and run on a
B200 by tests/golden/make_golden.py).  Each oracle stage is fed the
reference's own FP32 inputs and must reproduce the reference's outputs:
integer stages bit-exact, float stages within the tolerances of
tests/_parity.py.  Also pins the reference presets' constants bit for bit.
"""
import os

import numpy as np
import pytest

import sca2012_b200 as sph
from oracle import oracle as O
from tests._parity import check_close, check_equal

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
VARIANTS = {"2d": sph.PRESET_REF_2D, "3d2": sph.PRESET_REF_3D2, "3d4": sph.PRESET_REF_3D4}


def load(v):
    path = os.path.join(GOLDEN, f"ref_{v}.npz")
    assert os.path.exists(path), f"missing golden fixture {path} (run tests/golden/make_golden.py on a GPU)"
    return np.load(path)


def state(rec):
    st = {k: np.ascontiguousarray(rec[k]) for k in ("pos", "vel", "ev", "acc", "dens", "press", "energy", "level")}
    st["surface"] = np.ascontiguousarray(rec["surface"])
    return st


def cfg_of(v, split=0, merge=0):
    c = sph.preset(VARIANTS[v])
    c.use_split = split
    c.use_merge = merge
    return c


@pytest.mark.parametrize("v", list(VARIANTS))
def test_preset_constants_match_reference(v):
    g = load(v)
    p = g["params"]
    c = cfg_of(v)
    d = c.dim
    ours = [c.mass[0], c.mass[1], c.kernel[0], c.kernel[1], c.kernel2[0], c.kernel2[1], c.kernel6[0],
            c.kernel6[1], c.radius[0], c.radius[1], c.poly6[0], c.poly6[1], c.spiky[0], c.spiky[1],
            c.visco[0], c.visco[1], c.grad_poly6[0], c.grad_poly6[1], c.lapc_poly6[0], c.lapc_poly6[1]]
    if d == 3:
        ours += [c.poly6_radius[0], c.poly6_radius[1]]
    else:
        ours += [0.0, 0.0]
    ours += [c.cell_size] + [c.world[a] for a in range(d)]
    ours += [c.rest_density, c.gas_constant, c.time_step, c.viscosity, c.surface_threshold, c.co_surface,
             c.co_energy, c.split_criteria, c.merge_criteria] + [c.gravity[a] for a in range(d)] + [c.wall_damping]
    if d == 3:
        ours += [c.den_size]
    ours = np.array(ours, np.float32)
    assert len(ours) == len(p)
    check_equal("reference constants", ours.view(np.uint32), p.view(np.uint32))


@pytest.mark.parametrize("v", list(VARIANTS))
def test_oracle_stages_match_reference(v):
    g = load(v)
    cfg = cfg_of(v)
    s0 = state(g["s0"])
    s1 = state(g["s1_off"])
    n = len(s0["pos"])
    assert len(s1["pos"]) == n

    key, idx, cs, ce = O.sort(cfg, s0["pos"])
    check_equal("cell keys", g["off_hash"], key)
    check_equal("sorted index", g["off_index"], idx)
    check_equal("cell_start", g["off_cell_start"], cs)
    check_equal("cell_end", g["off_cell_end"], ce)

    dens, press, nbr = O.density(cfg, s0["pos"], s0["level"], idx, cs, ce)
    check_close("density", s1["dens"], dens)
    check_close("pressure", s1["press"], press)

    acc, surf, amb = O.force(cfg, s0["pos"], s0["ev"], s0["level"], dens, press, idx, cs, ce)
    p64, v64, e64, a64, amb2 = O.integrate(cfg, s0["pos"], s0["vel"], s0["ev"], s0["level"], acc, dens)
    ok = ~(amb | amb2)
    check_close("surface |grad c|", s1["surface"], surf)
    check_close("acceleration", s1["acc"], a64, ok)
    check_close("velocity", s1["vel"], v64, ok)
    check_close("eval velocity", s1["ev"], e64, ok)
    check_close("position", s1["pos"], p64, ok)

    en, tv = O.energy(cfg, s1["pos"], s1["vel"], s0["level"], idx, cs, ce)
    check_close("energy", s1["energy"], en)
    check_close("trans_vel", g["off_trans_vel"], tv)


@pytest.mark.parametrize("v", list(VARIANTS))
def test_oracle_adapt_matches_reference(v):
    g = load(v)
    cfg_on = cfg_of(v, 1, 1)
    s0 = state(g["s0"])
    pre = state(g["s1_off"])
    key, idx, cs, ce = O.sort(cfg_on, s0["pos"])
    _, _, nbr = O.density(cfg_on, s0["pos"], s0["level"], idx, cs, ce)
    exp, split, rem = O.adapt(cfg_on, pre, nbr, idx, cs, ce, cap=cfg_on.max_particle)
    got = state(g["s1_on"])
    n = len(s0["pos"])
    assert len(got["pos"]) == len(exp["pos"]), "particle count after split/merge"
    check_equal("levels", got["level"], exp["level"])
    for k in ("pos", "vel", "ev", "acc", "energy"):
        check_close(f"adapted {k}", got[k], exp[k])
    # the 3D reference leaves a child's dens/press/surface unwritten
    # (SPH-3D-2/sph_system.cu:1594-1607): compare them for the old particles
    n_child = int(split.sum()) * (cfg_on.split_ways - 1)
    live_old = len(exp["pos"]) - n_child
    m = np.ones(len(exp["pos"]), bool)
    if cfg_on.dim == 3:
        m[live_old:] = False
    for k in ("dens", "press", "surface"):
        check_close(f"adapted {k}", got[k], exp[k], mask=m)
    assert split.sum() > 0 or rem.sum() > 0 or n < 100, "fixture exercises neither split nor merge"


def grid_of(g):
    """Dense density grid and normals from the sparse fixture layout."""
    G = int(g["grid_nodes"])
    dens = np.zeros(G, np.float32)
    dens[g["grid_dens_idx"]] = g["grid_dens_val"]
    nrm = np.zeros((G, 3), np.float32)
    nrm[g["grid_normal_idx"]] = g["grid_normal_val"]
    return dens, nrm


@pytest.mark.parametrize("v", ["3d2", "3d4"])
def test_oracle_density_grid_matches_reference(v):
    g = load(v)
    cfg = cfg_of(v)
    s0 = state(g["s0"])
    s1 = state(g["s1_off"])   # the grid is splatted from the post-integration positions
    key, idx, cs, ce = O.sort(cfg, s0["pos"])
    dens, nrm = O.density_grid(cfg, s1["pos"], s0["level"], idx, cs, ce)
    gd, gn = grid_of(g)
    check_close("grid density", gd, dens)
    # normals of the FP32 grid (the reference differentiates its own floats)
    check_close("grid normals", gn, _normals(cfg, gd), rtol=2e-5)


@pytest.mark.parametrize("v", ["3d2", "3d4"])
def test_reference_cpu_marching_cubes_reproduces_reference_mesh(v):
    """The MC oracle is the reference's own CPU marching cubes
    (oracle/_ref/libref_<v>_mc.so); it must rebuild, from the fixture grid,
    the exact mesh the reference produced in its own run."""
    from tests._mc_ref import ref_mc, mesh_sha256
    g = load(v)
    gd, gn = grid_of(g)
    mesh = ref_mc(v, gd, gn)
    if mesh is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    assert len(mesh) == int(g["mesh_triangles"])
    assert mesh_sha256(mesh) == str(g["mesh_sha256"])


def _normals(cfg, dens):
    R, Cc, L = (int(cfg.ndens[a]) for a in range(3))
    d = dens.astype(np.float64).reshape(L, Cc, R)
    out = np.zeros((L, Cc, R, 3))
    for a, ax in enumerate((2, 1, 0)):
        lo = np.roll(d, 1, axis=ax)
        hi = np.roll(d, -1, axis=ax)
        sl_first = [slice(None)] * 3
        sl_first[ax] = 0
        sl_last = [slice(None)] * 3
        sl_last[ax] = -1
        lo[tuple(sl_first)] = 0.0
        hi[tuple(sl_last)] = 0.0
        out[..., a] = (lo - hi) / float(np.float32(cfg.den_size))
    ln = np.sqrt((out ** 2).sum(-1, keepdims=True))
    out = np.where(ln > 0, out / np.where(ln > 0, ln, 1), 0.0)
    return out.reshape(-1, 3)
