"""FP64 conserved-quantity reductions on the device (sph_conserved): equal to
FP64 host sums of the same state; mass exact through split and merge;
momentum kept by the pair forces when nothing external acts."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu


def _host_sums(cfg, st):
    m = np.where(st["level"] == 1, np.float64(cfg.mass[0]), np.float64(cfg.mass[1]))
    v = st["vel"].astype(np.float64)
    x = st["pos"].astype(np.float64)
    g = np.array(cfg.gravity[: cfg.dim], np.float64)
    return dict(mass=m.sum(), momentum=(m[:, None] * v).sum(0), kinetic=0.5 * (m * (v * v).sum(1)).sum(),
                potential=-(m * (x @ g)).sum())


@pytest.mark.parametrize("preset", [sph.PRESET_DAM_3D2, sph.PRESET_DAM_2D])
def test_sums_match_host(gpu, preset):
    cfg = sph.preset(preset)
    cfg.use_split = cfg.use_merge = 1
    pos, _, lvl = scenes.dam_3d2(cfg) if cfg.dim == 3 else scenes.dam_2d(cfg)
    vel = np.random.default_rng(1).normal(0, 0.1, pos.shape).astype(np.float32)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    m0 = s.conserved()["mass"]
    s.step(30)
    c = s.conserved()
    h = _host_sums(cfg, s.get_state())
    for k in ("mass", "kinetic", "potential"):
        assert abs(c[k] - h[k]) <= 1e-12 * abs(h[k]), k
    np.testing.assert_allclose(c["momentum"][: cfg.dim], h["momentum"], rtol=1e-12, atol=1e-15)
    assert abs(c["mass"] - m0) <= 1e-12 * m0   # split and merge conserve mass exactly
    assert np.isclose(c["energy"], c["kinetic"] + c["potential"])
    s.close()


def test_momentum_conserved_without_external_forces(gpu):
    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    cfg.gravity[0] = cfg.gravity[1] = cfg.gravity[2] = 0.0
    cfg.use_split = cfg.use_merge = 0
    pos, _, lvl = scenes.block_3d(cfg, counts=(16, 16, 16), spacing=0.01)
    pos = pos + np.float32(0.24)   # far from the walls
    vel = np.random.default_rng(2).normal(0, 0.05, pos.shape).astype(np.float32)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    p0 = s.conserved()["momentum"]
    scale = float(np.abs(vel).sum()) * cfg.mass[0]
    s.step(50)
    p1 = s.conserved()["momentum"]
    assert np.abs(p1 - p0).max() <= 1e-5 * scale, (p0, p1, scale)
    s.close()
