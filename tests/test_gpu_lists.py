"""Neighbour lists against the stencil walks: the density pass records each
particle's neighbour candidates (within 1.05 h_max of its start-of-step
position), and the force and energy passes filter that list instead of
walking the 3^DIM-cell stencil whenever it holds the walk's pairs.  With
walk_only = 1 every pass walks.  Both must give the same particles, bit for
bit, over many steps with splits and merges: at rest (the lists serve almost
every particle), with fast random velocities (some particles move farther
than the lists' margin allows or change cell, and walk), and so fast that no
list may be used."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level", "interior")


def _run(cfg, st, steps, walk_only, boxes=None):
    c = cfg.copy()
    c.walk_only = walk_only
    s = sph.Solver(c)
    if boxes is not None:
        s.set_scenes(boxes)
    s.set_state(st)
    s.step(steps)
    assert s.sync_status() == 0
    out = s.get_state()
    s.close()
    return out


def _same_runs(cfg, st, steps, boxes=None):
    a = _run(cfg, st, steps, 0, boxes)
    b = _run(cfg, st, steps, 1, boxes)
    assert len(a["pos"]) == len(b["pos"])
    for f in FIELDS:
        assert a[f].tobytes() == b[f].tobytes(), f"{f} differs between lists and walks"
    return a


@pytest.mark.parametrize("sigma", [0.0, 3.0, 40.0])
def test_lists_equal_walks_3d_four_way(gpu, sigma):
    cfg = sph.preset(sph.PRESET_DAM_3D4)
    pos, _, lvl = scenes.block_3d(cfg, counts=(32, 32, 24), spacing=0.005, seed=1)
    pos = (pos + np.float32(0.2)).astype(np.float32)
    vel = np.random.default_rng(1).normal(0.0, sigma, pos.shape).astype(np.float32)
    cfg.max_particle = 4 * len(pos)
    out = _same_runs(cfg, dict(pos=pos, vel=vel, level=lvl), 30)
    assert (out["level"] == 2).any(), "no split happened; the case does not cover adaptivity"


def test_lists_equal_walks_2d(gpu):
    cfg = sph.preset(sph.PRESET_DAM_2D)
    cfg.use_split = cfg.use_merge = 1
    cfg.merge_interior_steps = 10
    pos, vel, lvl = scenes.dam_2d(cfg, seed=2)
    vel = vel + np.random.default_rng(2).normal(0.0, 2.0, vel.shape).astype(np.float32)
    cfg.max_particle = 2 * len(pos)
    _same_runs(cfg, dict(pos=pos, vel=vel, level=lvl), 40)


def test_lists_equal_walks_batched(gpu):
    base = sph.preset(sph.PRESET_DAM_3D2)
    base.use_split = base.use_merge = 1
    base.merge_interior_steps = 20
    cfg, boxes, pos, vel, lvl, scene, _ = scenes.batch_scenes(base, 6, seed=4, n_min=512, n_max=4096)
    vel = vel + np.random.default_rng(4).normal(0.0, 2.0, vel.shape).astype(np.float32)
    _same_runs(cfg, dict(pos=pos, vel=vel, level=lvl, scene=scene), 40, boxes)


def _with_blob(pos, lvl, blob_counts, blob_spacing, seed):
    """Adds a dense lattice blob just above the block: its particles have far
    more than 128 candidates within 1.05 h_max, so their lists overflow and
    every consumer walks for them, next to particles that use their lists."""
    blob = scenes.lattice(blob_counts, blob_spacing, np.zeros(3), seed)
    lo = pos.min(0)
    top = pos[:, 1].max()
    blob = (blob + np.array([lo[0] + 0.02, top + 0.004, lo[2] + 0.02], np.float32)).astype(np.float32)
    return np.concatenate([pos, blob]), np.concatenate([lvl, np.ones(len(blob), np.uint32)])


def test_overflowing_lists_equal_walks(gpu):
    cfg = sph.preset(sph.PRESET_DAM_3D4)
    cfg.gas_constant = 0.05   # keeps the compressed blob's pressure finite over the run
    pos, _, lvl = scenes.block_3d(cfg, counts=(24, 24, 16), spacing=0.005, seed=5)
    pos = (pos + np.float32(0.2)).astype(np.float32)
    pos, lvl = _with_blob(pos, lvl, (8, 8, 8), 0.003, 6)
    vel = np.zeros_like(pos)
    cfg.max_particle = 4 * len(pos)
    # the blob's density neighbours (within h, inside the lists' 1.05 h_max)
    # already exceed the 128 entries a list holds
    s = sph.Solver(cfg)
    s.set_debug(True)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(1)
    assert s.get_debug()["nbr_count"].max() > 128
    s.close()
    _same_runs(cfg, dict(pos=pos, vel=vel, level=lvl), 12)


def test_adjoint_lists_equal_walks(gpu):
    """The backward pass rebuilds each taped step's candidate lists; with
    walk_only = 1 its force and density adjoints walk the stencil instead.
    The velocity and position gradients must agree bit for bit (each slot
    sums its pairs in walk order either way); the parameter gradients are
    FP64 atomics summed in arrival order, so they agree to rounding."""
    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    cfg.gas_constant = 0.5
    pos, _, lvl = scenes.block_3d(cfg, counts=(8, 8, 8), spacing=0.01, seed=7)
    pos = (pos + np.float32(0.1)).astype(np.float32)
    pos, lvl = _with_blob(pos, lvl, (7, 7, 7), 0.004, 8)
    vel = np.random.default_rng(7).normal(0.0, 0.1, pos.shape).astype(np.float32)
    grid_n, origin, spacing = (32, 32, 32), (0.01, 0.01, 0.01), 0.02
    target = np.zeros(np.prod(grid_n), np.float32)
    out = []
    for walk_only in (0, 1):
        c = cfg.copy()
        c.walk_only = walk_only
        s = sph.Solver(c)
        s.set_state(dict(pos=pos, vel=vel, level=lvl))
        s.rollout_forward(30, 10)
        loss, _ = s.splat_loss(grid_n, origin, spacing, target)
        g = s.rollout_backward(len(pos))
        assert s.sync_status() == 0
        s.close()
        out.append((loss, g))
    (l0, g0), (l1, g1) = out
    assert l0 == l1
    assert g0["d_vel0"].tobytes() == g1["d_vel0"].tobytes()
    assert g0["d_pos0"].tobytes() == g1["d_pos0"].tobytes()
    np.testing.assert_allclose(g0["d_params"], g1["d_params"], rtol=1e-12)
