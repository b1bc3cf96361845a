"""Batched scenes (sph_set_scenes): many dam-break scenes with their own
boxes, viscosities and stiffnesses advance in the same launches, and every
scene's particles come out bit-identical to that scene run alone in a handle
with the same world and box.  Splits and merges stay on, so the per-scene
order of survivors, children and compaction is covered too."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level", "interior")


def _run(cfg, boxes, pos, vel, lvl, scene, steps, graph=False):
    s = sph.Solver(cfg)
    s.set_scenes(boxes)
    s.set_state(dict(pos=pos, vel=vel, level=lvl, scene=scene))
    if graph:
        s.set_graph(True)
    s.step(steps)
    assert s.sync_status() == 0
    st = s.get_state()
    s.close()
    return st


def _same(a, b):
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("preset,count,steps", [(sph.PRESET_DAM_3D2, 6, 60), (sph.PRESET_DAM_2D, 8, 60)])
def test_batched_equals_alone(gpu, preset, count, steps):
    base = sph.preset(preset)
    base.use_split = base.use_merge = 1
    base.merge_interior_steps = 20   # so merges happen inside the run
    cfg, boxes, pos, vel, lvl, scene, counts = scenes.batch_scenes(base, count, seed=3, n_min=512, n_max=4096)
    batched = _run(cfg, boxes, pos, vel, lvl, scene, steps)
    assert set(np.unique(batched["scene"])) == set(range(count))
    total_split = 0
    first = np.concatenate([[0], np.cumsum(counts)])
    for k in range(count):
        c1 = cfg.copy()
        c1.max_particle = int(4 * counts[k])
        sl = slice(first[k], first[k + 1])
        alone = _run(c1, [boxes[k]], pos[sl], vel[sl], lvl[sl], np.zeros(counts[k], np.uint32), steps)
        mine = batched["scene"] == k
        assert mine.sum() == len(alone["pos"]), f"scene {k}: particle count differs"
        for f in FIELDS:
            assert _same(batched[f][mine], alone[f]), f"scene {k}: {f} differs"
        total_split += int((alone["level"] == 2).sum())
    assert total_split > 0, "no split happened; the case does not cover adaptivity"


def test_batched_graph_equals_eager(gpu):
    base = sph.preset(sph.PRESET_DAM_3D2)
    base.use_split = base.use_merge = 1
    cfg, boxes, pos, vel, lvl, scene, _ = scenes.batch_scenes(base, 12, seed=5, n_min=512, n_max=4096)
    a = _run(cfg, boxes, pos, vel, lvl, scene, 30)
    b = _run(cfg, boxes, pos, vel, lvl, scene, 30, graph=True)
    for f in FIELDS + ("scene",):
        assert _same(a[f], b[f]), f


def test_scene_walls_hold(gpu):
    """Every particle stays inside its own box (walls at lo + r, hi - r)."""
    base = sph.preset(sph.PRESET_DAM_3D2)
    base.use_split = base.use_merge = 1
    cfg, boxes, pos, vel, lvl, scene, _ = scenes.batch_scenes(base, 10, seed=7, n_min=512, n_max=2048)
    st = _run(cfg, boxes, pos, vel, lvl, scene, 200)
    lo = np.array([b[0] for b in boxes], np.float32)[st["scene"]]
    hi = np.array([b[1] for b in boxes], np.float32)[st["scene"]]
    assert (st["pos"] >= lo).all() and (st["pos"] <= hi).all()
    assert np.isfinite(st["pos"]).all()


def test_scene_errors(gpu):
    base = sph.preset(sph.PRESET_DAM_3D2)
    cfg, boxes, pos, vel, lvl, scene, _ = scenes.batch_scenes(base, 4, seed=1, n_min=512, n_max=1024)
    s = sph.Solver(cfg)
    # overlapping boxes
    lo, hi, mu, k = boxes[0]
    with pytest.raises(sph.SphError):
        s.set_scenes([boxes[0], (lo, hi, mu, k)])
    # a box outside the world
    with pytest.raises(sph.SphError):
        s.set_scenes([([0.0, 0.0, 0.0], [cfg.world[0] * 2, 0.5, 0.5], mu, k)])
    s.set_scenes(boxes)
    bad = scene.copy()
    bad[0] = len(boxes)
    with pytest.raises(sph.SphError):
        s.set_state(dict(pos=pos, vel=vel, level=lvl, scene=bad))
    s.set_state(dict(pos=pos, vel=vel, level=lvl, scene=scene))
    # fewer scenes than the particles name
    with pytest.raises(sph.SphError):
        s.set_scenes(boxes[:2])
    # the record format has no scene index
    rec = s.read_particles()
    with pytest.raises(sph.SphError):
        s.write_particles_from(rec.ctypes.data, len(rec))
    s.close()
