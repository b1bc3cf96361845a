"""Steps replayed as CUDA graphs give bit-identical states to eager steps,
across buffer parities, splits, merges, a config change (recapture) and a
surface-building step (which runs uncaptured)."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu


def _run(cfg, st, graph, steps, change_at=None):
    s = sph.Solver(cfg)
    s.set_graph(graph)
    s.set_state(st)
    for k in range(steps):
        if change_at is not None and k == change_at:
            c2 = cfg.copy()
            c2.viscosity = cfg.viscosity * 1.5
            c2.grid_every = 3 if cfg.dim == 3 else 0
            s.set_config(c2)
        s.step(1)
    assert s.sync_status() == 0
    out = s.read_particles()
    s.close()
    return out


@pytest.mark.parametrize("preset,scene", [(sph.PRESET_REF_3D2, scenes.ref_box_3d2),
                                          (sph.PRESET_REF_2D, scenes.ref_init_2d),
                                          (sph.PRESET_REF_3D4, scenes.ref_box_3d4)])
def test_graph_replay_matches_eager(preset, scene, gpu):
    cfg = sph.preset(preset)
    cfg.use_split = cfg.use_merge = 1
    pos, vel, lvl = scene(cfg)
    st = dict(pos=pos, vel=vel, level=lvl)
    a = _run(cfg, st, False, 9, change_at=4)
    b = _run(cfg, st, True, 9, change_at=4)
    assert len(a) == len(b)
    assert a.tobytes() == b.tobytes()
