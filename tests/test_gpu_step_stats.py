"""sph_last_step_stats: the last step's particle counts agree with the state
and with the split/merge bookkeeping, on every launch path (separate
launches, graph replay, persistent launches of several steps)."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["eager", "graph", "persistent"])
def test_step_stats_match_the_state(mode, gpu):
    cfg = sph.preset(sph.PRESET_DAM_3D4)
    pos, vel, lvl = scenes.block_3d(cfg, (24, 24, 12), 0.005, seed=3)
    cfg.max_particle = 4 * len(pos)
    cfg.grid_every = 0
    cfg.merge_interior_steps = 3   # merges within the run
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.set_graph(mode == "graph")
    s.set_persistent(mode == "persistent")
    ways = 4 if cfg.split_ways == 4 else 2
    splits = merges = 0
    for _ in range(12):
        n0 = s.num_particles()
        s.step(1)
        st = s.last_step_stats()
        state = s.get_state()
        assert st["error"] == 0
        assert st["n_start"] == n0
        assert st["n_end"] == st["n_start"] + st["n_split"] * (ways - 1) - st["n_removed"]
        assert st["n_end"] == s.num_particles() == len(state["level"])
        assert st["n_level2"] == int((state["level"] == 2).sum())
        splits += st["n_split"]
        merges += st["n_removed"]
    s.close()
    assert splits > 0


def test_step_stats_after_a_multi_step_launch(gpu):
    pos, vel, lvl = scenes.dam_2d(sph.preset(sph.PRESET_DAM_2D))
    cfg = sph.preset(sph.PRESET_DAM_2D)
    cfg.use_split = cfg.use_merge = 0
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    with pytest.raises(sph.SphError):
        s.last_step_stats()          # no step since the state was set
    s.set_persistent(True)
    s.step(10)
    assert s.last_launch_count() == 1
    st = s.last_step_stats()
    assert st == dict(n_start=len(pos), n_split=0, n_removed=0, n_end=len(pos), n_level2=0,
                      split_suppressed=0, error=0)
    s.close()
