"""Failure reporting without faulting the GPU: a non-finite particle is
reported by sph_sync (SPH_ERR_NONFINITE) and the handle stays usable; a
split that would exceed the capacity is skipped and reported
(SPH_ERR_CAPACITY); work can be bound to a caller's stream."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "ev", "dens", "press", "level")


def test_nonfinite_reported_and_handle_usable(gpu):
    cfg = sph.preset(sph.PRESET_DAM_2D)
    pos, vel, lvl = scenes.dam_2d(cfg)
    vel = vel.copy()
    vel[17, 0] = np.nan
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(2)
    assert s.sync_status() == sph.SPH_ERR_NONFINITE
    assert s.sync_status() == 0          # reported once, then cleared
    pos2, vel2, lvl2 = scenes.dam_2d(cfg)
    s.set_state(dict(pos=pos2, vel=vel2, level=lvl2))
    s.step(2)
    assert s.sync_status() == 0
    assert np.isfinite(s.get_state()["pos"]).all()
    s.close()


def test_capacity_guard(gpu):
    cfg = sph.preset(sph.PRESET_DAM_3D2)
    pos, vel, lvl = scenes.block_3d(cfg, (16, 16, 8), 0.01)
    cfg.max_particle = len(pos) + 8      # no room for the surface splits
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(1)
    assert s.sync_status() == sph.SPH_ERR_CAPACITY
    assert s.num_particles() == len(pos)  # the splits were skipped
    s.close()


def test_caller_stream(gpu):
    import torch
    cfg = sph.preset(sph.PRESET_DAM_2D)
    pos, vel, lvl = scenes.dam_2d(cfg)
    a, b = sph.Solver(cfg), sph.Solver(cfg)
    for h in (a, b):
        h.set_state(dict(pos=pos, vel=vel, level=lvl))
    st = torch.cuda.Stream()
    b.set_stream(st.cuda_stream)
    assert b.stream_ptr == st.cuda_stream
    a.step(10)
    b.step(10)
    st.synchronize()
    sa, sb = a.get_state(), b.get_state()
    for f in FIELDS:
        assert sa[f].tobytes() == sb[f].tobytes(), f
    b.set_stream(0)
    assert b.stream_ptr != st.cuda_stream
    a.close()
    b.close()
