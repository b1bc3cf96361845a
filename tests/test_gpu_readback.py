"""Asynchronous readback into mapped page-locked memory equals the
synchronous readback of the same states, while steps keep running."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu


def test_async_readback_matches_sync(gpu):
    import torch
    cfg = sph.preset(sph.PRESET_REF_3D2)
    cfg.use_split = cfg.use_merge = 1
    pos, vel, lvl = scenes.ref_box_3d2(cfg)

    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    sync = []
    for _ in range(3):
        s.step(1)
        sync.append(s.read_particles().copy())
    s.close()

    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    rec = s.record_size
    nbytes = cfg.max_particle * rec
    bufs = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(3)]
    cnts = [torch.zeros(1, dtype=torch.int32, pin_memory=True) for _ in range(3)]
    for k in range(3):
        s.step(1)
        rc = s._lib.sph_read_particles_async(s._h, bufs[k].data_ptr(), nbytes, cnts[k].data_ptr())
        assert rc == 0, s._lib.sph_last_error(s._h)
    assert s._lib.sph_readback_wait(s._h) == 0
    assert s.sync_status() == 0
    s.close()
    for k in range(3):
        n = int(cnts[k].numpy().view(np.uint32)[0])
        assert n == len(sync[k])
        got = bufs[k].numpy()[: n * rec].tobytes()
        assert got == sync[k].tobytes(), f"readback {k} differs"
