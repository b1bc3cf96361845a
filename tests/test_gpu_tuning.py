"""Launch-shape autotuner (sph_autotune / sph_set_tuning): it leaves the state
as it found it, its choices are valid shapes, and stepping with any shape
gives results bit-identical to the default shapes."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level", "interior")


def _solver():
    cfg = sph.preset(sph.PRESET_DAM_3D2)
    pos, vel, lvl = scenes.dam_3d2(cfg)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(5)
    return s


def test_autotune_keeps_state_and_results(gpu):
    a = _solver()
    before = a.get_state()
    t = a.autotune(reps=2)
    after = a.get_state()
    for f in FIELDS:
        assert before[f].tobytes() == after[f].tobytes(), f
    for k, st in enumerate(t["stages"]):
        assert t["block"][k] in (128, 256, 512)
        if st in ("force_integrate", "energy_split"):
            assert t["block"][k] in (128, 256)
        assert t["blocks_per_sm"][k] in (2, 4, 8, 16, 32, 64)
    assert t["step_ms_after"] <= t["step_ms_before"] * 1.1
    b = _solver()
    a.step(20)
    b.step(20)
    sa, sb = a.get_state(), b.get_state()
    for f in FIELDS:
        assert sa[f].tobytes() == sb[f].tobytes(), f
    a.close()
    b.close()


def test_extreme_shapes_same_results(gpu):
    a, b = _solver(), _solver()
    n = 8
    a.set_tuning([128] * n, [2] * n)
    b.set_tuning([512, 512, 512, 512, 256, 256, 512, 512], [32] * n, [0, 0, 0, 0, 1, 0, 0, 0])
    b.set_graph(True)
    a.step(15)
    b.step(15)
    sa, sb = a.get_state(), b.get_state()
    for f in FIELDS:
        assert sa[f].tobytes() == sb[f].tobytes(), f
    with pytest.raises(sph.SphError):
        a.set_tuning([256, 256, 256, 256, 512, 256, 256, 256], [8] * n)   # force tops out at 256
    with pytest.raises(sph.SphError):
        a.set_tuning([256] * n, [0] * n)
    a.close()
    b.close()
