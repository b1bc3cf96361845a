"""CUDA path vs the CPU oracle, stage by stage, through the C-ABI.

For each reference preset (2D, 3D-2 two-way, 3D-4 four-way) and the SI
workload presets: a state S0 is produced on the GPU by a few warm-up steps of
the CUDA solver itself; then from S0 one step runs with split/merge off and
one with them on, and every stage is checked against the oracle fed the same
FP32 inputs (see tests/_parity.py for the tolerances).
"""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes
from oracle import oracle as O
from tests._parity import check_close, check_equal

pytestmark = pytest.mark.gpu

def _obstacles(c):
    c.use_cylinder = 1       # the reference's three spheres (SPH-3D-2/sph_system.cu:242-282)
    c.push_left = 1          # push force (SPH-3D-2/sph_system.cu:229-236)


def _push_right(c):
    c.push_right = 1         # the 3D-4 push force from the right (SPH-3D-4/sph_system.cu:236-242)


def _mouse(c):
    c.extern_force_on = 1    # 2D mouse force (SPH-2D/sph_system.cu:781-789)
    c.extern_click[0], c.extern_click[1] = 8.0, 8.0
    c.extern_force[0], c.extern_force[1] = 3.0, -2.0


CASES = {
    "ref_2d": (sph.PRESET_REF_2D, scenes.ref_init_2d, 10),
    "ref_3d2": (sph.PRESET_REF_3D2, scenes.ref_box_3d2, 8),
    "ref_3d4": (sph.PRESET_REF_3D4, lambda c: _crop(scenes.ref_box_3d4(c), 14.0), 4),
    "dam_2d": (sph.PRESET_DAM_2D, scenes.dam_2d, 3),
    "dam_3d2_small": (sph.PRESET_DAM_3D2, lambda c: scenes.block_3d(c, (24, 24, 12), 0.01, seed=3), 3),
    "ref_3d2_obstacles": (sph.PRESET_REF_3D2, scenes.ref_box_3d2, 8, _obstacles),
    # the right third of the 3D-4 slab, where the push from the right acts (x > 2W/3)
    "ref_3d4_push_right": (sph.PRESET_REF_3D4, lambda c: _crop_right(scenes.ref_box_3d4(c), 30.0), 4,
                           _push_right),
    "ref_2d_mouse": (sph.PRESET_REF_2D, scenes.ref_init_2d, 10, _mouse),
    # the benchmark workload at full size: 1,114,112 particles, four-way
    "dam_3d4_full": (sph.PRESET_DAM_3D4, scenes.dam_3d4, 2),
}


def _crop(scene, xmax):
    pos, vel, lvl = scene
    m = pos[:, 0] < xmax
    return pos[m], vel[m], lvl[m]


def _crop_right(scene, xmin):
    pos, vel, lvl = scene
    m = pos[:, 0] > xmin
    return pos[m], vel[m], lvl[m]


def _cfg(preset, split, merge, n, extra=None):
    c = sph.preset(preset)
    c.use_split = int(split)
    c.use_merge = int(merge)
    c.max_particle = max(4 * n * (c.split_ways - 1) + n, 1024)
    if extra:
        extra(c)
    return c


def step_pair(s, cfg_on, cfg_off, s0):
    """From state s0: one step with split/merge off, then the same step with
    them on (the solver is left after the second)."""
    s.set_config(cfg_off)
    s.set_state(s0)
    s.step(1)
    assert s.sync_status() == 0
    s1 = s.get_state()
    dbg = s.get_debug()
    s.set_config(cfg_on)
    s.set_state(s0)
    s.step(1)
    assert s.sync_status() == 0
    return s1, dbg, s.get_state(), s.get_debug()


def run_case(name):
    preset, scene, warm, *more = CASES[name]
    extra = more[0] if more else None
    pos, vel, lvl = scene(sph.preset(preset))
    cfg_on = _cfg(preset, 1, 1, len(pos), extra)
    cfg_off = _cfg(preset, 0, 0, len(pos), extra)
    s = sph.Solver(cfg_on)
    s.set_debug(True)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(warm)
    assert s.sync_status() == 0
    s0 = s.get_state()
    s1, dbg, s1_on, dbg_on = step_pair(s, cfg_on, cfg_off, s0)
    s.close()
    return cfg_on, cfg_off, s0, s1, dbg, s1_on, dbg_on


@pytest.mark.parametrize("name", list(CASES))
def test_step_parity(name, gpu):
    verify_step(name, *run_case(name))


# Per-step parity deep into the configured runs: the GPU advances the whole
# run; before each checked step its FP32 state is taken and that step is
# checked stage by stage against the oracle fed that state.
DEEP = {
    # 2D plain dam break, 4,096 particles, no adaptivity, the 1,000-step run
    "dam_2d_run": (sph.PRESET_DAM_2D, scenes.dam_2d, 0, (1, 250, 500, 1000)),
    # 3D two-way dam break at full size (131,072 particles), split and merge
    # on, the 500-step run
    "dam_3d2_run": (sph.PRESET_DAM_3D2, scenes.dam_3d2, 1, (1, 100, 300, 500)),
    # the 1.1M-particle four-way benchmark workload (block + falling sphere),
    # the 200-step run, with its surface built every 10 steps as configured
    "dam_3d4_run": (sph.PRESET_DAM_3D4, scenes.dam_3d4, 1, (1, 100, 200)),
}


@pytest.mark.parametrize("name", list(DEEP))
def test_run_parity(name, gpu):
    preset, scene, adapt, checks = DEEP[name]
    pos, vel, lvl = scene(sph.preset(preset), seed=0)
    cfg_on = _cfg(preset, adapt, adapt, len(pos))
    cfg_off = _cfg(preset, 0, 0, len(pos))
    s = sph.Solver(cfg_on)
    s.set_debug(True)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    done = 0
    for k in checks:
        s.step(k - 1 - done)
        assert s.sync_status() == 0
        s0 = s.get_state()
        s1, dbg, s1_on, dbg_on = step_pair(s, cfg_on, cfg_off, s0)
        done = k
        verify_step(f"{name}@{k}", cfg_on, cfg_off, s0, s1, dbg, s1_on, dbg_on)
    s.close()


def verify_step(name, cfg_on, cfg, s0, s1, dbg, s1_on, dbg_on):
    n = len(s0["pos"])
    assert dbg["n"] == n and len(s1["pos"]) == n

    # (a) hash, stable sort, cell ranges: bit-exact
    key, idx, cs, ce = O.sort(cfg, s0["pos"])
    check_equal("cell keys", dbg["hash"], key)
    check_equal("sorted index", dbg["index"], idx)
    check_equal("cell_start", dbg["cell_start"], cs)
    check_equal("cell_end", dbg["cell_end"], ce)

    # (b) density / pressure / neighbour counts
    dens, press, nbr = O.density(cfg, s0["pos"], s0["level"], idx, cs, ce)
    check_equal("neighbour counts", dbg["nbr_count"], nbr)
    check_close(f"{name}/density", s1["dens"], dens)
    check_close(f"{name}/pressure", s1["press"], press)

    # (c) forces + integration
    acc, surf, amb = O.force(cfg, s0["pos"], s0["ev"], s0["level"], dens, press, idx, cs, ce)
    p64, v64, e64, a64, amb2 = O.integrate(cfg, s0["pos"], s0["vel"], s0["ev"], s0["level"], acc, dens)
    ok = ~(amb | amb2)
    check_close(f"{name}/surface |grad c|", s1["surface"], surf)
    check_close(f"{name}/acceleration", s1["acc"], a64, ok)
    check_close(f"{name}/velocity", s1["vel"], v64, ok)
    check_close(f"{name}/eval velocity", s1["ev"], e64, ok)
    check_close(f"{name}/position", s1["pos"], p64, ok)

    # (d) wavelet energy on the stale lists with the GPU's new positions
    en, tv = O.energy(cfg, s1["pos"], s1["vel"], s0["level"], idx, cs, ce)
    check_close(f"{name}/energy", s1["energy"], en)
    check_close(f"{name}/trans_vel", dbg["trans_vel"], tv)

    # (e) split + merge + compaction from the same post-energy state
    pre = {k: s1[k] for k in ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level")}
    pre["interior"] = s0["interior"]
    pre["sibling"] = s0["sibling"]
    exp, split, rem = O.adapt(cfg_on, pre, nbr, idx, cs, ce, cap=cfg_on.max_particle)
    check_equal("split flags", dbg_on["split_flag"], split)
    check_equal("merge flags", dbg_on["removed"], rem)
    assert len(s1_on["pos"]) == len(exp["pos"]), "particle count after split/merge"
    check_equal("levels", s1_on["level"], exp["level"])
    check_equal("interior counters", s1_on["interior"], exp["interior"])
    check_equal("split-group links", s1_on["sibling"], exp["sibling"])
    for k in ("pos", "vel", "ev", "acc", "energy"):
        check_close(f"{name}/adapted {k}", s1_on[k], exp[k])
    for k in ("dens", "press", "surface"):
        check_close(f"{name}/adapted {k}", s1_on[k], exp[k])
