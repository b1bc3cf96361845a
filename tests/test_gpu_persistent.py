"""The persistent step (sph_set_persistent): the whole step as one
cooperative launch with grid-wide barriers.  It must give the ordinary
launches' results bit for bit -- plain and adaptive, 2D and 3D, reference
and SI presets, batched scenes, compensated positions -- and a barrier whose
wait runs out must end the launch with SPH_ERR_TIMEOUT and leave the handle
usable (the wait is made to run out by a poll limit of 0, so no GPU ever
hangs).  Steps without splits run several to a launch, with a barrier
between two steps.  Scenes of up to 4,096 particles run as one thread-block cluster
with hardware barriers; larger ones, and any wait limit other than the
default, use the polled barriers.  Without split and merge a persistent step
also hashes the state it wrote for the next one; that hash must be dropped
whenever anything else touches the state, the config or the cell counts."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level", "interior")


def _same(a, b):
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def _cfg(preset, adapt, n):
    c = sph.preset(preset)
    c.use_split = c.use_merge = adapt
    c.max_particle = max(4 * n, 1024)
    c.grid_every = 0
    return c


CASES = {
    "dam_2d_plain": (sph.PRESET_DAM_2D, scenes.dam_2d, 0, 200),
    "dam_2d_adaptive": (sph.PRESET_DAM_2D, scenes.dam_2d, 1, 60),
    "ref_2d": (sph.PRESET_REF_2D, scenes.ref_init_2d, 1, 30),
    "ref_3d2": (sph.PRESET_REF_3D2, scenes.ref_box_3d2, 1, 30),
    "ref_3d4": (sph.PRESET_REF_3D4, scenes.ref_box_3d4, 1, 20),
    "dam_3d2_block": (sph.PRESET_DAM_3D2, lambda c: scenes.block_3d(c, (24, 24, 12), 0.01, seed=2), 1, 60),
    "rollout_preset": (sph.PRESET_ROLLOUT_3D, lambda c: scenes.block_3d(c, (16, 16, 16), 0.01, seed=4), 1, 40),
    # above 16K particles: the polled barriers with 256-thread blocks, plain
    "dam_3d2_plain_32k": (sph.PRESET_DAM_3D2, lambda c: scenes.block_3d(c, (40, 40, 20), 0.01, seed=5), 0, 60),
}


def _run(cfg, st0, steps, persistent, scene_boxes=None, debug=False, spin_limit=sph._abi.PERSISTENT_SPIN_DEFAULT):
    s = sph.Solver(cfg)
    if scene_boxes is not None:
        s.set_scenes(scene_boxes)
    s.set_state(st0)
    s.set_persistent(persistent, spin_limit)
    s.set_debug(debug)
    s.step(steps)
    assert s.sync_status() == 0
    st = s.get_state()
    dbg = s.get_debug() if debug else None
    launches = s.last_launch_count()
    s.close()
    return st, dbg, launches


@pytest.mark.parametrize("name", list(CASES))
def test_persistent_equals_ordinary_launches(name, gpu):
    preset, scene, adapt, steps = CASES[name]
    pos, vel, lvl = scene(sph.preset(preset))
    cfg = _cfg(preset, adapt, len(pos))
    st0 = dict(pos=pos, vel=vel, level=lvl)
    a, da, la = _run(cfg, st0, steps, False, debug=True)
    b, db, lb = _run(cfg, st0, steps, True, debug=True)
    # steps without splits share launches (up to 256 each); with splits, one launch per step
    assert lb == (steps if adapt else -(-steps // 256)), lb
    assert la > lb
    for f in FIELDS:
        assert _same(a[f], b[f]), f"{name}: {f} differs"
    for f in ("hash", "index", "nbr_count", "split_flag", "removed", "cell_start", "cell_end", "trans_vel"):
        assert _same(np.asarray(da[f]), np.asarray(db[f])), f"{name}: debug {f} differs"
    if adapt:
        assert (b["level"] == 2).any() or name == "ref_3d4", "no split happened"


def test_persistent_polled_and_cluster_barriers_agree(gpu):
    """4,096 particles fit one 16-block cluster (hardware cluster barriers);
    a wait limit other than the default selects the polled barriers."""
    pos, vel, lvl = scenes.dam_2d(sph.preset(sph.PRESET_DAM_2D))
    cfg = _cfg(sph.PRESET_DAM_2D, 0, len(pos))
    st0 = dict(pos=pos, vel=vel, level=lvl)
    a, _, _ = _run(cfg, st0, 100, False)
    b, _, _ = _run(cfg, st0, 100, True)
    c, _, _ = _run(cfg, st0, 100, True, spin_limit=1 << 21)
    for f in FIELDS:
        assert _same(a[f], b[f]) and _same(a[f], c[f]), f


def test_persistent_batched_scenes(gpu):
    base = sph.preset(sph.PRESET_DAM_3D2)
    base.use_split = base.use_merge = 1
    base.merge_interior_steps = 20
    cfg, boxes, pos, vel, lvl, scene, _ = scenes.batch_scenes(base, 8, seed=9, n_min=512, n_max=4096)
    st0 = dict(pos=pos, vel=vel, level=lvl, scene=scene)
    a, _, _ = _run(cfg, st0, 50, False, boxes)
    b, _, _ = _run(cfg, st0, 50, True, boxes)
    for f in FIELDS + ("scene",):
        assert _same(a[f], b[f]), f


def test_persistent_barrier_timeout_is_reported_and_recoverable(gpu):
    pos, vel, lvl = scenes.dam_2d(sph.preset(sph.PRESET_DAM_2D))
    cfg = _cfg(sph.PRESET_DAM_2D, 0, len(pos))
    st0 = dict(pos=pos, vel=vel, level=lvl)
    ref, _, _ = _run(cfg, st0, 5, False)
    s = sph.Solver(cfg)
    s.set_state(st0)
    s.set_persistent(True, spin_limit=0)   # every barrier wait gives up at its first poll
    s.step(3)                              # the first step gives up, the next two do nothing
    assert s.sync_status() == sph.SPH_ERR_TIMEOUT
    # the handle is usable: restore the state and step normally
    s.set_state(st0)
    s.set_persistent(True)
    s.step(5)
    assert s.sync_status() == 0
    got = s.get_state()
    s.close()
    for f in FIELDS:
        assert _same(got[f], ref[f]), f


def test_persistent_precomputed_hash_follows_state_changes(gpu):
    """Plain persistent steps interleaved with graph replays, eager steps,
    a config change, a state reload and a switch of barrier kind give the
    ordinary launches' bits at every checkpoint."""
    pos, vel, lvl = scenes.dam_2d(sph.preset(sph.PRESET_DAM_2D))
    cfg = _cfg(sph.PRESET_DAM_2D, 0, len(pos))
    st0 = dict(pos=pos, vel=vel, level=lvl)
    cfg2 = _cfg(sph.PRESET_DAM_2D, 0, len(pos))
    cfg2.viscosity = cfg.viscosity * 1.5

    def script(s, persistent):
        out = []
        s.set_state(st0)
        s.set_persistent(persistent)
        s.step(7)
        out.append(s.get_state())
        s.set_persistent(False)          # graph replay from a hashed state
        s.step(3)
        s.set_persistent(persistent)
        s.step(4)
        s.set_graph(False)               # eager launches in between
        s.set_persistent(False)
        s.step(2)
        s.set_graph(True)
        s.set_persistent(persistent)
        s.step(5)
        out.append(s.get_state())
        s.set_config(cfg2)               # the config changes between two persistent steps
        s.step(6)
        out.append(s.get_state())
        s.set_persistent(persistent, 1 << 21)   # polled barriers from a hash the cluster path left
        s.step(6)
        mid = s.get_state()
        out.append(mid)
        s.set_state(dict(pos=mid["pos"], vel=mid["vel"] * 0.5, level=mid["level"]))   # reload
        s.step(5)
        out.append(s.get_state())
        assert s.sync_status() == 0
        return out

    sa = sph.Solver(cfg)
    a = script(sa, False)
    sa.close()
    sb = sph.Solver(cfg)
    b = script(sb, True)
    sb.close()
    for k, (x, y) in enumerate(zip(a, b)):
        for f in FIELDS:
            assert _same(x[f], y[f]), f"checkpoint {k}: {f} differs"


def test_persistent_multi_step_launch_waits_for_readbacks(gpu):
    """An asynchronous readback of the current state, then three steps in one
    launch (which writes both state buffers), then another readback: both
    equal the synchronous readbacks of an ordinary run."""
    import torch
    pos, vel, lvl = scenes.dam_2d(sph.preset(sph.PRESET_DAM_2D))
    cfg = _cfg(sph.PRESET_DAM_2D, 0, len(pos))
    st0 = dict(pos=pos, vel=vel, level=lvl)
    s = sph.Solver(cfg)
    s.set_state(st0)
    want = []
    for k in (1, 3):
        s.step(k)
        want.append(s.read_particles())   # a view of its own buffer (a copy drops the pad bytes)
    s.close()
    s = sph.Solver(cfg)
    s.set_state(st0)
    s.set_persistent(True)
    nbytes = cfg.max_particle * s.record_size
    bufs = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    cnts = [torch.zeros(1, dtype=torch.int32, pin_memory=True) for _ in range(2)]
    for j, k in enumerate((1, 3)):
        s.step(k)
        s.read_particles_async_into(bufs[j].data_ptr(), nbytes, cnts[j].data_ptr())
    s.readback_wait()
    assert s.sync_status() == 0
    assert s.last_launch_count() == 1
    s.close()
    rec = want[0].dtype.itemsize
    for j in range(2):
        n = int(cnts[j].numpy().view(np.uint32)[0])
        assert n == len(want[j])
        assert bufs[j].numpy()[: n * rec].tobytes() == want[j].tobytes(), f"readback {j} differs"


def test_persistent_runs_break_at_surface_steps(gpu):
    """Plain 3D steps with a density grid and marching cubes every 5 steps:
    the persistent launches stop before each surface step (which runs the
    ordinary launches) and resume after it; state and the last mesh equal the
    ordinary path's."""
    import ctypes as C
    cfg = sph.preset(sph.PRESET_DAM_3D2)
    pos, vel, lvl = scenes.block_3d(cfg, (20, 20, 10), 0.01, seed=3)
    cfg.use_split = cfg.use_merge = 0
    cfg.grid_every = 5
    cfg.max_particle = 4 * len(pos)
    G = int(np.prod([cfg.ndens[a] for a in range(3)]))
    mx = min(3 * G, int(cfg.max_triangles)) if cfg.max_triangles else 3 * G

    def run(persistent):
        s = sph.Solver(cfg)
        s.set_state(dict(pos=pos, vel=vel, level=lvl))
        s.set_persistent(persistent)
        s.step(23)   # surface steps 0, 5, 10, 15, 20
        assert s.sync_status() == 0
        launches = s.last_launch_count()
        bufs = [np.zeros((mx, 3), np.float32) for _ in range(6)]
        mv = sph.MeshView()
        mv.max_triangles = mx
        for k, b in zip(("v0", "v1", "v2", "n0", "n1", "n2"), bufs):
            setattr(mv, k, b.ctypes.data_as(C.POINTER(C.c_float)))
        assert s._lib.sph_extract_surface(s._h, C.byref(mv)) == 0
        nt = int(mv.num_triangles)
        mesh = np.stack([b[:nt] for b in bufs], 1)
        st = s.get_state()
        s.close()
        return st, mesh, launches

    a, ma, la = run(False)
    b, mb, lb = run(True)
    for f in FIELDS:
        assert _same(a[f], b[f]), f
    assert len(ma) > 100 and _same(ma, mb)
    assert lb < la
