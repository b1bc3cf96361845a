"""Differentiable rollout on the GPU (sph_rollout_forward / sph_splat_loss /
sph_rollout_backward), the differentiable-rollout workload at a reduced
size (512 particles instead of 32,768; 200 steps, checkpoints every 20): a
jittered lattice block with initial velocities drawn N(0, 0.1^2), two-way
split and merge on, a 32^3 density-grid loss against the grid of a run with
viscosity 0.15 and stiffness 4.  Checked against the FP64 host
replay of the recorded topology (its own adjoint, which test_rollout_ref.py
checks against finite differences) and against FP64 central finite
differences of that replay: gradients within 1e-3 relative."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

GRID_N = (32, 32, 32)
ORIGIN = (0.01, 0.01, 0.01)
SPACING = 0.02
FIELDS = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level", "interior")


def _case(counts, seed, merge_steps):
    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    cfg.merge_interior_steps = merge_steps
    # level-2 particles of a cell paired in sorted order: this rule merges far
    # more often than the preset's split-group rule, so the adjoint's merge
    # path gets the most exercise, and its gradient is large enough that the
    # 1e-3 relative bound per direction sits above the FP32 trajectory's
    # rounding (tests/test_gpu_gradcheck_full.py runs the split-group rule)
    cfg.merge_rule = sph._abi.MERGE_INTERIOR
    pos, _, lvl = scenes.block_3d(cfg, counts=counts, spacing=0.01, seed=seed)
    pos = pos + np.float32(0.1)   # away from the low walls
    rng = np.random.default_rng(seed)
    vel = rng.normal(0.0, 0.1, pos.shape).astype(np.float32)
    return cfg, pos, vel, lvl


def _target(cfg, pos, vel, lvl, T):
    t = cfg.copy()
    t.viscosity, t.gas_constant = 0.15, 4.0
    s = sph.Solver(t)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(T)
    _, grid = s.splat_loss(GRID_N, ORIGIN, SPACING, np.zeros(np.prod(GRID_N), np.float32))
    s.close()
    return grid


@pytest.fixture(scope="module")
def rollout():
    from oracle import oracle as O
    T, every = 200, 20
    cfg, pos, vel, lvl = _case((8, 8, 8), 3, 5)
    target = _target(cfg, pos, vel, lvl, T)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.rollout_forward(T, every)
    L, grid = s.splat_loss(GRID_N, ORIGIN, SPACING, target)
    g = s.rollout_backward(len(pos))
    final = s.get_state()
    topo = [s.rollout_topology(t) for t in range(T)]
    g2 = s.rollout_backward(len(pos))
    after = s.get_state()
    s.close()
    rep = O.Rollout64(cfg, topo, GRID_N, ORIGIN, SPACING, target)
    return dict(cfg=cfg, pos=pos, vel=vel, lvl=lvl, T=T, L=L, g=g, g2=g2, final=final, after=after,
                topo=topo, rep=rep, target=target)


def test_taping_leaves_forward_unchanged(gpu, rollout):
    r = rollout
    s = sph.Solver(r["cfg"])
    s.set_state(dict(pos=r["pos"], vel=r["vel"], level=r["lvl"]))
    s.step(r["T"])
    plain = s.get_state()
    s.close()
    for f in FIELDS:
        assert plain[f].tobytes() == r["final"][f].tobytes(), f
        assert plain[f].tobytes() == r["after"][f].tobytes(), f
    # the case covers adaptivity
    assert sum(int(t["split"].sum()) for t in r["topo"]) > 0
    assert sum(int((t["merge_leader"] != 0xFFFFFFFF).sum()) for t in r["topo"]) > 0


def test_backward_is_repeatable(gpu, rollout):
    r = rollout
    assert r["g"]["d_vel0"].tobytes() == r["g2"]["d_vel0"].tobytes()
    np.testing.assert_allclose(r["g"]["d_params"], r["g2"]["d_params"], rtol=1e-12)


def test_gradient_matches_fp64_replay(gpu, rollout):
    r = rollout
    cfg = r["cfg"]
    mu, k = float(cfg.viscosity), float(cfg.gas_constant)
    L64, g64 = r["rep"].grad(r["pos"].astype(np.float64), r["vel"].astype(np.float64), mu, k)
    assert abs(r["L"] - L64) <= 1e-3 * abs(L64), (r["L"], L64)
    g = r["g"]
    for key in ("d_vel0", "d_pos0"):
        a, b = g[key].astype(np.float64), g64[key]
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err <= 1e-3, (key, err)
    assert abs(g["d_params"][0, 0] - g64["d_mu"]) <= 1e-3 * abs(g64["d_mu"]), (g["d_params"][0, 0], g64["d_mu"])
    assert abs(g["d_params"][0, 1] - g64["d_k"]) <= 1e-3 * abs(g64["d_k"]), (g["d_params"][0, 1], g64["d_k"])


def test_gradient_matches_finite_differences(gpu, rollout):
    """FP64 central differences (eps 1e-6) of the replay on random
    directions in (initial velocities, viscosity, stiffness)."""
    r = rollout
    cfg = r["cfg"]
    mu, k = float(cfg.viscosity), float(cfg.gas_constant)
    x0 = r["pos"].astype(np.float64)
    v0 = r["vel"].astype(np.float64)
    L = r["rep"].loss(x0, v0, mu, k)
    rng = np.random.default_rng(11)
    eps = 1e-6
    noise = 50 * np.finfo(np.float64).eps * abs(L) / eps
    g = r["g"]
    for _ in range(8):
        dv = rng.normal(size=v0.shape)
        dmu, dk = rng.normal() * 0.1, rng.normal()
        nrm = np.sqrt((dv * dv).sum() + dmu * dmu + dk * dk)
        dv, dmu, dk = dv / nrm, dmu / nrm, dk / nrm
        lp = r["rep"].loss(x0, v0 + eps * dv, mu + eps * dmu, k + eps * dk)
        lm = r["rep"].loss(x0, v0 - eps * dv, mu - eps * dmu, k - eps * dk)
        fd = (lp - lm) / (2 * eps)
        ad = (g["d_vel0"] * dv).sum() + g["d_params"][0, 0] * dmu + g["d_params"][0, 1] * dk
        assert abs(ad - fd) <= 1e-3 * abs(fd) + noise, (ad, fd)


def test_rollout_errors(gpu):
    cfg = sph.preset(sph.PRESET_REF_3D2)   # reference integrator: not covered
    s = sph.Solver(cfg)
    pos, vel, lvl = scenes.ref_box_3d2(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    with pytest.raises(sph.SphError):
        s.rollout_forward(4, 2)
    s.close()
    cfg, pos, vel, lvl = _case((4, 4, 4), 1, 50)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    with pytest.raises(sph.SphError):   # no rollout yet
        s.rollout_backward(len(pos))
    s.rollout_forward(4, 2)
    with pytest.raises(sph.SphError):   # no loss yet
        s.rollout_backward(len(pos))
    s.splat_loss(GRID_N, ORIGIN, SPACING, np.zeros(np.prod(GRID_N), np.float32))
    s.step(1)
    with pytest.raises(sph.SphError):   # the state moved on
        s.rollout_backward(len(pos))
    s.close()


def _rollout_2d(T=120, every=25):
    cfg = sph.preset(sph.PRESET_DAM_2D)
    cfg.use_split = cfg.use_merge = 1
    cfg.merge_interior_steps = 5
    cfg.compensated_positions = 1
    pos = scenes.lattice((16, 16), 0.01, np.array([0.1, 0.1]), 5)
    lvl = np.ones(len(pos), np.uint32)
    vel = np.random.default_rng(5).normal(0.0, 0.1, pos.shape).astype(np.float32)
    gn, org, sp = (64, 64, 1), (0.005, 0.005, 0.0), 0.01
    t = cfg.copy()
    t.viscosity, t.gas_constant = 0.15, 4.0
    s = sph.Solver(t)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(T)
    _, target = s.splat_loss(gn, org, sp, np.zeros(64 * 64, np.float32))
    s.close()
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.rollout_forward(T, every)
    L, _ = s.splat_loss(gn, org, sp, target)
    g = s.rollout_backward(len(pos))
    topo = [s.rollout_topology(k, states=True) for k in range(T)]
    x_final = s.get_state()["pos"]
    s.close()
    return cfg, pos, vel, L, g, topo, (gn, org, sp, target), x_final


def test_rollout_2d_matches_fp64(gpu):
    """2D (plain volume means in merges, no z) against the FP64 replay."""
    from oracle import oracle as O
    cfg, pos, vel, L, g, topo, (gn, org, sp, target), x_final = _rollout_2d()
    assert sum(int(t["split"].sum()) for t in topo) > 0
    rep = O.Rollout64(cfg, topo, gn, org, sp, target)
    mu, k = float(cfg.viscosity), float(cfg.gas_constant)
    # the adjoint arithmetic alone: FP64 adjoint about the GPU's trajectory
    La, ga = rep.grad_along(pos.astype(np.float64), vel.astype(np.float64), mu, k, x_final)
    L64, g64 = rep.grad(pos.astype(np.float64), vel.astype(np.float64), mu, k)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    info = dict(L=L, La=La, L64=L64, along=rel(g["d_vel0"], ga["d_vel0"]), fp64=rel(g["d_vel0"], g64["d_vel0"]),
                mu=(g["d_params"][0, 0], g64["d_mu"]), k=(g["d_params"][0, 1], g64["d_k"]))
    assert info["along"] <= 5e-4, info
    assert abs(L - L64) <= 1e-3 * abs(L64), info
    assert info["fp64"] <= 1e-3, info
    assert abs(g["d_params"][0, 0] - g64["d_mu"]) <= 1e-3 * abs(g64["d_mu"]), info
    assert abs(g["d_params"][0, 1] - g64["d_k"]) <= 1e-3 * abs(g64["d_k"]), info


def test_batched_rollout_equals_alone(gpu):
    """Batched scenes through the adjoint: each scene's velocity gradient is
    bit-identical to the scene's own rollout in the same world (targets with
    disjoint support, so the batched loss is the sum of the scenes' losses),
    and the per-scene viscosity / stiffness gradients agree to FP64
    rounding (their sums use FP64 atomics)."""
    base = sph.preset(sph.PRESET_DAM_3D2)
    base.use_split = base.use_merge = 1
    base.merge_interior_steps = 5
    cfg, boxes, pos, vel0, lvl, scene, counts = scenes.batch_scenes(base, 4, seed=9, n_min=512, n_max=2048)
    vel = np.random.default_rng(9).normal(0.0, 0.1, pos.shape).astype(np.float32)
    T, every = 40, 10
    gn = tuple(int(cfg.ncell[a]) for a in range(3))
    org = tuple(0.5 * float(cfg.cell_size) for _ in range(3))
    sp = float(cfg.cell_size)
    N = int(np.prod(gn))
    # target: each scene run with its constants perturbed
    tb = [(lo, hi, mu * 1.5, k + 1.0) for lo, hi, mu, k in boxes]
    s = sph.Solver(cfg)
    s.set_scenes(tb)
    s.set_state(dict(pos=pos, vel=vel, level=lvl, scene=scene))
    s.step(T)
    _, target = s.splat_loss(gn, org, sp, np.zeros(N, np.float32))
    s.close()
    s = sph.Solver(cfg)
    s.set_scenes(boxes)
    s.set_state(dict(pos=pos, vel=vel, level=lvl, scene=scene))
    s.rollout_forward(T, every)
    Lb, _ = s.splat_loss(gn, org, sp, target)
    gb = s.rollout_backward(len(pos), nscenes=len(boxes))
    s.close()
    first = np.concatenate([[0], np.cumsum(counts)])
    La = 0.0
    for k in range(len(boxes)):
        c1 = cfg.copy()
        c1.max_particle = int(4 * counts[k])
        sl = slice(first[k], first[k + 1])
        s = sph.Solver(c1)
        s.set_scenes([boxes[k]])
        s.set_state(dict(pos=pos[sl], vel=vel[sl], level=lvl[sl]))
        s.rollout_forward(T, every)
        L, _ = s.splat_loss(gn, org, sp, target)   # other scenes' target nodes add a constant
        g = s.rollout_backward(int(counts[k]))
        s.close()
        assert g["d_vel0"].tobytes() == gb["d_vel0"][sl].tobytes(), f"scene {k}: d_vel0 differs"
        np.testing.assert_allclose(g["d_params"][0], gb["d_params"][k], rtol=1e-10)
        La += L
    assert np.isfinite(Lb)
