"""The FP64 rollout replay (oracle/sph_rollout_ref.c) that checks the GPU
adjoint: its hand-written adjoint must equal central finite differences of
its own forward, on a hand-built topology with a split, a merge and wall
contacts (no GPU needed)."""
import numpy as np
import pytest

import sca2012_b200 as sph
from oracle import oracle as O

EMPTY = 0xFFFFFFFF


def _pairs(cfg, x, level):
    """Density and force lists of positions x (FP64) under the step's rules."""
    n = len(x)
    h = np.array([cfg.kernel[0 if l == 1 else 1] for l in level], np.float64)
    d_off, d_nbr, f_off, f_nbr = [0], [], [0], []
    for i in range(n):
        r2 = ((x - x[i]) ** 2).sum(1)
        for j in range(n):
            if j != i and r2[j] < h[i] ** 2:
                d_nbr.append(j)
        for j in range(n):
            if j != i and r2[j] < max(h[i], h[j]) ** 2 and r2[j] >= cfg.close_r2:
                r = np.sqrt(r2[j])
                f_nbr.append(j | (int(h[i] - r > 0) << 30) | (int(h[j] - r > 0) << 31))
        d_off.append(len(d_nbr))
        f_off.append(len(f_nbr))
    u = lambda a: np.array(a if len(a) else [0], np.uint32)
    return dict(dens_off=u(d_off), dens_nbr=u(d_nbr), force_off=u(f_off), force_nbr=u(f_nbr))


def _topology(cfg, x0, T):
    """T steps on a 4x4x4 block: particle 0 splits at step 1, it and its
    child merge back at step 3 (leader 0), particle 5 touches the low x wall
    at step 2."""
    hs2 = cfg.kernel[1] / 2
    x = x0.astype(np.float64).copy()
    level = np.ones(len(x), np.uint32)
    steps = []
    for t in range(T):
        n = len(x)
        d = dict(n=n, split_on=1, level=level.copy(), wall=np.zeros(n, np.uint32),
                 split=np.zeros(n, np.uint32), dst=np.arange(n, dtype=np.uint32),
                 child=np.full(n, n, np.uint32), merge_leader=np.full(n, EMPTY, np.uint32))
        d.update(_pairs(cfg, x, level))
        n_next = n
        if t == 1:
            d["split"][0] = 1
            n_next = n + 1
            c = x[0].copy()
            c[0] -= hs2
            x[0, 0] += hs2
            x = np.vstack([x, c])
            level = np.append(level, 2).astype(np.uint32)
            level[0] = 2
        elif t == 2:
            d["wall"][5] = 2      # low wall of x
        elif t == 3:
            d["merge_leader"][0] = 0
            d["merge_leader"][n - 1] = 0
            d["dst"][n - 1] = EMPTY
            n_next = n - 1
            x = x[:-1]
            level = level[:-1].copy()
            level[0] = 1
        d["n_next"] = n_next
        steps.append(d)
    return steps


@pytest.fixture(scope="module")
def case():
    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    rng = np.random.default_rng(4)
    g = np.indices((4, 4, 4)).reshape(3, -1).T
    x0 = 0.2 + g * 0.0098 + rng.uniform(-1e-4, 1e-4, g.shape)
    v0 = rng.normal(0, 0.1, x0.shape)
    steps = _topology(cfg, x0, 5)
    n = (8, 8, 8)
    rep = O.Rollout64(cfg, steps, n, (0.18, 0.18, 0.18), 0.01, np.zeros(np.prod(n)))
    # target: the grid of the same rollout with viscosity 0.15 and stiffness 4
    _, rep.target = rep.loss(x0, v0, 0.15, 4.0, want_grid=True)
    return rep, x0, v0


def test_adjoint_matches_finite_differences(case):
    """Central differences agree to 1e-6 relative, up to their own rounding
    noise (about eps_mach * |L| / eps)."""
    rep, x0, v0 = case
    mu, k = 0.1, 3.0
    L, g = rep.grad(x0, v0, mu, k)
    assert np.isclose(L, rep.loss(x0, v0, mu, k), rtol=1e-14)
    rng = np.random.default_rng(7)
    eps = 1e-5
    noise = 50 * np.finfo(np.float64).eps * abs(L) / eps
    for _ in range(6):
        dx = rng.normal(size=x0.shape) * 1e-3
        dv = rng.normal(size=v0.shape) * 0.1
        dmu, dk = rng.normal() * 0.05, rng.normal()
        lp = rep.loss(x0 + eps * dx, v0 + eps * dv, mu + eps * dmu, k + eps * dk)
        lm = rep.loss(x0 - eps * dx, v0 - eps * dv, mu - eps * dmu, k - eps * dk)
        fd = (lp - lm) / (2 * eps)
        ad = (g["d_pos0"] * dx).sum() + (g["d_vel0"] * dv).sum() + g["d_mu"] * dmu + g["d_k"] * dk
        assert abs(ad - fd) <= 1e-6 * abs(fd) + noise, (ad, fd)
    # each parameter alone
    for which, h in (("mu", 1e-4), ("k", 1e-4)):
        a = dict(mu=mu, k=k)
        a[which] += h
        lp = rep.loss(x0, v0, a["mu"], a["k"])
        a[which] -= 2 * h
        lm = rep.loss(x0, v0, a["mu"], a["k"])
        fd = (lp - lm) / (2 * h)
        tol = 1e-5 * abs(fd) + 50 * np.finfo(np.float64).eps * abs(L) / h
        assert abs(g["d_" + which] - fd) <= tol, (which, g["d_" + which], fd)
