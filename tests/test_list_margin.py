"""The margin argument behind the energy pass's use of the candidate lists,
checked in FP32 (no GPU needed).

The density pass lists every neighbour j with r2_old(i, j) < R^2, R^2 the
FP32 value (1 + 0.05)^2 h_max^2.  The energy pass accepts pairs with
r2_new(i, j) < h^2 (h <= h_max) and reads a particle's list only when
|d_i| + D <= 0.99 * 0.05 * h_max, D the step's largest displacement.  Then
every pair it would accept must be on the list.  Here r^2 is evaluated as the
kernels do (round-to-nearest subtractions, then fma(dz, dz, fma(dx, dx,
dy*dy))); the displacements push each pair apart as far as the budget allows
and the new distances sit just inside h, the worst case for the argument."""
import numpy as np

MARGIN = np.float32(0.05)


def _fma32(a, b, c):
    # float32 inputs: a*b is exact in float64, so only the sum rounds there
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def _r2(a, b):
    d = (a - b).astype(np.float32)   # float32 subtraction rounds to nearest
    t = _fma32(d[:, 0], d[:, 0], (d[:, 1] * d[:, 1]).astype(np.float32))
    return _fma32(d[:, 2], d[:, 2], t)


def _case(h, hmax, n, rng):
    h, hmax = np.float32(h), np.float32(hmax)
    hmax2 = np.float32(hmax * hmax)
    r = np.float32(np.float32(1.0) + MARGIN)
    re2 = np.float32(hmax2 * np.float32(r * r))
    budget = np.float32(np.float32(0.99) * MARGIN * np.sqrt(hmax2))
    # new positions: j at a distance just inside h of i, random direction
    xi_new = rng.uniform(0.2, 0.8, (n, 3)).astype(np.float32)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    dist = h * (1.0 - rng.uniform(0.0, 1e-6, n))
    xj_new = (xi_new + u * dist[:, None]).astype(np.float32)
    # displacements along the pair axis, apart, using the whole budget:
    # |d_i| + |d_j| <= |d_i| + D <= budget
    share = rng.uniform(0.0, 1.0, n)
    di = (budget * share)[:, None] * u
    dj = (budget * (1.0 - share))[:, None] * u
    xi_old = (xi_new + di).astype(np.float32)
    xj_old = (xj_new - dj).astype(np.float32)
    accepted = _r2(xi_new, xj_new) < np.float32(h * h)
    listed = _r2(xj_old, xi_old) < re2   # the density pass takes r2_of(p_j, p_i)
    return accepted, listed


def test_every_accepted_energy_pair_is_listed():
    rng = np.random.default_rng(11)
    cases = [(0.01, 0.01), (0.0063, 0.01), (1.0, 1.0), (0.8, 1.0), (0.02, 0.02), (1.2, 1.2)]
    for h, hmax in cases:
        accepted, listed = _case(h, hmax, 200_000, rng)
        assert accepted.sum() > 100_000
        assert not (accepted & ~listed).any(), (h, hmax)


def test_the_margin_is_needed():
    # without the margin (lists cut at h_max) such pairs would be missed
    rng = np.random.default_rng(12)
    h = np.float32(0.01)
    accepted, _ = _case(h, h, 100_000, rng)
    xi = rng.uniform(0.2, 0.8, (1000, 3)).astype(np.float32)
    u = rng.normal(size=(1000, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    xj_new = (xi + u * (0.999 * h)).astype(np.float32)
    xj_old = (xj_new + u * (0.04 * h)).astype(np.float32)   # it moved 0.04 h closer
    assert (_r2(xj_old, xi) >= np.float32(h * h)).all()
    assert accepted.any()
