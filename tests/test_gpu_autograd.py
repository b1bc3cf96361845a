"""The differentiable rollout behind a torch.autograd.Function (test harness
only; the library itself takes and returns host arrays).  The Function's
forward runs sph_rollout_forward + sph_splat_loss, its backward returns
sph_rollout_backward's gradients: torch.autograd then gives the same numbers
as the C-ABI, and a few steps of gradient descent on viscosity and stiffness
toward the target grid's values (0.15, 4) lower the loss."""
import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import scenes

pytestmark = pytest.mark.gpu

GRID_N = (32, 32, 32)
ORIGIN = (0.01, 0.01, 0.01)
SPACING = 0.02
STEPS, EVERY = 120, 20


def _scene():
    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    pos, _, lvl = scenes.block_3d(cfg, counts=(8, 8, 8), spacing=0.01, seed=2)
    pos = pos + np.float32(0.1)
    vel = np.random.default_rng(2).normal(0.0, 0.1, pos.shape).astype(np.float32)
    return cfg, pos, lvl, vel


def _run(cfg, pos, lvl, vel, mu, k, target):
    c = cfg.copy()
    c.viscosity, c.gas_constant = float(mu), float(k)
    s = sph.Solver(c)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.rollout_forward(STEPS, EVERY)
    loss, _ = s.splat_loss(GRID_N, ORIGIN, SPACING, target)
    g = s.rollout_backward(len(pos))
    s.close()
    return loss, g


def _rollout_function(torch, cfg, pos, lvl, target):
    class RolloutLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, vel0, params):
            loss, g = _run(cfg, pos, lvl, vel0.detach().cpu().numpy().astype(np.float32),
                           params[0].item(), params[1].item(), target)
            ctx.save_for_backward(torch.from_numpy(g["d_vel0"]).to(vel0.dtype),
                                  torch.from_numpy(g["d_params"][0].copy()).to(params.dtype))
            return vel0.new_tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            d_vel0, d_params = ctx.saved_tensors
            return gout.to(d_vel0.dtype) * d_vel0, gout.to(d_params.dtype) * d_params

    return RolloutLoss.apply


def _target(cfg, pos, lvl, vel):
    t = cfg.copy()
    t.viscosity, t.gas_constant = 0.15, 4.0
    s = sph.Solver(t)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(STEPS)
    _, grid = s.splat_loss(GRID_N, ORIGIN, SPACING, np.zeros(np.prod(GRID_N), np.float32))
    s.close()
    return grid


def test_autograd_function_matches_the_c_abi(gpu):
    import torch
    cfg, pos, lvl, vel = _scene()
    target = _target(cfg, pos, lvl, vel)
    f = _rollout_function(torch, cfg, pos, lvl, target)
    vel0 = torch.tensor(vel, requires_grad=True)
    params = torch.tensor([0.1, 3.0], dtype=torch.float64, requires_grad=True)
    loss = f(vel0, params)
    loss.backward()
    L, g = _run(cfg, pos, lvl, vel, 0.1, 3.0, target)
    assert loss.item() == L
    assert vel0.grad.numpy().tobytes() == g["d_vel0"].tobytes()
    np.testing.assert_allclose(params.grad.numpy(), g["d_params"][0], rtol=1e-12)


def test_gradient_descent_on_constants_lowers_the_loss(gpu):
    import torch
    cfg, pos, lvl, vel = _scene()
    target = _target(cfg, pos, lvl, vel)
    f = _rollout_function(torch, cfg, pos, lvl, target)
    vel0 = torch.tensor(vel)
    # sign descent with halving relative steps (a direction check, not an
    # optimiser): each step must lower the loss
    params = torch.tensor([0.1, 3.0], dtype=torch.float64, requires_grad=True)
    losses = []
    for step in (0.2, 0.1, 0.05, None):
        params.grad = None
        loss = f(vel0, params)
        loss.backward()
        losses.append(loss.item())
        if step is not None:
            with torch.no_grad():
                params -= step * params.abs() * torch.sign(params.grad)
    assert all(b < a for a, b in zip(losses, losses[1:])), losses
