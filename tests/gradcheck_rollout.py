"""Full-size gradient check of the differentiable rollout (needs a GPU; a
script, not collected by pytest):

    python tests/gradcheck_rollout.py [--steps 200] [--dirs 64] [--out FILE]

Workload: a 32^3 block (32,768 particles, spacing 0.01) in the 0.64^3 box,
initial velocities N(0, 0.1^2), two-way split and merge on, 200 steps with
checkpoints every 20, loss = mean squared difference of the final 32^3
density grid from the grid of a run with viscosity 0.15 and stiffness 4.
The GPU gradient (FP32 forward and adjoint) is compared with the FP64 host
replay of the recorded topology -- its adjoint, and FP64 central finite
differences (eps 1e-6) on random unit directions in (initial velocities,
viscosity, stiffness) and on viscosity and stiffness alone.  Prints one JSON
line of error statistics.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def gradcheck(steps=200, every=20, block=32, dirs=64, eps=1e-6, seed=0):
    """Runs the check and returns its statistics (the JSON line's dict);
    tests/test_gpu_gradcheck_full.py calls it with 8 directions."""
    a = argparse.Namespace(steps=steps, every=every, block=block, dirs=dirs, eps=eps, seed=seed)
    import sca2012_b200 as sph
    from sca2012_b200 import scenes
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)

    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    pos, _, lvl = scenes.block_3d(cfg, counts=(a.block,) * 3, spacing=0.01, seed=a.seed)
    vel = np.random.default_rng(a.seed).normal(0.0, 0.1, pos.shape).astype(np.float32)
    gn, org, sp = (32, 32, 32), (0.01, 0.01, 0.01), 0.02
    tcfg = cfg.copy()
    tcfg.viscosity, tcfg.gas_constant = 0.15, 4.0
    ts = sph.Solver(tcfg)
    ts.set_state(dict(pos=pos, vel=vel, level=lvl))
    ts.step(a.steps)
    _, target = ts.splat_loss(gn, org, sp, np.zeros(32 ** 3, np.float32))
    ts.close()

    t0 = time.perf_counter()
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.rollout_forward(a.steps, a.every)
    L_gpu, _ = s.splat_loss(gn, org, sp, target)
    g = s.rollout_backward(len(pos))
    t_gpu = time.perf_counter() - t0
    topo = [s.rollout_topology(t, states=True) for t in range(a.steps)]
    x_final = s.get_state()["pos"]
    n_final = s.num_particles()
    s.close()
    splits = int(sum(int(t["split"].sum()) for t in topo))
    merges = int(sum(int((t["merge_leader"] != 0xFFFFFFFF).sum()) for t in topo))
    walls = int(sum(int((t["wall"] != 0).sum()) for t in topo))

    rep = O.Rollout64(cfg, topo, gn, org, sp, target)
    mu, k = float(cfg.viscosity), float(cfg.gas_constant)
    x0, v0 = pos.astype(np.float64), vel.astype(np.float64)
    t0 = time.perf_counter()
    L64, g64 = rep.grad(x0, v0, mu, k)
    t_ref = time.perf_counter() - t0
    # the same FP64 adjoint about the GPU's FP32 trajectory: isolates the
    # adjoint arithmetic from the forward's FP32 rounding
    La, ga = rep.grad_along(x0, v0, mu, k, x_final)

    def rel(a_, b_):
        return float(np.linalg.norm(np.asarray(a_, np.float64) - b_) / np.linalg.norm(b_))

    rng = np.random.default_rng(a.seed + 1)
    eps = a.eps
    noise = 50 * np.finfo(np.float64).eps * abs(L64) / eps
    dirs = []
    t0 = time.perf_counter()
    for _ in range(a.dirs):
        dv = rng.normal(size=v0.shape)
        dmu, dk = rng.normal(), rng.normal()
        nrm = np.sqrt((dv * dv).sum() + dmu * dmu + dk * dk)
        dv, dmu, dk = dv / nrm, dmu / nrm, dk / nrm
        fd = (rep.loss(x0, v0 + eps * dv, mu + eps * dmu, k + eps * dk) -
              rep.loss(x0, v0 - eps * dv, mu - eps * dmu, k - eps * dk)) / (2 * eps)
        ad = float((g["d_vel0"] * dv).sum() + g["d_params"][0, 0] * dmu + g["d_params"][0, 1] * dk)
        ad64 = float((g64["d_vel0"] * dv).sum() + g64["d_mu"] * dmu + g64["d_k"] * dk)
        dirs.append((ad, ad64, fd))
    par = {}
    for name, idx in (("viscosity", 0), ("gas_constant", 1)):
        h = eps
        args_p = [mu + h, k] if idx == 0 else [mu, k + h]
        args_m = [mu - h, k] if idx == 0 else [mu, k - h]
        fd = (rep.loss(x0, v0, *args_p) - rep.loss(x0, v0, *args_m)) / (2 * h)
        par[name] = {"gpu": float(g["d_params"][0, idx]), "fp64_adjoint": g64["d_mu" if idx == 0 else "d_k"],
                     "fp64_fd": fd, "rel_gpu_vs_fd": abs(g["d_params"][0, idx] - fd) / abs(fd)}
    t_fd = time.perf_counter() - t0
    d = np.array(dirs)
    rel_gpu = np.abs(d[:, 0] - d[:, 2]) / np.abs(d[:, 2])
    rel_64 = np.abs(d[:, 1] - d[:, 2]) / np.abs(d[:, 2])
    # the same errors against the gradient's norm (directions are unit
    # vectors, so a direction nearly orthogonal to the gradient has a small
    # |fd| and an inflated relative error)
    gnorm = float(np.sqrt((g64["d_vel0"] ** 2).sum() + g64["d_mu"] ** 2 + g64["d_k"] ** 2))
    nrm_gpu = np.abs(d[:, 0] - d[:, 2]) / gnorm
    out = {
        "workload": f"{a.block}^3 block, {a.steps} steps, checkpoints every {a.every}, 32^3 grid loss",
        "particles_initial": len(pos), "particles_final": n_final,
        "splits": splits, "merge_members": merges, "wall_contacts": walls,
        "loss_gpu": L_gpu, "loss_fp64": L64, "loss_rel": abs(L_gpu - L64) / abs(L64),
        "d_vel0_rel_vs_fp64_adjoint": rel(g["d_vel0"], g64["d_vel0"]),
        "d_pos0_rel_vs_fp64_adjoint": rel(g["d_pos0"], g64["d_pos0"]),
        "along_fp32_trajectory": {
            "loss_rel": abs(L_gpu - La) / abs(La),
            "d_vel0_rel": rel(g["d_vel0"], ga["d_vel0"]), "d_pos0_rel": rel(g["d_pos0"], ga["d_pos0"]),
            "d_viscosity_rel": abs(g["d_params"][0, 0] - ga["d_mu"]) / abs(ga["d_mu"]),
            "d_gas_constant_rel": abs(g["d_params"][0, 1] - ga["d_k"]) / abs(ga["d_k"])},
        "params": par,
        "directions": a.dirs, "eps": eps, "fd_noise_floor": noise,
        "dir_rel_gpu_vs_fd_max": float(rel_gpu.max()), "dir_rel_gpu_vs_fd_median": float(np.median(rel_gpu)),
        "dir_rel_fp64_adjoint_vs_fd_max": float(rel_64.max()),
        "dirs_within_1e-3": int((np.abs(d[:, 0] - d[:, 2]) <= 1e-3 * np.abs(d[:, 2]) + noise).sum()),
        "dir_err_over_grad_norm_max": float(nrm_gpu.max()),
        "dir_abs_fd_over_grad_norm_min": float(np.abs(d[:, 2]).min() / gnorm),
        "seconds": {"gpu_forward_backward": t_gpu, "fp64_adjoint": t_ref, "fp64_fd": t_fd},
        "omp_threads": O.get_threads(),
    }
    out["dir_rel_gpu_vs_fd"] = rel_gpu.tolist()
    out["dir_err_over_grad_norm"] = nrm_gpu.tolist()
    out["dir_abs_fd_over_grad_norm"] = (np.abs(d[:, 2]) / gnorm).tolist()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--every", type=int, default=20)
    ap.add_argument("--block", type=int, default=32)
    ap.add_argument("--dirs", type=int, default=64)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    out = gradcheck(a.steps, a.every, a.block, a.dirs, a.eps, a.seed)
    line = json.dumps(out)
    print(line, flush=True)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
