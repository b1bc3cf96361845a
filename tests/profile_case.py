"""Fixed workload runner for profiling the step's kernels under ncu (test tooling).

    python tests/profile_case.py [--particles N] [--steps K] [--adaptive 0|1]
                                 [--block B0,..,B7 --bpsm P0,..,P7] [--persistent]
                                 [--workload dam_3d4|dam_2d]

Runs the four-way dam-break workload for K steps on cuda:0 and exits 0.  By
default the block is shrunk to about 300,000 particles (inputs still larger
than L2, about 0.5 GB on the device), which is the size for multi-pass
captures; --particles 0 runs the full 1,114,112-particle workload, which is
only for one-pass captures (the launch list).  Every step issues each kernel
once, so with K steps:

    # launch list (one pass per launch)
    ncu --metrics gpu__time_duration.sum --clock-control none --csv \
        --log-file launches.csv python tests/profile_case.py --particles 0
    # one kernel, one launch, all sections (about 40 passes)
    ncu --set full --clock-control none -k regex:k_density -s <K-1> -c 1 \
        -o prof python tests/profile_case.py

Always pass --clock-control none: without it ncu locks the GPU clocks.
Device memory stays near 450 bytes per particle of capacity (capacity = 1.5 x
the initial count).  --block/--bpsm set the launch shapes per tuned stage (the
order of sph_tuning: hash, scatter, reorder, density, force, energy, merge,
write), e.g. the ones the benchmark's autotuner reported.
"""
import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import sca2012_b200 as sph  # noqa: E402
from sca2012_b200 import scenes  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=300000, help="0 = the full 1,114,112-particle workload")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--adaptive", type=int, default=1)
    ap.add_argument("--block", default="")
    ap.add_argument("--bpsm", default="")
    ap.add_argument("--regcap", default="")
    ap.add_argument("--workload", default="dam_3d4", choices=["dam_3d4", "dam_2d"],
                    help="dam_2d: the 4,096-particle 2D dam (no adaptivity), stepped K steps twice")
    ap.add_argument("--persistent", action="store_true",
                    help="persistent launches (dam_2d: one launch per K steps; dam_3d4: one per step)")
    a = ap.parse_args()
    if a.workload == "dam_2d":
        cfg = sph.preset(sph.PRESET_DAM_2D)
        pos, vel, lvl = scenes.dam_2d(cfg, seed=0)
        s = sph.Solver(cfg)
        s.set_persistent(a.persistent)
        s.set_state(dict(pos=pos, vel=vel, level=lvl))
        for _ in range(2):   # persistent: two launches of K steps each (K <= 256)
            s.step(a.steps)
        rc = s.sync_status()
        s.close()
        print(f"profile_case: 2D dam, 2 x {a.steps} steps, persistent {a.persistent}, status {rc}")
        return 0 if rc == 0 else 1
    cfg = sph.preset(sph.PRESET_DAM_3D4)
    pos, vel, lvl = scenes.dam_3d4(cfg)
    if a.particles and a.particles < len(pos):
        keep = np.argsort(pos[:, 0], kind="stable")[: a.particles]
        keep.sort()
        pos, vel, lvl = pos[keep], vel[keep], lvl[keep]
    cfg.use_split = a.adaptive
    cfg.use_merge = a.adaptive
    cfg.max_particle = int(len(pos) * 1.5) + 1024
    s = sph.Solver(cfg)
    s.set_persistent(a.persistent)
    if a.block or a.bpsm or a.regcap:
        t = s.get_tuning()
        block = [int(x) for x in a.block.split(",")] if a.block else t["block"]
        bpsm = [int(x) for x in a.bpsm.split(",")] if a.bpsm else t["blocks_per_sm"]
        cap = [int(x) for x in a.regcap.split(",")] if a.regcap else t["reg_cap"]
        s.set_tuning(block, bpsm, cap)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    for k in range(a.steps):   # the particle count each step starts with (launch k of each kernel)
        print(f"profile_case: step {k + 1} starts with {s.num_particles()} particles")
        s.step(1)
    rc = s.sync_status()
    n = s.num_particles()
    s.close()
    print(f"profile_case: {len(pos)} -> {n} particles after {a.steps} steps, status {rc}")
    return 0 if rc == 0 else 1


if __name__ == "__main__":
    sys.exit(main())
