"""The N > 1 bench path on CPU: two gloo ranks run independent replicas, and
the whole-job numbers are the slowest rank's time and the sum of the units
(bench.reduce_over_ranks); the replicas' workloads differ by seed."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as tdist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, u = bench.reduce_over_ranks(10.0 + rank, 1000.0 * (rank + 1), True, "cpu")
        tdist.barrier()
        q.put((rank, t, u))
    finally:
        tdist.destroy_process_group()


def test_reduce_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for _, t, u in got:
        assert t == 11.0 and u == 3000.0


def test_single_rank_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(5.0, 7.0, False, "cpu") == (5.0, 7.0)


def test_replica_seeds_differ():
    sys.path.insert(0, ROOT)
    import bench
    if not os.path.exists(os.path.join(ROOT, "sca2012_b200", "libsca2012_b200.so")):
        pytest.skip("library not built")
    _, p0, _, _ = bench.load_workload(0)
    _, p1, _, _ = bench.load_workload(1)
    assert p0.shape == p1.shape and (p0 != p1).any()


@pytest.mark.parametrize("world", [2, 3, 8])
@pytest.mark.parametrize("dim", [2, 3])
def test_sharded_scenes_reproduce_the_full_set(world, dim):
    """bench.py's N-rank batched run gives rank r the scenes k with
    k mod N == r (scenes.batch_scenes(subset=...)).  Over all ranks that is
    every scene of the full set exactly once, each with the same particle
    count, box size, viscosity and stiffness bit for bit, and the same
    particles relative to its box (up to the rounding of the box offset,
    which differs between packings)."""
    sys.path.insert(0, ROOT)
    from oracle import presets
    from sca2012_b200 import scenes
    base = presets.preset(presets.PRESET_DAM_2D if dim == 2 else presets.PRESET_DAM_3D2)
    base.use_split = base.use_merge = 1
    count, seed = 24, 7
    full = scenes.batch_scenes(base, count, seed=seed)
    _, fboxes, fpos, _, _, fscene, fcounts = full
    cs = float(base.cell_size)
    seen = []
    for r in range(world):
        mine = [k for k in range(count) if k % world == r]
        seen += mine
        if not mine:
            continue
        _, boxes, pos, _, _, scene, counts = scenes.batch_scenes(base, count, seed=seed, subset=mine)
        assert len(boxes) == len(mine)
        for j, k in enumerate(mine):
            assert counts[j] == fcounts[k]
            lo, hi, mu, st = boxes[j]
            flo, fhi, fmu, fst = fboxes[k]
            assert mu == fmu and st == fst
            ext = [round((hi[a] - lo[a]) / cs) for a in range(dim)]
            fext = [round((fhi[a] - flo[a]) / cs) for a in range(dim)]
            assert ext == fext
            rel = pos[scene == j].astype(np.float64) - np.asarray(lo, np.float64)
            frel = fpos[fscene == k].astype(np.float64) - np.asarray(flo, np.float64)
            world_len = max(float(base.world[a]) for a in range(dim)) + max(hi) + max(fhi)
            assert np.abs(rel - frel).max() <= 4 * np.spacing(np.float32(world_len))
    assert sorted(seen) == list(range(count))
