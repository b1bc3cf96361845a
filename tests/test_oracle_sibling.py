"""The oracle's split-group merge (SPH_MERGE_SIBLING, the SI presets' rule)
on a hand-built state: a two-way group whose members have both been
interior long enough merges into its member of smaller index, a group with
a member that has not stays, and the surviving links follow the compaction.
The GPU kernels are checked against this restatement step by step in
tests/test_gpu_parity.py (split-group links, merge flags bit-exact)."""
import numpy as np

from oracle import oracle as O
from oracle import presets as P

NONE = O.NO_SIBLING


def test_sibling_groups_merge_back_when_all_members_are_interior():
    cfg = P.preset(P.PRESET_DAM_3D2)
    assert cfg.merge_rule == 3 and cfg.split_ways == 2
    n = 6
    pos = np.array([[0.100, 0.100, 0.100], [0.200, 0.200, 0.200], [0.300, 0.300, 0.300],
                    [0.104, 0.100, 0.100], [0.400, 0.100, 0.100], [0.404, 0.100, 0.100]], np.float32)
    st = dict(pos=pos, vel=np.zeros((n, 3), np.float32), ev=np.zeros((n, 3), np.float32),
              acc=np.zeros((n, 3), np.float32), dens=np.full(n, 1000.0, np.float32),
              press=np.zeros(n, np.float32), energy=np.zeros(n, np.float32), surface=np.zeros(n, np.float32),
              level=np.array([2, 1, 1, 2, 2, 2], np.uint32),
              interior=np.array([60, 0, 0, 60, 60, 10], np.uint32),
              sibling=np.array([3, NONE, NONE, 0, 5, 4], np.uint32))
    st["vel"][3, 0] = 1.0
    nbr = np.full(n, 26, np.uint32)     # no deficit: nothing splits, the counters grow
    key, idx, cs, ce = O.sort(cfg, pos)
    out, split, removed = O.adapt(cfg, st, nbr, idx, cs, ce, cap=4 * n)
    assert not split.any()
    assert removed.tolist() == [0, 0, 0, 1, 0, 0]          # the group {0, 3} merged into 0
    assert len(out["pos"]) == 5
    assert out["level"].tolist() == [1, 1, 1, 2, 2]
    # survivors [0, 1, 2, 4, 5]: the merged particle has no group, {4, 5} keeps its ring
    assert out["sibling"].tolist() == [NONE, NONE, NONE, 4, 3]
    assert out["interior"].tolist() == [0, 1, 1, 61, 11]
    # equal densities: the two members' volume weights are m_large/rho and m_small/rho
    w0, w3 = cfg.mass[0] / 1000.0, cfg.mass[1] / 1000.0
    assert abs(out["pos"][0, 0] - (0.100 * w0 + 0.104 * w3) / (w0 + w3)) < 1e-7
    assert abs(out["vel"][0, 0] - w3 / (w0 + w3)) < 1e-7


def test_split_makes_a_ring_of_parent_and_children():
    cfg = P.preset(P.PRESET_DAM_3D4)
    assert cfg.split_ways == 4
    n = 3
    pos = np.array([[0.1, 0.1, 0.1], [0.3, 0.3, 0.3], [0.5, 0.5, 0.5]], np.float32)
    st = dict(pos=pos, vel=np.zeros((n, 3), np.float32), ev=np.zeros((n, 3), np.float32),
              acc=np.zeros((n, 3), np.float32), dens=np.full(n, 1000.0, np.float32),
              press=np.zeros(n, np.float32), energy=np.zeros(n, np.float32), surface=np.zeros(n, np.float32),
              level=np.ones(n, np.uint32), interior=np.zeros(n, np.uint32))
    nbr = np.array([26, 5, 26], np.uint32)   # particle 1 has a neighbour deficit: it splits
    key, idx, cs, ce = O.sort(cfg, pos)
    out, split, removed = O.adapt(cfg, st, nbr, idx, cs, ce, cap=16)
    assert split.tolist() == [0, 1, 0]
    assert len(out["pos"]) == 6
    # parent 1 -> children 3, 4, 5 -> parent
    assert out["sibling"].tolist() == [NONE, 3, NONE, 4, 5, 1]
    assert out["level"].tolist() == [1, 2, 1, 2, 2, 2]
