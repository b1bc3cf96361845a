"""Marching cubes restated in FP64 numpy (TEST INFRASTRUCTURE).

Follows SPHSystem::marching_cube / marching_cube_cell
(SPH-3D-2/sph_system.cpp:406-542, the same in SPH-3D-4/sph_system.cpp:455-591):
cubes are visited x outer, y, z inner; corner v of the cube at node (x, y, z)
sits at node (x, y, z) + CORNERS[v]; corner bit v of the case is set when the
node density is above the iso value (:459-466); each cut edge gets a vertex
and a normal (the mean of its two node normals); triangles are appended in
cube order, up to five per cube, from the case table.  The reference places
a vertex at the edge midpoint (interpolation commented out, :479-482); with
`mc_interpolate` set the vertex is the linear interpolation at the iso value,
p = pa + s (pb - pa) with s = (iso - da) / (db - da), which is the config-mode
surface.  All arithmetic after the case decision is FP64.

The case table is the one sca2012_b200/csrc/gen_mc_tables.py derives from the
cube geometry (tests/test_mc_tables.py checks its polygon loops against the
reference's own table case by case).
"""
import importlib.util
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_tables = None


def tables():
    """(corner offsets [8, 3], edge corners [12, 2], triangle edges [256, 15]
    with -1 padding, triangle count [256])."""
    global _tables
    if _tables is None:
        path = os.path.join(os.path.dirname(_HERE), "sca2012_b200", "csrc", "gen_mc_tables.py")
        spec = importlib.util.spec_from_file_location("_oracle_mc_tables", path)
        g = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(g)
        tri = -np.ones((256, 15), np.int64)
        cnt = np.zeros(256, np.int64)
        for c in range(256):
            t = g.triangles(c)
            cnt[c] = len(t)
            for k, edges3 in enumerate(t):
                tri[c, 3 * k: 3 * k + 3] = edges3
        _tables = (np.array(g.CORNERS, np.int64), np.array(g.EDGES, np.int64), tri, cnt)
    return _tables


def cube_cases(cfg, dens):
    """Case (8 corner bits) of every cube, in the reference's cube order."""
    corners, _, _, _ = tables()
    R, Cn, L = (int(cfg.ndens[a]) for a in range(3))
    above = (np.asarray(dens).reshape(L, Cn, R) > np.float32(cfg.iso_value)).transpose(2, 1, 0)   # [x, y, z]
    flags = np.zeros((R - 1, Cn - 1, L - 1), np.int64)
    for v, (ox, oy, oz) in enumerate(corners):
        flags |= above[ox:R - 1 + ox, oy:Cn - 1 + oy, oz:L - 1 + oz].astype(np.int64) << v
    return flags.reshape(-1)


def marching_cubes(cfg, dens, normal):
    """Triangles (nt x 6 x 3: v0 v1 v2 n0 n1 n2, FP64) and the per-cube
    triangle counts of the surface of the node grid `dens` (node g =
    z*R*C + y*R + x) with node normals `normal` (G x 3 or G x 4)."""
    corners, edges, tri, cnt = tables()
    R, Cn, L = (int(cfg.ndens[a]) for a in range(3))
    dens64 = np.asarray(dens, np.float64).reshape(-1)
    nrm64 = np.asarray(normal, np.float64).reshape(len(dens64), -1)[:, :3]
    h = float(cfg.den_size)
    iso = float(cfg.iso_value)
    case = cube_cases(cfg, dens)
    per_cube = cnt[case]
    q = np.repeat(np.arange(len(case)), per_cube)               # cube of every triangle, in cube order
    first = np.repeat(np.cumsum(per_cube) - per_cube, per_cube)
    k = np.arange(len(q)) - first                                # triangle slot inside its cube
    cx = q // ((Cn - 1) * (L - 1))
    cy = (q // (L - 1)) % (Cn - 1)
    cz = q % (L - 1)
    out = np.zeros((len(q), 6, 3))
    for j in range(3):
        e = tri[case[q], 3 * k + j]
        a, b = edges[e, 0], edges[e, 1]
        na = np.stack([cx + corners[a, 0], cy + corners[a, 1], cz + corners[a, 2]], 1)
        nb = np.stack([cx + corners[b, 0], cy + corners[b, 1], cz + corners[b, 2]], 1)
        ga = na[:, 2] * R * Cn + na[:, 1] * R + na[:, 0]
        gb = nb[:, 2] * R * Cn + nb[:, 1] * R + nb[:, 0]
        # node position = index * den_size in FP32, as the grid defines it
        pa = (na.astype(np.float32) * np.float32(h)).astype(np.float64)
        pb = (nb.astype(np.float32) * np.float32(h)).astype(np.float64)
        if cfg.mc_interpolate:
            da, db = dens64[ga], dens64[gb]
            s = np.where(db != da, (iso - da) / np.where(db != da, db - da, 1.0), 0.5)
            out[:, j] = pa + s[:, None] * (pb - pa)
        else:
            out[:, j] = 0.5 * (pa + pb)
        out[:, 3 + j] = 0.5 * (nrm64[ga] + nrm64[gb])
    return out, per_cube
