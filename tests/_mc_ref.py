"""Access to the reference's own CPU marching cubes (oracle/_ref/libref_<v>_mc.so,
built from SPH-3D-2/sph_system.cpp and SPH-3D-4/sph_system.cpp by
oracle/build_ref.sh) — the marching-cubes oracle."""
import ctypes as C
import hashlib
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_libs = {}


def _lib(v):
    if v in _libs:
        return _libs[v]
    path = os.path.join(ROOT, "oracle", "_ref", f"libref_{v}_mc.so")
    if not os.path.exists(path):
        _libs[v] = None
        return None
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.mc_create.restype = vp
    lib.mc_grid_dims.argtypes = [vp, vp]
    lib.mc_run.argtypes = [vp, vp, vp] + [vp] * 6 + [C.c_uint]
    lib.mc_run.restype = C.c_uint
    lib.mc_tables.argtypes = [vp, vp]
    h = C.c_void_p(lib.mc_create())
    _libs[v] = (lib, h)
    return _libs[v]


def ref_mc(v, dens, normal):
    """Triangles (nt x 6 x 3: v0 v1 v2 n0 n1 n2) of the reference's
    SPHSystem::marching_cube() on the given node densities and normals."""
    got = _lib(v)
    if got is None:
        return None
    lib, h = got
    dens = np.ascontiguousarray(dens, np.float32)
    normal = np.ascontiguousarray(normal, np.float32).reshape(-1, 3)
    mx = 3 * len(dens)
    bufs = [np.zeros((mx, 3), np.float32) for _ in range(6)]
    nt = lib.mc_run(h, dens.ctypes.data, normal.ctypes.data, *[b.ctypes.data for b in bufs], mx)
    return np.stack([b[:nt] for b in bufs], 1)


def ref_tables(v="3d2"):
    got = _lib(v)
    if got is None:
        return None, None
    lib, h = got
    ef = np.zeros(256, np.int32)
    tt = np.zeros((256, 16), np.int32)
    lib.mc_tables(ef.ctypes.data, tt.ctypes.data)
    return ef, tt


def mesh_sha256(mesh):
    return hashlib.sha256(np.ascontiguousarray(mesh, np.float32).tobytes()).hexdigest()
