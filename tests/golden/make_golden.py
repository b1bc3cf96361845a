"""Generates the golden fixtures in tests/golden/ by running the UNMODIFIED
reference solver (oracle/_ref/libref_<variant>_gpu.so, built from the
reference sources by oracle/build_ref.sh) on a CUDA GPU.

    python tests/golden/make_golden.py OUT_DIR

For each variant (SPH-2D, SPH-3D-2, SPH-3D-4) it builds the reference's own
default scene, runs a few warm-up steps with split and merge on, snapshots
the state S0, then from S0 runs one step with split/merge off and one with
them on, recording the resulting states and the step's intermediate device
buffers (cell keys, sorted index, cell ranges, wavelet-transformed velocity).
For the 3D variants a third step from S0 with the density-grid display mode
records the grid, its normals and the reference's CPU marching-cubes mesh.
It also records the constants the reference constructor computed.

The fixtures pin the CPU oracle (tests/test_oracle_golden.py) and the CUDA
path (tests/test_gpu_parity.py).  Nothing reads the reference tree here.
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref")

# variant: (dim, warm-up steps, crop x below this value or None)
VARIANTS = {"2d": (2, 10, None), "3d2": (3, 8, 6.0), "3d4": (3, 4, 10.0)}


def particle_dtype(dim, size):
    if dim == 3:
        d = np.dtype({"names": ["pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "tension", "level"],
                      "formats": [("<f4", 3)] * 4 + ["<f4"] * 5 + ["<u4"],
                      "offsets": [0, 12, 24, 36, 48, 52, 56, 60, 64, 68], "itemsize": size})
    else:
        d = np.dtype({"names": ["pos", "vel", "ev", "acc", "dens", "press", "energy", "level", "surface"],
                      "formats": [("<f4", 2)] * 4 + ["<f4"] * 3 + ["<u4", "<f4"],
                      "offsets": [0, 8, 16, 24, 32, 36, 40, 44, 48], "itemsize": size})
    return d


def load(v):
    lib = C.CDLL(os.path.join(REF, f"libref_{v}_gpu.so"))
    vp = C.c_void_p
    lib.ref_create.restype = vp
    for name, args in [("ref_add_default_scene", [vp, C.c_int]), ("ref_set_state", [vp, vp, C.c_uint]),
                       ("ref_set_flags", [vp, C.c_int, C.c_int, C.c_int]), ("ref_step", [vp]),
                       ("ref_read_particles", [vp, vp]), ("ref_param_floats", [vp, vp]),
                       ("ref_read_debug", [vp, C.c_uint, vp, vp, vp, vp, vp])]:
        getattr(lib, name).argtypes = args
    lib.ref_num_particles.argtypes = [vp]
    lib.ref_num_particles.restype = C.c_uint
    lib.ref_total_cell.argtypes = [vp]
    lib.ref_total_cell.restype = C.c_uint
    lib.ref_step.restype = C.c_int
    lib.ref_param_floats.restype = C.c_int
    if v != "2d":
        lib.ref_grid_nodes.argtypes = [vp]
        lib.ref_grid_nodes.restype = C.c_uint
        lib.ref_grid_dims.argtypes = [vp, vp]
        lib.ref_read_grid.argtypes = [vp, vp, vp]
        lib.ref_read_mesh.argtypes = [vp] + [vp] * 6
        lib.ref_read_mesh.restype = C.c_uint
    return lib


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def read_state(lib, h, dt):
    n = lib.ref_num_particles(h)
    buf = np.zeros(n, dt)
    lib.ref_read_particles(h, ptr(buf))
    return buf


def read_debug(lib, h, n, dim, ncell):
    d = {k: np.zeros(n, np.uint32) for k in ("hash", "index")}
    d["cell_start"] = np.zeros(ncell, np.uint32)
    d["cell_end"] = np.zeros(ncell, np.uint32)
    d["trans_vel"] = np.zeros((n, dim), np.float32)
    lib.ref_read_debug(h, n, ptr(d["hash"]), ptr(d["index"]), ptr(d["cell_start"]), ptr(d["cell_end"]),
                       ptr(d["trans_vel"]))
    return d


def step_checked(lib, h):
    rc = lib.ref_step(h)
    if rc == -1:
        raise RuntimeError("reference parameter upload failed; step not run")
    if rc in (-2, -3):
        raise RuntimeError("state outside the box or with an unknown level; step not run")
    if rc != 0:
        raise RuntimeError(f"reference step reported CUDA error {rc}")


def check_state(buf, dim, world):
    p = buf["pos"]
    if not np.all(np.isfinite(p)):
        raise RuntimeError("non-finite position in the reference state; stopping before the next step")
    if (p < 0).any() or (p > np.asarray(world[:dim])).any():
        raise RuntimeError("position outside the box; stopping before the next step")


def mesh_digest(mesh):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(mesh, np.float32).tobytes()).hexdigest()


def compact(out):
    """Fixture layout: the density grid and its normals sparse (non-zero
    nodes only), the marching-cubes mesh as its triangle count and SHA-256
    (the reference's own CPU marching cubes, oracle/_ref/libref_*_mc.so,
    must reproduce it from the grid), and no copy of the grid-step state
    (identical to s1_off: same input, split/merge off)."""
    res = {k: v for k, v in out.items() if k not in ("grid_dens", "grid_normal", "mesh", "s1_grid", "init")}
    if "grid_dens" in out:
        d, nrm = out["grid_dens"], out["grid_normal"]
        if not np.array_equal(out["s1_grid"].view(np.uint8), out["s1_off"].view(np.uint8)):
            raise RuntimeError("grid step state differs from the split/merge-off step state")
        nz = np.flatnonzero(d).astype(np.uint32)
        res["grid_dens_idx"], res["grid_dens_val"] = nz, d[nz]
        nn = np.flatnonzero(np.any(nrm != 0, axis=1)).astype(np.uint32)
        res["grid_normal_idx"], res["grid_normal_val"] = nn, nrm[nn]
        res["grid_nodes"] = np.uint32(len(d))
        res["mesh_triangles"] = np.uint32(len(out["mesh"]))
        res["mesh_sha256"] = np.array(mesh_digest(out["mesh"]))
    return res


def run_variant(v, out_dir):
    dim, warm, crop = VARIANTS[v]
    lib = load(v)
    size = C.CDLL(os.path.join(REF, f"libref_{v}_gpu.so")).ref_particle_size()
    dt = particle_dtype(dim, size)
    h = C.c_void_p(lib.ref_create())
    params = np.zeros(64, np.float32)
    npar = lib.ref_param_floats(h, ptr(params))
    params = params[:npar]
    world = params[23:23 + dim]
    ncell = lib.ref_total_cell(h)

    lib.ref_add_default_scene(h, 0)
    n0 = lib.ref_num_particles(h)
    # the host copy holds the scene add_*() built; re-upload it (cropped) as the state
    init = np.zeros(n0, dt)
    lib.ref_read_particles(h, ptr(init))
    if crop is not None:
        init = init[init["pos"][:, 0] < crop].copy()
    lib.ref_set_state(h, ptr(init), len(init))
    lib.ref_set_flags(h, 1, 1, 1)
    for _ in range(warm):
        step_checked(lib, h)
        check_state(read_state(lib, h, dt), dim, world)
    s0 = read_state(lib, h, dt)
    n = len(s0)

    out = {"params": params, "init": init, "s0": s0}
    for tag, flags in (("off", (0, 0, 1)), ("on", (1, 1, 1))):
        lib.ref_set_state(h, ptr(s0), n)
        lib.ref_set_flags(h, *flags)
        step_checked(lib, h)
        out[f"s1_{tag}"] = read_state(lib, h, dt)
        dbg = read_debug(lib, h, n, dim, ncell)
        for k, a in dbg.items():
            out[f"{tag}_{k}"] = a
    if dim == 3:
        lib.ref_set_state(h, ptr(s0), n)
        lib.ref_set_flags(h, 0, 0, 2)
        step_checked(lib, h)
        G = lib.ref_grid_nodes(h)
        dims = np.zeros(3, np.uint32)
        lib.ref_grid_dims(h, ptr(dims))
        dens = np.zeros(G, np.float32)
        nrm = np.zeros((G, 3), np.float32)
        lib.ref_read_grid(h, ptr(dens), ptr(nrm))
        mx = 3 * G
        tri = [np.zeros((mx, 3), np.float32) for _ in range(6)]
        nt = lib.ref_read_mesh(h, *[ptr(t) for t in tri])
        out["grid_dims"] = dims
        out["grid_dens"] = dens
        out["grid_normal"] = nrm
        out["mesh"] = np.stack([t[:nt] for t in tri], 1)   # nt x 6 x 3 (v0 v1 v2 n0 n1 n2)
        out["s1_grid"] = read_state(lib, h, dt)
    path = os.path.join(out_dir, f"ref_{v}.npz")
    np.savez_compressed(path, **compact(out))
    print(f"{v}: n={n} -> off {len(out['s1_off'])}, on {len(out['s1_on'])}; wrote {path} "
          f"({os.path.getsize(path) / 1e6:.2f} MB)")


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden")
    os.makedirs(out_dir, exist_ok=True)
    only = sys.argv[2] if len(sys.argv) > 2 else None
    if only:
        run_variant(only, out_dir)
        return
    # one process per variant: each reference build carries its own runtime
    import subprocess
    rc = 0
    for v in VARIANTS:
        rc |= subprocess.run([sys.executable, os.path.abspath(__file__), out_dir, v]).returncode
    sys.exit(rc)


if __name__ == "__main__":
    main()
