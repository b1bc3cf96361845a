"""sca2012_b200 — B200-native adaptive SPH step behind the reference's SPHSystem API.

`Solver` is a thin Python owner of one C-ABI handle (include/sph/sph.h).  It
mirrors the reference host class's operations (SPH-3D-2/sph_system.h:26-154):
construct from constants, add particles, advance with `animation()` /
`step()`, read the particle state back.  All compute runs in the in-tree CUDA
library; if that library or a GPU is missing the calls raise — there is no
CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._abi import Config, StateView, DebugView, MeshView  # noqa: F401
from ._abi import (SPH_OK, SPH_ERR_INVALID, SPH_ERR_CAPACITY, SPH_ERR_CUDA, SPH_ERR_NO_DEVICE,  # noqa: F401
                   SPH_ERR_NONFINITE, SPH_ERR_RANGE, SPH_ERR_TIMEOUT)
from ._abi import (PRESET_REF_2D, PRESET_REF_3D2, PRESET_REF_3D4, PRESET_DAM_2D,  # noqa: F401
                   PRESET_DAM_3D2, PRESET_DAM_3D4, PRESET_ROLLOUT_3D)

__all__ = ["Solver", "Config", "preset", "SphError", "lib"]


class SphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sph error {code}: {msg}")
        self.code = code


def lib():
    return _abi.load()


def preset(which):
    """Config of a preset (SPH_PRESET_*)."""
    c = Config()
    rc = lib().sph_config_preset(int(which), C.byref(c))
    if rc:
        raise SphError(rc, f"unknown preset {which}")
    return c


def _f(a):
    return a.ctypes.data_as(_abi.FP) if a is not None else None


def _u(a):
    return a.ctypes.data_as(_abi.UP) if a is not None else None


STATE_FIELDS = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "level", "interior", "scene",
                "sibling")
_U32_FIELDS = ("level", "interior", "scene", "sibling")
NO_SIBLING = 0xFFFFFFFF   # sibling of a particle outside any split group


def particle_dtype(dim):
    """numpy dtype of the reference's Particle record (SPH-3D-2/sph_system.h:8-24,
    SPH-2D/sph_system.h:7-22)."""
    if dim == 3:
        return np.dtype({"names": ["pos", "vel", "ev", "acc", "dens", "press", "energy", "surface", "tension",
                                   "level"],
                         "formats": [("<f4", 3)] * 4 + ["<f4"] * 5 + ["<u4"],
                         "offsets": [0, 12, 24, 36, 48, 52, 56, 60, 64, 68], "itemsize": 72})
    return np.dtype({"names": ["pos", "vel", "ev", "acc", "dens", "press", "energy", "level", "surface"],
                     "formats": [("<f4", 2)] * 4 + ["<f4"] * 3 + ["<u4", "<f4"],
                     "offsets": [0, 8, 16, 24, 32, 36, 40, 44, 48], "itemsize": 56})


class Solver:
    """One solver instance on the current CUDA device."""

    def __init__(self, cfg):
        self._lib = lib()
        self.cfg = cfg.copy()
        self.dim = int(cfg.dim)
        h = _abi.H()
        rc = self._lib.sph_create(C.byref(self.cfg), C.byref(h))
        if rc:
            raise SphError(rc, "sph_create failed (no CUDA device, or invalid config)")
        self._h = h

    # -- lifecycle ------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.sph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = self._lib.sph_last_error(self._h)
            raise SphError(rc, f"{what}: {msg.decode() if msg else ''}")

    # -- configuration --------------------------------------------------
    def set_config(self, cfg):
        self._check(self._lib.sph_set_config(self._h, C.byref(cfg)), "sph_set_config")
        self.cfg = cfg.copy()

    def set_debug(self, on=True):
        self._check(self._lib.sph_set_debug(self._h, 1 if on else 0), "sph_set_debug")

    def set_graph(self, on=True):
        """Replay steps as captured CUDA graphs (same results, fewer launches)."""
        self._check(self._lib.sph_set_graph(self._h, 1 if on else 0), "sph_set_graph")

    def set_persistent(self, on=True, spin_limit=_abi.PERSISTENT_SPIN_DEFAULT):
        """Run each step as one cooperative launch (same results as the
        ordinary launches); spin_limit bounds every barrier wait."""
        self._check(self._lib.sph_set_persistent(self._h, 1 if on else 0, int(spin_limit)), "sph_set_persistent")

    def set_scenes(self, boxes):
        """Batched scenes: boxes is a list of (lo, hi, viscosity, gas_constant)
        with lo/hi of length dim; a particle's `scene` state field indexes it.
        An empty list returns to the single box [0, world]."""
        arr = (_abi.Scene * max(1, len(boxes)))()
        for s, (lo, hi, mu, k) in enumerate(boxes):
            for d in range(self.dim):
                arr[s].lo[d] = float(lo[d])
                arr[s].hi[d] = float(hi[d])
            arr[s].viscosity = float(mu)
            arr[s].gas_constant = float(k)
        self._check(self._lib.sph_set_scenes(self._h, len(boxes), arr), "sph_set_scenes")

    def set_stream(self, stream_ptr):
        """Runs the handle's work on the caller's CUDA stream (0 = its own)."""
        self._check(self._lib.sph_set_stream(self._h, C.c_void_p(int(stream_ptr) or None)), "sph_set_stream")

    @property
    def stream_ptr(self):
        return self._lib.sph_get_stream(self._h)

    # -- particles -------------------------------------------------------
    def add_particles(self, pos, vel, level):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, self.dim)
        vel = np.ascontiguousarray(vel, np.float32).reshape(-1, self.dim)
        level = np.ascontiguousarray(level, np.uint32).reshape(-1)
        n = pos.shape[0]
        self._check(self._lib.sph_add_particles(self._h, n, _f(pos), _f(vel), _u(level)), "sph_add_particles")

    def set_state(self, st):
        """st: dict with pos/vel/ev/acc (n x dim) and optional scalars, level (n);
        `sibling` (the split-group ring) defaults to none."""
        pos = np.ascontiguousarray(st["pos"], np.float32)
        n = pos.shape[0]
        keep = {}
        v = StateView()
        v.n = n
        for k in STATE_FIELDS:
            a = st.get(k)
            if a is None:
                continue
            a = np.ascontiguousarray(a, np.uint32 if k in _U32_FIELDS else np.float32)
            keep[k] = a
            setattr(v, k, _u(a) if k in _U32_FIELDS else _f(a))
        self._check(self._lib.sph_set_state(self._h, C.byref(v)), "sph_set_state")

    def num_particles(self):
        n = C.c_uint32()
        self._check(self._lib.sph_get_num_particles(self._h, C.byref(n)), "sph_get_num_particles")
        return int(n.value)

    def get_state(self):
        n = self.num_particles()
        d = self.dim
        out = {k: np.zeros((n, d), np.float32) for k in ("pos", "vel", "ev", "acc")}
        for k in ("dens", "press", "energy", "surface"):
            out[k] = np.zeros(n, np.float32)
        out["level"] = np.zeros(n, np.uint32)
        out["interior"] = np.zeros(n, np.uint32)
        out["scene"] = np.zeros(n, np.uint32)
        out["sibling"] = np.full(n, NO_SIBLING, np.uint32)
        v = StateView()
        v.n = n
        for k in STATE_FIELDS:
            setattr(v, k, _u(out[k]) if k in _U32_FIELDS else _f(out[k]))
        self._check(self._lib.sph_get_state(self._h, C.byref(v)), "sph_get_state")
        return out

    def get_debug(self):
        n_guess = self.cfg.max_particle
        ncell = int(np.prod([self.cfg.ncell[a] for a in range(self.dim)]))
        dv = DebugView()
        dv.n_sorted = 0
        # first call with no arrays to learn n
        arr = {k: np.zeros(n_guess, np.uint32) for k in ("hash", "index", "nbr_count", "split_flag", "removed")}
        arr["cell_start"] = np.zeros(ncell, np.uint32)
        arr["cell_end"] = np.zeros(ncell, np.uint32)
        arr["trans_vel"] = np.zeros(n_guess * self.dim, np.float32)
        for k, a in arr.items():
            setattr(dv, k, _f(a) if k == "trans_vel" else _u(a))
        self._check(self._lib.sph_get_debug(self._h, C.byref(dv)), "sph_get_debug")
        n = int(dv.n_sorted)
        out = {k: a[:n].copy() for k, a in arr.items() if k not in ("cell_start", "cell_end", "trans_vel")}
        out["cell_start"] = arr["cell_start"]
        out["cell_end"] = arr["cell_end"]
        out["trans_vel"] = arr["trans_vel"][: n * self.dim].reshape(n, self.dim).copy()
        out["n"] = n
        return out

    # -- reference-layout records (SPHSystem::m_host_mem) ------------------
    @property
    def record_size(self):
        return int(self._lib.sph_particle_record_size(self._h))

    def read_particles_into(self, host_ptr, capacity_bytes):
        """Copies the state as reference Particle records to host memory at
        host_ptr (ideally page-locked); returns the record count."""
        n = C.c_uint32()
        self._check(self._lib.sph_read_particles(self._h, C.c_void_p(host_ptr), int(capacity_bytes), C.byref(n)),
                    "sph_read_particles")
        return int(n.value)

    def write_particles_from(self, host_ptr, n):
        self._check(self._lib.sph_write_particles(self._h, C.c_void_p(host_ptr), int(n)), "sph_write_particles")

    def read_particles_async_into(self, mapped_ptr, capacity_bytes, mapped_count_ptr):
        """Starts the asynchronous readback of the current state as reference
        Particle records into mapped page-locked memory (4-byte aligned), the
        record count into *mapped_count_ptr; returns at once (sph_read_particles_async)."""
        self._check(self._lib.sph_read_particles_async(self._h, C.c_void_p(mapped_ptr), int(capacity_bytes),
                                                       C.c_void_p(mapped_count_ptr)), "sph_read_particles_async")

    def readback_wait(self):
        """Blocks until every asynchronous readback has landed in host memory."""
        self._check(self._lib.sph_readback_wait(self._h), "sph_readback_wait")

    def read_particles(self):
        """Reference-layout records as a numpy structured array."""
        n = self.num_particles()
        buf = np.zeros(max(n, 1) * self.record_size, np.uint8)
        got = self.read_particles_into(buf.ctypes.data, buf.nbytes)
        return buf[: got * self.record_size].view(particle_dtype(self.dim))

    def conserved(self):
        """FP64 device sums: mass, momentum (3), kinetic, potential, total energy."""
        out = np.zeros(7, np.float64)
        self._check(self._lib.sph_conserved(self._h, out.ctypes.data_as(_abi.DP)), "sph_conserved")
        return dict(mass=out[0], momentum=out[1:4].copy(), kinetic=out[4], potential=out[5], energy=out[6])

    # -- launch tuning -----------------------------------------------------
    def autotune(self, reps=3):
        """Times launch shapes per stage on the current state (restored
        afterwards) and keeps the fastest; returns the choice and the mean
        step time before and after."""
        t = _abi.Tuning()
        self._check(self._lib.sph_autotune(self._h, int(reps), C.byref(t)), "sph_autotune")
        return self._tuning_dict(t)

    def get_tuning(self):
        t = _abi.Tuning()
        self._check(self._lib.sph_get_tuning(self._h, C.byref(t)), "sph_get_tuning")
        return self._tuning_dict(t)

    def set_tuning(self, block, blocks_per_sm, reg_cap=None):
        """reg_cap None keeps the handle's register caps."""
        if reg_cap is None:
            reg_cap = self.get_tuning()["reg_cap"]
        t = _abi.Tuning()
        for k in range(_abi.TUNE_STAGES):
            t.block[k] = int(block[k])
            t.blocks_per_sm[k] = int(blocks_per_sm[k])
            t.reg_cap[k] = int(reg_cap[k])
        self._check(self._lib.sph_set_tuning(self._h, C.byref(t)), "sph_set_tuning")

    @staticmethod
    def _tuning_dict(t):
        return dict(block=list(t.block), blocks_per_sm=list(t.blocks_per_sm), reg_cap=list(t.reg_cap),
                    stages=list(_abi.TUNE_STAGE_NAMES), step_ms_before=t.step_ms_before,
                    step_ms_after=t.step_ms_after)

    # -- differentiable rollout --------------------------------------------
    def rollout_forward(self, nsteps, checkpoint_every):
        """Advances nsteps keeping checkpoints every `checkpoint_every` steps."""
        self._check(self._lib.sph_rollout_forward(self._h, int(nsteps), int(checkpoint_every)),
                    "sph_rollout_forward")

    def splat_loss(self, n, origin, spacing, target):
        """mean((G - target)^2) of the current state's density grid G (nodes
        origin + i * spacing, x fastest); returns (loss, G)."""
        g = _abi.LossGrid()
        for d in range(3):
            g.n[d] = int(n[d]) if d < self.dim else 1
            g.origin[d] = float(origin[d]) if d < self.dim else 0.0
        g.spacing = float(spacing)
        tgt = np.ascontiguousarray(target, np.float32).reshape(-1)
        grid = np.zeros_like(tgt)
        loss = C.c_double()
        self._check(self._lib.sph_splat_loss(self._h, C.byref(g), _f(tgt), _f(grid), C.byref(loss)),
                    "sph_splat_loss")
        return float(loss.value), grid

    def rollout_backward(self, n0, nscenes=1):
        """Gradient of the last splat_loss with respect to the initial
        velocities and positions (n0 x dim) and the per-scene viscosity and
        gas constant (nscenes x 2)."""
        gv = np.zeros((n0, self.dim), np.float32)
        gx = np.zeros((n0, self.dim), np.float32)
        gp = np.zeros(2 * max(1, nscenes), np.float64)
        self._check(self._lib.sph_rollout_backward(self._h, _f(gv), _f(gx), gp.ctypes.data_as(_abi.DP), len(gp)),
                    "sph_rollout_backward")
        return dict(d_vel0=gv, d_pos0=gx, d_params=gp.reshape(-1, 2))

    def rollout_topology(self, step, states=False):
        """Recorded topology of forward step `step` (particle indices of that
        step); states=True adds the FP32 state the step started from."""
        v = _abi.TopologyView()
        self._check(self._lib.sph_rollout_topology(self._h, int(step), C.byref(v)), "sph_rollout_topology")
        n, nd, nf = v.n, v.n_dens_pairs, v.n_force_pairs
        out = {k: np.zeros(n, np.uint32) for k in ("level", "wall", "split", "dst", "child", "merge_leader")}
        out["dens_off"] = np.zeros(n + 1, np.uint32)
        out["force_off"] = np.zeros(n + 1, np.uint32)
        out["dens_nbr"] = np.zeros(max(nd, 1), np.uint32)
        out["force_nbr"] = np.zeros(max(nf, 1), np.uint32)
        v.dens_cap, v.force_cap = nd, nf
        for k, a in out.items():
            setattr(v, k, _u(a))
        if states:
            for k in ("pos", "vel", "ev"):
                out[k] = np.zeros((n, self.dim), np.float32)
                setattr(v, k, _f(out[k]))
        self._check(self._lib.sph_rollout_topology(self._h, int(step), C.byref(v)), "sph_rollout_topology")
        out.update(n=v.n, n_next=v.n_next, n_split=v.n_split, n_removed=v.n_removed, split_on=v.split_on)
        return out

    # -- profiling ---------------------------------------------------------
    def set_profiling(self, on=True):
        self._check(self._lib.sph_set_profiling(self._h, 1 if on else 0), "sph_set_profiling")

    def stage_times(self):
        ms = (C.c_float * 32)()
        names = (C.c_char_p * 32)()
        cnt = C.c_int()
        self._check(self._lib.sph_stage_times(self._h, ms, names, 32, C.byref(cnt)), "sph_stage_times")
        return [(names[k].decode(), float(ms[k])) for k in range(min(cnt.value, 32))]

    # -- stepping ----------------------------------------------------------
    def step(self, nsteps=1):
        self._check(self._lib.sph_step(self._h, int(nsteps)), "sph_step")

    def sync(self):
        rc = self._lib.sph_sync(self._h)
        if rc:
            self._check(rc, "sph_sync")

    def sync_status(self):
        """Synchronises and returns the device status code (0 = ok) without raising."""
        return int(self._lib.sph_sync(self._h))

    def last_step_stats(self):
        """Counts of the last step: n_start, n_split, n_removed, n_end,
        n_level2, split_suppressed, error (sph_last_step_stats)."""
        st = _abi.StepStats()
        self._check(self._lib.sph_last_step_stats(self._h, C.byref(st)), "sph_last_step_stats")
        return {k: int(getattr(st, k)) for k, _ in st._fields_}

    def last_launch_count(self):
        n = C.c_uint32()
        self._check(self._lib.sph_last_launch_count(self._h, C.byref(n)), "sph_last_launch_count")
        return int(n.value)

    # reference spelling: SPHSystem::animation() advances one step
    def animation(self):
        self.step(1)
