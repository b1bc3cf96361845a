"""Python loader for the CPU oracle (oracle/libsph_oracle.so).

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module, as the checker or as the timed CPU port
of the reference step — never as the product path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsph_oracle.so")

_lib = None


class RefTopo(C.Structure):
    """ref_topo of sph_rollout_ref.c: one recorded step."""
    _fields_ = [("n", C.c_uint32), ("n_next", C.c_uint32), ("split_on", C.c_uint32)] + [
        (k, C.POINTER(C.c_uint32)) for k in ("level", "dens_off", "dens_nbr", "force_off", "force_nbr", "wall",
                                            "split", "dst", "child", "merge_leader")] + [
        (k, C.POINTER(C.c_float)) for k in ("x_rec", "v_rec", "ev_rec")]


def abi():
    """The ctypes mirror of sph.h's structs (sca2012_b200/_abi.py).  When the
    package is already imported its module is used, so that structs built by
    either side have the same types; otherwise the file is loaded on its own,
    without importing the package or loading its CUDA library."""
    import sys
    mod = sys.modules.get("sca2012_b200._abi")
    if mod is not None:
        return mod
    mod = sys.modules.get("_oracle_abi_mirror")
    if mod is None:
        import importlib.util
        path = os.path.join(os.path.dirname(HERE), "sca2012_b200", "_abi.py")
        spec = importlib.util.spec_from_file_location("_oracle_abi_mirror", path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules["_oracle_abi_mirror"] = mod
        spec.loader.exec_module(mod)
    return mod


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("oracle/libsph_oracle.so not built (make -C oracle)")
    A = abi()
    StateView, DebugView = A.StateView, A.DebugView
    lib = C.CDLL(LIB_PATH)
    PC = C.c_void_p   # sph_config*, from any mirror of the struct (passed by byref)
    U = C.POINTER(C.c_uint32)
    F = C.POINTER(C.c_float)
    D = C.POINTER(C.c_double)
    B = C.POINTER(C.c_uint8)
    lib.oracle_set_threads.argtypes = [C.c_int]
    lib.oracle_get_threads.restype = C.c_int
    lib.oracle_sort.argtypes = [PC, C.c_uint32, F, U, U, U, U]
    lib.oracle_density.argtypes = [PC, C.c_uint32, F, U, U, U, U, D, D, U]
    lib.oracle_force.argtypes = [PC, C.c_uint32, F, F, U, D, D, U, U, U, D, D, B]
    lib.oracle_integrate.argtypes = [PC, C.c_uint32, F, F, F, U, D, D, D, D, D, D, B]
    lib.oracle_energy.argtypes = [PC, C.c_uint32, F, F, U, U, U, U, D, D]
    lib.oracle_adapt.argtypes = [PC, C.c_uint32, C.c_uint32, C.POINTER(StateView), U, U, U, U,
                                 C.POINTER(StateView), U, U]
    lib.oracle_adapt.restype = C.c_int64
    lib.oracle_step.argtypes = [PC, C.c_uint32, C.c_uint32, C.POINTER(StateView), C.POINTER(StateView),
                                C.POINTER(DebugView)]
    lib.oracle_step.restype = C.c_int64
    lib.oracle_density_grid.argtypes = [PC, C.c_uint32, F, U, U, U, U, D, D]
    PT = C.POINTER(RefTopo)
    PG = C.POINTER(A.LossGrid)
    lib.ref_rollout_forward.argtypes = [PC, PT, C.c_uint32, C.c_uint32, D, D, C.c_double, C.c_double, PG, D, D]
    lib.ref_rollout_forward.restype = C.c_double
    lib.ref_rollout_grad.argtypes = [PC, PT, C.c_uint32, C.c_uint32, D, D, C.c_double, C.c_double, PG, D,
                                     D, D, D, D]
    lib.ref_rollout_grad.restype = C.c_double
    lib.ref_rollout_grad_along.argtypes = [PC, PT, C.c_uint32, C.c_uint32, D, D, C.c_double, C.c_double, PG, D,
                                           F, D, D, D, D]
    lib.ref_rollout_grad_along.restype = C.c_double
    _lib = lib
    return lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


def _f(a):
    return _p(a, C.c_float)


def _u(a):
    return _p(a, C.c_uint32)


def _d(a):
    return _p(a, C.c_double)


def _b(a):
    return _p(a, C.c_uint8)


def set_threads(n):
    load().oracle_set_threads(int(n))


def get_threads():
    return int(load().oracle_get_threads())


def ncells(cfg):
    return int(np.prod([cfg.ncell[a] for a in range(cfg.dim)]))


def f32(a, d=None):
    a = np.ascontiguousarray(a, np.float32)
    return a if d is None else a.reshape(-1, d)


def sort(cfg, pos):
    lib = load()
    pos = f32(pos)
    n = pos.shape[0]
    C_ = ncells(cfg)
    key = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    cs = np.zeros(C_, np.uint32)
    ce = np.zeros(C_, np.uint32)
    lib.oracle_sort(C.byref(cfg), n, _f(pos), _u(key), _u(idx), _u(cs), _u(ce))
    return key, idx, cs, ce


def density(cfg, pos, level, idx, cs, ce):
    lib = load()
    pos = f32(pos)
    level = np.ascontiguousarray(level, np.uint32)
    n = pos.shape[0]
    dens = np.zeros(n)
    press = np.zeros(n)
    nbr = np.zeros(n, np.uint32)
    lib.oracle_density(C.byref(cfg), n, _f(pos), _u(level), _u(idx), _u(cs), _u(ce), _d(dens), _d(press), _u(nbr))
    return dens, press, nbr


def force(cfg, pos, ev, level, dens, press, idx, cs, ce):
    lib = load()
    pos, ev = f32(pos), f32(ev)
    level = np.ascontiguousarray(level, np.uint32)
    dens = np.ascontiguousarray(dens, np.float64)
    press = np.ascontiguousarray(press, np.float64)
    n = pos.shape[0]
    acc = np.zeros((n, cfg.dim))
    surf = np.zeros(n)
    amb = np.zeros(n, np.uint8)
    lib.oracle_force(C.byref(cfg), n, _f(pos), _f(ev), _u(level), _d(dens), _d(press), _u(idx), _u(cs), _u(ce),
                     _d(acc), _d(surf), _b(amb))
    return acc, surf, amb.astype(bool)


def integrate(cfg, pos, vel, ev, level, acc, dens):
    lib = load()
    pos, vel, ev = f32(pos), f32(vel), f32(ev)
    level = np.ascontiguousarray(level, np.uint32)
    acc = np.ascontiguousarray(acc, np.float64)
    dens = np.ascontiguousarray(dens, np.float64)
    n = pos.shape[0]
    out = [np.zeros((n, cfg.dim)) for _ in range(4)]
    amb = np.zeros(n, np.uint8)
    lib.oracle_integrate(C.byref(cfg), n, _f(pos), _f(vel), _f(ev), _u(level), _d(acc), _d(dens),
                         *[_d(o) for o in out], _b(amb))
    return out[0], out[1], out[2], out[3], amb.astype(bool)


def energy(cfg, pos_new, vel_new, level, idx, cs, ce):
    lib = load()
    pos_new, vel_new = f32(pos_new), f32(vel_new)
    level = np.ascontiguousarray(level, np.uint32)
    n = pos_new.shape[0]
    e = np.zeros(n)
    tv = np.zeros((n, cfg.dim))
    lib.oracle_energy(C.byref(cfg), n, _f(pos_new), _f(vel_new), _u(level), _u(idx), _u(cs), _u(ce), _d(e), _d(tv))
    return e, tv


_STATE_F = ("pos", "vel", "ev", "acc", "dens", "press", "energy", "surface")
_STATE_U = ("level", "interior", "sibling")
NO_SIBLING = 0xFFFFFFFF


def _view(st, n, keep):
    v = abi().StateView()
    v.n = n
    for k in _STATE_F + ("level", "interior", "sibling"):
        a = st.get(k)
        if a is None:
            continue
        a = np.ascontiguousarray(a, np.uint32 if k in _STATE_U else np.float32)
        keep.append(a)
        setattr(v, k, _u(a) if k in _STATE_U else _f(a))
    return v


def _alloc_state(cfg, cap):
    d = cfg.dim
    st = {k: np.zeros((cap, d), np.float32) for k in ("pos", "vel", "ev", "acc")}
    for k in ("dens", "press", "energy", "surface"):
        st[k] = np.zeros(cap, np.float32)
    st["level"] = np.zeros(cap, np.uint32)
    st["interior"] = np.zeros(cap, np.uint32)
    st["sibling"] = np.full(cap, NO_SIBLING, np.uint32)
    return st


def _pad(st, cap, cfg):
    """Copies a state dict into capacity-sized arrays (slots >= n zero)."""
    out = _alloc_state(cfg, cap)
    n = len(st["pos"])
    for k, a in st.items():
        if k in out and a is not None:
            out[k][:n] = np.asarray(a).reshape(out[k][:n].shape)
    return out


def adapt(cfg, st, nbr, idx, cs, ce, cap=None):
    """Split + merge + compaction on a post-energy state dict (n particles)."""
    lib = load()
    n = len(st["pos"])
    cap = cap or max(n * (4 if cfg.split_ways == 4 else 2), 1)
    keep = []
    pin = _pad(st, cap, cfg)
    vin = _view(pin, n, keep)
    out = _alloc_state(cfg, cap)
    vout = _view(out, n, [])
    split = np.zeros(max(n, 1), np.uint32)
    rem = np.zeros(max(n, 1), np.uint32)
    nbr = np.ascontiguousarray(nbr, np.uint32) if nbr is not None else np.zeros(max(n, 1), np.uint32)
    n_out = lib.oracle_adapt(C.byref(cfg), n, cap, C.byref(vin), _u(nbr), _u(idx), _u(cs), _u(ce),
                             C.byref(vout), _u(split), _u(rem))
    if n_out < 0:
        raise RuntimeError("oracle_adapt: capacity exceeded")
    res = {k: v[:n_out].copy() for k, v in out.items()}
    return res, split[:n], rem[:n]


def step(cfg, st, cap=None):
    """One whole oracle step on a state dict; returns (new state, debug)."""
    DebugView = abi().DebugView
    lib = load()
    n = len(st["pos"])
    cap = cap or max(n * (4 if cfg.split_ways == 4 else 2), 1)
    keep = []
    pin = _pad(st, cap, cfg)
    vin = _view(pin, n, keep)
    out = _alloc_state(cfg, cap)
    vout = _view(out, n, [])
    C_ = ncells(cfg)
    dbg = {k: np.zeros(max(n, 1), np.uint32) for k in ("hash", "index", "nbr_count", "split_flag", "removed")}
    dbg["cell_start"] = np.zeros(C_, np.uint32)
    dbg["cell_end"] = np.zeros(C_, np.uint32)
    dbg["trans_vel"] = np.zeros((max(n, 1), cfg.dim), np.float32)
    dv = DebugView()
    for k, a in dbg.items():
        setattr(dv, k, _f(a) if k == "trans_vel" else _u(a))
    n_out = lib.oracle_step(C.byref(cfg), n, cap, C.byref(vin), C.byref(vout), C.byref(dv))
    if n_out < 0:
        raise RuntimeError("oracle_step: capacity exceeded")
    res = {k: v[:n_out].copy() for k, v in out.items()}
    for k in ("hash", "index", "nbr_count", "split_flag", "removed", "trans_vel"):
        dbg[k] = dbg[k][:n]
    return res, dbg


def density_grid(cfg, pos, level, idx, cs, ce):
    lib = load()
    pos = f32(pos)
    level = np.ascontiguousarray(level, np.uint32)
    G = int(cfg.ndens[0] * cfg.ndens[1] * cfg.ndens[2])
    dens = np.zeros(G)
    nrm = np.zeros((G, 3))
    lib.oracle_density_grid(C.byref(cfg), pos.shape[0], _f(pos), _u(level), _u(idx), _u(cs), _u(ce),
                            _d(dens), _d(nrm))
    return dens, nrm


# ----------------------------------------------------------------- FP64 rollout replay
class Rollout64:
    """FP64 replay of a GPU rollout with its recorded topology held fixed
    (sph_rollout_ref.c); `topo` is the list of Solver.rollout_topology()
    dicts of steps 0..T-1."""

    def __init__(self, cfg, topo, grid_n, origin, spacing, target):
        LossGrid = abi().LossGrid
        self.lib = load()
        self.cfg = cfg
        self.keep = topo
        self.steps = (RefTopo * len(topo))()
        for t, d in enumerate(topo):
            st = self.steps[t]
            st.n, st.n_next, st.split_on = d["n"], d["n_next"], d["split_on"]
            for k in ("level", "dens_off", "dens_nbr", "force_off", "force_nbr", "wall", "split", "dst", "child",
                      "merge_leader"):
                setattr(st, k, _u(d[k]))
            for k, src in (("x_rec", "pos"), ("v_rec", "vel"), ("ev_rec", "ev")):
                if src in d:
                    setattr(st, k, _f(d[src]))
        self.grid = LossGrid()
        for a in range(3):
            self.grid.n[a] = int(grid_n[a])
            self.grid.origin[a] = float(origin[a])
        self.grid.spacing = float(spacing)
        self.target = np.ascontiguousarray(target, np.float64).reshape(-1)

    def loss(self, x0, v0, mu, k, want_grid=False):
        x0 = np.ascontiguousarray(x0, np.float64)
        v0 = np.ascontiguousarray(v0, np.float64)
        grid = np.zeros_like(self.target) if want_grid else None
        L = self.lib.ref_rollout_forward(C.byref(self.cfg), self.steps, len(self.keep), len(x0), _d(x0), _d(v0),
                                         float(mu), float(k), C.byref(self.grid), _d(self.target), _d(grid))
        return (L, grid) if want_grid else L

    def grad(self, x0, v0, mu, k):
        x0 = np.ascontiguousarray(x0, np.float64)
        v0 = np.ascontiguousarray(v0, np.float64)
        gx = np.zeros_like(x0)
        gv = np.zeros_like(v0)
        gmu, gk = C.c_double(), C.c_double()
        L = self.lib.ref_rollout_grad(C.byref(self.cfg), self.steps, len(self.keep), len(x0), _d(x0), _d(v0),
                                      float(mu), float(k), C.byref(self.grid), _d(self.target), _d(gx), _d(gv),
                                      C.byref(gmu), C.byref(gk))
        return L, dict(d_pos0=gx, d_vel0=gv, d_mu=gmu.value, d_k=gk.value)

    def grad_along(self, x0, v0, mu, k, x_final):
        """FP64 adjoint linearised about the recorded FP32 trajectory (the
        topology dicts must carry pos/vel/ev; x_final = the final positions)."""
        x0 = np.ascontiguousarray(x0, np.float64)
        v0 = np.ascontiguousarray(v0, np.float64)
        xf = np.ascontiguousarray(x_final, np.float32)
        gx = np.zeros_like(x0)
        gv = np.zeros_like(v0)
        gmu, gk = C.c_double(), C.c_double()
        L = self.lib.ref_rollout_grad_along(C.byref(self.cfg), self.steps, len(self.keep), len(x0), _d(x0), _d(v0),
                                            float(mu), float(k), C.byref(self.grid), _d(self.target), _f(xf),
                                            _d(gx), _d(gv), C.byref(gmu), C.byref(gk))
        return L, dict(d_pos0=gx, d_vel0=gv, d_mu=gmu.value, d_k=gk.value)
