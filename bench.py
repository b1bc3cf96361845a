"""Benchmark of the adaptive SPH step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the 1.1M-particle four-way adaptive configuration): a 128x128x64
block at spacing 0.005 plus a 65 536-particle sphere falling at 2 m/s in a
1.28 x 1.28 x 0.64 box (128x128x64 cells of h = 0.01), SI constants
(rho0 1000, k 3, mu 0.1, dt 2.5e-5), four-way split/merge on.  Synthetic,
seeded inputs (no dataset exists for this workload).

A step = one call of the C-ABI step: hash, counting sort, stable reorder,
density, force + integration, wavelet energy + split decision, merge,
compaction.  `value` = particle-steps/s with the state resident in HBM,
timed per step with CUDA events on the solver's stream; L2 (126 MB) is
flushed by a 256 MB write between timed steps, outside the events.  `e2e`
= the same metric through the host API a reference user calls: each step
uploads the state from page-locked memory in the reference's Particle
layout, steps, and reads it back (SPHSystem::animation()'s readback).
For N > 1 each rank runs an independent replica (the single-scene step has
no data-parallel split without a halo exchange): weak scaling, value = sum
of particle-steps / max over ranks of the timed duration.

--impl reference times the CPU oracle (the FP64 port of the reference step)
on the host cores on the same workload, rank 0 only.  That arm loads no part
of the package's CUDA library: its configuration comes from the oracle's
restatement of the preset (oracle/presets.py, checked byte for byte against
the library's) and its particles from the numpy scene generator.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D particle-steps/s @1M"
UNIT = "particle-steps/s"
WORKLOAD = ("dam_3d4: 1,048,576-particle block (s=0.005) + 65,536-particle sphere, 1.28x1.28x0.64 box, "
            "128x128x64 cells, four-way split/merge, dt=2.5e-5, SI constants")

# Algorithmic (compulsory) bytes per particle of each stage, every array read
# or written once (neighbour data re-reads are cache traffic, not counted).
STAGE_BYTES = {
    "hash": 16 + 4 + 4 + 4,                  # pos in; key, slot out; count atomics (only a state no
                                             # step wrote: the write-out hashes the next state)
    "scatter": 4 + 4 + 4 + 4,                # key, slot, offset in; index out
    "reorder": 4 + 4 + 48 + 4 + 4 + 4,       # index, key, pos/vel/ev in; sidx, skey, inv out
    "density": 16 + 4 + 8,                   # pos, m in; rho, p out (the unfused figure per stage)
    "force_integrate": 16 * 4 + 16 * 4 + 4,  # pos, ev, aux, vel in; pos, vel, ev, acc, surface out
    "energy_split": 16 + 16 + 4 + 16 + 4 + 4 + 4 + 4 + 4,  # new pos, vel, surf, aux, nbr, idx; energy, flags
    "write": 4 * 16 + 16 + 4 * 4 + 4 * 4 + 4 * 16 + 5 * 4 + 4 + 4,  # sorted state + flags in; canonical state,
                                                                        # next step's key and slot out
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-sample-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    p.add_argument("--batch-scenes", type=int, default=256, help="0 skips the batched-scenes comparison")
    p.add_argument("--batch-steps", type=int, default=500, help="batched steps timed (the 500-step run)")
    p.add_argument("--single-steps", type=int, default=20, help="steps of the one-handle-per-scene baselines")
    p.add_argument("--rollout-steps", type=int, default=200, help="0 skips the differentiable-rollout timing")
    p.add_argument("--other-configs", type=int, default=1, help="0 skips the smaller workloads and CPU detail")
    return p.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region:
    through NVML every 2 ms (read-only queries), else nvidia-smi every 200 ms."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []
        self.running = False

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:   # the CUDA device's own GPU, whatever the visible-device mapping
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self):
        nv, h = self.nvml
        while self.running:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((sm, reasons))
            except Exception:
                break
            time.sleep(0.002)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self.sm_max = self.nvml[0].nvmlDeviceGetMaxClockInfo(self.nvml[1], self.nvml[0].NVML_CLOCK_SM)
            self.running = True
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.running = False
            self.thread.join(timeout=5)
            sm = [float(v) for v, _ in self.samples]
            reasons = sorted({name for _, r in self.samples for bit, name in self.REASONS.items() if r & bit})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(self.sm_max),
                    "reasons": reasons, "samples": len(sm), "source": "NVML, every 2 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r.split(", ") for r in self.lines if r.count(",") >= 8]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, every 200 ms"}


# ----------------------------------------------------------------- helpers
def load_workload(seed):
    import sca2012_b200 as sph
    from sca2012_b200 import scenes
    cfg = sph.preset(sph.PRESET_DAM_3D4)
    pos, vel, lvl = scenes.dam_3d4(cfg, seed=seed)
    return cfg, pos, vel, lvl


def load_workload_host_only(seed):
    """The same workload for the CPU reference arm without the package: the
    configuration from the oracle's restatement of the preset, the particles
    from the scene generator's file loaded on its own (plain numpy).  Nothing
    of the CUDA library is loaded."""
    import importlib.util
    from oracle import presets
    spec = importlib.util.spec_from_file_location("_bench_scenes", os.path.join(ROOT, "sca2012_b200", "scenes.py"))
    scenes = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(scenes)
    cfg = presets.preset(presets.PRESET_DAM_3D4)
    pos, vel, lvl = scenes.dam_3d4(cfg, seed=seed)
    return cfg, pos, vel, lvl


def workload_config(cfg, n0):
    """The `config` of both arms' JSON lines: what defines the workload."""
    return {"workload": WORKLOAD, "particles_initial": int(n0),
            "cells": int(cfg.ncell[0] * cfg.ncell[1] * cfg.ncell[2]),
            "max_particle": int(cfg.max_particle)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def profiled_counters(stage):
    """Per-launch DRAM bytes and warp instructions of `stage` from the
    committed ncu summary, with the particle count of that launch (None where
    absent)."""
    path = os.path.join(ROOT, "profiles", f"{stage}_dam3d4.txt")
    if not os.path.exists(path):
        return None, None, None
    txt = open(path).read()
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    i = re.search(r"smsp__inst_executed.sum\s+([0-9.]+) M", txt)
    n = re.search(r"particles:\s*([0-9]+)", txt)
    return ((float(m.group(1)) if m else None), (float(i.group(1)) * 1e6 if i else None),
            (int(n.group(1)) if n else None))


def issue_fraction(inst, n_prof, n_now, ms, sm_mhz, sms=148):
    """Warp instructions issued (scaled by particle count) over the issue slots
    of the launch: SMs x 4 schedulers x SM clock x duration."""
    if not (inst and n_prof and ms and sm_mhz):
        return None
    return inst * (n_now / n_prof) / (sms * 4 * sm_mhz * 1e6 * ms * 1e-3)


def cpu_baseline(cfg, pos, vel, lvl, steps, threads=None):
    """The oracle (FP64 port of the reference step) on the host cores."""
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    st = dict(pos=pos, vel=vel, level=lvl)
    cap = len(pos) * 4
    t_total, ps = 0.0, 0
    for _ in range(steps):
        n = len(st["pos"])
        t0 = time.perf_counter()
        st, _ = O.step(cfg, st, cap=cap)
        t_total += time.perf_counter() - t0
        ps += n
    return ps / t_total, O.get_threads(), t_total


# ----------------------------------------------------------------- our arm
def reduce_over_ranks(t_ms, units, dist, device):
    """Whole-job timing of independent replicas: the slowest rank's time and
    the units all ranks processed (every rank calls it, in the same order)."""
    if not dist:
        return t_ms, units
    import torch
    import torch.distributed as tdist
    t = torch.tensor([t_ms], device=device, dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    u = torch.tensor([units], device=device, dtype=torch.float64)
    tdist.all_reduce(u)
    return float(t.item()), float(u.item())


def run_ours(args, rank, world, local_rank):
    import torch
    import sca2012_b200 as sph
    torch.cuda.set_device(local_rank)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
    cfg, pos, vel, lvl = load_workload(args.seed + rank)
    n0 = len(pos)
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    stream = torch.cuda.ExternalStream(s.stream_ptr)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)

    for _ in range(args.warmup):
        s.step(1)
    if s.sync_status():
        raise RuntimeError("solver reported an error during warm-up")
    # launch shapes picked by the autotuner on this state (restored afterwards)
    tuning = None if args.no_autotune else s.autotune(reps=3)
    # the timed steps replay each step from a CUDA graph (sph_set_graph; the
    # surface steps launch directly): one untimed step per buffer parity
    # captures both graphs first
    s.set_graph(True)
    for _ in range(2):
        s.step(1)
    cons0 = s.conserved()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    counts = []
    launches = 0
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    for k in range(args.steps):
        flush_l2()
        counts.append(s.num_particles())   # synchronises; outside the events
        ev[k][0].record(stream)
        s.step(1)
        ev[k][1].record(stream)
        launches += s.last_launch_count()
    torch.cuda.synchronize()
    clk = clocks.stop()
    last_step = s.last_step_stats()   # synchronises; after the timed steps
    s.set_graph(False)
    status = s.sync_status()
    cons1 = s.conserved()
    conserved = {"mass_rel_drift": (cons1["mass"] - cons0["mass"]) / cons0["mass"],
                 "momentum_start": cons0["momentum"].tolist(), "momentum_end": cons1["momentum"].tolist(),
                 "energy_start": cons0["energy"], "energy_end": cons1["energy"],
                 "note": "FP64 device sums over the timed steps; gravity and walls act, so only mass is conserved"}
    times = [a.elapsed_time(b) for a, b in ev]
    t_ms = float(sum(times))
    ps = float(sum(counts))
    t_ms, ps = reduce_over_ranks(t_ms, ps, dist, "cuda")
    value = ps / (t_ms * 1e-3)

    # --- per-stage durations (separate profiled steps, same stream)
    s.set_profiling(True)
    stage_ms = {}
    prof_steps = 5
    n_prof = []
    for _ in range(prof_steps):
        flush_l2()
        n_prof.append(s.num_particles())
        s.step(1)
        for name, ms in s.stage_times():
            stage_ms.setdefault(name, []).append(ms)
    s.set_profiling(False)
    stage_avg = {k: float(np.mean(v)) for k, v in stage_ms.items()}
    # the dominant per-step kernel (the surface stage runs every grid_every-th
    # step only and has no per-particle byte count)
    top = max((k for k in stage_avg if k in STAGE_BYTES), key=stage_avg.get)
    n_avg = float(np.mean(n_prof))
    peak, peak_src = measured_peaks()
    alg = STAGE_BYTES.get(top, 0) * n_avg
    achieved = alg / (stage_avg[top] * 1e-3) / 1e9
    traffic_full, _, n_full = profiled_counters(top)
    traffic = traffic_full * (n_avg / n_full) if traffic_full and n_full else None
    # the three neighbour loops together against their compulsory bytes
    # (density 28 + force 64 + energy 36 = 128 B per particle-step), and each
    # against the two bounds it can hit: HBM bytes and instruction issue
    nl_ms = sum(stage_avg.get(k, 0.0) for k in ("density", "force_integrate", "energy_split"))
    nl_gbs = 128.0 * n_avg / (nl_ms * 1e-3) / 1e9 if nl_ms else None
    sm_mhz = clk.get("sm_mhz") or 1965.0
    per_kernel = {}
    for k, nb in (("density", 28), ("force_integrate", 64), ("energy_split", 36)):
        if k not in stage_avg:
            continue
        tr, inst, n_p = profiled_counters(k)
        a = nb * n_avg / (stage_avg[k] * 1e-3) / 1e9
        per_kernel[k] = {"ms": stage_avg[k], "algorithmic_bytes_per_particle": nb, "achieved_gbs": a,
                         "hbm_frac": a / peak,
                         "dram_traffic_per_launch": tr * (n_avg / n_p) if tr and n_p else None,
                         "issue_frac": issue_fraction(inst, n_p, n_avg, stage_avg[k], sm_mhz)}

    # --- plain (non-adaptive) step on the same state, for the "vs plain" ratio
    plain = cfg.copy()
    plain.use_split = 0
    plain.use_merge = 0
    s.set_config(plain)
    pt, pc = [], []
    for _ in range(min(args.steps, 20)):
        flush_l2()
        pc.append(s.num_particles())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.step(1)
        b.record(stream)
        b.synchronize()
        pt.append(a.elapsed_time(b))
    plain_value = sum(pc) / (sum(pt) * 1e-3)
    s.set_config(cfg)

    # --- end to end through the host API (reference Particle records)
    rec = s.record_size
    cap_bytes = cfg.max_particle * rec
    host = torch.empty(cap_bytes, dtype=torch.uint8, pin_memory=True)
    n_cur = s.read_particles_into(host.data_ptr(), cap_bytes)
    e2e_t, e2e_ps, h2d, d2h = 0.0, 0.0, 0, 0
    e2e_steps = min(args.steps, 20)
    for _ in range(e2e_steps):
        flush_l2()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.write_particles_from(host.data_ptr(), n_cur)
        s.step(1)
        n_next = s.read_particles_into(host.data_ptr(), cap_bytes)
        b.record(stream)
        b.synchronize()
        e2e_t += a.elapsed_time(b)
        e2e_ps += n_cur
        h2d += n_cur * rec
        d2h += n_next * rec + 4
        n_cur = n_next
    e2e_t, e2e_ps = reduce_over_ranks(e2e_t, e2e_ps, dist, "cuda")
    e2e_value = e2e_ps / (e2e_t * 1e-3)

    # --- the reference app's frame loop: a step, then the step's records read
    # back for display (SPH-3D-2/sph_main.cpp:613-733), no upload.  Synchronous
    # (sph_read_particles) and asynchronous (sph_read_particles_async into
    # mapped page-locked memory, two buffers, overlapping the next step).
    frame = {}
    fbufs = [host, torch.empty(cap_bytes, dtype=torch.uint8, pin_memory=True)]
    fcnts = [torch.zeros(1, dtype=torch.int32, pin_memory=True) for _ in range(2)]
    for mode in ("sync", "async"):
        torch.cuda.synchronize()
        n_sum, d2h_f = 0, 0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        n_first = s.num_particles()
        for k in range(e2e_steps):
            s.step(1)
            if mode == "sync":
                n_here = s.read_particles_into(host.data_ptr(), cap_bytes)
                n_sum += n_here
                d2h_f += n_here * rec
            else:
                s.read_particles_async_into(fbufs[k & 1].data_ptr(), cap_bytes, fcnts[k & 1].data_ptr())
        if mode == "async":
            s.readback_wait()
        b.record(stream)
        b.synchronize()
        if mode == "async":   # the count moves by well under 1 % over these steps
            n_sum = e2e_steps * (n_first + s.num_particles()) // 2
            d2h_f = n_sum * rec
        ft, fps = reduce_over_ranks(a.elapsed_time(b), n_sum, dist, "cuda")
        frame[mode] = {"value": fps / (ft * 1e-3), "unit": UNIT, "ms_per_step": ft / e2e_steps,
                       "d2h_bytes_per_step": d2h_f // e2e_steps}
    frame["api"] = ("sph_step + sph_read_particles (sync) / sph_read_particles_async into mapped memory "
                    "(async); the L2 is not flushed between these steps")
    status |= s.sync_status()
    s.close()

    # --- the reference's own default 3D-2 scene (7,220 particles, split and
    # merge on): launch-bound, so eager launches vs CUDA-graph replay
    from sca2012_b200 import scenes as _sc
    small = {}
    rcfg = sph.preset(sph.PRESET_REF_3D2)
    rcfg.use_split = rcfg.use_merge = 1
    rpos, rvel, rlvl = _sc.ref_box_3d2(rcfg)
    for mode in ("eager", "graph"):
        rs = sph.Solver(rcfg)
        rs.set_graph(mode == "graph")
        rs.set_state(dict(pos=rpos, vel=rvel, level=rlvl))
        rs.step(5)
        rst = torch.cuda.ExternalStream(rs.stream_ptr)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(rst)
        rs.step(50)
        b.record(rst)
        b.synchronize()
        small[mode + "_ms_per_step"] = a.elapsed_time(b) / 50
        status |= rs.sync_status()
        rs.close()
    small["particles_initial"] = len(rpos)

    batched = batched_scenes(args, rank, world) if args.batch_scenes else None
    others = small_configs(args) if (world == 1 and not args.no_cpu_baseline and args.other_configs) else None
    roll = rollout_bench(args) if (world == 1 and args.rollout_steps) else None

    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, cores, tt = cpu_baseline(cfg, pos, vel, lvl, args.cpu_sample_steps)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                   "sample": f"{args.cpu_sample_steps} full steps of the same workload from its initial state "
                             f"({tt:.1f} s), FP64 oracle, OpenMP"}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(cfg, n0),
            "timing": {"particles_timed_mean": ps / args.steps / world,
                       "l2": "flushed (256 MB write) between timed steps",
                       "launch": "CUDA graph replay per step (surface steps launch directly)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "plain_value": plain_value, "adaptive_vs_plain": value / plain_value,
            "last_timed_step": last_step,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // e2e_steps,
                    "d2h_bytes_per_step": d2h // e2e_steps,
                    "api": "sph_write_particles + sph_step + sph_read_particles (page-locked host)",
                    "frame_loop": frame},
            "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_particle": STAGE_BYTES.get(top),
                         "launch_ms": stage_avg[top], "peak_source": peak_src,
                         "note": ("neighbour loops are bound by FP32 issue (density) and dependent-load latency "
                                  "(force, energy): the HBM fraction is low by design"),
                         "neighbour_loops": {"stages": ["density", "force_integrate", "energy_split"],
                                             "bytes_per_particle": 128, "ms": nl_ms, "achieved": nl_gbs,
                                             "frac": nl_gbs / peak if nl_gbs else None,
                                             "per_kernel": per_kernel,
                                             "issue_frac_note": ("ncu smsp__inst_executed.sum of the committed "
                                                                 "profiles/<kernel>_dam3d4.txt, scaled by particle "
                                                                 "count, / (148 SMs x 4 x median SM clock x live "
                                                                 "kernel time)")}},
            "stages_ms": stage_avg,
            "tuning": tuning,
            "conserved": conserved,
            "ref_3d2_default_scene": small,
            "batched_scenes": batched,
            "other_configs": others,
            "rollout": roll,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": launches,
            "status": status,
        }
    return out


# ----------------------------------------------------------------- other configurations
def small_configs(args):
    """The 2D plain dam break (4,096 particles, no adaptivity, 1,000-step
    config) and the 3D two-way dam break (131,072 particles, 500-step config)
    on the GPU, eager, CUDA-graph and persistent (one cooperative launch per
    step), 200 timed steps each; and the FP64
    oracle on the host, one thread and all threads, a few steps of each of
    the three workloads (particle-steps/s)."""
    import torch
    import sca2012_b200 as sph
    from sca2012_b200 import scenes as sc
    from oracle import oracle as O
    cases = {"dam_2d_4096": (sph.PRESET_DAM_2D, sc.dam_2d, 0), "dam_3d2_131072": (sph.PRESET_DAM_3D2, sc.dam_3d2, 1)}
    gpu, cpu = {}, {}
    for name, (pre, make, adapt) in cases.items():
        cfg = sph.preset(pre)
        cfg.use_split = cfg.use_merge = adapt
        pos, vel, lvl = make(cfg, seed=args.seed)
        for mode in ("eager", "graph", "persistent"):
            s = sph.Solver(cfg)
            s.set_graph(mode == "graph")
            s.set_persistent(mode == "persistent")
            s.set_state(dict(pos=pos, vel=vel, level=lvl))
            s.step(5)
            st = torch.cuda.ExternalStream(s.stream_ptr)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            n_before = s.num_particles()
            a.record(st)
            s.step(200)
            b.record(st)
            b.synchronize()
            n_after = s.num_particles()
            gpu.setdefault(name, {})[mode] = 200 * 0.5 * (n_before + n_after) / (a.elapsed_time(b) * 1e-3)
            s.close()
        for th in (1, os.cpu_count() or 1):
            v, used, _ = cpu_baseline(cfg, pos, vel, lvl, 3 if adapt else 10, threads=th)
            cpu.setdefault(name, {})[f"threads_{used}"] = v
    cfg, pos, vel, lvl = load_workload(args.seed)
    for th in (1, os.cpu_count() or 1):
        v, used, _ = cpu_baseline(cfg, pos, vel, lvl, 1, threads=th)
        cpu.setdefault("dam_3d4_1114112", {})[f"threads_{used}"] = v
    O.set_threads(0)
    return {"gpu_particle_steps_per_s": gpu, "cpu_oracle_particle_steps_per_s": cpu,
            "cpu_cores": os.cpu_count(), "note": "GPU: CUDA events, count averaged over the window"}


# ----------------------------------------------------------------- batched scenes
def batched_scenes(args, rank=0, world=1):
    """256 independent dam-break scenes (128 2D, 128 3D two-way; sizes
    log-uniform in [1024, 65536], per-scene viscosity and stiffness), split
    and merge on.  Batched: one handle per dimensionality holding all its
    scenes, each step replayed as a CUDA graph, over the 500-step run (the
    same steps are also timed with plain launches and as one persistent
    launch per step).  Baselines (rates over --single-steps): one handle per
    scene in its own box-sized world with plain (eager) launches, stepped
    (a) one scene at a time, each synchronised before the next, and (b) all
    handles' streams at once.  Scene-steps/s by wall clock around
    synchronised loops (the baselines span 256 streams).  With N > 1 ranks
    the scenes are sharded (scene k on rank k mod N, no collective in the
    step) and only the batched figure is taken: all scenes / the slowest
    rank's time."""
    import torch
    import sca2012_b200 as sph
    from sca2012_b200 import scenes as sc
    half = args.batch_scenes // 2
    steps = args.batch_steps
    batches = []
    for pre, seed in ((sph.PRESET_DAM_2D, args.seed + 11), (sph.PRESET_DAM_3D2, args.seed + 12)):
        base = sph.preset(pre)
        base.use_split = base.use_merge = 1
        mine = [k for k in range(half) if k % world == rank]
        batches.append(sc.batch_scenes(base, half, seed=seed, subset=mine if world > 1 else None))

    def timed_call(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    def timed(solvers, k, per_scene_sync=False):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            for h in solvers:
                h.step(1)
                if per_scene_sync:
                    h.sync()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    # batched
    bs = []
    particles = 0
    for cfg, boxes, pos, vel, lvl, scene, counts in batches:
        h = sph.Solver(cfg)
        h.set_scenes(boxes)
        h.set_state(dict(pos=pos, vel=vel, level=lvl, scene=scene))
        h.set_graph(True)
        bs.append(h)
        particles += len(pos)
    timed(bs, 3)
    # launch shapes picked by the autotuner on each handle's state (restored afterwards)
    tuned = [None if args.no_autotune else h.autotune(reps=2) for h in bs]
    t_batched = timed(bs, steps)
    # the same steps with plain launches: what graph replay saves, i.e. the
    # launch overhead a single persistent launch per step could remove at most
    for h in bs:
        h.set_graph(False)
    t_eager = timed(bs, steps)
    # and as one persistent launch per step (sph_set_persistent)
    for h in bs:
        h.set_persistent(True)
    t_persist = timed(bs, steps)
    for h in bs:
        h.set_persistent(False)
        h.set_graph(True)
    status = 0
    if world > 1:
        n_mine = sum(len(b[1]) for b in batches)
        t_all, n_all = reduce_over_ranks(t_batched, float(n_mine), True, "cuda")
        for h in bs:
            status |= h.sync_status()
            h.close()
        return {"scenes": int(n_all), "ranks": world, "steps": steps, "sharding": "scene k on rank k mod N",
                "batched_scene_steps_per_s": n_all * steps / t_all, "status": status,
                "timing": "wall clock around synchronised step loops, slowest rank"}
    # the adjoint of the last 50 steps, batched: checkpointed forward, a
    # density-grid loss over every scene (nodes at cell centres), backward
    t_fwd = t_bwd = 0.0
    adj_steps = 50
    # the plain batched step at this state (graph replay), the ratio's denominator
    t_plain_here = timed(bs, adj_steps)
    for h, (cfg, boxes, *_rest) in zip(bs, batches):
        gn = tuple(int(cfg.ncell[a]) for a in range(3))
        org = tuple(0.5 * float(cfg.cell_size) for _ in range(3))
        h.rollout_forward(adj_steps, 10)   # allocates checkpoints and tape (untimed)
        n_start = h.num_particles()
        t_fwd += timed_call(lambda: h.rollout_forward(adj_steps, 10))
        h.splat_loss(gn, org, float(cfg.cell_size), np.zeros(int(np.prod(gn)), np.float32))
        t_bwd += timed_call(lambda: h.rollout_backward(n_start, nscenes=len(boxes)))
    for h in bs:
        status |= h.sync_status()
        h.close()
    # one handle per scene
    singles = []
    for cfg, boxes, pos, vel, lvl, scene, counts in batches:
        first = np.concatenate([[0], np.cumsum(counts)])
        for k, (lo, hi, mu, stiff) in enumerate(boxes):
            c1 = cfg.copy()
            for a in range(int(cfg.dim)):
                c1.ncell[a] = int(round((hi[a] - lo[a]) / float(cfg.cell_size)))
                c1.world[a] = np.float32(c1.ncell[a]) * np.float32(cfg.cell_size)
            c1.viscosity, c1.gas_constant = mu, stiff
            c1.max_particle = int(4 * counts[k])
            h = sph.Solver(c1)
            sl = slice(first[k], first[k + 1])
            h.set_state(dict(pos=pos[sl] - np.asarray(lo, np.float32), vel=vel[sl], level=lvl[sl]))
            singles.append(h)
    # the baselines are rates over fewer steps (256 handles one after another
    # take about 40 ms a step)
    timed(singles, 2)
    s_steps = args.single_steps
    t_seq = timed(singles, s_steps, per_scene_sync=True)
    t_conc = timed(singles, s_steps)
    for h in singles:
        status |= h.sync_status()
        h.close()
    n_sc = len(singles)
    v_b = n_sc * steps / t_batched
    v_s = n_sc * s_steps / t_seq
    v_c = n_sc * s_steps / t_conc
    return {"scenes": n_sc, "particles_initial": particles, "steps": steps, "baseline_steps": s_steps,
            "batched_scene_steps_per_s": v_b, "sequential_scene_steps_per_s": v_s,
            "concurrent_streams_scene_steps_per_s": v_c,
            "batched_vs_sequential": v_b / v_s, "batched_vs_concurrent_streams": v_b / v_c,
            "batched_ms_per_step": t_batched / steps * 1e3,
            "batched_eager_launches_ms_per_step": t_eager / steps * 1e3,
            "batched_persistent_ms_per_step": t_persist / steps * 1e3,
            "batched_persistent_scene_steps_per_s": n_sc * steps / t_persist, "status": status,
            "tuning": [None if t is None else {"block": t["block"], "blocks_per_sm": t["blocks_per_sm"]}
                       for t in tuned],
            "adjoint_last_50": {"forward_ms_per_step": t_fwd / adj_steps * 1e3,
                                "backward_ms_per_step": t_bwd / adj_steps * 1e3,
                                "backward_vs_forward": t_bwd / t_fwd,
                                "plain_batched_ms_per_step_here": t_plain_here / adj_steps * 1e3,
                                "backward_vs_plain_batched_step": t_bwd / t_plain_here,
                                "loss": "mean squared density grid (nodes at cell centres), per-scene gradients"},
            "timing": "wall clock around synchronised step loops"}


# ----------------------------------------------------------------- differentiable rollout
def rollout_bench(args):
    """Differentiable-rollout workload: a 32^3 block (spacing 0.01) in the
    0.64^3 box, initial velocities N(0, 0.1^2), two-way split/merge on, 200
    steps with checkpoints every 20, a 32^3 density-grid loss against the
    grid of a run with viscosity 0.15 and stiffness 4.  Reports the plain
    forward (eager steps), the checkpointed forward, and the backward (the
    taped replay of every interval plus the adjoint kernels), each per step;
    wall clock around synchronised calls."""
    import torch
    import sca2012_b200 as sph
    from sca2012_b200 import scenes as sc
    T, every = args.rollout_steps, 20
    cfg = sph.preset(sph.PRESET_ROLLOUT_3D)
    pos, _, lvl = sc.block_3d(cfg, counts=(32, 32, 32), spacing=0.01, seed=args.seed)
    vel = np.random.default_rng(args.seed).normal(0.0, 0.1, pos.shape).astype(np.float32)
    gn, org, sp = (32, 32, 32), (0.01, 0.01, 0.01), 0.02
    tcfg = cfg.copy()
    tcfg.viscosity, tcfg.gas_constant = 0.15, 4.0
    ts = sph.Solver(tcfg)
    ts.set_state(dict(pos=pos, vel=vel, level=lvl))
    ts.step(T)
    _, target = ts.splat_loss(gn, org, sp, np.zeros(32 ** 3, np.float32))
    ts.close()

    def wall(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(3)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    t_plain = wall(lambda: (s.step(T), s.sync()))
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.rollout_forward(T, every)     # warm-up (allocations)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    t_fwd = wall(lambda: s.rollout_forward(T, every))
    n_final = s.num_particles()
    loss = [None]
    t_loss = wall(lambda: loss.__setitem__(0, s.splat_loss(gn, org, sp, target)[0]))
    g = [None]
    t_bwd = wall(lambda: g.__setitem__(0, s.rollout_backward(len(pos))))
    status = s.sync_status()
    s.close()
    dp = g[0]["d_params"][0]
    return {"particles_initial": len(pos), "particles_final": n_final, "steps": T, "checkpoint_every": every,
            "plain_forward_ms_per_step": t_plain / T * 1e3,
            "rollout_forward_ms_per_step": t_fwd / T * 1e3,
            "backward_ms_per_step": t_bwd / T * 1e3,
            "backward_vs_plain_forward": t_bwd / t_plain,
            "loss": loss[0], "loss_ms": t_loss * 1e3,
            "d_viscosity": float(dp[0]), "d_gas_constant": float(dp[1]),
            "d_vel0_norm": float(np.linalg.norm(g[0]["d_vel0"])), "status": status,
            "timing": "wall clock around synchronised calls"}


# ----------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return None
    cfg, pos, vel, lvl = load_workload_host_only(args.seed)
    from oracle import oracle as O
    st = dict(pos=pos, vel=vel, level=lvl)
    cap = len(pos) * 4
    # bounded sample: each step is one full oracle step of the workload
    for _ in range(args.warmup if args.warmup < 2 else 1):
        st, _ = O.step(cfg, st, cap=cap)
    t, ps = 0.0, 0.0
    for _ in range(args.steps):
        n = len(st["pos"])
        t0 = time.perf_counter()
        st, _ = O.step(cfg, st, cap=cap)
        t += time.perf_counter() - t0
        ps += n
    v = ps / t
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(cfg, len(pos)),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": O.get_threads(), "kind": "port",
                             "sample": f"{args.steps} full steps of the workload, FP64 oracle, OpenMP, "
                                       f"after {min(args.warmup, 1)} warm-up step(s)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        out = run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()
    if out:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
