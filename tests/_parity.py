"""Stage-by-stage parity checks shared by the oracle-vs-reference and
CUDA-vs-oracle tests.

Tolerances (stated once, used everywhere):
  * integer outputs (cell keys, sorted index, cell ranges, neighbour counts,
    split flags, merge flags, levels, particle counts): bit-exact;
  * float outputs vs the FP64 oracle: per particle
        |x - x64| <= RTOL * max(|x64|, rms(x64))
    with RTOL = 1e-5, |.| the Euclidean norm for vectors and rms taken over
    all particles of that field.  A particle whose value is at least the
    field's RMS is held to 1e-5 of its own value; one whose value is a
    near-total cancellation of its neighbour sum (the colour-field gradient
    deep inside the fluid, the pressure k((rho/rho0)^3 - 1) at rho ~ rho0)
    is held to 1e-5 of the field's typical size, because an FP32 sum's
    rounding error scales with its terms, not with what is left after they
    cancel;
  * particles whose FP64 value sits within 1e-5 of a discontinuity the FP32
    code decides (the surface-tension switch, a wall) are reported as
    ambiguous and excluded from the value comparison of that stage.
"""
import json
import os

import numpy as np

RTOL = 1e-5
FLOOR = 1.0

# One record per check_close call: how many particles were compared, how
# many were held to the field's RMS instead of their own value (|x64| below
# FLOOR * rms), how many of those pass only because of that floor (error
# against their own value above RTOL), how many were excluded as ambiguous,
# and the largest error against its own value among the particles above the
# RMS.  Written as JSON
# lines to $SPH_PARITY_REPORT when that is set.
REPORT = []


def norm_rows(a):
    a = np.asarray(a, np.float64)
    return np.abs(a) if a.ndim == 1 else np.sqrt((a * a).sum(-1))


def rel_err(x, ref, floor=FLOOR):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    d = norm_rows(x - ref)
    r = norm_rows(ref)
    rms = np.sqrt(np.mean(r[np.isfinite(r)] ** 2)) if np.isfinite(r).any() else 0.0
    scale = np.maximum(r, floor * rms)
    scale = np.where(scale > 0, scale, 1.0)
    return d / scale


def check_close(name, x, ref, mask=None, rtol=RTOL, floor=FLOOR):
    """Asserts the per-particle relative error bound; NaN must match NaN."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    nx = ~np.isfinite(x) if x.ndim == 1 else ~np.isfinite(x).all(-1)
    nr = ~np.isfinite(ref) if ref.ndim == 1 else ~np.isfinite(ref).all(-1)
    sel = np.ones(len(x), bool) if mask is None else np.asarray(mask, bool)
    bad_nan = sel & (nx != nr)
    assert not bad_nan.any(), f"{name}: NaN pattern differs at {np.flatnonzero(bad_nan)[:10]}"
    ok = sel & ~nr
    xs = np.where(nx[:, None] if x.ndim > 1 else nx, 0, x)
    rs = np.where(nr[:, None] if ref.ndim > 1 else nr, 0, ref)
    e = rel_err(xs, rs, floor)
    e = np.where(ok, e, 0.0)
    r = norm_rows(rs)
    rms = np.sqrt(np.mean(r[ok] ** 2)) if ok.any() else 0.0
    below = ok & (r < floor * rms)
    own = np.where(ok & (r > 0), norm_rows(xs - rs) / np.where(r > 0, r, 1.0), 0.0)
    # particles that pass only because of the floor: their error against
    # their own value is above rtol
    needs_floor = ok & (own > rtol)
    rec = {"name": name, "compared": int(ok.sum()), "held_to_rms": int(below.sum()),
           "pass_only_by_floor": int(needs_floor.sum()),
           "excluded_ambiguous": int((~sel).sum()), "non_finite_matched": int((sel & nr).sum()),
           "max_err_bound": float(e.max(initial=0.0)),
           "max_err_own_value_above_rms": float(np.where(below, 0.0, own).max(initial=0.0))}
    REPORT.append(rec)
    path = os.environ.get("SPH_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rec) + "\n")
    worst = int(np.argmax(e)) if len(e) else 0
    assert e.max(initial=0.0) <= rtol, (
        f"{name}: max rel err {e.max():.3e} > {rtol:.0e} at particle {worst} "
        f"(got {x[worst]}, ref {ref[worst]}); {rec['held_to_rms']} of {rec['compared']} held to the RMS, "
        f"{rec['excluded_ambiguous']} excluded")
    return rec["max_err_bound"]


def check_equal(name, x, ref):
    x = np.asarray(x)
    ref = np.asarray(ref)
    assert x.shape == ref.shape, f"{name}: shape {x.shape} vs {ref.shape}"
    bad = np.flatnonzero((x != ref).reshape(len(x), -1).any(-1)) if x.size else []
    assert len(bad) == 0, f"{name}: {len(bad)} mismatches, first at {bad[:10]}: {x[bad[:5]]} vs {ref[bad[:5]]}"
