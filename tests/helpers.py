"""Shared helpers of the parity tests: run a field through the CPU oracle and
through the C ABI side by side."""
from __future__ import annotations

import numpy as np

from oracle import pyoracle as po

STATE = ["x", "y", "u", "v", "r", "h", "theta", "omega"]
DIAG = ["tfx", "tfy", "fcx", "fcy", "fbx", "fby", "m", "mc", "mb", "tsigxx", "tsigyy",
        "tsigxy", "tsigyx", "tp"]


def oracle_for(f, ridge_mode=po.RIDGE_DEFERRED):
    return po.Oracle(f.params, f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v,
                     bonds=f.bonds, damage=f.damage, field=f.forcing, ridge_mode=ridge_mode)


def gpu_for(f, precision=0):
    from godar_b200.lib import Stepper
    s = Stepper(f.params, f.n, precision)
    s.upload(f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, bonds=f.bonds, damage=f.damage)
    if f.forcing is not None:
        s.set_field(f.forcing)
    return s


def run_both(f, nsteps, chunks=1, precision=0):
    """Advances oracle and GPU by nsteps (in `chunks` calls); returns both."""
    o = oracle_for(f)
    g = gpu_for(f, precision)
    per = nsteps // chunks
    t = 1
    for c in range(chunks):
        k = per if c < chunks - 1 else nsteps - per * (chunks - 1)
        o.step(k)
        g.step(t, 0, k)
        t += k
    return o, g


def max_rel(a, b, scale=None):
    a = np.asarray(a)
    b = np.asarray(b)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def pairset(pi, pj):
    return set(zip(pi.tolist(), pj.tolist()))


def _wrapped(d, L, periodic):
    d = np.asarray(d, dtype=np.float64)
    return d - L * np.round(d / L) if periodic else d


def position_error(f, xa, ya, xb, yb):
    """Largest distance between two runs' positions of the same floes
    (nearest image along periodic axes), in metres, and the largest
    displacement of run b from the field's initial positions: the motion a
    tolerance must be tighter than."""
    from godar_b200.params import BC_PERIODIC_X, BC_PERIODIC_Y
    px = bool(f.params.boundary & BC_PERIODIC_X)
    py = bool(f.params.boundary & BC_PERIODIC_Y)
    dx = _wrapped(xa - xb, f.params.nx, px)
    dy = _wrapped(ya - yb, f.params.ny, py)
    mx = _wrapped(xb - f.x, f.params.nx, px)
    my = _wrapped(yb - f.y, f.params.ny, py)
    return float(np.max(np.hypot(dx, dy))), float(np.max(np.hypot(mx, my)))


# The mixed path's position tolerance, relative to the largest displacement
# of any floe over the run (the target: positions within 1e-5 of the FP64
# path's, relative), so that a mixed run that did not move the floes fails.
MIXED_POS_REL = 1e-5
# Fields where contacts form during the run: a pair whose gap crosses zero
# within the two runs' position difference (about 1e-9 m) touches one step
# earlier in one of them, and that floe's error jumps to the effect of one
# step of contact force.  Measured: on the 65,536-floe sheltering + ridging
# field 9 floes of 65,536 beyond 1e-5 of the motion after 1,000 steps (the
# largest 1.0e-4); on a 500-floe field one floe at 2.2e-3 after 100 steps.
# Such fields are held to 1e-5 for all but ONSET_FRACTION of the floes and
# to ONSET_MAX for the rest.
ONSET_FRACTION = 0.01
ONSET_MAX = 1e-2


def check_mixed_positions(f, s32, s64, onsets=False):
    """Asserts the mixed run s32 against the FP64 run s64 of field f;
    returns (largest error, largest displacement, floes beyond 1e-5)."""
    from godar_b200.params import BC_PERIODIC_X, BC_PERIODIC_Y
    err, moved = position_error(f, s32.field("x"), s32.field("y"), s64.field("x"), s64.field("y"))
    px = bool(f.params.boundary & BC_PERIODIC_X)
    py = bool(f.params.boundary & BC_PERIODIC_Y)
    e = np.hypot(_wrapped(s32.field("x") - s64.field("x"), f.params.nx, px),
                 _wrapped(s32.field("y") - s64.field("y"), f.params.ny, py))
    beyond = int(np.sum(e > MIXED_POS_REL * moved))
    print(f"{f.name}: position error {err:.3e} m, largest displacement {moved:.3e} m, "
          f"{beyond} of {f.n} floes beyond {MIXED_POS_REL:g} of it")
    assert moved > 0.0
    if onsets:
        assert beyond <= ONSET_FRACTION * f.n, (beyond, f.n)
        assert err <= ONSET_MAX * moved, (err, moved)
    else:
        assert err <= MIXED_POS_REL * moved, (err, moved)
    return err, moved, beyond
