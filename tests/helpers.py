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
