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
