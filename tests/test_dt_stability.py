"""The time step of the bonded fields.

The benchmark states dt = 0.5 s for its bonded fields, but the reference's
explicit scheme - symplectic Euler with critically damped beam dashpots
(bonds.f90:113-138), integration.f90:1-38 - is unstable there for 6 GPa beams
on floes of a few hundred metres: the oracle's velocities grow by orders of
magnitude per step and overflow within 20 steps.  The bonded fields
therefore run at dt = 0.05 s (generators.DT_BONDED), where the same field
stays bounded.  The GPU side (a run that blows up comes back as
GODAR_ERR_NAN) is in test_gpu_edge.py."""
import numpy as np

from godar_b200 import generators as gen

from .helpers import oracle_for


def _speeds(dt, steps):
    f = gen.bonded_field(n=400, seed=5, nsteps=steps, dt=dt)
    o = oracle_for(f)
    out = []
    for _ in range(steps):
        o.step(1)
        fl = o.floes()
        out.append(float(np.max(np.hypot(fl["u"], fl["v"]))))
    o.close()
    return out


def test_stated_step_diverges_within_twenty_steps():
    s = _speeds(0.5, 20)
    assert s[0] < 1e-2                       # it starts at rest under wind
    assert not np.isfinite(s[-1]) or s[-1] > 1e6, s[-1]
    first_bad = next(k for k, v in enumerate(s) if not (np.isfinite(v) and v < 1e3))
    assert first_bad < 20


def test_used_step_stays_bounded():
    s = _speeds(0.05, 200)
    assert all(np.isfinite(s))
    assert max(s) < 0.05, max(s)
