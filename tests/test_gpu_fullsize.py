"""The benchmark's fields at their full sizes.

- the bonded field (4,096 floes): the FP64 path against the oracle, bit for
  bit, over its full 2,000 steps (state, forces, stresses and bonds checked
  after 50, 1,000 and 2,000 steps);
- the polydisperse field (65,536 floes with sheltering, ridging and a
  wall): the FP64 path against the oracle, bit for bit, over 100 steps
  (about two minutes of the single-threaded oracle);
- the polydisperse field: the mixed path within 1e-5 of the FP64 path over
  1,000 steps, relative to the largest displacement of any floe, for all
  but a few floes whose contacts start one step apart in the two runs
  (helpers.check_mixed_positions);
- the 512-field ensemble (2.2 M floes): every member evolves inside the
  batch exactly as it does alone (mixed path: all sums are per floe in a
  fixed order), and the internal forces of each field cancel (Newton's third
  law, up to FP32 rounding)."""
import os

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import Batch, Stepper
from godar_b200.params import PREC_FP64, PREC_MIXED
from oracle import pyoracle as po

from .helpers import DIAG, STATE, check_mixed_positions, gpu_for, oracle_for, pairset

pytestmark = pytest.mark.gpu


def assert_bits(o, g, names):
    of = o.floes()
    for k in names:
        a, b = g.field(k), of[k]
        bad = np.nonzero(a.view(np.int64) != b.view(np.int64))[0]
        assert bad.size == 0, f"{k}: {bad.size} floes differ"


def test_bonded_field_full_size_bit_exact():
    f = gen.bonded_field(nsteps=2000)
    assert f.n == 4096
    o, g = oracle_for(f), gpu_for(f)
    t = 1
    for k in (50, 950, 1000):
        o.step(k)
        g.step(t, 0, k)
        t += k
        assert_bits(o, g, STATE + DIAG)
        ob, gb = o.pairs(po.P_BONDS), g.pairs(2)
        assert pairset(ob[0], ob[1]) == pairset(gb[0], gb[1])
    assert t == 2001


@pytest.fixture(scope="module")
def polydisperse():
    return gen.polydisperse_field(nsteps=1000)


def test_polydisperse_full_size_bit_exact(polydisperse):
    f = polydisperse
    assert f.n == 65536
    o, g = oracle_for(f), gpu_for(f)
    t = 1
    for k in (3, 97):
        o.step(k)
        g.step(t, 0, k)
        t += k
        assert_bits(o, g, STATE + DIAG)
    oc, gc = o.pairs(po.P_CONTACTS), g.pairs(1)
    assert pairset(oc[0], oc[1]) == pairset(gc[0], gc[1])


def test_polydisperse_full_size_mixed_within_tolerance(polydisperse):
    f = polydisperse
    s64, s32 = gpu_for(f, PREC_FP64), gpu_for(f, PREC_MIXED)
    for s in (s64, s32):
        s.step(1, 0, 1000)
    check_mixed_positions(f, s32, s64, onsets=True)
    for k in ("r", "h"):
        assert np.max(np.abs(s32.field(k) - s64.field(k)) / s64.field(k)) <= 1e-5, k


def test_ensemble_members_evolve_as_alone_and_internal_forces_cancel():
    from bench import make_ensemble
    fields = make_ensemble(512, 0, 1, os.cpu_count() or 1)
    assert sum(f.n for f in fields) > 2_000_000
    b = Batch(PREC_MIXED)
    hs = [b.add_field(f) for f in fields]
    b.step(20)
    sizes = [f.n for f in fields]
    for k in sorted({int(np.argmin(sizes)), int(np.argsort(sizes)[len(sizes) // 2]), int(np.argmax(sizes))}):
        f = fields[k]
        s = Stepper(f.params, f.n, PREC_MIXED)
        s.upload(f.x, f.y, f.r, f.h)
        s.step(1, 0, 20)
        for name in ("x", "y", "u", "v"):
            assert np.array_equal(b.field(hs[k], name).view(np.int64), s.field(name).view(np.int64)), (k, name)
        s.close()
    # contact and bond forces are equal and opposite on the two floes of a
    # pair: their sum over a field vanishes up to FP32 rounding
    for k in range(0, len(fields), 37):
        fx = b.field(hs[k], "fcx") + b.field(hs[k], "fbx")
        fy = b.field(hs[k], "fcy") + b.field(hs[k], "fby")
        scale = float(np.sum(np.abs(fx)) + np.sum(np.abs(fy))) or 1.0
        assert abs(float(np.sum(fx))) + abs(float(np.sum(fy))) <= 1e-5 * scale, k
    b.close()
