"""GPU parity: the FP64 path through the C ABI against the CPU oracle.

The FP64 step reproduces the reference's sequential summation order and uses
the same deterministic transcendentals as the oracle, so the bar here is
bit-identical state, forces and pair topology."""

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.params import make_params, BC_PERIODIC_X, BC_PERIODIC_Y
from oracle import pyoracle as po

from .helpers import DIAG, STATE, pairset, run_both

pytestmark = pytest.mark.gpu


def assert_bit_equal(o, g, fields):
    of = o.floes()
    for k in fields:
        a = g.field(k)
        b = of[k]
        bad = np.nonzero(a.view(np.int64) != b.view(np.int64))[0]
        assert bad.size == 0, f"{k}: {bad.size} floes differ, first {bad[:5]}: gpu {a[bad[:3]]} oracle {b[bad[:3]]}"


def two_disk_field(periodic: bool, gap: float = 1.0, speed: float = 0.5):
    L = 1e5
    p = make_params(L, L, cohesion=0, shelter=0, ridging=0, dt=0.05, rtree=1000.0, lat=0.0,
                    boundary=(BC_PERIODIC_X | BC_PERIODIC_Y) if periodic else 0)
    x = np.array([50000.0, 52000.0 + gap])
    y = np.array([50000.0, 50000.0 + 30.0])
    r = np.array([1000.0, 1000.0])
    h = np.array([1.0, 1.2])
    f = gen.Field("two", p, x, y, r, h, 2000, u=np.array([speed, -speed]), v=np.zeros(2))
    return f


@pytest.mark.parametrize("periodic", [True, False])
def test_two_disk_collision_bit_exact(periodic):
    f = two_disk_field(periodic)
    o, g = run_both(f, 1500, chunks=3)
    assert_bit_equal(o, g, STATE + DIAG)


def test_lattice_periodic_bit_exact_1000_steps():
    f = gen.lattice_field(periodic=True)
    o, g = run_both(f, 1000, chunks=4)
    assert_bit_equal(o, g, STATE + DIAG)
    oi, oj, _ = o.pairs(po.P_CANDIDATES)
    gi, gj, _ = g.pairs(0)
    assert pairset(oi, oj) == pairset(gi, gj)


def test_lattice_walls_bit_exact():
    f = gen.lattice_field(periodic=False)
    o, g = run_both(f, 600, chunks=2)
    assert_bit_equal(o, g, STATE + DIAG)


def test_bonded_field_bit_exact():
    f = gen.bonded_field(n=300, nsteps=300)
    o, g = run_both(f, 300, chunks=3)
    assert_bit_equal(o, g, STATE + DIAG)
    ob = o.pairs(po.P_BONDS)
    gb = g.pairs(2)
    assert pairset(ob[0], ob[1]) == pairset(gb[0], gb[1])
    oc = o.pairs(po.P_CANDIDATES)
    gc = g.pairs(0)
    assert pairset(oc[0], oc[1]) == pairset(gc[0], gc[1])


def test_large_bonded_field_bit_exact():
    """10000 floes: the bond table is built in chunks of floes on several
    host threads and must be the oracle's, bond for bond."""
    f = gen.bonded_field(n=10000, nsteps=6)
    o, g = run_both(f, 6, chunks=2)
    assert_bit_equal(o, g, STATE)
    ob = o.pairs(po.P_BONDS)
    gb = g.pairs(2)
    assert len(ob[0]) > 10000
    assert pairset(ob[0], ob[1]) == pairset(gb[0], gb[1])


def test_polydisperse_shelter_ridging_bit_exact():
    f = gen.polydisperse_field(n=600, nsteps=200)
    o, g = run_both(f, 200, chunks=2)
    assert_bit_equal(o, g, STATE + DIAG)
    oc = o.pairs(po.P_CONTACTS)
    gc = g.pairs(1)
    assert pairset(oc[0], oc[1]) == pairset(gc[0], gc[1])
