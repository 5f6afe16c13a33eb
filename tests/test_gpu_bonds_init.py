"""Bond creation on the device at admission (bonds_init.cu): the bonds of
time step 1 (stepper.f90:93-101) and their geometry (bond_properties,
bonds.f90:237-269), read back bit for bit through a checkpoint of the fresh
field and compared with the same rule restated here in numpy over all
pairs i < j:

    dist <= r_i + rtree  and  (r_i + r_j) - dist >= -(bond_lim + bond_lim_rel (r_i + r_j))
    [and hash(seed, i, j) / 2^32 < bond_frac  when 0 < bond_frac < 1]

    rb = lambda_rb min(r_i, r_j), hb = (h_i + h_j) / 2, lb = dist,
    sb = 2 rb hb, ib = 2/3 hb rb^3

and with the oracle's bond list after its first step.  Fields: the relative
limit of the bonded fields (doubly periodic, pairs across the boundary), the
hashed 10 % of the polydisperse field (a wall, open side), the reference's
absolute limit with four walls, and fields admitted together into one batch
beside a resident one."""
import struct

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import Batch, Stepper
from godar_b200.params import BC_PERIODIC_X, BC_PERIODIC_Y, PREC_FP64, PREC_MIXED, make_params
from oracle import pyoracle as po

from .helpers import oracle_for, pairset

pytestmark = pytest.mark.gpu


def _expected(f):
    """Bond table of the rule, in (i, j) order: arrays i, j, rb, hb, lb, sb, ib."""
    p = f.params
    x, y, r, h = f.x, f.y, f.r, f.h
    px, py = bool(p.boundary & BC_PERIODIC_X), bool(p.boundary & BC_PERIODIC_Y)
    out = []
    for i in range(f.n - 1):
        j = np.arange(i + 1, f.n)
        dx = x[i] - x[j]
        dy = y[i] - y[j]
        if px:
            dx = np.where(dx > 0.5 * p.nx, dx - p.nx, np.where(dx < -0.5 * p.nx, dx + p.nx, dx))
        if py:
            dy = np.where(dy > 0.5 * p.ny, dy - p.ny, np.where(dy < -0.5 * p.ny, dy + p.ny, dy))
        dist = np.sqrt(dx * dx + dy * dy)
        lim = p.bond_lim + p.bond_lim_rel * (r[i] + r[j])
        ok = (dist <= r[i] + p.rtree) & (((r[i] + r[j]) - dist) >= -lim)
        for k in np.nonzero(ok)[0]:
            out.append((i, int(j[k]), float(dist[k])))
    return out


def _geometry(p, r, h, i, j, dist):
    ri, rj = r[i], r[j]
    rb = p.lambda_rb * (ri if ri < rj else rj)
    hb = (h[i] + h[j]) / 2.0
    sb = (2.0 * rb) * hb
    ib = ((2.0 / 3.0) * hb) * ((rb * rb) * rb)
    return rb, hb, dist, sb, ib


def _table(data):
    """Bond table of a checkpoint: list of (i, j, flag, rb, hb, lb, sb, ib, dmg)."""
    magic, ver, prec, n, nb, nh, _ = struct.unpack_from("8s6i", data, 0)
    assert magic == b"GODARCK1"
    o = 32 + 12 * 8 * n
    out = []
    for _ in range(nb):
        i, j, flag, _ = struct.unpack_from("4i", data, o)
        v = struct.unpack_from("10d", data, o + 16)
        out.append((i, j, flag) + v[:5] + (v[9],))
        o += 16 + 80
    return out


def _device_table(f, precision=PREC_FP64):
    s = Stepper(f.params, f.n, precision)
    s.upload(f.x, f.y, f.r, f.h)
    if f.forcing is not None:
        s.set_field(f.forcing)
    s.step(1, 0, 0)     # admits the field (time step 1, not a restart) without stepping
    t = _table(s.checkpoint())
    s.close()
    return t


def _check_against_rule(f, t):
    want = _expected(f)
    assert [(a[0], a[1]) for a in t] == [(i, j) for i, j, _ in want]
    for row, (i, j, dist) in zip(t, want):
        g = _geometry(f.params, f.r, f.h, i, j, dist)
        assert row[2] == 1 and row[8] == 0.0
        assert all(np.float64(a).view(np.int64) == np.float64(b).view(np.int64) for a, b in zip(row[3:8], g)), (i, j)


def _check_against_oracle(f, t):
    o = oracle_for(f)
    o.step(1)
    bi, bj, _ = o.pairs(po.P_BONDS)
    o.close()
    assert pairset(bi, bj) == {(a[0], a[1]) for a in t}


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_relative_limit_periodic(precision):
    f = gen.bonded_field(n=1200, seed=3, nsteps=10)
    t = _device_table(f, precision)
    assert len(t) > f.n
    _check_against_rule(f, t)
    _check_against_oracle(f, t)


def test_hashed_fraction_with_a_wall():
    f = gen.polydisperse_field(n=3000, seed=2, nsteps=10)
    assert 0.0 < f.params.bond_frac < 1.0
    t = _device_table(f)
    assert len(t) > 0
    # the hashed selection is the oracle's: its first-step bond list
    _check_against_oracle(f, t)
    # and every listed bond satisfies the geometric rule, with its geometry
    full = {(i, j): d for i, j, d in _expected(f)}
    assert len(t) < len(full)
    for row in t:
        d = full[(row[0], row[1])]
        g = _geometry(f.params, f.r, f.h, row[0], row[1], d)
        assert all(np.float64(a).view(np.int64) == np.float64(b).view(np.int64) for a, b in zip(row[3:8], g))


def test_absolute_limit_four_walls():
    rng = np.random.default_rng(11)
    n = 900
    r = rng.uniform(150.0, 400.0, n)
    h = rng.uniform(0.5, 2.0, n)
    # non-overlapping disks at 60 % area fraction, inside the four walls
    x, y, L, _, _ = gen.place_fraction(r, 0.6, 1.0, False, False, 11)
    assert np.all(x - r >= 0) and np.all(x + r <= L) and np.all(y - r >= 0) and np.all(y + r <= L)
    p = make_params(L, L, cohesion=1, shelter=0, ridging=0, dt=0.02, rtree=800.0, bond_lim=120.0,
                    bond_lim_rel=0.0, boundary=0)
    f = gen.Field("walls", p, x, y, r, h, 10)
    t = _device_table(f)
    assert len(t) > 0
    _check_against_rule(f, t)
    _check_against_oracle(f, t)


def test_fields_admitted_together_beside_a_resident_one():
    resident = gen.bonded_field(n=500, seed=21, nsteps=10)
    fresh = [gen.bonded_field(n=n, seed=30 + k, nsteps=10) for k, n in enumerate((300, 800, 450))]
    nocoh = gen.lattice_field(n_side=8, periodic=True, nsteps=10)
    b = Batch(PREC_FP64)
    b.add_field(resident)
    b.step(3)
    hs = [b.add_field(f) for f in fresh[:2]] + [b.add_field(nocoh)] + [b.add_field(fresh[2])]
    b.step(2)
    for h_, f in zip(hs, fresh[:2] + [nocoh] + [fresh[2]]):
        alone = Stepper(f.params, f.n, PREC_FP64)
        alone.upload(f.x, f.y, f.r, f.h)
        if f.forcing is not None:
            alone.set_field(f.forcing)
        alone.step(1, 0, 2)
        for k in ("x", "y", "u", "v", "omega"):
            assert np.array_equal(b.field(h_, k).view(np.int64), alone.field(k).view(np.int64)), (f.name, k)
        alone.close()
    b.close()
