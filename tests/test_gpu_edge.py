"""Edge cases of the device path: a single floe, floes out of each other's
reach, rejected inputs, and restart bonds given by the caller (as ini_get
reads them, ini_get.f90:129-130)."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import GodarError, Stepper
from godar_b200.params import BC_PERIODIC_X, BC_PERIODIC_Y, PREC_FP64, PREC_MIXED, make_params
from oracle import pyoracle as po

from .helpers import DIAG, STATE, check_mixed_positions, gpu_for

pytestmark = pytest.mark.gpu

GODAR_ERR_BAD_INPUT = 2
GODAR_ERR_NAN = 4


def field_of(x, y, r, h, periodic=False, u=None, v=None, **kw):
    L = 1e5
    opts = dict(cohesion=0, shelter=0, ridging=0, dt=0.05, rtree=1000.0, lat=0.0,
                boundary=(BC_PERIODIC_X | BC_PERIODIC_Y) if periodic else 0)
    opts.update(kw)
    p = make_params(L, L, **opts)
    n = len(x)
    return gen.Field("edge", p, np.asarray(x, float), np.asarray(y, float), np.asarray(r, float),
                     np.asarray(h, float), 100,
                     u=np.zeros(n) if u is None else np.asarray(u, float),
                     v=np.zeros(n) if v is None else np.asarray(v, float))


def run_pair(f, steps, precision, restart=0):
    o = po.Oracle(f.params, f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, bonds=f.bonds, damage=f.damage)
    g = Stepper(f.params, f.n, precision)
    g.upload(f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, bonds=f.bonds, damage=f.damage)
    o.step(steps, restart=restart)
    g.step(1, restart, steps)
    return o, g


@pytest.mark.parametrize("periodic", [False, True])
def test_single_floe_bit_exact(periodic):
    f = field_of([50000.0], [50000.0], [800.0], [1.2], periodic=periodic, u=[0.3], v=[-0.1])
    o, g = run_pair(f, 200, PREC_FP64)
    of = o.floes()
    for k in STATE + DIAG:
        assert np.array_equal(g.field(k).view(np.int64), of[k].view(np.int64)), k
    assert len(g.pairs(0)[0]) == 0


def test_single_floe_mixed_close_to_fp64():
    f = field_of([50000.0], [50000.0], [800.0], [1.2], u=[0.3], v=[-0.1])
    _, g64 = run_pair(f, 200, PREC_FP64)
    g32 = Stepper(f.params, 1, PREC_MIXED)
    g32.upload(f.x, f.y, f.r, f.h, u=f.u, v=f.v)
    g32.step(1, 0, 200)
    _, moved, _ = check_mixed_positions(f, g32, g64)
    assert moved > 1.0


def test_out_of_reach_floes_have_no_pairs():
    # centres 20 km apart, radii 1 km, rtree 1 km: no candidate pair
    x = [20000.0, 40000.0, 60000.0, 80000.0]
    f = field_of(x, [50000.0] * 4, [1000.0] * 4, [1.0] * 4)
    o, g = run_pair(f, 100, PREC_FP64)
    of = o.floes()
    for k in STATE:
        assert np.array_equal(g.field(k).view(np.int64), of[k].view(np.int64)), k
    for which in (0, 1, 2):
        assert len(g.pairs(which)[0]) == 0


@pytest.mark.parametrize("bad", ["nan_x", "zero_r", "negative_h", "bond_index"])
def test_bad_inputs_are_rejected(bad):
    x = np.array([40000.0, 42500.0])
    y = np.array([50000.0, 50000.0])
    r = np.array([1000.0, 1000.0])
    h = np.array([1.0, 1.0])
    bonds = None
    if bad == "nan_x":
        x[1] = np.nan
    elif bad == "zero_r":
        r[0] = 0.0
    elif bad == "negative_h":
        h[1] = -1.0
    else:
        bonds = np.array([[0, 5]])
    f = field_of(x, y, r, h)
    g = Stepper(f.params, 2, PREC_FP64)
    with pytest.raises(GodarError) as e:
        g.upload(x, y, r, h, bonds=bonds)
    assert e.value.status == GODAR_ERR_BAD_INPUT


def test_periodic_domain_smaller_than_the_search_radius_is_rejected():
    # 2 (r_max + rtree + skin) = 2 (400 + 1000 + 14) m > 2500 m
    p = make_params(2500.0, 2500.0, cohesion=0, shelter=0, ridging=0, dt=0.05, rtree=1000.0, lat=0.0,
                    boundary=BC_PERIODIC_X | BC_PERIODIC_Y)
    g = Stepper(p, 2, PREC_FP64)
    g.upload(np.array([500.0, 2000.0]), np.array([500.0, 500.0]), np.array([400.0, 400.0]), np.ones(2))
    # the field is checked when it is admitted, at its first step
    with pytest.raises(GodarError) as e:
        g.step(1, 0, 1)
    assert e.value.status == GODAR_ERR_BAD_INPUT


def test_restart_bonds_given_by_the_caller_bit_exact():
    # a chain of four touching floes bonded explicitly, with damage carried in
    x = [40000.0, 41990.0, 43980.0, 45970.0]
    f = field_of(x, [50000.0] * 4, [1000.0] * 4, [1.0, 1.2, 0.9, 1.1], u=[0.2, 0.0, 0.0, -0.2],
                 cohesion=1)
    f.bonds = np.array([[0, 1], [1, 2], [2, 3]], dtype=np.int32)
    f.damage = np.array([0.0, 0.25, 0.5])
    o, g = run_pair(f, 300, PREC_FP64, restart=1)
    of = o.floes()
    for k in STATE + DIAG:
        assert np.array_equal(g.field(k).view(np.int64), of[k].view(np.int64)), k
    gb = g.pairs(2)
    ob = o.pairs(2)
    assert sorted(zip(gb[0].tolist(), gb[1].tolist())) == sorted(zip(ob[0].tolist(), ob[1].tolist()))
    assert np.array_equal(np.sort(gb[2]).view(np.int64), np.sort(ob[2]).view(np.int64))


def test_download_matches_the_single_field_calls():
    f = gen.bonded_field(n=300, seed=7, nsteps=50)
    g = gpu_for(f, PREC_FP64)
    g.step(1, 0, 30)
    outs, pairs = g.download(which=2)
    for k, a in outs.items():
        assert np.array_equal(a.view(np.int64), g.field(k).view(np.int64)), k
    ref = g.pairs(2)
    for a, b in zip(pairs, ref):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    outs2, none = g.download(names=["x", "tfx"])
    assert none is None and set(outs2) == {"x", "tfx"}


def test_set_precision_before_the_first_step_only():
    f = gen.bonded_field(n=300, seed=7, nsteps=50)
    a = gpu_for(f, PREC_FP64)
    a.set_precision(PREC_MIXED)
    a.step(1, 0, 40)
    b = gpu_for(f, PREC_MIXED)
    b.step(1, 0, 40)
    for k in STATE:
        assert np.array_equal(a.field(k).view(np.int64), b.field(k).view(np.int64)), k
    with pytest.raises(GodarError) as e:
        a.set_precision(PREC_FP64)
    assert e.value.status == 7


def test_fp64_without_diagnostics_still_bit_exact():
    f = gen.bonded_field(n=300, seed=9, nsteps=60)
    o = po.Oracle(f.params, f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, field=f.forcing)
    g = gpu_for(f, PREC_FP64)
    g.set_diagnostics(False)
    t = 1
    for k in (5, 17, 38):
        g.step(t, 0, k)
        t += k
    o.step(60)
    of = o.floes()
    for k in STATE:
        assert np.array_equal(g.field(k).view(np.int64), of[k].view(np.int64)), k


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_unstable_step_returns_nan_status(precision):
    """The bonded field at the benchmark's stated dt = 0.5 s blows up (the
    explicit beam dashpots are unstable there; the oracle's velocities
    overflow within 20 steps, test_dt_stability.py): the step call reports
    GODAR_ERR_NAN instead of returning non-finite state as a result."""
    f = gen.bonded_field(n=400, seed=5, nsteps=60, dt=0.5)
    g = gpu_for(f, precision)
    with pytest.raises(GodarError) as e:
        g.step(1, 0, 60)
    assert e.value.status == GODAR_ERR_NAN
    g.close()


GODAR_ERR_TIMEOUT = 5


def test_device_wait_that_runs_out_returns_timeout(monkeypatch):
    """Every wait of the step kernels is bounded.  With the test seam
    GODAR_TEST_WAIT_SPINS the bulk-copy bond kernel first waits a few tries
    on a barrier that nothing completes: the wait gives up, the kernel
    reports ST_TIMEOUT and returns, and the step call reports
    GODAR_ERR_TIMEOUT instead of hanging; the device stays usable (the same
    field then steps in a fresh context)."""
    f = gen.bonded_field(n=300, seed=5, nsteps=10)
    monkeypatch.setenv("GODAR_BOND_VARIANT", "1")
    monkeypatch.setenv("GODAR_TEST_WAIT_SPINS", "2000")
    s = gpu_for(f, PREC_MIXED)
    monkeypatch.delenv("GODAR_TEST_WAIT_SPINS")
    with pytest.raises(GodarError) as e:
        s.step(1, 0, 5)
    assert e.value.status == GODAR_ERR_TIMEOUT
    s.close()
    g = gpu_for(f, PREC_MIXED)
    g.step(1, 0, 5)
    assert np.all(np.isfinite(g.field("x")))
    g.close()
