"""godar_batch_step_async: steps queued without waiting give the results of
godar_batch_step bit for bit - through neighbour-list expiries (the steps
queued behind an expiring one do nothing and are run again after the
rebuild) and with a uniform forcing that changes every call - and the
summaries read back after queued steps are those of the synchronous run
(to 1e-12: a summary sums over the floes' memory order, which a rebuild
changes, and a queued run reads a summary before it learns of the expiry
that the synchronous run rebuilt after at once).  An error raised by a
queued step is returned by a later call.  The single-field context's
godar_gpu_step_async, called one step at a time as the replacement stepper
calls it, gives the outputs of godar_gpu_step bit for bit."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import GodarError
from godar_b200.params import PREC_FP64, PREC_MIXED

from .helpers import gpu_for

pytestmark = pytest.mark.gpu

NAMES = ["x", "y", "u", "v", "r", "h", "theta", "omega"]
GODAR_ERR_NAN = 4
# one-step calls (the pipelined case), then calls of several steps
CALLS = [1] * 40 + [3, 1, 5, 2, 1, 8, 1, 1, 4, 1]


def _fields():
    out = []
    for k, n in enumerate((3000, 1200, 700)):
        f = gen.bonded_field(n=n, seed=60 + k, nsteps=100, wind_field=False, wind_dir_deg=30.0 * k)
        rng = np.random.default_rng(70 + k)
        ang = rng.uniform(0.0, 2.0 * np.pi, f.n)
        f.u = 2.0 * np.cos(ang)
        f.v = 2.0 * np.sin(ang)
        out.append(f)
    return out


def _forcing(k, ni):
    a = np.deg2rad(10.0 * k)
    uvw = np.zeros(4 * ni)
    for i in range(ni):
        uvw[4 * i:4 * i + 4] = (12.0 * np.cos(a + i), 12.0 * np.sin(a + i), 0.1 * np.cos(a), 0.1 * np.sin(a))
    return uvw


def _run(fields, precision, queued, monkeypatch):
    import torch
    from godar_b200.lib import Batch
    # a 1 m Verlet skin: at 2 m/s the neighbour list expires every few steps
    monkeypatch.setenv("GODAR_SKIN_FRAC", "0")
    b = Batch(precision)
    try:
        hids = [b.add_field(f) for f in fields]
        b.step(20)   # the autotuner's steps run synchronously either way
        ni = len(fields)
        bufs = [torch.empty(4 * ni, dtype=torch.float64).pin_memory().numpy() for _ in range(2)]
        sums = []
        for k, n in enumerate(CALLS):
            b.set_uniform_forcing(_forcing(k, ni))
            if queued:
                b.step_async(n)
            else:
                b.step(n)
            b.summary_async(bufs[k & 1])
            if k > 0:
                sums.append(bufs[(k - 1) & 1].copy())
        b.wait()
        sums.append(bufs[(len(CALLS) - 1) & 1].copy())
        state = {h: {k: b.field(h, k) for k in NAMES} for h in hids}
        rebuilds = b.stats()["rebuilds"]
    finally:
        b.close()
    return state, sums, rebuilds


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_queued_steps_equal_synchronous_steps(precision, monkeypatch):
    fields = _fields()
    a, sa, ra = _run(fields, precision, False, monkeypatch)
    q, sq, rq = _run(fields, precision, True, monkeypatch)
    print(f"rebuilds: synchronous {ra}, queued {rq}")
    assert ra == rq and ra >= 5
    for h in a:
        for k in NAMES:
            assert np.isfinite(a[h][k]).all(), (h, k)
            assert np.array_equal(a[h][k].view(np.int64), q[h][k].view(np.int64)), (h, k)
    assert len(sa) == len(sq) == len(CALLS)
    for i, (s1, s2) in enumerate(zip(sa, sq)):
        s1, s2 = s1.reshape(-1, 4), s2.reshape(-1, 4)
        scale = np.max(np.abs(s1), axis=0)
        assert np.all(np.abs(s1 - s2) <= 1e-12 * scale), i
        assert np.array_equal(s1[:, 3], s2[:, 3]), i   # the largest speed: order-free


def test_error_of_a_queued_step_is_returned_by_a_later_call(monkeypatch):
    """The bonded field at dt = 0.5 s blows up within about 20 steps."""
    from godar_b200.lib import Batch
    monkeypatch.setenv("GODAR_TUNE", "0")
    f = gen.bonded_field(n=400, seed=5, nsteps=60, dt=0.5)
    b = Batch(PREC_MIXED)
    try:
        b.add_field(f)
        b.step(1)
        with pytest.raises(GodarError) as e:
            for _ in range(60):
                b.step_async(1)
            b.wait()
        assert e.value.status == GODAR_ERR_NAN
    finally:
        b.close()


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_admission_and_removal_between_queued_steps(precision, monkeypatch):
    """A field admitted while steps are queued (the forcing upload that
    follows commits the new layout) and one removed later: the queued steps
    are read before the relayout, and every field ends as with synchronous
    calls."""
    from godar_b200.lib import Batch
    monkeypatch.setenv("GODAR_SKIN_FRAC", "0")
    base = _fields()
    extra = gen.bonded_field(n=900, seed=66, nsteps=100, wind_field=False, wind_dir_deg=75.0)

    def run(queued):
        b = Batch(precision)
        try:
            hids = [b.add_field(f) for f in base[:2]]
            b.step(20)
            count = 2
            for k in range(36):
                if k == 8:
                    hids.append(b.add_field(extra))
                    count += 1
                if k == 24:
                    b.remove(hids.pop(0))
                    count -= 1
                b.set_uniform_forcing(_forcing(k, count))
                if queued:
                    b.step_async(1)
                else:
                    b.step(1)
            b.wait()
            out = {i: {k: b.field(h, k) for k in NAMES} for i, h in enumerate(hids)}
            return out, b.stats()["rebuilds"]
        finally:
            b.close()

    a, ra = run(False)
    q, rq = run(True)
    print(f"rebuilds: synchronous {ra}, queued {rq}")
    assert ra == rq
    for i in a:
        for k in NAMES:
            assert np.array_equal(a[i][k].view(np.int64), q[i][k].view(np.int64)), (i, k)


FIELDS_OUT = ["x", "y", "u", "v", "r", "h", "theta", "omega", "tfx", "tfy", "fcx", "fcy", "fbx", "fby",
              "m", "mc", "mb", "tsigxx", "tsigyy", "tsigxy", "tsigyx", "tp"]


def _shim_run(f, precision, queued, monkeypatch, steps=100, comp=7):
    """The replacement stepper's pattern: one step a call, diagnostics on
    output steps only, every output and the bond and contact lists read
    back on output steps."""
    from godar_b200.lib import Stepper
    monkeypatch.setenv("GODAR_SKIN_FRAC", "0")
    s = Stepper(f.params, f.n, precision)
    s.upload(f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, bonds=f.bonds, damage=f.damage)
    if f.forcing is not None:
        s.set_field(f.forcing)
    outs = []
    for t in range(1, steps + 1):
        out = t % comp == 0 or t == 1
        s.set_diagnostics(out)
        if queued:
            s.step_async(t, 0, 1)
        else:
            s.step(t, 0, 1)
        if out:
            fl, bonds = s.download(FIELDS_OUT, which=2)
            contacts = s.pairs(1)
            outs.append((t, fl, bonds, contacts))
    final = s.floes()
    s.close()
    return outs, final


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_queued_single_field_steps_equal_synchronous_steps(precision, monkeypatch):
    """godar_gpu_step_async one step a call, as the replacement stepper calls
    it, through neighbour-list expiries (a 1 m skin at 2 m/s): every output
    step's floe outputs, bond and contact lists, and the final state equal
    those of godar_gpu_step bit for bit."""
    f = _fields()[0]
    a, fa = _shim_run(f, precision, False, monkeypatch)
    q, fq = _shim_run(f, precision, True, monkeypatch)
    moved = np.max(np.hypot(fa["x"] - f.x, fa["y"] - f.y))
    assert moved > 5.0   # many times the 1 m skin: the rows were rebuilt often
    assert len(a) == len(q)
    for (t, fl1, b1, c1), (_, fl2, b2, c2) in zip(a, q):
        for k in FIELDS_OUT:
            assert np.isfinite(fl1[k]).all(), (t, k)
            assert np.array_equal(fl1[k].view(np.int64), fl2[k].view(np.int64)), (t, k)
        for l1, l2 in ((b1, b2), (c1, c2)):
            for x1, x2 in zip(l1, l2):
                assert np.array_equal(x1, x2), t
    for k in fa:
        assert np.array_equal(fa[k].view(np.int64), fq[k].view(np.int64)), k


def test_error_of_a_queued_single_field_step_is_returned_by_a_later_call():
    f = gen.bonded_field(n=400, seed=5, nsteps=60, dt=0.5)
    s = gpu_for(f, PREC_MIXED)
    with pytest.raises(GodarError) as e:
        for t in range(1, 61):
            s.step_async(t, 0, 1)
        s.field("x")
    assert e.value.status == GODAR_ERR_NAN
