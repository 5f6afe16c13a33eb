"""Batches and precision modes on the GPU.

- every instance of a batch evolves exactly as it does alone (FP64: bit for
  bit; the order of floes inside a batch never changes a floe's own sums);
- the mixed-precision path stays within 1e-5 of the FP64 path (positions,
  relative to the largest displacement over the run);
- instances can be removed and added between steps without disturbing the
  others (continuous batching)."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import Batch, Stepper
from godar_b200.params import PREC_FP64, PREC_MIXED

from .helpers import STATE, check_mixed_positions

pytestmark = pytest.mark.gpu


def small_fields():
    return [gen.bonded_field(n=150, seed=3, nsteps=120),
            gen.lattice_field(n_side=8, periodic=True),
            gen.bonded_field(n=220, seed=4, nsteps=120, wind_field=False, wind_dir_deg=33.0)]


def alone(f, nsteps, prec=PREC_FP64):
    s = Stepper(f.params, f.n, prec)
    s.upload(f.x, f.y, f.r, f.h)
    if f.forcing is not None:
        s.set_field(f.forcing)
    s.step(1, 0, nsteps)
    return s


def test_batch_equals_alone_fp64():
    fields = small_fields()
    b = Batch(PREC_FP64)
    hs = [b.add_field(f) for f in fields]
    b.step(60)
    b.step(60)
    for f, hid in zip(fields, hs):
        s = alone(f, 120)
        for k in STATE:
            a = b.field(hid, k)
            ref = s.field(k)
            assert np.array_equal(a.view(np.int64), ref.view(np.int64)), (f.name, k)
        assert b.steps_done(hid) == 120


def test_batch_add_remove_between_steps():
    fields = small_fields()
    b = Batch(PREC_FP64)
    h0 = b.add_field(fields[0])
    h1 = b.add_field(fields[1])
    b.step(40)
    b.remove(h1)
    h2 = b.add_field(fields[2])
    b.step(80)
    s0 = alone(fields[0], 120)
    s2 = alone(fields[2], 80)
    for k in STATE:
        assert np.array_equal(b.field(h0, k).view(np.int64), s0.field(k).view(np.int64)), k
        assert np.array_equal(b.field(h2, k).view(np.int64), s2.field(k).view(np.int64)), k


def test_mixed_precision_within_tolerance():
    f = gen.bonded_field(n=400, seed=5, nsteps=400)
    s64 = alone(f, 400, PREC_FP64)
    s32 = alone(f, 400, PREC_MIXED)
    check_mixed_positions(f, s32, s64)
    for k in ("u", "v"):
        ref = s64.field(k)
        scale = float(np.max(np.abs(ref)))
        assert scale > 0.0
        assert np.max(np.abs(s32.field(k) - ref)) <= 1e-3 * scale, k


def test_async_read_back_matches_sync_reads():
    import torch
    fields = [gen.bonded_field(n=n, seed=20 + k, nsteps=50) for k, n in enumerate((300, 500, 420))]
    b = Batch(PREC_MIXED)
    for f in fields:
        b.add_field(f)
    nf = sum(f.n for f in fields)
    ox = torch.empty(nf, dtype=torch.float64).pin_memory().numpy()
    ov = torch.empty(nf, dtype=torch.float64).pin_memory().numpy()
    for it in range(5):
        b.step(1)
        b.get_all_async(["x", "v"], [ox, ov])
        b.wait()
        rx = np.empty(nf)
        rv = np.empty(nf)
        b.get_all("x", rx)
        b.get_all("v", rv)
        assert np.array_equal(ox.view(np.int64), rx.view(np.int64)), it
        assert np.array_equal(ov.view(np.int64), rv.view(np.int64)), it
    # a read-back left pending while the next steps run still lands intact
    b.step(1)
    b.get_all_async(["x"], [ox])
    b.step(1)
    b.step(3)
    b.wait()
    b2 = Batch(PREC_MIXED)
    for f in fields:
        b2.add_field(f)
    for k in (1, 1, 1, 1, 1, 1):
        b2.step(k)
    ref = np.empty(nf)
    b2.get_all("x", ref)
    assert np.array_equal(ox.view(np.int64), ref.view(np.int64))


def test_reserved_pool_and_repeated_relayouts_stay_exact():
    """A batch whose memory pool was grown ahead of time and whose membership
    changes many times (each change re-lays every buffer out, reusing the
    previous layout's memory) still steps every field exactly as alone."""
    fields = small_fields()
    b = Batch(PREC_FP64)
    b.reserve(256 << 20)
    h = [b.add_field(f) for f in fields]
    extra = gen.bonded_field(n=180, seed=9, nsteps=120)
    for r in range(6):
        he = b.add_field(extra)
        b.step(10)
        b.remove(he)
        b.step(10)
    for f, hid in zip(fields, h):
        s = alone(f, 120)
        for k in STATE:
            assert np.array_equal(b.field(hid, k).view(np.int64), s.field(k).view(np.int64)), (f.name, k)


def test_pipelined_read_backs_of_consecutive_steps():
    """Read-backs of consecutive steps into alternating buffers, two in
    flight: each call's buffers hold that step's state once the next call
    has returned."""
    import torch
    fields = [gen.bonded_field(n=n, seed=40 + k, nsteps=50) for k, n in enumerate((350, 280))]
    b, ref = Batch(PREC_MIXED), Batch(PREC_MIXED)
    for f in fields:
        b.add_field(f)
        ref.add_field(f)
    nf = sum(f.n for f in fields)
    bufs = [[torch.empty(nf, dtype=torch.float64).pin_memory().numpy() for _ in range(2)] for _ in range(2)]
    expect = []
    for k in range(8):
        b.step(1)
        b.get_all_async(["x", "u"], bufs[k & 1])
        ref.step(1)
        ex, eu = np.empty(nf), np.empty(nf)
        ref.get_all("x", ex)
        ref.get_all("u", eu)
        expect.append((ex, eu))
        if k > 0:
            px, pu = bufs[(k - 1) & 1]
            assert np.array_equal(px.view(np.int64), expect[k - 1][0].view(np.int64)), k
            assert np.array_equal(pu.view(np.int64), expect[k - 1][1].view(np.int64)), k
    b.wait()
    lx, lu = bufs[7 & 1]
    assert np.array_equal(lx.view(np.int64), expect[7][0].view(np.int64))
    assert np.array_equal(lu.view(np.int64), expect[7][1].view(np.int64))


def test_instance_summary_matches_the_fields():
    """godar_batch_summary_async: per instance the momentum, kinetic energy
    and largest speed of the current state, equal (to rounding of the sum
    order) to the same sums over the fields read back; the same bits for the
    same state and memory order (no rebuild since admission here), whatever
    else the batch holds."""
    fields = [gen.bonded_field(n=n, seed=40 + k, nsteps=30) for k, n in enumerate((260, 510, 380))]
    b = Batch(PREC_MIXED)
    hs = [b.add_field(f) for f in fields]
    b.step(25)
    s = b.summary()
    assert s.shape == (3, 4)
    for k, (h, f) in enumerate(zip(hs, fields)):
        u, v, om = b.field(h, "u"), b.field(h, "v"), b.field(h, "omega")
        r, hh = b.field(h, "r"), b.field(h, "h")
        m = ((f.params.rhoice * f.params.pi) * hh) * (r * r)
        inert = (0.5 * m) * (r * r)
        want = np.array([np.sum(m * u), np.sum(m * v),
                         np.sum(0.5 * m * (u * u + v * v) + 0.5 * inert * om * om),
                         np.max(np.hypot(u, v))])
        scale = np.array([np.sum(np.abs(m * u)), np.sum(np.abs(m * v)), want[2], want[3]])
        assert np.all(np.abs(s[k] - want) <= 1e-12 * scale + 1e-300), (k, s[k], want)
        assert s[k, 2] > 0.0 and s[k, 3] > 0.0
    # the same field alone: the same bits
    alone = Batch(PREC_MIXED)
    ha = alone.add_field(fields[1])
    alone.step(25)
    assert np.array_equal(alone.summary()[0].view(np.int64), s[1].view(np.int64))
    alone.close()
    b.close()
