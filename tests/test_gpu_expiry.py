"""A step that raises the neighbour-list expiry is kept, so every floe must be
updated in it: the floe-update kernel stops only on an expiry raised at an
earlier step, not on one raised by another block of its own launch.

The candidate set is decided by the exact FP64 test every step and every sum
runs in an order set by reference ids, so no result depends on the Verlet
skin, that is on when the rows are rebuilt.  A field of 300,000 floes (far
more blocks than fit on the GPU at once, so blocks of the floe update start
after others have finished) moving at 2 m/s is run with a 1 m skin (a
rebuild every few steps) and with a skin that never expires in the window;
both runs must end in the same bits."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.params import PREC_FP64, PREC_MIXED

pytestmark = pytest.mark.gpu

NAMES = ["x", "y", "u", "v", "r", "h", "theta", "omega"]
STEPS = 40


@pytest.fixture(scope="module")
def field():
    f = gen.bonded_field(n=300000, seed=7, device="gpu")
    rng = np.random.default_rng(8)
    ang = rng.uniform(0.0, 2.0 * np.pi, f.n)
    f.u = 2.0 * np.cos(ang)
    f.v = 2.0 * np.sin(ang)
    return f


def _run(f, precision, skin_frac, monkeypatch):
    from godar_b200.lib import Batch
    monkeypatch.setenv("GODAR_SKIN_FRAC", skin_frac)
    b = Batch(precision)
    try:
        h = b.add_field(f)
        b.step(STEPS)
        out = {k: b.field(h, k) for k in NAMES}
        rebuilds = b.stats()["rebuilds"]
    finally:
        b.close()
    return out, rebuilds


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_expiring_steps_update_every_floe(field, precision, monkeypatch):
    tight, rb_tight = _run(field, precision, "0", monkeypatch)
    wide, rb_wide = _run(field, precision, "0.05", monkeypatch)
    print(f"rebuilds: 1 m skin {rb_tight}, 300 m skin {rb_wide}")
    assert rb_tight >= rb_wide + 4
    moved = np.max(np.hypot(tight["x"] - field.x, tight["y"] - field.y))
    assert moved > 2.0
    for k in NAMES:
        assert np.isfinite(tight[k]).all(), k
        assert np.array_equal(tight[k].view(np.int64), wide[k].view(np.int64)), k
