"""godar_batch_set_phase_timing: which steps of godar_batch_step are timed
kernel by kernel with CUDA events (none by default, every step with an
interval of 1, some with a larger interval), and timing changes no result."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.params import PREC_FP64, PREC_MIXED

pytestmark = pytest.mark.gpu

NAMES = ["x", "y", "u", "v", "omega"]


def _run(precision, every, monkeypatch):
    from godar_b200.lib import Batch
    monkeypatch.setenv("GODAR_TUNE", "0")
    b = Batch(precision)
    try:
        hs = [b.add_field(gen.bonded_field(n=n, seed=40 + n, nsteps=100)) for n in (1500, 600)]
        b.step(4)
        b.set_phase_timing(every)
        s0 = b.stats()
        b.step(64)
        s1 = b.stats()
        out = {h: {k: b.field(h, k) for k in NAMES} for h in hs}
    finally:
        b.close()
    timed = s1["timed_steps"] - s0["timed_steps"]
    steps = s1["launches"] - s0["launches"]
    phase = [a - c for a, c in zip(s1["phase_ms"], s0["phase_ms"])]
    return out, timed, steps, phase


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_phase_timing_counts_its_steps_and_changes_no_result(precision, monkeypatch):
    ref, t0, n0, p0 = _run(precision, 0, monkeypatch)
    assert n0 == 64 and t0 == 0 and all(p == 0.0 for p in p0)
    for every in (1, 8):
        out, t, n, p = _run(precision, every, monkeypatch)
        assert n == 64
        if every == 1:
            assert t == 64
        else:
            assert 64 // every <= t < 64
        assert all(x > 0.0 for x in p), p
        for h in ref:
            for k in NAMES:
                assert np.array_equal(ref[h][k].view(np.int64), out[h][k].view(np.int64)), (every, h, k)
