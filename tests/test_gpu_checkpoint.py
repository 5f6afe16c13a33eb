"""Checkpoint and restart: a field stopped, saved with godar_gpu_checkpoint
and loaded into a new context with godar_gpu_restore continues exactly as if
it had never stopped (bit for bit in both precisions) - floe state, wall
histories, bonds with their strain and damage, and contact histories all
travel."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import GodarError, Stepper
from godar_b200.params import PREC_FP64, PREC_MIXED

from .helpers import STATE, gpu_for

pytestmark = pytest.mark.gpu

FORCES = ["tfx", "tfy", "fcx", "fcy", "fbx", "fby", "m", "mc", "mb"]

FIELDS = {
    "bonded": lambda: gen.bonded_field(n=400, seed=5, nsteps=100),
    "shelter_ridging_wall": lambda: gen.polydisperse_field(n=500, seed=2, nsteps=100),
}


def resumed(f, precision, first, second):
    a = gpu_for(f, precision)
    a.step(1, 0, first)
    data = a.checkpoint()
    c = Stepper(f.params, f.n, precision)
    c.restore(data)
    if f.forcing is not None:
        c.set_field(f.forcing)
    c.step(first + 1, 1, second)
    return c, data


@pytest.mark.parametrize("name", sorted(FIELDS))
def test_fp64_restart_continues_bit_for_bit(name):
    f = FIELDS[name]()
    ref = gpu_for(f, PREC_FP64)
    ref.step(1, 0, 80)
    c, data = resumed(f, PREC_FP64, 40, 40)
    assert len(data) > 0
    for k in STATE + FORCES:
        assert np.array_equal(c.field(k).view(np.int64), ref.field(k).view(np.int64)), k
    rb, cb = ref.pairs(2), c.pairs(2)
    assert sorted(zip(rb[0].tolist(), rb[1].tolist(), rb[2].tolist())) == \
        sorted(zip(cb[0].tolist(), cb[1].tolist(), cb[2].tolist()))
    rc, cc = ref.pairs(1), c.pairs(1)
    assert sorted(zip(rc[0].tolist(), rc[1].tolist())) == sorted(zip(cc[0].tolist(), cc[1].tolist()))


def test_mixed_restart_continues_bit_for_bit():
    f = FIELDS["bonded"]()
    ref = gpu_for(f, PREC_MIXED)
    ref.step(1, 0, 80)
    c, _ = resumed(f, PREC_MIXED, 40, 40)
    # the restore rebuilds the neighbour rows where the uninterrupted run
    # did not; the mixed sums' order does not depend on the rows' build, so
    # the continuation is exact
    for k in STATE:
        assert np.array_equal(c.field(k).view(np.int64), ref.field(k).view(np.int64)), k
    rb, cb = ref.pairs(2), c.pairs(2)
    assert sorted(zip(rb[0].tolist(), rb[1].tolist())) == sorted(zip(cb[0].tolist(), cb[1].tolist()))


def test_checkpoint_is_stable_and_restore_checks_its_input():
    f = FIELDS["bonded"]()
    a = gpu_for(f, PREC_FP64)
    a.step(1, 0, 20)
    d1 = a.checkpoint()
    assert a.checkpoint() == d1
    # a restored field checkpointed again after zero further steps is the same
    c = Stepper(f.params, f.n, PREC_FP64)
    c.restore(d1)
    c.set_field(f.forcing)
    c.step(21, 1, 0)
    assert c.checkpoint() == d1
    bad = Stepper(f.params, f.n + 1, PREC_FP64)
    with pytest.raises(GodarError) as e:
        bad.restore(d1)
    assert e.value.status == 2
    with pytest.raises(GodarError):
        c.restore(b"not a checkpoint" + d1[16:])
    with pytest.raises(GodarError):
        c.restore(d1[:-8])
