"""Served request stream on the GPU: results are the same alone and in the
mix, bit for bit in both precisions (every per-floe sum runs in an order set
by the reference ids alone, so neither the other fields of the batch nor the
times at which the batch rebuilt its neighbour rows change a field's
result), the HBM budget bounds how many fields are resident, and fields that
leave the batch do not disturb the others."""
import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import Batch, Stepper
from godar_b200.params import PREC_FP64, PREC_MIXED
from godar_b200.serve import Request, serve

pytestmark = pytest.mark.gpu


def stream(nsteps=60, sizes=(300, 700, 220, 500, 410, 260)):
    out = []
    for k, n in enumerate(sizes):
        f = gen.bonded_field(n=n, seed=100 + k, nsteps=nsteps, wind_field=(k % 2 == 0),
                        wind_dir_deg=40.0 * k, wind_speed=9.0 + k)
        out.append(Request(rid=k, arrival=0.01 * k, fld=f, nsteps=nsteps - 7 * (k % 3)))
    return out


def alone(f, nsteps, prec):
    s = Stepper(f.params, f.n, prec)
    s.upload(f.x, f.y, f.r, f.h)
    if f.forcing is not None:
        s.set_field(f.forcing)
    s.step(1, 0, nsteps)
    return s.field("x"), s.field("y")


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_served_equals_alone(prec):
    reqs = stream()
    st = serve(reqs, precision=prec, chunk=16, realtime=False)
    assert st.completed == len(reqs)
    for rq in reqs:
        x, y = alone(rq.fld, rq.nsteps, prec)
        assert np.array_equal(rq.result["x"].view(np.int64), x.view(np.int64)), rq.rid
        assert np.array_equal(rq.result["y"].view(np.int64), y.view(np.int64)), rq.rid


def test_budget_bounds_resident_fields():
    reqs = stream(nsteps=30, sizes=(400,) * 6)
    per = Batch.instance_bytes(400, 4 * 400)     # FP64 estimate of a fresh bonded field
    st = serve(reqs, precision=PREC_FP64, hbm_budget=int(2.2 * per), chunk=10, realtime=False)
    assert st.completed == len(reqs)
    assert st.max_resident <= 2


def test_removing_the_first_field_keeps_the_rest_exact():
    fs = [gen.bonded_field(n=n, seed=200 + k, nsteps=90) for k, n in enumerate((260, 340, 180))]
    b = Batch(PREC_FP64)
    h = [b.add_field(f) for f in fs]
    b.step(30)
    b.remove(h[0])
    b.step(60)
    for k in (1, 2):
        x, y = alone(fs[k], 90, PREC_FP64)
        assert np.array_equal(b.field(h[k], "x").view(np.int64), x.view(np.int64))
        assert np.array_equal(b.field(h[k], "y").view(np.int64), y.view(np.int64))
