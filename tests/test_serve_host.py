"""Host logic of the serving loop (godar_b200/serve.py) over a fake batch on
the CPU: admission against the HBM budget, waiting requests joining as
fields retire, chunks cut at the first completion, results read before the
field is removed, and errors other than the budget raised to the caller."""
from types import SimpleNamespace

import numpy as np
import pytest

from godar_b200 import serve
from godar_b200.lib import GodarError

BYTES_PER_FLOE = 1000


class FakeBatch:
    """Stands in for godar_b200.lib.Batch: a field of n floes costs
    n * BYTES_PER_FLOE bytes of the budget; godar_batch_add's budget refusal
    is status 8."""

    instances = []

    def __init__(self, precision, budget):
        self.budget = budget
        self.used = 0
        self.fields = {}          # hid -> [n, steps done, tag]
        self.next_hid = 0
        self.steps = []           # nsteps of every step call
        self.resident = []        # resident hids at every step call
        self.reads = []           # (hid, name) in order
        self.removed = []
        self.log = []             # reads and removals in call order
        self.reserved = None
        self.closed = False
        FakeBatch.instances.append(self)

    def reserve(self, nbytes):
        self.reserved = nbytes

    def add_field(self, fld):
        cost = fld.n * BYTES_PER_FLOE
        if fld.n == 0:
            raise GodarError(2, "empty field")
        if self.used + cost > self.budget:
            raise GodarError(serve.GODAR_ERR_BUDGET, "over budget")
        hid = self.next_hid
        self.next_hid += 1
        self.used += cost
        self.fields[hid] = [fld.n, 0, fld.tag]
        return hid

    def step(self, k):
        self.steps.append(k)
        self.resident.append(sorted(self.fields))
        for v in self.fields.values():
            v[1] += k

    def sync(self):
        return 0.5

    def field(self, hid, name):
        self.reads.append((hid, name))
        self.log.append(("read", hid))
        n, done, tag = self.fields[hid]
        return np.full(n, float(done * 1000 + tag))

    def remove(self, hid):
        self.log.append(("remove", hid))
        n = self.fields.pop(hid)[0]
        self.used -= n * BYTES_PER_FLOE
        self.removed.append(hid)

    def close(self):
        self.closed = True


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.instances.clear()
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    return FakeBatch


def _req(rid, n, nsteps, arrival=0.0):
    return serve.Request(rid=rid, arrival=arrival, fld=SimpleNamespace(n=n, tag=rid), nsteps=nsteps)


def test_every_request_completes_with_its_own_step_count(fake):
    reqs = [_req(0, 10, 120), _req(1, 20, 50), _req(2, 5, 75), _req(3, 7, 200)]
    st = serve.serve(reqs, hbm_budget=10**9, chunk=50, realtime=False, reserve=0)
    b = fake.instances[0]
    assert st.completed == 4 and b.closed and not b.fields
    for rq in reqs:
        # each field's result was read after exactly its own number of steps
        assert np.all(rq.result["x"] == rq.nsteps * 1000 + rq.rid)
        assert rq.done >= rq.admitted >= 0.0
    # chunks never exceed `chunk` and stop at the first field to finish
    assert max(b.steps) <= 50 and sum(b.steps) == 200
    assert b.steps == [50, 25, 45, 50, 30]
    assert st.floe_steps == sum(r.n * r.nsteps for r in reqs)
    assert st.gpu_ms == pytest.approx(0.5 * len(b.steps))
    assert st.max_resident == 4


def test_budget_holds_requests_until_fields_retire(fake):
    # budget for 30 floes: requests of 20, 20 and 10 floes
    reqs = [_req(0, 20, 100), _req(1, 20, 40), _req(2, 10, 40)]
    st = serve.serve(reqs, hbm_budget=30 * BYTES_PER_FLOE, chunk=100, realtime=False, reserve=0)
    b = fake.instances[0]
    assert st.completed == 3
    # request 1 waits behind request 0 (first come, first served: request 2
    # does not overtake it), and joins once request 0 has retired
    assert b.resident[0] == [0]
    assert b.removed[0] == 0
    assert all(0 not in r for r in b.resident[1:])
    assert b.used == 0 and st.max_resident == 2
    for rq in reqs:
        assert np.all(rq.result["x"] == rq.nsteps * 1000 + rq.rid)


def test_results_are_read_before_any_field_of_the_chunk_is_removed(fake):
    reqs = [_req(0, 4, 30), _req(1, 4, 30), _req(2, 4, 60)]
    serve.serve(reqs, hbm_budget=10**9, chunk=100, realtime=False, reserve=0, keep=("x", "y"))
    b = fake.instances[0]
    assert b.removed[:2] == [0, 1]
    # both finished fields' reads come before the first removal of the chunk
    assert b.log[:6] == [("read", 0), ("read", 0), ("read", 1), ("read", 1), ("remove", 0), ("remove", 1)]
    assert b.reads[:4] == [(0, "x"), (0, "y"), (1, "x"), (1, "y")]


def test_reserve_is_capped_by_the_budget(fake):
    serve.serve([_req(0, 3, 10)], hbm_budget=5 << 20, realtime=False, reserve=16 << 30)
    assert fake.instances[0].reserved == 5 << 20


def test_a_request_larger_than_the_whole_budget_is_an_error(fake):
    reqs = [_req(0, 50, 10)]
    with pytest.raises(GodarError) as e:
        serve.serve(reqs, hbm_budget=10 * BYTES_PER_FLOE, realtime=False, reserve=0)
    assert e.value.status == serve.GODAR_ERR_BUDGET
    assert fake.instances[0].closed


def test_errors_other_than_the_budget_are_raised(fake):
    reqs = [_req(0, 10, 10), _req(1, 0, 10)]
    with pytest.raises(GodarError) as e:
        serve.serve(reqs, hbm_budget=10**9, realtime=False, reserve=0)
    assert e.value.status == 2
    # the batch is closed on the error path too
    assert fake.instances[0].closed


def test_on_complete_sees_every_request_once(fake):
    seen = []
    reqs = [_req(k, 3 + k, 10 * (k + 1)) for k in range(6)]
    st = serve.serve(reqs, hbm_budget=10**9, realtime=False, reserve=0, on_complete=lambda r: seen.append(r.rid))
    assert sorted(seen) == list(range(6)) and st.completed == 6
    # shorter requests finish first
    assert seen == list(range(6))
