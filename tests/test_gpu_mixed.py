"""The mixed-precision path: agreement with the FP64 path (positions,
velocities, per-floe forces, pair topology), and independence of the result
from how a run is cut into calls (diagnostic steps at the end of each call,
CUDA-graph chunks) and from the kernels' block sizes (the autotuner).

The mixed step is deterministic: every force is summed per floe in a fixed
order, so any two ways of running the same steps must agree bit for bit."""
import os

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200.lib import Batch, Stepper
from godar_b200.params import PREC_FP64, PREC_MIXED

from .helpers import STATE, check_mixed_positions, pairset

pytestmark = pytest.mark.gpu


def run(f, precision, chunks, env=None):
    old = {}
    for k, v in (env or {}).items():
        old[k] = os.environ.get(k)
        os.environ[k] = v
    try:
        s = Stepper(f.params, f.n, precision)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    s.upload(f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, bonds=f.bonds, damage=f.damage)
    if f.forcing is not None:
        s.set_field(f.forcing)
    t = 1
    for k in chunks:
        s.step(t, 0, k)
        t += k
    return s


FIELDS = {
    "bonded": lambda: gen.bonded_field(n=400, seed=5, nsteps=200),
    "shelter_ridging": lambda: gen.polydisperse_field(n=500, seed=2, nsteps=200),
}


def run_batch(f, chunks, prepare=False):
    b = Batch(PREC_MIXED)
    h = b.add_field(f)
    for k in chunks:
        if prepare:
            b.prepare(k)
        b.step(k)
    b.sync()
    return b, h


@pytest.mark.parametrize("name", sorted(FIELDS))
def test_mixed_is_independent_of_chunking_graphs_and_blocks(name):
    f = FIELDS[name]()
    a = run(f, PREC_MIXED, [60])
    b = run(f, PREC_MIXED, [7, 13, 1, 39])
    c = run(f, PREC_MIXED, [60], env={"GODAR_BLOCK": "64", "GODAR_GRAPHS": "0"})
    o = run(f, PREC_MIXED, [60], env={"GODAR_OVERLAP_BONDS": "1"})
    # the bond kernel's other variant: records streamed through shared
    # memory by bulk copies
    v1 = run(f, PREC_MIXED, [7, 53], env={"GODAR_BOND_VARIANT": "1"})
    # without diagnostic steps (positions-only callers)
    nd = run(f, PREC_MIXED, [], env=None)
    nd.set_diagnostics(False)
    for t0, k in ((1, 7), (8, 13), (21, 40)):
        nd.step(t0, 0, k)
    # repeated chunk shapes run as captured graphs (from the second use, or
    # at once after prepare)
    d, hd = run_batch(f, [12, 16, 16, 16])
    e, he = run_batch(f, [12, 48], prepare=True)
    assert d.stats()["graph_launches"] > 0 and e.stats()["graph_launches"] > 0
    for k in STATE:
        va = a.field(k).view(np.int64)
        assert np.array_equal(va, b.field(k).view(np.int64)), (k, "chunking")
        assert np.array_equal(va, c.field(k).view(np.int64)), (k, "blocks, no graphs")
        assert np.array_equal(va, o.field(k).view(np.int64)), (k, "bond kernel on a second stream")
        assert np.array_equal(va, v1.field(k).view(np.int64)), (k, "bond tiles by bulk copies")
        assert np.array_equal(va, nd.field(k).view(np.int64)), (k, "no diagnostics")
        assert np.array_equal(va, d.field(hd, k).view(np.int64)), (k, "graphs")
        assert np.array_equal(va, e.field(he, k).view(np.int64)), (k, "prepared graphs")


@pytest.mark.parametrize("name", sorted(FIELDS))
def test_mixed_against_fp64_state_forces_topology(name):
    f = FIELDS[name]()
    chunks = [10, 25, 25, 40]
    s64 = run(f, PREC_FP64, chunks)
    s32 = run(f, PREC_MIXED, chunks)
    # contacts form in the sheltering + ridging field during the run
    check_mixed_positions(f, s32, s64, onsets=(name == "shelter_ridging"))
    for k in ("u", "v"):
        scale = max(np.max(np.abs(s64.field(k))), 1e-6)
        err = np.max(np.abs(s32.field(k) - s64.field(k))) / scale
        assert err <= 1e-3, (k, err)
    # per-floe forces of the last (diagnostic) step, FP32 sums against FP64
    for k in ("tfx", "tfy", "fcx", "fcy", "fbx", "fby"):
        ref = s64.field(k)
        scale = max(np.max(np.abs(ref)), 1.0)
        err = np.max(np.abs(s32.field(k) - ref)) / scale
        assert err <= 1e-3, (k, err)
    for which in (0, 1, 2):
        p64 = s64.pairs(which)
        p32 = s32.pairs(which)
        assert pairset(p64[0], p64[1]) == pairset(p32[0], p32[1]), which
