"""Committed regression fixtures (tests/golden/, made by make_golden.py with
the oracle): the oracle must still reproduce them bit for bit, and so must
the FP64 GPU path through the C ABI."""
import glob
import json
import os

import numpy as np
import pytest

from godar_b200.params import GodarParams
from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
STATE = ["x", "y", "u", "v", "r", "h", "theta", "omega"]
DIAG = ["tfx", "tfy", "fcx", "fcy", "fbx", "fby", "m", "mc", "mb", "tsigxx", "tsigyy", "tsigxy",
        "tsigyx", "tp"]


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    p = GodarParams()
    for k, v in meta["params"].items():
        setattr(p, k, v)
    return z, meta, p


def inputs(z):
    g = lambda k: z[k] if k in z.files else None
    return g("in_x"), g("in_y"), g("in_r"), g("in_h"), g("in_u"), g("in_v"), g("forcing")


def same(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def test_oracle_reproduces_fixture(path):
    z, meta, p = load(path)
    x, y, r, h, u, v, fld = inputs(z)
    o = po.Oracle(p, x, y, r, h, u=u, v=v, field=fld)
    o.step(meta["nsteps"])
    out = o.floes()
    for k in STATE + DIAG:
        assert same(out[k], z["out_" + k]), k
    ci, cj, _ = o.pairs(po.P_CANDIDATES)
    assert np.array_equal(ci, z["cand_i"]) and np.array_equal(cj, z["cand_j"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def test_gpu_reproduces_fixture(path):
    from godar_b200.lib import Stepper, P_BONDS, P_CANDIDATES
    z, meta, p = load(path)
    x, y, r, h, u, v, fld = inputs(z)
    s = Stepper(p, len(x))
    s.upload(x, y, r, h, u=u, v=v)
    if fld is not None:
        s.set_field(fld)
    s.step(1, 0, meta["nsteps"])
    for k in STATE + DIAG:
        assert same(s.field(k), z["out_" + k]), k
    ci, cj, _ = s.pairs(P_CANDIDATES)
    assert np.array_equal(ci, z["cand_i"]) and np.array_equal(cj, z["cand_j"])
    bi, bj, bv = s.pairs(P_BONDS)
    assert np.array_equal(bi, z["bond_i"]) and np.array_equal(bj, z["bond_j"])
    assert same(bv, z["bond_dmg"])
