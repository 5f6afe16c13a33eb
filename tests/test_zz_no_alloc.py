"""The allocation-free candidate search (godar_gpu_candidates_noalloc).

It serves callers that cannot call cudaMalloc: the test owns every device
buffer (inputs and outputs) and checks that two calls in a row give the same
candidate pairs as the regular entry point (a Stepper's candidate list after
its first step, computed from the same positions).  Kept in a file pytest
collects last."""
import ctypes

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200 import lib as L
from godar_b200.lib import Stepper


def _regular(f):
    s = Stepper(f.params, f.n)
    s.upload(f.x, f.y, f.r, f.h)
    if f.forcing is not None:
        s.set_field(f.forcing)
    s.step(1, 0, 1)
    pi, pj, _ = s.pairs(L.P_CANDIDATES)
    s.close()
    return sorted(zip(pi.tolist(), pj.tolist()))


def _noalloc(f, cap):
    import torch
    dev = torch.device("cuda:0")
    x = torch.tensor(f.x, dtype=torch.float64, device=dev)
    y = torch.tensor(f.y, dtype=torch.float64, device=dev)
    r = torch.tensor(f.r, dtype=torch.float64, device=dev)
    pi = torch.full((cap,), -1, dtype=torch.int32, device=dev)
    pj = torch.full((cap,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    cnt = ctypes.c_int(0)
    st = L.load().godar_gpu_candidates_noalloc(
        x.data_ptr(), y.data_ptr(), r.data_ptr(), f.n, f.params.nx, f.params.ny, f.params.rtree,
        f.params.boundary, pi.data_ptr(), pj.data_ptr(), cap, ctypes.byref(cnt))
    assert st == 0, st
    m = cnt.value
    return sorted(zip(pi[:m].cpu().tolist(), pj[:m].cpu().tolist()))


@pytest.mark.gpu
def test_noalloc_candidates_match_regular_entry_point_twice():
    import torch
    torch.cuda.set_device(0)
    fields = [gen.polydisperse_field(n=3000, nsteps=1), gen.bonded_field(n=1500, nsteps=1)]
    for f in fields:
        want = _regular(f)
        got = _noalloc(f, cap=4 * len(want) + 16)
        assert len(want) > 0
        assert got == want, f.name


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_table():
    cnt = ctypes.c_int(0)
    n = 65537
    st = L.load().godar_gpu_candidates_noalloc(1, 1, 1, n, 1e4, 1e4, 100.0, 0, 1, 1, 10, ctypes.byref(cnt))
    assert st == 3            # GODAR_ERR_CAPACITY, before any device work
