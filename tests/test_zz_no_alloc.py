"""The allocation-free candidate search (godar_gpu_candidates_noalloc).

It serves callers that cannot call cudaMalloc: a host program whose own
allocator already holds the GPU's memory, or a loop that must not pay
cudaMalloc's implicit synchronisation.  These tests own every device buffer
(inputs and outputs) and check that:

- two calls in a row on the same field, made after a larger field has left
  its contents in the shared scratch array, give the candidate pairs of the
  regular entry point (a Stepper's candidate list after its first step);
- a result larger than the caller's capacity returns GODAR_ERR_CAPACITY with
  the full count and writes only pairs of the full list;
- positions several periods outside a periodic domain give the same pairs
  as the oracle's candidate list of the same field inside the domain;
- a field whose search grid hits the 256 x 256 cell cap gives the oracle's
  candidate list;
- a warmed-up call leaves the device's free memory unchanged.

Kept in a file pytest collects last."""
import ctypes

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200 import lib as L
from godar_b200.lib import Stepper
from godar_b200.params import BC_PERIODIC_X, BC_PERIODIC_Y, make_params
from oracle import pyoracle as po

ERR_CAPACITY = 3


def _regular(f):
    s = Stepper(f.params, f.n)
    s.upload(f.x, f.y, f.r, f.h)
    if f.forcing is not None:
        s.set_field(f.forcing)
    s.step(1, 0, 1)
    pi, pj, _ = s.pairs(L.P_CANDIDATES)
    s.close()
    return sorted(zip(pi.tolist(), pj.tolist()))


def _oracle(p, x, y, r, h):
    o = po.Oracle(p, x, y, r, h)
    o.step(1)
    pi, pj, _ = o.pairs(po.P_CANDIDATES)
    o.close()
    return sorted(zip(pi.tolist(), pj.tolist()))


def _call(x, y, r, p, cap):
    """One call through the C ABI on device buffers; (status, count, pairs)."""
    import torch
    dev = torch.device("cuda:0")
    xd = torch.tensor(np.asarray(x), dtype=torch.float64, device=dev)
    yd = torch.tensor(np.asarray(y), dtype=torch.float64, device=dev)
    rd = torch.tensor(np.asarray(r), dtype=torch.float64, device=dev)
    pi = torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev)
    pj = torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    cnt = ctypes.c_int(-1)
    st = L.load().godar_gpu_candidates_noalloc(
        xd.data_ptr(), yd.data_ptr(), rd.data_ptr(), len(x), p.nx, p.ny, p.rtree, p.boundary,
        pi.data_ptr(), pj.data_ptr(), cap, ctypes.byref(cnt))
    m = min(cnt.value, cap)
    return st, cnt.value, sorted(zip(pi[:m].cpu().tolist(), pj[:m].cpu().tolist()))


def _noalloc(f, cap):
    st, cnt, got = _call(f.x, f.y, f.r, f.params, cap)
    assert st == 0, st
    assert cnt == len(got)
    return got


def _setup():
    import torch
    torch.cuda.set_device(0)
    cnt = ctypes.c_int(-1)
    assert L.load().godar_gpu_candidates_noalloc(None, None, None, 0, 0.0, 0.0, 0.0, 0, None, None, 0,
                                                 ctypes.byref(cnt)) == 0
    assert cnt.value == 0


@pytest.mark.gpu
def test_noalloc_candidates_match_regular_entry_point_twice():
    _setup()
    big = gen.polydisperse_field(n=3000, nsteps=1)
    small = gen.bonded_field(n=1500, nsteps=1)
    want_big, want_small = _regular(big), _regular(small)
    assert want_big and want_small
    # the larger field first, so that the smaller one's calls find its
    # cell ranges and counts left in the scratch array
    assert _noalloc(big, 4 * len(want_big) + 16) == want_big
    for _ in range(2):
        assert _noalloc(small, 4 * len(want_small) + 16) == want_small
    assert _noalloc(big, len(want_big)) == want_big


@pytest.mark.gpu
def test_noalloc_result_beyond_capacity():
    _setup()
    f = gen.bonded_field(n=1500, nsteps=1)
    want = _regular(f)
    cap = len(want) // 2
    st, cnt, got = _call(f.x, f.y, f.r, f.params, cap)
    assert st == ERR_CAPACITY
    assert cnt == len(want)
    assert len(got) == cap and set(got) <= set(want)


def _quantised_field(n, L, rlo, rhi, rtree, boundary, seed):
    """Floes with positions on a 1/64 m grid (so that shifts by whole periods
    and the wrap back are exact in FP64); overlaps do not matter here."""
    rng = np.random.default_rng(seed)
    x = np.round(rng.uniform(0.0, L, n) * 64.0) / 64.0
    y = np.round(rng.uniform(0.0, L, n) * 64.0) / 64.0
    x[x >= L] = 0.0
    y[y >= L] = 0.0
    r = rng.uniform(rlo, rhi, n)
    h = np.ones(n)
    p = make_params(L, L, rtree=rtree, boundary=boundary, dt=0.1)
    return p, x, y, r, h


@pytest.mark.gpu
def test_noalloc_wraps_periodic_positions_outside_the_domain():
    _setup()
    L_ = 40000.0
    p, x, y, r, h = _quantised_field(2000, L_, 200.0, 600.0, 600.0, BC_PERIODIC_X | BC_PERIODIC_Y, 7)
    want = _oracle(p, x, y, r, h)
    assert len(want) > 500
    rng = np.random.default_rng(8)
    kx = rng.choice([-3, -1, 0, 1, 2], len(x))
    ky = rng.choice([-2, 0, 1, 4], len(y))
    xs, ys = x + kx * L_, y + ky * L_
    assert np.array_equal(xs - kx * L_, x) and np.array_equal(ys - ky * L_, y)   # exact shifts
    st, cnt, got = _call(xs, ys, r, p, 4 * len(want) + 16)
    assert st == 0 and cnt == len(want)
    assert got == want


@pytest.mark.gpu
def test_noalloc_grid_at_its_cell_cap():
    _setup()
    # search radius <= 80 m in a 30 km domain: 375 cells per axis wanted,
    # 256 used (cells wider than the radius)
    p, x, y, r, h = _quantised_field(60000, 30000.0, 20.0, 40.0, 40.0, 0, 9)
    want = _oracle(p, x, y, r, h)
    assert len(want) > 10000
    st, cnt, got = _call(x, y, r, p, len(want) + 16)
    assert st == 0 and cnt == len(want)
    assert got == want


@pytest.mark.gpu
def test_noalloc_call_leaves_device_memory_unchanged():
    import torch
    _setup()
    f = gen.bonded_field(n=1500, nsteps=1)
    dev = torch.device("cuda:0")
    xd = torch.tensor(f.x, dtype=torch.float64, device=dev)
    yd = torch.tensor(f.y, dtype=torch.float64, device=dev)
    rd = torch.tensor(f.r, dtype=torch.float64, device=dev)
    cap = 64 * f.n
    pi = torch.empty(cap, dtype=torch.int32, device=dev)
    pj = torch.empty(cap, dtype=torch.int32, device=dev)
    cnt = ctypes.c_int(-1)
    fn = L.load().godar_gpu_candidates_noalloc
    args = (xd.data_ptr(), yd.data_ptr(), rd.data_ptr(), f.n, f.params.nx, f.params.ny, f.params.rtree,
            f.params.boundary, pi.data_ptr(), pj.data_ptr(), cap, ctypes.byref(cnt))
    assert fn(*args) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert fn(*args) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_table():
    cnt = ctypes.c_int(0)
    n = 65537
    st = L.load().godar_gpu_candidates_noalloc(1, 1, 1, n, 1e4, 1e4, 100.0, 0, 1, 1, 10, ctypes.byref(cnt))
    assert st == ERR_CAPACITY            # before any device work
