"""The GPU initial-condition generator (godar_gpu_place): every disk placed
inside the domain without overlap (periodic axes by minimum image), the
result a function of the inputs and the seed only, at the dense fractions of
configurations 2 and 3."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from godar_b200 import generators as gen
from godar_b200.lib import place_disks

pytestmark = pytest.mark.gpu


def assert_valid(x, y, r, Lx, Ly, px, py):
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(y))
    if px:
        assert np.all((x >= 0) & (x < Lx))
    else:
        assert np.all(x - r >= -1e-9 * Lx) and np.all(x + r <= Lx * (1 + 1e-12))
    if py:
        assert np.all((y >= 0) & (y < Ly))
    else:
        assert np.all(y - r >= -1e-9 * Ly) and np.all(y + r <= Ly * (1 + 1e-12))
    box = [Lx if px else 4 * Lx, Ly if py else 4 * Ly]
    pts = np.stack([np.mod(x, box[0]), np.mod(y, box[1])], axis=1)
    t = cKDTree(pts, boxsize=box)
    pairs = np.array(sorted(t.query_pairs(2 * r.max())), dtype=np.int64).reshape(-1, 2)
    if len(pairs):
        d = pts[pairs[:, 0]] - pts[pairs[:, 1]]
        for k, (L, per) in enumerate(((Lx, px), (Ly, py))):
            if per:
                d[:, k] -= L * np.round(d[:, k] / L)
        dist = np.hypot(d[:, 0], d[:, 1])
        sep = r[pairs[:, 0]] + r[pairs[:, 1]]
        assert np.all(dist >= sep * (1 - 1e-12)), int(np.sum(dist < sep))


def test_bonded_field_on_the_gpu():
    f = gen.bonded_field(nsteps=10, device="gpu")
    Lx, Ly = f.meta["domain_m"]
    assert f.meta["area_fraction"] >= 0.66
    assert_valid(f.x, f.y, f.r, Lx, Ly, True, True)
    g = gen.bonded_field(nsteps=10, device="gpu")
    assert np.array_equal(f.x.view(np.int64), g.x.view(np.int64))
    assert np.array_equal(f.y.view(np.int64), g.y.view(np.int64))


def test_polydisperse_field_on_the_gpu():
    f = gen.polydisperse_field(nsteps=10, device="gpu")
    Lx, Ly = f.meta["domain_m"]
    assert f.n == 65536 and f.meta["area_fraction"] >= 0.75
    assert_valid(f.x, f.y, f.r, Lx, Ly, False, True)


def test_gap_and_unplaceable_disks():
    rng = np.random.default_rng(0)
    r = rng.uniform(50.0, 100.0, 500)
    x, y, placed = place_disks(r, 6000.0, 6000.0, True, False, seed=3, gap=5.0)
    assert placed == 500
    assert_valid(x, y, r + 2.5, 6000.0, 6000.0, True, False)
    # far more disk area than domain: some cannot be placed, and say so
    x, y, placed = place_disks(np.full(200, 100.0), 1000.0, 1000.0, False, False, seed=1, max_rounds=8)
    assert placed < 200
    assert int(np.sum(np.isfinite(x))) == placed
