"""Synthetic benchmark fields: reproducible, overlap-free, at the stated area
fraction, and writable in the reference's input format."""
import os

import numpy as np

from godar_b200 import generators as gen


def overlaps(f, periodic):
    return gen._overlaps(f.x, f.y, f.r, f.params.nx, f.params.ny, periodic, periodic)


def test_lattice_no_overlap_and_seeded():
    a = gen.lattice_field()
    b = gen.lattice_field()
    assert a.n == 256 and np.array_equal(a.x, b.x)
    assert not overlaps(a, True)
    assert a.params.rtree == 1500.0 and a.params.dt == 1.0
    assert abs(a.params.sin_lat - 1.0) < 1e-15


def test_bonded_field_fraction_and_no_overlap():
    f = gen.bonded_field(n=800)
    assert abs(f.meta["area_fraction"] - 0.70) < 0.02
    assert not overlaps(f, True)
    assert f.r.min() >= 200 and f.r.max() <= 3000
    assert f.forcing.shape == (4, 2, 257)


def test_polydisperse_field_wall():
    f = gen.polydisperse_field(n=1500)
    assert f.meta["area_fraction"] > 0.75
    assert np.all(f.x - f.r >= -1e-9)      # wall at x = 0 respected
    assert f.params.shelter == 1 and f.params.ridging == 1 and f.params.bond_frac == 0.1


def test_ensemble_sizes_log_uniform():
    s = gen.ensemble_sizes(512)
    assert s.min() >= 256 and s.max() < 16384
    assert 3000 < np.mean(s) < 5000      # (b - a) / ln(b / a) = 3878


def test_reference_input_files(tmp_path):
    f = gen.lattice_field(n_side=4)
    f.write_reference_inputs(str(tmp_path))
    x = np.loadtxt(os.path.join(tmp_path, "x.dat"))
    assert np.array_equal(x, f.x)
    assert len(open(os.path.join(tmp_path, "omega.dat")).read().split()) == f.n


def _max_overlap(f):
    L = f.params.nx
    worst = 0.0
    for a in range(f.n):
        dx = f.x[a] - f.x
        dy = f.y[a] - f.y
        dx -= L * np.round(dx / L)
        dy -= L * np.round(dy / L)
        d = np.hypot(dx, dy)
        d[a] = np.inf
        worst = max(worst, float(np.max(f.r[a] + f.r - d)))
    return worst


def test_ensemble_members_overlap_free_across_periodic_edges():
    """Small periodic domains: disks straddling the edges must not overlap
    their wrapped neighbours."""
    sizes = gen.ensemble_sizes(512)
    for i in (7, 51, 53):
        f = gen.ensemble_member(i, int(sizes[i]))
        assert _max_overlap(f) <= 1e-6, i
