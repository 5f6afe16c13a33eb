"""Output records (sea_ice_post, diagnostics_outputs.f90:1-189) on the CPU:
the library's list-directed formatter against gfortran's known outputs and
against the restatement in oracle/posts.py, plus the round trip that lets
np.loadtxt read the files back bit for bit."""
import math
import os

import numpy as np
import pytest

from godar_b200 import lib
from oracle import posts

# list-directed outputs of gfortran for REAL(8) values (one item per record)
KNOWN = {
    1.0: "   1.0000000000000000     \n",
    0.1: "  0.10000000000000001     \n",
    -2.5: "  -2.5000000000000000     \n",
    0.0: "   0.0000000000000000     \n",
    1.0e-3: "   1.0000000000000000E-003\n",
    12345.678: "   12345.678000000000     \n",
    2.0 ** 80: "   1.2089258196146292E+024\n",
}


@pytest.mark.parametrize("x", sorted(KNOWN))
def test_known_gfortran_records(x):
    assert lib.format_reals([x]) == KNOWN[x]
    assert posts.record([x]) == KNOWN[x]


def test_integer_and_mixed_records():
    assert posts.record([1, 2, 3]) == "           1           2           3\n"
    assert posts.record([0, 12, 7, 0.5]) == "           0          12           7  0.50000000000000000     \n"


def edge_values():
    rng = np.random.default_rng(3)
    v = [0.1, np.nextafter(0.1, 0), np.nextafter(0.1, 1), 1e17, np.nextafter(1e17, 0), 9.999999999999999e16,
         99999999999999999.0, 0.09999999999999999, -0.0, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
         -1e-300, 1.0 / 3.0, 2.0 / 3.0, 1e16, 123456789012345678.0, 0.5, -0.1]
    mags = 10.0 ** rng.uniform(-30, 30, 400)
    v += list(mags * rng.choice([-1.0, 1.0], 400))
    v += list(rng.standard_normal(200))
    return np.array(v, dtype=np.float64)


def test_formatter_matches_restatement():
    v = edge_values()
    rec = lib.format_reals(v)
    assert rec == posts.record([float(x) for x in v])
    assert len(rec) == 26 * len(v) + 1


def test_special_values():
    rec = lib.format_reals([math.inf, -math.inf, math.nan])
    assert rec == posts.record([math.inf, -math.inf, math.nan])
    assert rec.split() == ["Infinity", "-Infinity", "NaN"]


def test_round_trip_is_exact():
    v = edge_values()
    back = np.array([float(t) for t in lib.format_reals(v).split()])
    assert np.array_equal(back.view(np.int64), v.view(np.int64))


def test_clear_posts_removes_the_files(tmp_path):
    d = str(tmp_path)
    for name in posts.ALL_FILES + ["info"]:
        open(os.path.join(d, name + ".07"), "w").write("x\n")
    open(os.path.join(d, "x.08"), "w").write("keep\n")
    lib.clear_posts(d, "07")
    assert sorted(os.listdir(d)) == ["x.08"]
    lib.clear_posts(d, "07")           # nothing left to delete: not an error


def test_unwritable_directory_reports_io_error(tmp_path):
    # a directory that does not exist: deleting nothing is fine, appending is
    # an i/o error reported by status (no GPU needed to reach it)
    lib.clear_posts(str(tmp_path / "missing"), "01")
    L = lib.load()
    assert L.godar_gpu_clear_posts(None, None) == 2        # GODAR_ERR_BAD_INPUT
    assert "i/o" in L.godar_gpu_errstr(11).decode()
