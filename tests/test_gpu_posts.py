"""The output step on the GPU: godar_gpu_write_posts appends the reference's
25 text files (sea_ice_post, diagnostics_outputs.f90:1-189) from the device
state; the same records written from the CPU oracle's state by the
restatement in oracle/posts.py must be byte-identical (the FP64 path is
bit-exact, so every digit must agree), over several output steps."""
import os

import numpy as np
import pytest

from godar_b200 import generators as gen
from godar_b200 import lib
from oracle import posts
from oracle import pyoracle as po

from .helpers import gpu_for, oracle_for
from .test_gpu_parity import two_disk_field

pytestmark = pytest.mark.gpu


def run_posts(f, tmp_path, outputs, comp):
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "oracle")
    os.makedirs(dg)
    os.makedirs(do)
    lib.clear_posts(dg, "01")
    o = oracle_for(f)
    g = gpu_for(f)
    t = 1
    for tstep in outputs:
        k = tstep - t + 1
        o.step(k)
        g.step(t, 0, k)
        t = tstep + 1
        g.write_posts(dg, "01", tstep, comp)
        posts.write_posts(do, "01", tstep, comp, o.floes(), o.pairs(po.P_BONDS), o.pairs(po.P_CONTACTS))
    for name in posts.ALL_FILES:
        a = open(posts.path_of(dg, name, "01"), "rb").read()
        b = open(posts.path_of(do, name, "01"), "rb").read()
        assert a == b, name
    return dg


def test_bonded_field_posts_match_oracle(tmp_path):
    f = gen.bonded_field(n=300, nsteps=60)
    d = run_posts(f, tmp_path, outputs=[1, 30, 60], comp=30.0)
    # the readers of the reference's tools: np.loadtxt per file
    x = np.loadtxt(posts.path_of(d, "x", "01"))
    assert x.shape == (3, f.n)
    b = np.loadtxt(posts.path_of(d, "bond", "01"), dtype=int)
    assert b.shape[1] == 3 and set(b[:, 0]) == {0, 1, 2}
    assert np.all(b[:, 1] > b[:, 2])


def test_colliding_pair_angle_posts(tmp_path):
    # rtree above the radii (as the reference advises, gridded_placement.py:
    # 272-275): a pair cannot leave the candidates while overlapping, so the
    # reference's stale deltan array and the current contact list agree
    f = two_disk_field(False)
    f.params.rtree = 1500.0
    d = run_posts(f, tmp_path, outputs=[1, 20, 40, 60], comp=20.0)
    lines = open(posts.path_of(d, "angle", "01")).read().splitlines()
    assert lines, "the two disks should be in contact at an output step"
