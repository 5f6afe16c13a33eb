"""Generates the regression fixtures in this directory with the CPU oracle.

Each fixture holds a small seeded floe field (inputs, parameters, forcing
grid) and the oracle's state, forces, stresses and pair lists after a number
of steps.  The CPU tests check that the oracle still reproduces them bit for
bit; the GPU tests check the C ABI against them without running the oracle.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from godar_b200 import generators as gen  # noqa: E402
from godar_b200.params import BC_PERIODIC_X, BC_PERIODIC_Y, make_params  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


def two_disks():
    L = 1e5
    p = make_params(L, L, cohesion=0, shelter=0, ridging=0, dt=0.05, rtree=1000.0, lat=0.0,
                    boundary=BC_PERIODIC_X | BC_PERIODIC_Y)
    f = gen.Field("two_disks", p, np.array([5e4, 5.2001e4]), np.array([5e4, 5.003e4]),
                  np.array([1000.0, 1000.0]), np.array([1.0, 1.2]), 1200,
                  u=np.array([0.5, -0.5]), v=np.zeros(2))
    return f


CASES = {
    "two_disks": (two_disks, 1200),
    "lattice_periodic_36": (lambda: gen.lattice_field(n_side=6, periodic=True), 300),
    "lattice_walls_36": (lambda: gen.lattice_field(n_side=6, periodic=False), 300),
    "bonded_120": (lambda: gen.bonded_field(n=120, nsteps=200), 200),
    "polydisperse_shelter_ridging_500": (lambda: gen.polydisperse_field(n=500, nsteps=80), 80),
}


def run(f, nsteps):
    o = po.Oracle(f.params, f.x, f.y, f.r, f.h, f.theta, f.omega, f.u, f.v, field=f.forcing)
    o.step(nsteps)
    out = o.floes()
    ci, cj, cv = o.pairs(po.P_CANDIDATES)
    bi, bj, bv = o.pairs(po.P_BONDS)
    return out, (ci, cj, cv), (bi, bj, bv)


def main():
    for name, (make, nsteps) in CASES.items():
        f = make()
        out, cand, bonds = run(f, nsteps)
        arrays = {"in_" + k: v for k, v in (("x", f.x), ("y", f.y), ("r", f.r), ("h", f.h)) if v is not None}
        for k, v in (("u", f.u), ("v", f.v)):
            if v is not None:
                arrays["in_" + k] = v
        if f.forcing is not None:
            arrays["forcing"] = f.forcing
        for k, v in out.items():
            arrays["out_" + k] = v
        arrays["cand_i"], arrays["cand_j"], arrays["cand_dn"] = cand
        arrays["bond_i"], arrays["bond_j"], arrays["bond_dmg"] = bonds
        meta = {"name": name, "nsteps": nsteps, "params": f.params.as_dict()}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=json.dumps(meta), **arrays)
        print(name, f.n, "floes", nsteps, "steps")


if __name__ == "__main__":
    main()
