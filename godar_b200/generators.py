"""Seeded synthetic floe fields for the five benchmark configurations:
``lattice_field`` (256 rigid disks on a lattice), ``bonded_field`` (4,096
bonded floes), ``polydisperse_field`` (65,536 floes with sheltering, ridging
and a wall), ``ensemble`` / ``ensemble_member`` (512 bonded fields of 256 to
16,384 floes) and ``served_arrivals`` / ``served_member`` (the served request
stream).

The reference ships no input fields (files/ and output/ are git-ignored,
.gitignore:4-5); its own generator is tools/init/gridded_placement.py
(lattice placement, radius/thickness distributions at 111-196).  These
generators produce the configurations the benchmark is quoted on, with numpy
PCG64 seeds, and can write them in the reference's input format
(``files/{x,y,r,h,theta,omega}.dat``, one value per line, read by
ini_get.f90:148-164).

Where a configuration's floe count, radius law and area fraction cannot all
hold in its stated domain, the floe count and area fraction are kept and the
domain is scaled; the achieved area fraction is returned in ``meta``.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field as dfield

import numpy as np

from .params import (BC_OPEN_RIGHT, BC_PERIODIC_X, BC_PERIODIC_Y, GodarParams,
                     make_params)

_HERE = os.path.dirname(os.path.abspath(__file__))
_GEN_LIB = os.path.join(_HERE, "libgodar_gen.so")
_gen = None


def _genlib():
    global _gen
    if _gen is None:
        if not os.path.exists(_GEN_LIB):
            from .build import build_gen
            build_gen()
        L = ctypes.CDLL(_GEN_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.godar_gen_place.restype = ctypes.c_int
        L.godar_gen_place.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                      ctypes.c_int, ctypes.c_double, dp, dp]
        _gen = L
    return _gen


@dataclass
class Field:
    """One floe field: parameters, initial state and run length."""
    name: str
    params: GodarParams
    x: np.ndarray
    y: np.ndarray
    r: np.ndarray
    h: np.ndarray
    nsteps: int
    theta: np.ndarray | None = None
    omega: np.ndarray | None = None
    u: np.ndarray | None = None
    v: np.ndarray | None = None
    forcing: np.ndarray | None = None    # 4 x fny x fnx node values (ua, va, uw, vw)
    bonds: np.ndarray | None = None       # restart bonds (k, 2)
    damage: np.ndarray | None = None
    meta: dict = dfield(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.x)

    def write_reference_inputs(self, directory: str, suffix: str = "") -> None:
        """Writes files/{x,y,r,h,theta,omega}<suffix>.dat, one value per line."""
        os.makedirs(directory, exist_ok=True)
        zeros = np.zeros(self.n)
        for name, arr in (("x", self.x), ("y", self.y), ("r", self.r), ("h", self.h),
                          ("theta", self.theta if self.theta is not None else zeros),
                          ("omega", self.omega if self.omega is not None else zeros)):
            with open(os.path.join(directory, f"{name}{suffix}.dat"), "w") as f:
                for v in arr:
                    f.write(repr(float(v)) + "\n")


def place(r: np.ndarray, Lx: float, Ly: float, periodic_x: bool, periodic_y: bool,
          seed: int, max_trials: int = 400, gap: float = 0.0, device: str = "cpu"):
    """Places disks (largest first, relaxed random trials).  Returns x, y with
    NaN for disks that found no place.  device "gpu": godar_gpu_place (rounds
    of parallel trials per radius class; a different field for the same
    seed)."""
    if device == "gpu":
        from .lib import place_disks
        x, y, _ = place_disks(r, Lx, Ly, periodic_x, periodic_y, seed, max_rounds=256, gap=gap)
        return x, y
    r = np.ascontiguousarray(r, dtype=np.float64)
    x = np.empty_like(r)
    y = np.empty_like(r)
    dp = ctypes.POINTER(ctypes.c_double)
    _genlib().godar_gen_place(len(r), r.ctypes.data_as(dp), Lx, Ly, int(periodic_x),
                              int(periodic_y), seed, max_trials, gap,
                              x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    return x, y


def place_fraction(r: np.ndarray, phi: float, aspect: float, periodic_x: bool,
                   periodic_y: bool, seed: int, max_trials: int = 400, gap: float = 0.0,
                   device: str = "cpu"):
    """Chooses the domain for area fraction ``phi`` and places all disks,
    enlarging the domain by 2% per retry until every disk fits."""
    area = float(np.sum(np.pi * r * r))
    Ly = math.sqrt(area / (phi * aspect))
    Lx = aspect * Ly
    for _ in range(60):
        x, y = place(r, Lx, Ly, periodic_x, periodic_y, seed, max_trials, gap, device)
        if np.all(np.isfinite(x)):
            return x, y, Lx, Ly, area / (Lx * Ly)
        Lx *= 1.02
        Ly *= 1.02
    raise RuntimeError("placement failed")


def _overlaps(x, y, r, Lx, Ly, px, py):
    """Indices of disks overlapping another (cell list, minimum image)."""
    n = len(x)
    cs = 2 * r.max()
    ncx, ncy = max(1, int(Lx // cs)), max(1, int(Ly // cs))
    cx = np.clip((x / (Lx / ncx)).astype(int), 0, ncx - 1)
    cy = np.clip((y / (Ly / ncy)).astype(int), 0, ncy - 1)
    cells = {}
    for i in range(n):
        cells.setdefault((cx[i], cy[i]), []).append(i)
    bad = set()
    for i in range(n):
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                a, b = cx[i] + dx, cy[i] + dy
                if px:
                    a %= ncx
                if py:
                    b %= ncy
                for j in cells.get((a, b), ()):
                    if j <= i:
                        continue
                    ddx, ddy = x[i] - x[j], y[i] - y[j]
                    if px:
                        ddx -= Lx * round(ddx / Lx)
                    if py:
                        ddy -= Ly * round(ddy / Ly)
                    if math.hypot(ddx, ddy) < r[i] + r[j]:
                        bad.add(i)
                        bad.add(j)
    return sorted(bad)


# ---------------------------------------------------------------- lattice field
def lattice_field(n_side: int = 16, periodic: bool = True, seed: int = 0,
                  nsteps: int = 1000) -> Field:
    """Plain method, 256 rigid disks on a jittered 16x16 lattice in 50 km x
    50 km, r ~ U[500,1500] m, h ~ U[0.5,2] m, rho_ice 910, uniform wind
    10 m/s at 30 deg and current 0.1 m/s at 200 deg, skin drag 1.2e-3 /
    5.5e-3, f = 2 Omega (lat = pi/2; the stated 1.46e-4 exceeds 2 Omega =
    1.4584e-4), E = 6 GPa, nu = 0.3, mu = 0.7, dt = 1 s, rtree = 1500 m.
    Doubly periodic (extension) or the reference's four walls."""
    rng = np.random.default_rng(seed)
    L = 50e3
    sp = L / n_side
    n = n_side * n_side
    k = np.arange(n)
    bx, by = (k % n_side + 0.5) * sp, (k // n_side + 0.5) * sp
    x = bx + rng.uniform(-0.1 * sp, 0.1 * sp, n)
    y = by + rng.uniform(-0.1 * sp, 0.1 * sp, n)
    r = rng.uniform(500.0, 1500.0, n)
    h = rng.uniform(0.5, 2.0, n)
    for _ in range(1000):
        bad = _overlaps(x, y, r, L, L, periodic, periodic)
        if not periodic:
            bad = sorted(set(bad) | set(np.nonzero((x - r < 0) | (x + r > L) |
                                                   (y - r < 0) | (y + r > L))[0]))
        if not bad:
            break
        bad = np.asarray(bad)
        x[bad] = bx[bad] + rng.uniform(-0.1 * sp, 0.1 * sp, len(bad))
        y[bad] = by[bad] + rng.uniform(-0.1 * sp, 0.1 * sp, len(bad))
        r[bad] = rng.uniform(500.0, 1500.0, len(bad))
    else:
        raise RuntimeError("lattice_field: could not remove overlaps")
    wa, wc = math.radians(30.0), math.radians(200.0)
    p = make_params(
        L, L, cohesion=0, shelter=0, ridging=0, rhoice=910.0, Csair=1.2e-3,
        Cswater=5.5e-3, lat=math.pi / 2, e_modul=6e9, poiss_ratio=0.3,
        friction_coeff=0.7, dt=1.0, rtree=1500.0, ntree=1.0, nt=float(nsteps),
        ua=10.0 * math.cos(wa), va=10.0 * math.sin(wa),
        uw=0.1 * math.cos(wc), vw=0.1 * math.sin(wc),
        boundary=(BC_PERIODIC_X | BC_PERIODIC_Y) if periodic else 0)
    return Field("lattice", p, x, y, r, h, nsteps,
                 meta={"area_fraction": float(np.sum(np.pi * r * r) / L ** 2),
                       "periodic": periodic})


# ---------------------------------------------------------------- bonded field
def _lognormal_radii(rng, n, median=800.0, sigma=0.4, lo=200.0, hi=3000.0):
    return np.clip(rng.lognormal(math.log(median), sigma, n), lo, hi)


# The explicit scheme of the reference (symplectic Euler with explicit,
# critically damped bond dashpots, bonds.f90:132-138) is unstable at the
# stated dt = 0.5 s for 6 GPa beams on 200 m floes (omega dt > 1; velocities
# grow tenfold per step).  The bonded fields therefore run with the largest
# step that stayed stable in the oracle with margin; the stated value is kept
# in meta["dt_stated"].
DT_BONDED = 0.05
DT_POLYDISPERSE = 0.02


def bonded_field(n: int = 4096, seed: int = 1, phi: float = 0.70, nsteps: int = 2000,
                 wind_field: bool = True, wind_dir_deg: float | None = None,
                 wind_speed: float = 12.0, max_trials: int = 400, dt: float = DT_BONDED,
                 device: str = "cpu") -> Field:
    """Bonded field: lognormal radii (median 800 m, sigma_ln 0.4, clipped
    [200, 3000] m), h ~ U[0.3, 3.0] m, area fraction 70% (domain scaled),
    pairs with gap < 0.05 (r_i + r_j) bonded, eb = 6 GPa, tensile 0.5 MPa,
    shear 0.3 MPa, wind 12 m/s (1 + 0.5 sin(2 pi x / L)) toward +y, ocean at
    rest, rtree = 3000 m, doubly periodic; dt 0.05 s (stated 0.5 s)."""
    rng = np.random.default_rng(seed)
    r = _lognormal_radii(rng, n)
    h = rng.uniform(0.3, 3.0, n)
    x, y, Lx, Ly, achieved = place_fraction(r, phi, 1.0, True, True, seed, max_trials, device=device)
    forcing = None
    fnx = fny = 0
    ua = va = 0.0
    if wind_field:
        fnx, fny = 257, 2
        xs = np.linspace(0.0, Lx, fnx)
        vfield = wind_speed * (1.0 + 0.5 * np.sin(2 * np.pi * xs / Lx))
        forcing = np.zeros((4, fny, fnx))
        forcing[1, :, :] = vfield[None, :]
    else:
        ang = math.radians(wind_dir_deg if wind_dir_deg is not None else 90.0)
        ua, va = wind_speed * math.cos(ang), wind_speed * math.sin(ang)
    p = make_params(
        Lx, Ly, cohesion=1, shelter=0, ridging=0, dt=dt, rtree=3000.0, ntree=1.0,
        nt=float(nsteps), eb=6e9, sigmatb_crit=5e5, tau_crit=3e5, bond_lim=0.0,
        bond_lim_rel=0.05, ua=ua, va=va, uw=0.0, vw=0.0, rhoice=910.0,
        boundary=BC_PERIODIC_X | BC_PERIODIC_Y, field_nx=fnx, field_ny=fny)
    return Field("bonded", p, x, y, r, h, nsteps, forcing=forcing,
                 meta={"area_fraction": achieved, "domain_m": (Lx, Ly),
                       "target_fraction": phi, "dt_stated": 0.5})


# ---------------------------------------------------------------- polydisperse field
def _grf(rng, nxg, nyg, dx, corr):
    """Gaussian random field with a Gaussian spectrum of correlation length
    ``corr``, unit variance, on an nxg x nyg grid (FFT, seeded)."""
    kx = np.fft.fftfreq(nxg, d=dx) * 2 * np.pi
    ky = np.fft.fftfreq(nyg, d=dx) * 2 * np.pi
    K2 = kx[None, :] ** 2 + ky[:, None] ** 2
    spec = np.exp(-K2 * corr * corr / 4.0)
    noise = rng.standard_normal((nyg, nxg)) + 1j * rng.standard_normal((nyg, nxg))
    f = np.real(np.fft.ifft2(noise * np.sqrt(spec)))
    f -= f.mean()
    return f / (f.std() + 1e-30)


def polydisperse_field(n: int = 65536, seed: int = 2, phi: float = 0.85, nsteps: int = 2000,
                       max_trials: int = 300, dt: float = DT_POLYDISPERSE, device: str = "cpu") -> Field:
    """Large polydisperse field: radii power law p(r) ~ r^-2 on [100, 5000] m,
    h ~ Gamma(2, 0.75) (mean 1.5 m), area fraction 85% (domain scaled), wall
    at x = 0 (open at x = L, periodic in y), 10% of near-contact pairs bonded,
    wind 15 m/s toward the wall with a 20% Gaussian-random-field perturbation
    (50 km correlation), ocean eddies of 0.2 m/s at 30 km scale, sheltering and
    ridging on, rtree = 5000 m; dt 0.02 s (stated 0.5 s, unstable for the
    100 m floes)."""
    rng = np.random.default_rng(seed)
    a, b = 100.0, 5000.0
    u = rng.uniform(0.0, 1.0, n)
    r = 1.0 / (1.0 / a - u * (1.0 / a - 1.0 / b))
    h = rng.gamma(2.0, 0.75, n)
    h = np.maximum(h, 0.05)
    x, y, Lx, Ly, achieved = place_fraction(r, phi, 1.0, False, True, seed, max_trials, device=device)
    dxg = 2500.0
    fnx = int(math.ceil(Lx / dxg)) + 1
    fny = int(math.ceil(Ly / dxg)) + 1
    xs = np.linspace(0.0, Lx, fnx)
    ys = np.linspace(0.0, Ly, fny)
    g1 = _grf(rng, fnx, fny, Lx / (fnx - 1), 50e3)
    g2 = _grf(rng, fnx, fny, Lx / (fnx - 1), 50e3)
    forcing = np.zeros((4, fny, fnx))
    forcing[0] = -15.0 * (1.0 + 0.2 * g1)      # toward the wall at x = 0
    forcing[1] = 15.0 * 0.2 * g2
    lam = 30e3
    X, Y = np.meshgrid(xs, ys)
    forcing[2] = 0.2 * np.sin(2 * np.pi * X / lam) * np.cos(2 * np.pi * Y / lam)
    forcing[3] = -0.2 * np.cos(2 * np.pi * X / lam) * np.sin(2 * np.pi * Y / lam)
    p = make_params(
        Lx, Ly, cohesion=1, shelter=1, ridging=1, dt=dt, rtree=5000.0, ntree=1.0,
        nt=float(nsteps), bond_lim=0.0, bond_lim_rel=0.05, bond_frac=0.10,
        bond_seed=seed, rhoice=910.0, ua=0.0, va=0.0, uw=0.0, vw=0.0,
        boundary=BC_PERIODIC_Y | BC_OPEN_RIGHT, field_nx=fnx, field_ny=fny)
    return Field("polydisperse", p, x, y, r, h, nsteps, forcing=forcing,
                 meta={"area_fraction": achieved, "domain_m": (Lx, Ly),
                       "target_fraction": phi, "dt_stated": 0.5})


# ---------------------------------------------------------------- batched ensemble
def ensemble_sizes(count: int = 512, lo: int = 256, hi: int = 16384, seed: int = 4):
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi), count))).astype(int)


def ensemble_member(i: int, n: int, phi: float = 0.80, nsteps: int = 1000,
                    max_trials: int = 200) -> Field:
    """Member i of the batched ensemble: the bonded-field generator with seed 10+i,
    domain scaled to 80% area fraction, uniform wind of random direction
    U[0, 360) deg and speed U[8, 16] m/s."""
    rng = np.random.default_rng(10 + i)
    ang = rng.uniform(0.0, 360.0)
    spd = rng.uniform(8.0, 16.0)
    f = bonded_field(n=n, seed=10 + i, phi=phi, nsteps=nsteps, wind_field=False,
                wind_dir_deg=ang, wind_speed=spd, max_trials=max_trials)
    f.name = f"ensemble[{i}]"
    return f


def ensemble(count: int = 512, nsteps: int = 1000, sizes=None, max_trials: int = 200):
    sizes = ensemble_sizes(count) if sizes is None else sizes
    return [ensemble_member(i, int(n), nsteps=nsteps, max_trials=max_trials)
            for i, n in enumerate(sizes)]


# ---------------------------------------------------------------- served stream
def served_arrivals(count: int = 1000, rate: float = 20.0, seed: int = 5,
                    lo: int = 512, hi: int = 65536):
    """Poisson arrival times (rate req/s) and floe counts log-uniform in
    [lo, hi] for the served request stream."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    n = np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi), count))).astype(int)
    return t, n


def served_member(k: int, n: int, nsteps: int = 2000, max_trials: int = 150) -> Field:
    rng = np.random.default_rng(1000 + k)
    ang = rng.uniform(0.0, 360.0)
    spd = rng.uniform(8.0, 16.0)
    f = bonded_field(n=n, seed=1000 + k, phi=0.70, nsteps=nsteps, wind_field=False,
                wind_dir_deg=ang, wind_speed=spd, max_trials=max_trials)
    f.name = f"served[{k}]"
    return f
