"""Run parameters: a ctypes mirror of ``godar_params`` in include/godar_gpu.h.

Field order and defaults follow the reference's namelist reader
``read_namelist`` (model/src/par_get.f90:130-155) and ``get_default``
(model/src/par_get.f90:16-109); the derived constants follow
par_get.f90:263-266.  Extensions (boundary flags, relative bond limit, bond
fraction, forcing grid) default to zero, which reproduces the reference.
"""
from __future__ import annotations

import ctypes
import math
import re

import numpy as np

BC_PERIODIC_X = 1
BC_PERIODIC_Y = 2
BC_OPEN_LEFT = 4
BC_OPEN_RIGHT = 8
BC_OPEN_BOTTOM = 16
BC_OPEN_TOP = 32

PREC_FP64 = 0
PREC_MIXED = 1

_I = ctypes.c_int32
_D = ctypes.c_double

_FIELDS = [
    # options_nml
    ("dynamics", _I), ("slipping", _I), ("thermodyn", _I), ("cohesion", _I),
    ("ridging", _I), ("shelter", _I),
    # numerical_param_nml
    ("rtree", _D), ("ntree", _D), ("dt", _D), ("nt", _D), ("comp", _D),
    # physical_param_nml
    ("Cdair", _D), ("Csair", _D), ("Cdwater", _D), ("Cswater", _D), ("z0w", _D),
    ("lat", _D), ("rhoair", _D), ("rhoice", _D), ("rhowater", _D),
    # disk_param_nml
    ("e_modul", _D), ("poiss_ratio", _D), ("friction_coeff", _D),
    ("rest_coeff", _D), ("sigmanc_crit", _D),
    # bond_param_nml
    ("eb", _D), ("lambda_rb", _D), ("lambda_lb", _D), ("sigmatb_crit", _D),
    ("sigmacb_crit", _D), ("tau_crit", _D), ("bond_lim", _D), ("dmax", _D),
    ("dtd", _D), ("dth", _D),
    # forcings_nml
    ("uw", _D), ("vw", _D), ("ua", _D), ("va", _D),
    # parameter.h
    ("nx", _D), ("ny", _D),
    # derived
    ("ec", _D), ("gc", _D), ("beta", _D), ("pi", _D), ("sin_lat", _D),
    # extensions
    ("boundary", _I), ("bond_seed", _I), ("bond_lim_rel", _D), ("bond_frac", _D),
    ("field_nx", _I), ("field_ny", _I),
]

NAMELIST_GROUPS = {
    "options_nml": ["dynamics", "slipping", "thermodyn", "cohesion", "ridging", "shelter"],
    "numerical_param_nml": ["rtree", "ntree", "dt", "nt", "comp"],
    "physical_param_nml": ["Cdair", "Csair", "Cdwater", "Cswater", "z0w", "lat",
                           "rhoair", "rhoice", "rhowater"],
    "disk_param_nml": ["e_modul", "poiss_ratio", "friction_coeff", "rest_coeff",
                       "sigmanc_crit"],
    "bond_param_nml": ["eb", "lambda_rb", "lambda_lb", "sigmatb_crit", "sigmacb_crit",
                       "tau_crit", "bond_lim", "dmax", "dtd", "dth"],
    "forcings_nml": ["uw", "vw", "ua", "va"],
}


class GodarParams(ctypes.Structure):
    _fields_ = _FIELDS

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in _FIELDS}

    def copy(self) -> "GodarParams":
        p = GodarParams()
        ctypes.pointer(p)[0] = self
        return p


def derive(p: GodarParams) -> GodarParams:
    """Recompute ec, gc, beta (par_get.f90:264-266), pi (par_get.f90:35) and
    sin(lat) (forcing.f90:202) with the reference's evaluation order."""
    p.pi = 4.0 * math.atan(1.0)
    nu = p.poiss_ratio
    p.ec = p.e_modul / (2.0 * (1.0 - nu * nu))
    p.gc = p.e_modul / ((4.0 * (1.0 - nu)) * (2.0 + nu))
    le = math.log(p.rest_coeff)
    p.beta = (10.0 * le) / math.sqrt(le * le + p.pi * p.pi)
    p.sin_lat = math.sin(p.lat)
    return p


def default_params(nx: float = 5e3, ny: float = 5e3) -> GodarParams:
    """``get_default`` (par_get.f90:16-109).  ``lat = 1.4`` there is a default
    (single-precision) REAL literal, so its value is float32(1.4)."""
    p = GodarParams()
    p.dynamics, p.slipping, p.thermodyn = 1, 1, 0
    p.cohesion, p.ridging, p.shelter = 1, 1, 1
    p.rtree, p.ntree, p.dt, p.nt, p.comp = 1e3, 1.0, 1e-3, 1e3, 1.0
    p.Cdair, p.Csair, p.Cdwater, p.Cswater = 3e-1, 5e-4, 3e-1, 2e-3
    p.z0w = 3.0e-4
    p.lat = float(np.float32(1.4))
    p.rhoair, p.rhoice, p.rhowater = 1.3, 9e2, 1026.0
    p.e_modul, p.poiss_ratio, p.friction_coeff = 6e9, 33e-2, 7e-1
    p.rest_coeff, p.sigmanc_crit = 88e-2, 1e6
    p.eb, p.lambda_rb, p.lambda_lb = 6e9, 8e-1, 1.0
    p.sigmatb_crit, p.sigmacb_crit, p.tau_crit = 1e5, 1e6, 1e6
    p.bond_lim, p.dmax, p.dtd, p.dth = 1e-2, 9e-1, 1.0, 1e5
    p.uw = p.vw = p.ua = p.va = 0.0
    p.nx, p.ny = nx, ny
    p.boundary = 0
    p.bond_seed = 0
    p.bond_lim_rel = 0.0
    p.bond_frac = 0.0
    p.field_nx = p.field_ny = 0
    return derive(p)


def make_params(nx: float, ny: float, **kw) -> GodarParams:
    """Defaults, then namelist-style overrides, then the derived constants."""
    p = default_params(nx, ny)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k!r}")
        setattr(p, k, v)
    return derive(p)


_FORTRAN_NUM = re.compile(r"^([+-]?(?:\d+\.?\d*|\.\d+))(?:[dDeE]([+-]?\d+))?$")


def _parse_value(tok: str):
    t = tok.strip().rstrip(",")
    tl = t.lower()
    if tl in (".true.", "t", ".t."):
        return 1
    if tl in (".false.", "f", ".f."):
        return 0
    if t.startswith(("'", '"')):
        return t.strip("'\"")
    m = _FORTRAN_NUM.match(t)
    if not m:
        raise ValueError(f"cannot parse namelist value {tok!r}")
    mant, exp = m.group(1), m.group(2)
    is_double = exp is not None and re.search(r"[dD]", t) is not None
    val = float(mant + (("e" + exp) if exp else ""))
    if not is_double and ("." in mant or exp is not None):
        # a default-kind REAL literal keeps single precision when read into a
        # double by the reference's own source defaults; namelist input is
        # read at full precision by gfortran, so only source literals matter.
        pass
    return val


def read_namelist(path: str, p: GodarParams | None = None,
                  nx: float = 5e3, ny: float = 5e3) -> GodarParams:
    """Reads a GODAR namelist file group by group like ``read_namelist``
    (par_get.f90:114-268): a group that fails to parse (for example one with
    an unknown variable, as generic/namelist_generic.nml:45 does) keeps its
    defaults entirely."""
    if p is None:
        p = default_params(nx, ny)
    text = open(path).read()
    for group, names in NAMELIST_GROUPS.items():
        m = re.search(r"&" + group + r"\b(.*?)\n\s*/", text, re.S | re.I)
        if not m:
            continue
        body = re.sub(r"!.*", "", m.group(1))
        vals = {}
        ok = True
        for part in re.split(r",?\s*\n", body):
            part = part.strip()
            if not part:
                continue
            if "=" not in part:
                ok = False
                break
            k, v = part.split("=", 1)
            k = k.strip()
            match = [n for n in names if n.lower() == k.lower()]
            if not match:
                ok = False
                break
            try:
                vals[match[0]] = _parse_value(v)
            except ValueError:
                ok = False
                break
        if ok:
            for k, v in vals.items():
                setattr(p, k, v)
    return derive(p)
