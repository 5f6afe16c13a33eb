"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes wrapper of oracle/liboracle.so.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker of the CUDA path; the godar_b200 package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

RIDGE_REFERENCE, RIDGE_DEFERRED = 0, 1
MATH_DET, MATH_LIBM = 0, 1
P_CANDIDATES, P_CONTACTS, P_BONDS = 0, 1, 2

FLOE_FIELDS = ["x", "y", "u", "v", "r", "h", "theta", "omega", "tfx", "tfy",
               "fcx", "fcy", "fbx", "fby", "m", "mc", "mb", "tsigxx", "tsigyy",
               "tsigxy", "tsigyx", "tp", "fax", "fay", "fwx", "fwy", "ma", "mw",
               "fcorx", "fcory", "fx_bc", "fy_bc", "m_bc", "hsfa", "hsfw", "mass"]

_lib = None


def build() -> str:
    src = [os.path.join(HERE, f) for f in ("godar_oracle.c", "godar_oracle.h", "detmath_oracle.h")]
    if (not os.path.exists(LIB) or
            any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in src if os.path.exists(s))):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        L.gdo_create.restype = ctypes.c_void_p
        L.gdo_create.argtypes = [ctypes.c_void_p, ctypes.c_int] + [dp] * 8 + [ctypes.c_int, ip, ip, dp, dp]
        L.gdo_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.gdo_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.gdo_set_modes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.gdo_get_floes.argtypes = [ctypes.c_void_p, dp]
        L.gdo_get_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int, ip, ip, dp, ctypes.c_int]
        L.gdo_get_pair_hist.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.gdo_destroy.argtypes = [ctypes.c_void_p]
        for f in ("gdo_exp", "gdo_log", "gdo_asin", "gdo_acos"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = [ctypes.c_double]
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class Oracle:
    """One floe field advanced by the C restatement of ``stepper``."""

    def __init__(self, params, x, y, r, h, theta=None, omega=None, u=None, v=None,
                 bonds=None, damage=None, field=None,
                 ridge_mode=RIDGE_DEFERRED, math_mode=MATH_DET):
        L = lib()
        assert L.gdo_params_size() == ctypes.sizeof(params), "params layout mismatch"
        self.n = n = len(x)
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        self._keep = [c(x), c(y), c(r), c(h), c(theta), c(omega), c(u), c(v)]
        nb = 0
        bi = bj = dmg = None
        if bonds is not None and len(bonds):
            b = np.asarray(bonds, dtype=np.int32).reshape(-1, 2)
            bi = np.ascontiguousarray(b[:, 0]); bj = np.ascontiguousarray(b[:, 1])
            nb = len(b)
            dmg = c(damage) if damage is not None else None
        fld = c(field)
        self._keep += [bi, bj, dmg, fld]
        self.params = params
        self.s = L.gdo_create(ctypes.byref(params), n, *[_dp(a) for a in self._keep[:8]],
                              nb, _ip(bi), _ip(bj), _dp(dmg), _dp(fld))
        L.gdo_set_modes(self.s, ridge_mode, math_mode)
        self.tstep = 1

    def step(self, nsteps=1, restart=0):
        lib().gdo_run(self.s, self.tstep, nsteps, restart)
        self.tstep += nsteps

    def floes(self) -> dict:
        out = np.empty(len(FLOE_FIELDS) * self.n, dtype=np.float64)
        lib().gdo_get_floes(self.s, _dp(out))
        out = out.reshape(len(FLOE_FIELDS), self.n)
        return {k: out[i].copy() for i, k in enumerate(FLOE_FIELDS)}

    def pairs(self, which):
        L = lib()
        cnt = L.gdo_get_pairs(self.s, which, None, None, None, 0)
        pi = np.empty(max(cnt, 1), np.int32); pj = np.empty(max(cnt, 1), np.int32)
        val = np.empty(max(cnt, 1), np.float64)
        L.gdo_get_pairs(self.s, which, _ip(pi), _ip(pj), _dp(val), cnt)
        return pi[:cnt], pj[:cnt], val[:cnt]

    def pair_hist(self, i, j):
        out = np.zeros(4)
        lib().gdo_get_pair_hist(self.s, i, j, _dp(out))
        return out

    def close(self):
        if self.s:
            lib().gdo_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
