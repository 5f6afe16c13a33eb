"""ORACLE / TEST INFRASTRUCTURE ONLY: the reference's output records restated
in Python, the checker of godar_gpu_write_posts.

sea_ice_post (model/src/diagnostics_outputs.f90:1-189) appends one
list-directed record (write(u,*)) per output step to 25 files named
"output/<name>.<expno>"; clear_posts (model/src/diagnostics_ini_io.f90:1-100)
deletes them (and the info file) before a run.  List-directed layout is the
compiler runtime's; the reference is built with gfortran
(godarCMakeFiles/gfortranFLAGS.cmake), whose libgfortran writes:

- a blank at the start of every record and one blank between items;
- INTEGER(4) right-justified in 11 columns;
- REAL(8) as G25.17E3 with scale factor 1: F editing with 17 significant
  digits, right-justified in 20 columns and followed by 5 blanks, when
  0.1 <= |x| < 1e17 after rounding (zero as 0.0000000000000000); otherwise
  1PE25.17E3 (one digit, the point, 16 digits, E, sign, 3 exponent digits)
  right-justified in 25 columns.  Digits are correctly rounded.

The reference ships no output files, so this layout is pinned by the
runtime's documented list-directed rules and known outputs (tests), not by
reference fixtures.
"""
from __future__ import annotations

import math
import os

PER_FLOE = ["x", "y", "u", "v", "r", "h", "theta", "omega", "tfx", "tfy", "fcx", "fcy", "fbx", "fby",
            "mom", "mc", "mb", "tsigxx", "tsigyy", "tsigxy", "tsigyx", "tp"]
# oracle field name of each per-floe file
ORACLE_KEY = {"mom": "m"}
ALL_FILES = ["x", "y", "u", "v", "r", "h", "theta", "omega", "bond", "tfx", "tfy", "fcx", "fcy", "fbx",
             "fby", "mom", "mc", "mb", "tsigxx", "tsigyy", "tsigxy", "tsigyx", "tp", "angle", "damage"]


def g25_17(x: float) -> str:
    """One REAL(8) list-directed field, 25 characters."""
    if math.isnan(x):
        return "NaN".rjust(25)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(25)
    e = "%.16e" % x
    neg = e.startswith("-")
    m, ex = e.lstrip("-").split("e")
    dig = m.replace(".", "")
    e10 = int(ex)
    sign = "-" if neg else ""
    if x == 0.0:
        return (sign + "0.0000000000000000").rjust(20) + " " * 5
    if -1 <= e10 <= 16:
        k = e10 + 1
        body = "0." + dig if k == 0 else dig[:k] + "." + dig[k:]
        return (sign + body).rjust(20) + " " * 5
    body = dig[0] + "." + dig[1:] + "E" + ("-" if e10 < 0 else "+") + "%03d" % abs(e10)
    return (sign + body).rjust(25)


def int11(v: int) -> str:
    return "%11d" % v


def record(items) -> str:
    """One list-directed record of ints and floats."""
    out = []
    for it in items:
        out.append(" " + (int11(it) if isinstance(it, (int,)) and not isinstance(it, bool) else g25_17(float(it))))
    return "".join(out) + "\n"


def path_of(d: str, name: str, expno: str) -> str:
    return os.path.join(d, name + "." + expno.strip())


def write_posts(d: str, expno: str, tstep: int, comp: float, floes: dict, bonds, contacts):
    """Appends one output step.  floes: the oracle's floe fields; bonds and
    contacts: (i, j, value) arrays with i < j, 0-based (value = damage, and
    deltan)."""
    out_no = int(tstep / comp)
    pi = 4.0 * math.atan(1.0)
    x, y = floes["x"], floes["y"]
    bi, bj, bv = bonds
    order = sorted(range(len(bi)), key=lambda q: (int(bi[q]), int(bj[q])))
    rb = "".join(record([out_no, int(bj[q]) + 1, int(bi[q]) + 1]) for q in order) + "\n"
    rd = "".join(record([out_no, int(bj[q]) + 1, int(bi[q]) + 1, float(bv[q])]) for q in order)
    ci, cj, cv = contacts
    ra = []
    for q in sorted(range(len(ci)), key=lambda q: (int(ci[q]), int(cj[q]))):
        lo, hi = int(ci[q]), int(cj[q])
        if not cv[q] > 0.0:
            continue
        ang = (math.atan2(float(y[hi]) - float(y[lo]), float(x[hi]) - float(x[lo])) * 180.0) / pi
        ra.append(record([out_no, hi + 1, lo + 1, ang]))
    for name in PER_FLOE:
        with open(path_of(d, name, expno), "a") as f:
            f.write(record([float(v) for v in floes[ORACLE_KEY.get(name, name)]]))
    for name, text in (("bond", rb), ("angle", "".join(ra)), ("damage", rd)):
        with open(path_of(d, name, expno), "a") as f:
            f.write(text)
