"""The Fortran binding (godar_b200/fortran/godar_gpu_mod.f90) read as text
against the C ABI: every bind(C) interface names a declared entry point with
the header's parameter count and kinds (by-value int / double / size_t, a
c_ptr by value, everything else by reference), and the bind(C) derived type
godar_params lists the C struct's fields in order with the same types.  The
image has no Fortran compiler, so the module is parsed rather than built."""
import ctypes
import os
import re

from godar_b200.params import GodarParams

from .test_capi import header_prototypes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOD = os.path.join(ROOT, "godar_b200", "fortran", "godar_gpu_mod.f90")


def _logical_lines(path):
    """Statements of a free-form Fortran file: comments dropped, '&'
    continuations joined."""
    out, cur = [], ""
    for raw in open(path):
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if s.startswith("&"):
            s = s[1:].lstrip()
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        out.append(cur + s)
        cur = ""
    return out


def fortran_interfaces():
    """bind name -> list of (kind) per dummy argument, in order."""
    lines = _logical_lines(MOD)
    res = {}
    k = 0
    while k < len(lines):
        m = re.match(r"(function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", lines[k], re.I)
        if not m:
            k += 1
            continue
        args = [a.strip().lower() for a in m.group(3).split(",") if a.strip()]
        decl = {}
        k += 1
        while not re.match(r"end\s+(function|subroutine)", lines[k], re.I):
            d = re.match(r"([^:]+)::(.*)", lines[k])
            if d:
                spec = d.group(1).lower().replace(" ", "")
                for nm in re.findall(r"(\w+)(?:\([^)]*\))?", d.group(2)):
                    decl[nm.lower()] = spec
            k += 1
        kinds = []
        for a in args:
            spec = decl[a]
            if ",value" not in spec:
                kinds.append("ptr")
            elif spec.startswith("type(c_ptr)"):
                kinds.append("ptr")
            elif spec.startswith("integer(c_int)") or spec.startswith("integer(c_int32_t)"):
                kinds.append("int")
            elif spec.startswith("real(c_double)"):
                kinds.append("double")
            elif spec.startswith("integer(c_size_t)") or spec.startswith("integer(c_int64_t)"):
                kinds.append("u64")
            else:
                raise AssertionError(f"unmapped declaration {spec} of {a} in {m.group(4)}")
        res[m.group(4)] = kinds
    return res


def _c_kind(t: str) -> str:
    if "*" in t:
        return "ptr"
    return {"int": "int", "size_t": "u64", "double": "double", "uint64_t": "u64"}[t.replace("const ", "")]


def test_every_fortran_interface_matches_the_header():
    protos = header_prototypes()
    ifs = fortran_interfaces()
    # the entry points the replacement stepper and sea_ice_post use
    for need in ("godar_gpu_derive_params", "godar_gpu_create", "godar_gpu_upload", "godar_gpu_step",
                 "godar_gpu_step_async", "godar_gpu_download", "godar_gpu_write_posts", "godar_gpu_clear_posts",
                 "godar_gpu_checkpoint", "godar_gpu_restore", "godar_gpu_set_diagnostics",
                 "godar_gpu_last_error", "godar_gpu_destroy"):
        assert need in ifs, need
    for name, kinds in ifs.items():
        assert name in protos, name
        assert kinds == [_c_kind(t) for t in protos[name][1]], name


def test_fortran_params_type_mirrors_the_c_struct():
    lines = _logical_lines(MOD)
    a = next(i for i, s in enumerate(lines) if re.match(r"type\s*,\s*bind\(C\)\s*::\s*godar_params", s, re.I))
    fields = []
    for s in lines[a + 1:]:
        if re.match(r"end\s+type", s, re.I):
            break
        spec, names = s.split("::")
        kind = {"integer(c_int32_t)": ctypes.c_int32, "real(c_double)": ctypes.c_double}[spec.strip().lower()]
        fields += [(n.strip(), kind) for n in names.split(",")]
    c_fields = [(n, t) for n, t in GodarParams._fields_]
    assert [n.lower() for n, _ in fields] == [n.lower() for n, _ in c_fields]
    for (n, t), (_, ct) in zip(fields, c_fields):
        assert ctypes.sizeof(t) == ctypes.sizeof(ct), n
        assert (t is ctypes.c_double) == (ct is ctypes.c_double), n


def _calls(path):
    """(name, argument count) of every godar_gpu_* call in a Fortran file."""
    out = []
    for s in _logical_lines(path):
        for m in re.finditer(r"\b(godar_gpu_\w+)\s*\(", s):
            if re.match(r"\s*(function|subroutine)\b", s, re.I):
                continue
            depth, k, args, cur = 1, m.end(), [], ""
            while depth:
                ch = s[k]
                if ch == "(":
                    depth += 1
                elif ch == ")":
                    depth -= 1
                if depth == 1 and ch == ",":
                    args.append(cur)
                    cur = ""
                elif depth:
                    cur += ch
                k += 1
            if cur.strip():
                args.append(cur)
            out.append((m.group(1), len(args)))
    return out


def test_replacement_routines_call_the_interfaces_with_their_arity():
    ifs = fortran_interfaces()
    seen = set()
    for f in ("stepper.f90", "sea_ice_post.f90"):
        for name, nargs in _calls(os.path.join(ROOT, "godar_b200", "fortran", f)):
            assert name in ifs, (f, name)
            assert nargs == len(ifs[name]), (f, name, nargs)
            seen.add(name)
    assert {"godar_gpu_create", "godar_gpu_upload", "godar_gpu_step_async", "godar_gpu_set_diagnostics",
            "godar_gpu_write_posts", "godar_gpu_clear_posts"} <= seen
