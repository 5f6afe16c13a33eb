"""The C ABI library, checked without a GPU: it loads, exports every entry
point include/godar_gpu.h declares, agrees with the Python params mirror, and
refuses to run (instead of falling back to the CPU) when no device is
visible."""
import ctypes
import os
import re

import numpy as np
import pytest

from godar_b200 import lib as L
from godar_b200.params import GodarParams, default_params, read_namelist

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "godar_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(godar_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(L.EXPORTS)


def test_params_layout_and_defaults_match():
    lib = L.load()
    assert lib.godar_gpu_params_size() == ctypes.sizeof(GodarParams)
    p = GodarParams()
    assert lib.godar_gpu_default_params(ctypes.byref(p)) == 0
    q = default_params()
    for name, _ in GodarParams._fields_:
        assert getattr(p, name) == getattr(q, name), name
    q.rest_coeff = 0.5
    q.poiss_ratio = 0.25
    lib.godar_gpu_derive_params(ctypes.byref(q))
    from godar_b200.params import derive
    r = default_params()
    r.rest_coeff = 0.5
    r.poiss_ratio = 0.25
    derive(r)
    assert (q.beta, q.ec, q.gc) == (r.beta, r.ec, r.gc)


def test_errors_are_reported_not_hidden():
    lib = L.load()
    h = ctypes.c_void_p()
    p = default_params()
    assert lib.godar_gpu_create(None, 10, 0, ctypes.byref(h)) == 2
    assert lib.godar_gpu_create(ctypes.byref(p), 0, 0, ctypes.byref(h)) == 2
    assert lib.godar_gpu_create(ctypes.byref(p), 10, 7, ctypes.byref(h)) == 2
    assert lib.godar_gpu_errstr(2) == b"bad input"


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(L.GodarError) as e:
        L.Stepper(default_params(), 8)
    assert e.value.status == 10
    # the allocation-free search's set-up call needs a device too
    cnt = ctypes.c_int(-1)
    assert L.load().godar_gpu_candidates_noalloc(None, None, None, 0, 0.0, 0.0, 0.0, 0, None, None, 0,
                                                 ctypes.byref(cnt)) == 10
    assert cnt.value == 0


def test_namelist_reader_group_fallback(tmp_path):
    """read_namelist keeps a whole group at its defaults when the group has a
    variable it does not declare (par_get.f90:184-245)."""
    nml = tmp_path / "n.nml"
    nml.write_text("""&options_nml
    shelter = .false.   ! comment
    ridging = .false.
    /
&numerical_param_nml
    rtree = 999d0
    dt = 2.5d-1
    /
&bond_param_nml
    eb = 1d9
    not_a_bond_variable = 3d0
    /
&forcings_nml
    ua = 4.5d0
    va = -1.0
    /
""")
    p = read_namelist(str(nml))
    d = default_params()
    assert p.shelter == 0 and p.ridging == 0 and p.cohesion == 1
    assert p.rtree == 999.0 and p.dt == 0.25
    assert p.eb == d.eb                      # whole group fell back
    assert p.ua == 4.5 and p.va == -1.0


@pytest.mark.parametrize("case", ["nan_r", "zero_r", "inf_L", "neg_L", "nan_gap", "gap_eats_radius", "rounds"])
def test_place_rejects_bad_inputs_before_touching_a_device(case):
    r = np.array([30.0, 20.0, 10.0])
    kw = dict(Lx=1000.0, Ly=800.0, periodic_x=True, periodic_y=False, seed=3, max_rounds=16, gap=0.0)
    if case == "nan_r":
        r[1] = np.nan
    elif case == "zero_r":
        r[2] = 0.0
    elif case == "inf_L":
        kw["Lx"] = np.inf
    elif case == "neg_L":
        kw["Ly"] = -5.0
    elif case == "nan_gap":
        kw["gap"] = np.nan
    elif case == "gap_eats_radius":
        kw["gap"] = -20.0          # r + gap / 2 = 0 for the smallest disk
    else:
        kw["max_rounds"] = 0
    with pytest.raises(L.GodarError) as e:
        L.place_disks(r, **kw)
    assert e.value.status == 2


def test_place_needs_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(L.GodarError) as e:
        L.place_disks(np.array([30.0, 20.0]), 1000.0, 800.0, True, True, 1, gap=-10.0)
    assert e.value.status == 10


def header_prototypes():
    """name -> (return type, [parameter types]) of every declaration in
    include/godar_gpu.h."""
    text = open(os.path.join(ROOT, "include", "godar_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(godar_\w+)\s*\(([^;{]*?)\)\s*;", text):
        ret = " ".join(m.group(1).split())
        params = [" ".join(p.split()) for p in m.group(3).split(",")]
        if params == ["void"]:
            params = []
        # drop the parameter name, keep the type
        types = [re.sub(r"\s*\b\w+$", "", p) if not p.endswith("*") else p for p in params]
        out[m.group(2)] = (ret, types)
    return out


def _kind_of_c(t: str) -> str:
    if "*" in t:
        return "ptr"
    t = t.replace("const ", "")
    # size_t and uint64_t are both 64-bit unsigned here (ctypes aliases them)
    return {"int": "int", "size_t": "u64", "double": "double", "uint64_t": "u64"}[t]


def _kind_of_ctypes(t) -> str:
    if t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
        return "ptr"
    return {ctypes.c_int: "int", ctypes.c_size_t: "u64", ctypes.c_double: "double",
            ctypes.c_uint64: "u64"}[t]


def test_python_binding_matches_every_prototype():
    """Each ctypes binding in godar_b200/lib.py passes the header's parameter
    kinds (pointer, int, double, 64-bit unsigned) in order, and functions that
    return size_t or a string have their result type set."""
    lib = L.load()
    protos = header_prototypes()
    assert set(protos) == set(header_functions())
    for name, (ret, params) in protos.items():
        fn = getattr(lib, name)
        want = [_kind_of_c(t) for t in params]
        if want:
            assert fn.argtypes is not None, name
            assert [_kind_of_ctypes(t) for t in fn.argtypes] == want, name
        if ret == "size_t":
            assert fn.restype == ctypes.c_size_t, name
        elif ret.endswith("*"):
            assert fn.restype == ctypes.c_char_p, name


def test_calls_on_a_null_handle_are_rejected():
    """Every call on a context or a batch, queued steps and the timing
    switches included, rejects a null handle with GODAR_ERR_BAD_INPUT
    before it touches a device."""
    lib = L.load()
    d = ctypes.c_double(0)
    i64 = (ctypes.c_int64 * 8)()
    n = ctypes.c_size_t(0)
    calls = [
        lambda: lib.godar_gpu_step(None, 1, 0, 1),
        lambda: lib.godar_gpu_step_async(None, 1, 0, 1),
        lambda: lib.godar_gpu_set_diagnostics(None, 1),
        lambda: lib.godar_gpu_stats(None, ctypes.byref(d), i64),
        lambda: lib.godar_gpu_get_floe_field(None, 0, None),
        lambda: lib.godar_gpu_checkpoint(None, None, 0, ctypes.byref(n)),
        lambda: lib.godar_gpu_set_precision(None, 0),
        lambda: lib.godar_batch_step(None, 1),
        lambda: lib.godar_batch_step_async(None, 1),
        lambda: lib.godar_batch_set_diagnostics(None, 1),
        lambda: lib.godar_batch_set_phase_timing(None, 16),
        lambda: lib.godar_batch_phase_stats(None, None, 0, None, None),
        lambda: lib.godar_batch_stats(None, None, None, None, None),
        lambda: lib.godar_batch_sync(None, ctypes.byref(d)),
        lambda: lib.godar_batch_wait(None),
    ]
    for k, call in enumerate(calls):
        assert call() == 2, k
