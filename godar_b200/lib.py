"""ctypes binding of libgodar_gpu.so (the C ABI in include/godar_gpu.h).

This is the host-side mirror of the reference's step interface: a
:class:`Stepper` wraps one floe field and is advanced the way GODAR's driver
calls ``stepper(tstep, restart)`` (model/src/godar.f90:191-193); a
:class:`Batch` advances many fields together.  There is no CPU fallback: if
the CUDA library cannot be loaded or no GPU is visible, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import GodarParams, PREC_FP64, PREC_MIXED

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgodar_gpu.so")

FLOE_FIELDS = ["x", "y", "u", "v", "r", "h", "theta", "omega", "tfx", "tfy", "fcx", "fcy",
               "fbx", "fby", "m", "mc", "mb", "tsigxx", "tsigyy", "tsigxy", "tsigyx", "tp"]
FIELD_ID = {k: i for i, k in enumerate(FLOE_FIELDS)}
P_CANDIDATES, P_CONTACTS, P_BONDS = 0, 1, 2

EXPORTS = [
    "godar_gpu_version", "godar_gpu_errstr", "godar_gpu_last_error", "godar_gpu_params_size",
    "godar_gpu_default_params", "godar_gpu_derive_params", "godar_gpu_create", "godar_gpu_upload",
    "godar_gpu_set_field", "godar_gpu_step", "godar_gpu_step_async", "godar_gpu_get_floe_field", "godar_gpu_get_pairs",
    "godar_gpu_download", "godar_gpu_place", "godar_gpu_write_posts", "godar_gpu_clear_posts", "godar_posts_format_reals",
    "godar_gpu_set_precision", "godar_gpu_checkpoint", "godar_gpu_restore", "godar_gpu_stats", "godar_gpu_destroy", "godar_batch_create", "godar_batch_instance_bytes",
    "godar_batch_add", "godar_batch_remove", "godar_batch_step", "godar_batch_step_async", "godar_batch_sync",
    "godar_batch_get_floe_field", "godar_batch_steps_done", "godar_batch_count",
    "godar_batch_bytes_in_use", "godar_batch_set_uniform_forcing", "godar_batch_get_all",
    "godar_batch_stats", "godar_batch_phase_stats", "godar_batch_set_phase_timing", "godar_batch_launch_config", "godar_batch_prepare", "godar_batch_reserve", "godar_batch_rebuild_stats",
    "godar_batch_set_diagnostics", "godar_gpu_set_diagnostics", "godar_batch_get_all_async", "godar_batch_summary_async", "godar_batch_wait",
    "godar_batch_destroy",
    "godar_gpu_candidates_noalloc",
]


NPHASES = 5


class GodarError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"godar status {status}: {msg}")
        self.status = status


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


def load():
    """Loads libgodar_gpu.so (built in-tree by godar_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing; run `python -m godar_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.godar_gpu_version.restype = ctypes.c_char_p
    L.godar_gpu_errstr.restype = ctypes.c_char_p
    L.godar_gpu_errstr.argtypes = [ctypes.c_int]
    L.godar_gpu_last_error.restype = ctypes.c_char_p
    L.godar_gpu_create.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.godar_gpu_upload.argtypes = [vp] + [_dp] * 8 + [ctypes.c_int, _ip, _ip, _dp]
    L.godar_gpu_set_field.argtypes = [vp, _dp]
    L.godar_gpu_step.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.godar_gpu_step_async.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.godar_gpu_get_floe_field.argtypes = [vp, ctypes.c_int, _dp]
    L.godar_gpu_get_pairs.argtypes = [vp, ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.godar_gpu_stats.argtypes = [vp, _dp, ctypes.POINTER(ctypes.c_int64)]
    L.godar_gpu_download.argtypes = [vp, vp, ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.godar_gpu_set_precision.argtypes = [vp, ctypes.c_int]
    L.godar_gpu_checkpoint.argtypes = [vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    L.godar_gpu_restore.argtypes = [vp, vp, ctypes.c_size_t]
    L.godar_gpu_destroy.argtypes = [vp]
    L.godar_gpu_default_params.argtypes = [vp]
    L.godar_gpu_derive_params.argtypes = [vp]
    L.godar_batch_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(vp)]
    L.godar_batch_instance_bytes.restype = ctypes.c_size_t
    L.godar_batch_instance_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
    L.godar_batch_add.argtypes = ([vp, vp, ctypes.c_int] + [_dp] * 8 + [ctypes.c_int, _ip, _ip, _dp, _dp,
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_int)])
    L.godar_batch_remove.argtypes = [vp, ctypes.c_int]
    L.godar_batch_step.argtypes = [vp, ctypes.c_int]
    L.godar_batch_step_async.argtypes = [vp, ctypes.c_int]
    L.godar_batch_sync.argtypes = [vp, _dp]
    L.godar_batch_get_floe_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, _dp]
    L.godar_batch_steps_done.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    L.godar_batch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]
    L.godar_batch_bytes_in_use.restype = ctypes.c_size_t
    L.godar_batch_bytes_in_use.argtypes = [vp]
    L.godar_batch_destroy.argtypes = [vp]
    L.godar_batch_set_uniform_forcing.argtypes = [vp, _dp]
    L.godar_batch_get_all.argtypes = [vp, ctypes.c_int, _dp]
    L.godar_batch_stats.argtypes = [vp, _dp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                    ctypes.POINTER(ctypes.c_int64)]
    L.godar_batch_phase_stats.argtypes = [vp, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int64)]
    L.godar_batch_set_phase_timing.argtypes = [vp, ctypes.c_int]
    L.godar_batch_launch_config.argtypes = [vp, _ip, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_int64)]
    L.godar_batch_prepare.argtypes = [vp, ctypes.c_int]
    L.godar_gpu_write_posts.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_double]
    L.godar_gpu_clear_posts.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    L.godar_gpu_place.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_uint64, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                  ctypes.POINTER(ctypes.c_int)]
    L.godar_posts_format_reals.argtypes = [_dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t)]
    L.godar_batch_reserve.argtypes = [vp, ctypes.c_size_t]
    L.godar_batch_rebuild_stats.argtypes = [vp, _dp] + [ctypes.POINTER(ctypes.c_int64)] * 3
    L.godar_batch_set_diagnostics.argtypes = [vp, ctypes.c_int]
    L.godar_batch_get_all_async.argtypes = [vp, ctypes.c_int, _ip, vp]
    L.godar_batch_wait.argtypes = [vp]
    L.godar_batch_summary_async.argtypes = [vp, vp]
    L.godar_gpu_set_diagnostics.argtypes = [vp, ctypes.c_int]
    L.godar_gpu_candidates_noalloc.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_int, vp, vp, ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_int)]
    if L.godar_gpu_params_size() != ctypes.sizeof(GodarParams):
        raise RuntimeError("godar_params layout differs between the library and params.py")
    _lib = L
    return L


def _check(st: int):
    if st != 0:
        L = load()
        raise GodarError(st, f"{L.godar_gpu_errstr(st).decode()}: {L.godar_gpu_last_error().decode()}")


def _arr(a, n=None, dtype=np.float64):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=dtype)
    if n is not None and a.shape[0] != n:
        raise ValueError("array length mismatch")
    return a


def _ptr(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def _bond_arrays(bonds, damage):
    if bonds is None or len(bonds) == 0:
        return 0, None, None, None
    b = np.asarray(bonds, dtype=np.int32).reshape(-1, 2)
    bi = np.ascontiguousarray(b[:, 0])
    bj = np.ascontiguousarray(b[:, 1])
    d = _arr(damage) if damage is not None else None
    return len(b), bi, bj, d


def _field_array(params: GodarParams, field):
    if field is None:
        return None
    f = np.ascontiguousarray(field, dtype=np.float64).reshape(-1)
    if f.size != 4 * params.field_nx * params.field_ny:
        raise ValueError("forcing grid size does not match field_nx * field_ny")
    return f


class Stepper:
    """One floe field on the GPU, advanced like ``call stepper(tstep, restart)``."""

    def __init__(self, params: GodarParams, n: int, precision: int = PREC_FP64):
        L = load()
        self.params = params
        self.n = n
        self._h = ctypes.c_void_p()
        _check(L.godar_gpu_create(ctypes.byref(params), n, precision, ctypes.byref(self._h)))
        self._keep = []

    def upload(self, x, y, r, h, theta=None, omega=None, u=None, v=None, bonds=None, damage=None):
        n = self.n
        arrs = [_arr(a, n) for a in (x, y, r, h, theta, omega, u, v)]
        nb, bi, bj, d = _bond_arrays(bonds, damage)
        _check(load().godar_gpu_upload(self._h, *[_ptr(a) for a in arrs], nb, _ptr(bi, _ip), _ptr(bj, _ip), _ptr(d)))

    def set_field(self, field):
        f = _field_array(self.params, field)
        _check(load().godar_gpu_set_field(self._h, _ptr(f)))

    def step(self, tstep: int, restart: int = 0, nsteps: int = 1):
        _check(load().godar_gpu_step(self._h, tstep, restart, nsteps))

    def step_async(self, tstep: int, restart: int = 0, nsteps: int = 1):
        """Queues the steps and returns; an error of a queued step is raised
        by the next call on this stepper."""
        _check(load().godar_gpu_step_async(self._h, tstep, restart, nsteps))

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        _check(load().godar_gpu_get_floe_field(self._h, FIELD_ID[name], _ptr(out)))
        return out

    def floes(self, names=None) -> dict:
        return {k: self.field(k) for k in (names or FLOE_FIELDS)}

    def set_diagnostics(self, on: bool):
        _check(load().godar_gpu_set_diagnostics(self._h, 1 if on else 0))

    def checkpoint(self) -> bytes:
        """The field's complete state as bytes (godar_gpu_checkpoint)."""
        n = ctypes.c_size_t(0)
        L = load()
        _check(L.godar_gpu_checkpoint(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(L.godar_gpu_checkpoint(self._h, buf, n.value, ctypes.byref(n)))
        return buf.raw[:n.value]

    def restore(self, data: bytes):
        """Loads a checkpoint (then step on with restart = 1)."""
        buf = ctypes.create_string_buffer(data, len(data))
        _check(load().godar_gpu_restore(self._h, buf, len(data)))

    def set_precision(self, precision: int):
        _check(load().godar_gpu_set_precision(self._h, precision))

    def download(self, names=None, which: int = -1):
        """Per-floe outputs (all, or `names`) and optionally one pair list in
        one call (godar_gpu_download)."""
        names = list(names or FLOE_FIELDS)
        outs = {k: np.empty(self.n, dtype=np.float64) for k in names}
        ptrs = (ctypes.c_void_p * len(FLOE_FIELDS))()
        for k, a in outs.items():
            ptrs[FIELD_ID[k]] = a.ctypes.data
        cnt = ctypes.c_int(0)
        L = load()
        if which < 0:
            _check(L.godar_gpu_download(self._h, ptrs, -1, None, None, None, 0, ctypes.byref(cnt)))
            return outs, None
        _check(L.godar_gpu_download(self._h, ptrs, which, None, None, None, 0, ctypes.byref(cnt)))
        m = cnt.value
        pi = np.empty(max(m, 1), np.int32)
        pj = np.empty(max(m, 1), np.int32)
        val = np.empty(max(m, 1), np.float64)
        _check(L.godar_gpu_download(self._h, None, which, _ptr(pi, _ip), _ptr(pj, _ip), _ptr(val), m,
                                    ctypes.byref(cnt)))
        return outs, (pi[:m], pj[:m], val[:m])

    def write_posts(self, dir: str | None, expno: str, tstep: int, comp: float):
        """Appends one output step to the reference's text files
        (sea_ice_post) in `dir` (None: "output")."""
        _check(load().godar_gpu_write_posts(self._h, dir.encode() if dir else None, expno.encode(), int(tstep),
                                            float(comp)))

    def pairs(self, which: int):
        L = load()
        cnt = ctypes.c_int(0)
        _check(L.godar_gpu_get_pairs(self._h, which, None, None, None, 0, ctypes.byref(cnt)))
        m = cnt.value
        pi = np.empty(max(m, 1), np.int32)
        pj = np.empty(max(m, 1), np.int32)
        val = np.empty(max(m, 1), np.float64)
        _check(L.godar_gpu_get_pairs(self._h, which, _ptr(pi, _ip), _ptr(pj, _ip), _ptr(val), m, ctypes.byref(cnt)))
        return pi[:m], pj[:m], val[:m]

    def stats(self):
        ms = ctypes.c_double(0)
        c = (ctypes.c_int64 * 4)()
        _check(load().godar_gpu_stats(self._h, ctypes.byref(ms), c))
        return ms.value, {"candidates": c[0], "contacts": c[1], "bonds": c[2], "plastic": c[3]}

    def close(self):
        if self._h:
            load().godar_gpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many floe fields advanced together on one GPU, admitted against an
    HBM budget (bytes; 0 = unlimited)."""

    def __init__(self, precision: int = PREC_MIXED, hbm_budget: int = 0):
        L = load()
        self._h = ctypes.c_void_p()
        _check(L.godar_batch_create(precision, hbm_budget, ctypes.byref(self._h)))
        self.sizes = {}

    @staticmethod
    def instance_bytes(n: int, nb: int = 0) -> int:
        return int(load().godar_batch_instance_bytes(n, nb))

    def add(self, params: GodarParams, x, y, r, h, theta=None, omega=None, u=None, v=None,
            bonds=None, damage=None, field=None, restart: int = 0) -> int:
        n = len(x)
        arrs = [_arr(a, n) for a in (x, y, r, h, theta, omega, u, v)]
        nb, bi, bj, d = _bond_arrays(bonds, damage)
        f = _field_array(params, field)
        hid = ctypes.c_int(-1)
        _check(load().godar_batch_add(self._h, ctypes.byref(params), n, *[_ptr(a) for a in arrs], nb,
                                      _ptr(bi, _ip), _ptr(bj, _ip), _ptr(d), _ptr(f), restart, ctypes.byref(hid)))
        self.sizes[hid.value] = n
        return hid.value

    def add_field(self, fld, restart: int = 0) -> int:
        """Adds a godar_b200.generators.Field."""
        return self.add(fld.params, fld.x, fld.y, fld.r, fld.h, fld.theta, fld.omega, fld.u, fld.v,
                        fld.bonds, fld.damage, fld.forcing, restart)

    def remove(self, hid: int):
        _check(load().godar_batch_remove(self._h, hid))
        self.sizes.pop(hid, None)

    def step(self, nsteps: int = 1):
        _check(load().godar_batch_step(self._h, nsteps))

    def step_async(self, nsteps: int = 1):
        """Queues nsteps time steps without waiting (godar_batch_step_async);
        an error of a queued step is raised by the next call."""
        _check(load().godar_batch_step_async(self._h, nsteps))

    def get_all_async(self, names, outs):
        """Queues the read-back of state fields `names` of every instance into
        `outs` (pinned float64 arrays); valid after wait()."""
        ids = (ctypes.c_int32 * len(names))(*[FIELD_ID[k] for k in names])
        ptrs = (ctypes.c_void_p * len(names))(*[o.ctypes.data for o in outs])
        # two read-backs can be in flight: keep both calls' arguments alive
        self._async_keep = [getattr(self, "_async_keep", [None])[-1], (ids, ptrs, outs)]
        _check(load().godar_batch_get_all_async(self._h, len(names), ids, ptrs))

    def summary_async(self, out):
        """Queues a per-instance summary of the current state into `out`
        (a pinned float64 array of 4 x instances: momentum x, y, kinetic
        energy, largest speed, in admission order); valid after wait()."""
        self._async_keep = [getattr(self, "_async_keep", [None])[-1], (out,)]
        _check(load().godar_batch_summary_async(self._h, out.ctypes.data))

    def summary(self) -> np.ndarray:
        """The per-instance summary, synchronously: an array (instances, 4)."""
        n = len(self.sizes)
        out = np.zeros(4 * max(n, 1))
        self.summary_async(out)
        self.wait()
        return out[:4 * n].reshape(n, 4)

    def wait(self):
        _check(load().godar_batch_wait(self._h))

    def set_diagnostics(self, on: bool):
        """Diagnostics on the last step of each step call (default on)."""
        _check(load().godar_batch_set_diagnostics(self._h, 1 if on else 0))

    def set_phase_timing(self, every: int):
        """Time the kernels of every `every`-th step of each chunk with CUDA
        events (0, the default: none beyond the autotuner's steps)."""
        _check(load().godar_batch_set_phase_timing(self._h, int(every)))

    def prepare(self, nsteps: int):
        """Captures the CUDA graphs of the next step(nsteps) ahead of time."""
        _check(load().godar_batch_prepare(self._h, nsteps))

    def reserve(self, nbytes: int):
        """Grows the batch's device memory pool to at least nbytes, so that a
        serving loop's admissions and relayouts do not reach the CUDA driver's
        allocator."""
        _check(load().godar_batch_reserve(self._h, int(nbytes)))

    def launch_config(self) -> dict:
        """Block size and variant of each step kernel (see
        godar_batch_launch_config) and whether CUDA graphs are in use."""
        st = self.stats()
        return {"blocks": [c & 0xffff for c in st["blocks"]], "variants": [c >> 16 for c in st["blocks"]],
                "graphs": st["graphs"]}

    def sync(self) -> float:
        ms = ctypes.c_double(0)
        _check(load().godar_batch_sync(self._h, ctypes.byref(ms)))
        return ms.value

    def field(self, hid: int, name: str) -> np.ndarray:
        out = np.empty(self.sizes[hid], dtype=np.float64)
        _check(load().godar_batch_get_floe_field(self._h, hid, FIELD_ID[name], _ptr(out)))
        return out

    def steps_done(self, hid: int) -> int:
        s = ctypes.c_int64(0)
        _check(load().godar_batch_steps_done(self._h, hid, ctypes.byref(s)))
        return s.value

    def count(self):
        ni = ctypes.c_int(0)
        nf = ctypes.c_int64(0)
        _check(load().godar_batch_count(self._h, ctypes.byref(ni), ctypes.byref(nf)))
        return ni.value, nf.value

    def bytes_in_use(self) -> int:
        return int(load().godar_batch_bytes_in_use(self._h))

    def set_uniform_forcing(self, uvw):
        a = np.ascontiguousarray(uvw, dtype=np.float64).reshape(-1)
        _check(load().godar_batch_set_uniform_forcing(self._h, _ptr(a)))

    def get_all(self, name: str, out=None) -> np.ndarray:
        _, nf = self.count()
        if out is None:
            out = np.empty(nf, dtype=np.float64)
        _check(load().godar_batch_get_all(self._h, FIELD_ID[name], _ptr(out)))
        return out

    def stats(self) -> dict:
        ms = ctypes.c_double(0)
        la = ctypes.c_int64(0)
        rb = ctypes.c_int64(0)
        c = (ctypes.c_int64 * 4)()
        _check(load().godar_batch_stats(self._h, ctypes.byref(ms), ctypes.byref(la), ctypes.byref(rb), c))
        ph = (ctypes.c_double * NPHASES)()
        kl = ctypes.c_int64(0)
        ts = ctypes.c_int64(0)
        _check(load().godar_batch_phase_stats(self._h, ph, NPHASES, ctypes.byref(kl), ctypes.byref(ts)))
        bl = (ctypes.c_int32 * NPHASES)()
        go = ctypes.c_int32(0)
        gl = ctypes.c_int64(0)
        _check(load().godar_batch_launch_config(self._h, bl, NPHASES, ctypes.byref(go), ctypes.byref(gl)))
        return {"kernel_ms": ms.value, "launches": la.value, "rebuilds": rb.value,
                "candidates": c[0], "contacts": c[1], "bonds": c[2], "plastic": c[3],
                "phase_ms": list(ph), "kernel_launches": kl.value, "timed_steps": ts.value,
                "blocks": [c & 0xffff for c in bl],
                "variants": [c >> 16 for c in bl],
                "graphs": bool(go.value), "graph_launches": gl.value, **self._rebuild_stats()}

    def _rebuild_stats(self) -> dict:
        ms = ctypes.c_double(0)
        rb, pr, cl = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        _check(load().godar_batch_rebuild_stats(self._h, ctypes.byref(ms), ctypes.byref(rb), ctypes.byref(pr),
                                                ctypes.byref(cl)))
        return {"rebuild_ms": ms.value, "pairs": pr.value, "contact_list": cl.value}

    def close(self):
        if self._h:
            load().godar_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def clear_posts(dir: str | None, expno: str):
    """Deletes an experiment's output files (clear_posts)."""
    _check(load().godar_gpu_clear_posts(dir.encode() if dir else None, expno.encode()))


def format_reals(values) -> str:
    """One list-directed output record of REAL(8) values, as the output files
    hold it."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    n = ctypes.c_size_t(0)
    L = load()
    _check(L.godar_posts_format_reals(_ptr(v), len(v), None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    _check(L.godar_posts_format_reals(_ptr(v), len(v), buf, n.value + 1, ctypes.byref(n)))
    return buf.value.decode()


def place_disks(r, Lx: float, Ly: float, periodic_x: bool, periodic_y: bool, seed: int,
                max_rounds: int = 256, gap: float = 0.0):
    """Non-overlapping disk centres on the GPU (godar_gpu_place); NaN for
    disks that found no place.  Returns x, y and the number placed."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    x = np.empty_like(r)
    y = np.empty_like(r)
    placed = ctypes.c_int(0)
    _check(load().godar_gpu_place(len(r), _ptr(r), float(Lx), float(Ly), int(periodic_x), int(periodic_y),
                                  int(seed) & 0xFFFFFFFFFFFFFFFF, int(max_rounds), float(gap), _ptr(x), _ptr(y),
                                  ctypes.byref(placed)))
    return x, y, placed.value

