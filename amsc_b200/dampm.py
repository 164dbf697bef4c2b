"""Python host side of the B200 MPM step, over the C ABI of
``include/dampm_cuda.h`` (``libdampm_cuda.so``, built in-tree).

:class:`Solver` mirrors how the reference drives its step:
``DATA data("DATA.json")`` then the ``while (fixed ? it < NSTEPS : t < T)``
loop of main/optim_par.cpp:281-668 (or main/gpu_offload.cpp:276-575 with
merge/split).  There is no CPU fallback: without the CUDA library or a GPU
every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Iterable, Optional

import numpy as np

from .data import DATA

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdampm_cuda.so")

# names of the persistent state arrays of dampm_set_state / dampm_get_state
STATE_FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "Mp", "Vp", "H")
# particle fields that are always available for download
CORE_FIELDS = STATE_FIELDS + ("F_21", "Ap", "mom_px", "mom_py", "Fb_x", "Fb_y",
                              "label", "level", "xp", "yp", "vpxL", "vpyL")
GRAD_FIELDS = ("vpx_dx", "vpx_dy", "vpy_dx", "vpy_dy")
RECORD_FIELDS = ("apx", "apy", "Zp", "hpZ", "dZxp", "dZyp", "Fpx", "Fpy",
                 "Fric_px", "Fric_py")


class dampm_grid(C.Structure):
    _fields_ = [("Nex", C.c_int), ("Ney", C.c_int), ("hx", C.c_double), ("hy", C.c_double)]


class dampm_params(C.Structure):
    _fields_ = [("g", C.c_double), ("T", C.c_double), ("rho", C.c_double),
                ("xi", C.c_double), ("mu", C.c_double), ("phi", C.c_double),
                ("tauy", C.c_double), ("BINGHAM_ON", C.c_double),
                ("FRICTION_ON", C.c_double), ("CFL", C.c_double),
                ("BC_FLAG", C.c_int), ("MERGE_SPLIT_ON", C.c_int),
                ("eq_level", C.c_double), ("DT_FIXED", C.c_double), ("NSTEPS", C.c_int)]


class dampm_ms_params(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("split_hp_min", C.c_double),
                ("shear_split", C.c_double), ("hp_min", C.c_double), ("max_dv", C.c_double),
                ("min_level", C.c_int), ("max_level", C.c_int),
                ("min_particles_per_cell", C.c_int), ("call_interval", C.c_int),
                ("max_ops", C.c_double), ("pair_dist", C.c_double)]


class DampmError(RuntimeError):
    pass


_lib = None

_DP = C.POINTER(C.c_double)


def _declare(lib):
    P = C.c_void_p
    sig = {
        "dampm_ctx_create": (C.c_int, [C.POINTER(dampm_grid), C.POINTER(dampm_params),
                                       C.POINTER(dampm_ms_params), C.c_int, C.c_longlong,
                                       P, C.POINTER(P)]),
        "dampm_ctx_destroy": (C.c_int, [P]),
        "dampm_upload_terrain": (C.c_int, [P, _DP, _DP, _DP]),
        "dampm_upload_particles": (C.c_int, [P, C.c_longlong] + [_DP] * 10),
        "dampm_step": (C.c_int, [P, C.c_int]),
        "dampm_run": (C.c_int, [P, C.c_longlong, C.c_int, C.POINTER(C.c_longlong)]),
        "dampm_sync": (C.c_int, [P]),
        "dampm_status": (C.c_int, [P, C.POINTER(C.c_int), _DP, _DP, C.POINTER(C.c_longlong)]),
        "dampm_enable_merge_split": (C.c_int, [P, C.c_int]),
        "dampm_merge_split": (C.c_int, [P, C.c_double, C.POINTER(C.c_longlong)]),
        "dampm_set_ms_variant": (C.c_int, [P, C.c_int, C.c_double]),
        "dampm_download": (C.c_int, [P, C.c_char_p, _DP]),
        "dampm_download_nodal": (C.c_int, [P, C.c_char_p, _DP]),
        "dampm_record_outputs": (C.c_int, [P, C.c_int]),
        "dampm_set_graphs": (C.c_int, [P, C.c_int]),
        "dampm_ledgers": (C.c_int, [P, _DP]),
        "dampm_ledger_history": (C.c_int, [P, C.c_longlong, C.c_int, _DP]),
        "dampm_set_state": (C.c_int, [P, C.c_longlong, C.POINTER(_DP)] + [_DP] * 5),
        "dampm_get_state": (C.c_int, [P, C.POINTER(_DP)]),
        "dampm_last_launch_count": (C.c_longlong, [P]),
        "dampm_last_timings": (C.c_int, [P, C.c_int, _DP]),
        "dampm_last_error": (C.c_char_p, [P]),
        "dampm_version": (C.c_char_p, []),
        "dampm_batch_create": (C.c_int, [C.c_longlong, C.c_longlong, C.c_int, C.c_int, P,
                                         C.POINTER(P)]),
        "dampm_batch_destroy": (C.c_int, [P]),
        "dampm_batch_add": (C.c_int, [P, C.POINTER(dampm_grid), C.POINTER(dampm_params), _DP,
                                      C.c_longlong] + [_DP] * 10 + [C.POINTER(C.c_int)]),
        "dampm_batch_remove": (C.c_int, [P, C.c_int]),
        "dampm_batch_compact": (C.c_int, [P]),
        "dampm_batch_step": (C.c_int, [P, C.c_int]),
        "dampm_batch_sync": (C.c_int, [P]),
        "dampm_batch_query": (C.c_int, [P, C.c_int, C.POINTER(C.c_int), _DP, _DP,
                                        C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
        "dampm_batch_download": (C.c_int, [P, C.c_int, C.c_char_p, _DP]),
        "dampm_batch_ledgers": (C.c_int, [P, C.c_int, _DP]),
        "dampm_batch_usage": (C.c_int, [P, C.POINTER(C.c_longlong)]),
        "dampm_batch_states": (C.c_int, [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), _DP, C.POINTER(C.c_int)]),
        "dampm_batch_last_error": (C.c_char_p, [P]),
        "dampm_batch_tune": (C.c_int, [P, C.c_int, C.c_int, C.c_int]),
        "dampm_stage_download": (C.c_int, [P, C.c_int, C.POINTER(C.c_char_p), C.POINTER(_DP),
                                           C.POINTER(C.c_longlong)]),
        "dampm_staged_wait": (C.c_int, [P]),
        "dampm_slab_record_doubles": (C.c_int, []),
        "dampm_slab_set": (C.c_int, [P, C.c_int, C.c_int]),
        "dampm_slab_set_index": (C.c_int, [P, C.POINTER(C.c_int)]),
        "dampm_slab_pass": (C.c_int, [P, C.c_int]),
        "dampm_slab_node_column": (C.c_int, [P, C.c_int, P, C.c_int]),
        "dampm_slab_cfl": (C.c_int, [P, _DP, C.c_int]),
        "dampm_slab_route": (C.c_int, [P, P, P, C.c_longlong, C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_longlong)]),
        "dampm_slab_ghosts": (C.c_int, [P, P, C.c_longlong, C.POINTER(C.c_longlong)]),
        "dampm_slab_import": (C.c_int, [P, P, C.c_longlong, C.c_int]),
        "dampm_slab_download": (C.c_int, [P, C.c_char_p, _DP, C.POINTER(C.c_longlong)]),
        "dampm_json_read": (C.c_int, [C.c_char_p, C.POINTER(P)]),
        "dampm_json_size": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_longlong)]),
        "dampm_json_kind": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_int)]),
        "dampm_json_get": (C.c_int, [P, C.c_char_p, _DP]),
        "dampm_json_error": (C.c_char_p, [P]),
        "dampm_json_free": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def load_library(path: str = LIB_PATH):
    """Loads libdampm_cuda.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise DampmError(f"{path} missing: build it with `python -m amsc_b200.build`")
        _lib = _declare(C.CDLL(path))
    return _lib


def pinned_array(n: int) -> np.ndarray:
    """A float64 array in page-locked host memory (device-to-host copies into
    it run asynchronously); plain memory where no CUDA device is present."""
    import torch
    if torch.cuda.is_available():
        return torch.empty(int(n), dtype=torch.float64, pin_memory=True).numpy()
    return np.empty(int(n), dtype=np.float64)


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_DP)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def make_structs(d: DATA):
    s = d.scalars
    g = dampm_grid(int(s["Nex"]), int(s["Ney"]), float(s["hx"]), float(s["hy"]))
    p = dampm_params(float(s["g"]), float(s["T"]), float(s["rho"]), float(s["xi"]),
                     float(s["mu"]), float(s["phi"]), float(s["tauy"]),
                     float(s["BINGHAM_ON"]), float(s["FRICTION_ON"]), float(s["CFL"]),
                     int(s["BC_FLAG"]), int(s["MERGE_SPLIT_ON"]), float(s["eq_level"]),
                     float(s.get("DT_FIXED", 0.0)), int(s.get("NSTEPS", 0)))
    m = dampm_ms_params(float(s["ms_alpha"]), float(s["ms_beta"]),
                        float(s["ms_split_hp_min"]), float(s["ms_shear_split"]),
                        float(s["ms_hp_min"]), float(s["ms_max_dv"]),
                        int(s["ms_min_level"]), int(s["ms_max_level"]),
                        int(s["ms_min_particles_per_cell"]), int(s["ms_call_interval"]),
                        float(s["ms_max_ops"]), float(s.get("ms_pair_dist", 0.0)))
    return g, p, m


class Solver:
    """One scenario resident on the GPU.

    ``merge_split=True`` applies ``adaptive_merge_split`` at the
    gpu_offload cadence (every ms_call_interval steps, main/gpu_offload.cpp
    :321) when the DATA's MERGE_SPLIT_ON is set; the default follows
    optim_par, which never splits or merges.
    """

    def __init__(self, d: DATA, capacity: int = 0, merge_split: bool = False,
                 record: bool = False, stream: Optional[int] = None):
        self.lib = load_library()
        self.data = d
        d.validate()
        self.nn = d.nnodes
        g, p, m = make_structs(d)
        h = C.c_void_p()
        rc = self.lib.dampm_ctx_create(C.byref(g), C.byref(p), C.byref(m), 0,
                                       int(capacity), C.c_void_p(stream or 0), C.byref(h))
        if rc != 0:
            raise DampmError(f"dampm_ctx_create failed ({rc})")
        self.h = h
        self._keep = [g, p, m]
        self._check(self.lib.dampm_enable_merge_split(self.h, 1 if merge_split else 0))
        # the ELFS merge/split variant (DATA key ms_variant = 1)
        if int(d.scalars.get("ms_variant", 0)) != 0:
            self._check(self.lib.dampm_set_ms_variant(
                self.h, int(d.scalars["ms_variant"]),
                float(d.scalars.get("ms_stretch_thresh", 1e7))))
        self._check(self.lib.dampm_record_outputs(self.h, 1 if record else 0))
        A = d.arrays
        self._check(self.lib.dampm_upload_terrain(self.h, _ptr(_f64(A["Z"])),
                                                  _ptr(_f64(A["dZdx"])),
                                                  _ptr(_f64(A["dZdy"]))))
        arrs = [_f64(A[k]) for k in ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp",
                                     "mom_px", "mom_py", "Vp")]
        self._check(self.lib.dampm_upload_particles(self.h, d.np, *[_ptr(a) for a in arrs]))

    # -- plumbing -------------------------------------------------------------
    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.dampm_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise DampmError(f"dampm call failed ({rc}): {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.dampm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- stepping -------------------------------------------------------------
    def set_graphs(self, enable: bool):
        """Runs of 16 identical passes replay a CUDA graph (default) or, with
        False, every pass is launched plainly; the results are the same."""
        self._check(self.lib.dampm_set_graphs(self.h, 1 if enable else 0))

    def step(self, n: int = 1):
        """Enqueues n passes of the loop body (asynchronous)."""
        self._check(self.lib.dampm_step(self.h, int(n)))

    def run(self, max_steps: int = 1 << 40, chunk: int = 64) -> int:
        """Runs while the reference loop condition holds; returns passes done."""
        done = C.c_longlong()
        self._check(self.lib.dampm_run(self.h, int(max_steps), int(chunk), C.byref(done)))
        return int(done.value)

    def sync(self):
        self._check(self.lib.dampm_sync(self.h))

    def _status(self):
        it = C.c_int()
        t = C.c_double()
        dt = C.c_double()
        n = C.c_longlong()
        rc = self.lib.dampm_status(self.h, C.byref(it), C.byref(t), C.byref(dt), C.byref(n))
        return rc, {"it": it.value, "t": t.value, "dt": dt.value, "np": int(n.value)}

    def status(self) -> Dict[str, float]:
        """Loop state; raises when the device status word is set (the run
        diverged or merge/split ran out of capacity)."""
        rc, st = self._status()
        self._check(rc)
        return st

    @property
    def failed(self) -> bool:
        """True once the device status word stopped the run."""
        return self._status()[0] == -5

    @property
    def num_particles(self) -> int:
        rc, st = self._status()
        if rc not in (0, -5):  # a diverged run still has its particles
            self._check(rc)
        return st["np"]

    def merge_split(self, dt: float):
        counts = (C.c_longlong * 4)()
        self._check(self.lib.dampm_merge_split(self.h, float(dt), counts))
        return [int(c) for c in counts]

    # -- data out -------------------------------------------------------------
    def download(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self.num_particles
        if out is None:
            out = np.empty(n, dtype=np.float64)
        self._check(self.lib.dampm_download(self.h, name.encode(), _ptr(out)))
        return out

    def stage_download(self, out: Dict[str, np.ndarray]) -> int:
        """Starts copying the named particle fields into the given float64
        arrays and returns at once; steps enqueued afterwards run meanwhile
        when the arrays are page-locked (pinned_array).  Call staged_wait()
        before reading them.  Returns the count of values each receives."""
        names = list(out)
        for k in names:
            a = out[k]
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size < self.num_particles:
                raise ValueError(f"{k}: needs a contiguous float64 array of >= np values")
        self._staged = [out[k] for k in names]  # kept alive until the copies end
        fields = (C.c_char_p * len(names))(*[k.encode() for k in names])
        ptrs = (_DP * len(names))(*[_ptr(out[k]) for k in names])
        n = C.c_longlong()
        self._check(self.lib.dampm_stage_download(self.h, len(names), fields, ptrs,
                                                  C.byref(n)))
        return int(n.value)

    def staged_wait(self):
        self._check(self.lib.dampm_staged_wait(self.h))
        self._staged = None

    def download_nodal(self, name: str) -> np.ndarray:
        out = np.empty(self.nn, dtype=np.float64)
        self._check(self.lib.dampm_download_nodal(self.h, name.encode(), _ptr(out)))
        return out

    def fields(self, names: Iterable[str]) -> Dict[str, np.ndarray]:
        return {k: self.download(k) for k in names}

    def ledger_history(self, first_it: int, n: int) -> np.ndarray:
        """Rows {t, err_mass, err_mom} of steps first_it .. first_it+n-1."""
        out = np.empty((n, 3), dtype=np.float64)
        self._check(self.lib.dampm_ledger_history(self.h, int(first_it), int(n), _ptr(out)))
        return out

    def ledgers(self) -> np.ndarray:
        out = np.empty(9, dtype=np.float64)
        self._check(self.lib.dampm_ledgers(self.h, _ptr(out)))
        return out

    def set_state(self, state: Dict[str, np.ndarray], fresh: Optional[Dict[str, np.ndarray]] = None):
        arrs = [_f64(state[k]) for k in STATE_FIELDS]
        ptrs = (_DP * 11)(*[_ptr(a) for a in arrs])
        fr = [None] * 5
        if fresh is not None:
            fr = [_f64(fresh[k]) for k in ("Ap", "mom_px", "mom_py", "Fb_x", "Fb_y")]
        self._keep_state = (arrs, fr)
        self._check(self.lib.dampm_set_state(self.h, arrs[0].shape[0], ptrs,
                                             *[_ptr(a) for a in fr]))

    def get_state(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        n = self.num_particles
        if out is None:
            out = {k: np.empty(n, dtype=np.float64) for k in STATE_FIELDS}
        ptrs = (_DP * 11)(*[_ptr(out[k]) for k in STATE_FIELDS])
        self._check(self.lib.dampm_get_state(self.h, ptrs))
        return out

    def last_launch_count(self) -> int:
        return int(self.lib.dampm_last_launch_count(self.h))

    def timings(self, enable: bool = True) -> np.ndarray:
        out = np.zeros(5, dtype=np.float64)
        self._check(self.lib.dampm_last_timings(self.h, 1 if enable else 0, _ptr(out)))
        return out
