"""Batches of independent scenarios on one GPU (``dampm_batch_*``).

Each scenario keeps its own grid, terrain, particles, physics and loop
(fixed dt for NSTEPS passes or CFL until T); one launch per kernel advances
all of them.  A scenario's numbers are the same alone (``Solver``) and in a
batch.  The reference runs one DATA per process (main/optim_par.cpp:128-682);
this is that loop body applied to many scenarios at once.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, Optional

import numpy as np

from .data import DATA
from .dampm import DampmError, _f64, _ptr, load_library, make_structs

BATCH_FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "Mp", "Vp", "H",
                "mom_px", "mom_py")


class Batch:
    """A set of scenarios resident in HBM, stepped together."""

    def __init__(self, particle_cap: int, node_cap: int, scenario_cap: int,
                 stream: Optional[int] = None, precision: str = "fp64"):
        """precision "fp64" is the plain path; "fp32" keeps particle and
        nodal fields in FP32 with compensated nodal sums (terrain, the
        well-balanced depth terms, ledgers and time stay FP64)."""
        self.lib = load_library()
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision is fp64 or fp32")
        self.precision = precision
        h = C.c_void_p()
        rc = self.lib.dampm_batch_create(int(particle_cap), int(node_cap), int(scenario_cap),
                                         1 if precision == "fp32" else 0,
                                         C.c_void_p(stream or 0), C.byref(h))
        if rc != 0:
            raise DampmError(f"dampm_batch_create failed ({rc})")
        self.h = h
        self.np: Dict[int, int] = {}
        self._tuning = (2, 192)  # the library's defaults

    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.dampm_batch_last_error(self.h).decode() if self.h else ""
            raise DampmError(f"dampm batch call failed ({rc}): {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.dampm_batch_destroy(self.h)
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

    @staticmethod
    def footprint(d: DATA) -> Dict[str, int]:
        """Capacity a scenario takes: particles and nodes."""
        return {"particles": d.np, "nodes": d.nnodes}

    def add(self, d: DATA) -> int:
        d.validate()
        g, p, _ = make_structs(d)
        A = d.arrays
        arrs = [_f64(A[k]) for k in ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp", "mom_px",
                                     "mom_py", "Vp")]
        Z = _f64(A["Z"])
        handle = C.c_int()
        self._check(self.lib.dampm_batch_add(self.h, C.byref(g), C.byref(p), _ptr(Z), d.np,
                                             *[_ptr(a) for a in arrs], C.byref(handle)))
        self.np[handle.value] = d.np
        return handle.value

    def remove(self, handle: int):
        self._check(self.lib.dampm_batch_remove(self.h, int(handle)))
        self.np.pop(handle, None)

    def compact(self):
        self._check(self.lib.dampm_batch_compact(self.h))

    def step(self, n: int = 1):
        self._check(self.lib.dampm_batch_step(self.h, int(n)))

    def sync(self):
        self._check(self.lib.dampm_batch_sync(self.h))

    def query(self, handle: int) -> Dict[str, float]:
        it, t, dt, run, np_ = C.c_int(), C.c_double(), C.c_double(), C.c_int(), C.c_longlong()
        self._check(self.lib.dampm_batch_query(self.h, int(handle), C.byref(it), C.byref(t),
                                               C.byref(dt), C.byref(run), C.byref(np_)))
        return {"it": it.value, "t": t.value, "dt": dt.value, "running": bool(run.value),
                "np": np_.value}

    def download(self, handle: int, name: str) -> np.ndarray:
        out = np.empty(self.np[handle], dtype=np.float64)
        self._check(self.lib.dampm_batch_download(self.h, int(handle), name.encode(), _ptr(out)))
        return out

    def ledgers(self, handle: int) -> np.ndarray:
        out = np.empty(9, dtype=np.float64)
        self._check(self.lib.dampm_batch_ledgers(self.h, int(handle), _ptr(out)))
        return out

    def tune(self, units_per_cta: int = 0, col_weight: int = 0, graphs: Optional[bool] = None):
        """P2G units per CTA, column weight of the unit plan, CUDA-graph
        replay of multi-pass steps (0 / None keeps a setting)."""
        g = -1 if graphs is None else (1 if graphs else 0)
        self._check(self.lib.dampm_batch_tune(self.h, int(units_per_cta), int(col_weight), g))

    def autotune(self, passes: int = 16, units=(1, 2, 4, 8), weights=(64, 192, 512),
                 margin: float = 0.03) -> Dict:
        """Coordinate search over the unit plan (units per CTA, then column
        weight) from the current setting.  Each trial times `passes` passes
        twice and keeps the better; a candidate replaces the current setting
        only when it is more than `margin` faster, so noise cannot make the
        choice worse.  The passes are real passes of the run: unit cuts
        change no result, only time."""
        def measure(u, w):
            self.tune(u, w)
            self.step(passes)  # capture of the graph for this setting
            self.sync()
            best = float("inf")
            for _ in range(2):
                t0 = time.perf_counter()
                self.step(passes)
                self.sync()
                best = min(best, (time.perf_counter() - t0) / passes)
            trials.append((u, w, round(1e3 * best, 4)))
            return best

        trials = []
        cu, cw = self._tuning
        cur = measure(cu, cw)
        for u in units:
            if u != cu:
                t = measure(u, cw)
                if t < cur * (1.0 - margin):
                    cu, cur = u, t
        for w in weights:
            if w != cw:
                t = measure(cu, w)
                if t < cur * (1.0 - margin):
                    cw, cur = w, t
        self.tune(cu, cw)
        self._tuning = (cu, cw)
        return {"units_per_cta": cu, "col_weight": cw, "ms_per_pass": 1e3 * cur,
                "passes": 3 * passes * len(trials), "trials": trials}

    def states(self) -> Dict[int, Dict[str, float]]:
        """Loop state of every live scenario, one synchronisation.  "failed":
        the scenario's state diverged (non-finite or negative) and its status
        word stopped it; the others are unaffected."""
        cap = max(len(self.np), 1)
        hs, run, its = (C.c_int * cap)(), (C.c_int * cap)(), (C.c_int * cap)()
        ts = (C.c_double * cap)()
        n = C.c_int()
        self._check(self.lib.dampm_batch_states(self.h, cap, hs, run, its, ts, C.byref(n)))
        return {hs[k]: {"running": run[k] == 1, "failed": run[k] < 0, "it": its[k],
                        "t": ts[k]}
                for k in range(n.value)}

    def usage(self) -> Dict[str, int]:
        out = (C.c_longlong * 8)()
        self._check(self.lib.dampm_batch_usage(self.h, out))
        keys = ("live", "removed", "particles", "particle_cap", "nodes", "node_cap",
                "scenario_cap", "launches")
        return dict(zip(keys, [int(v) for v in out]))
