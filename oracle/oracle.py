"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracle.

Loads ``oracle/_build/libdampm_oracle.so`` (the C++ restatement of the
reference step in ``dampm_oracle.cpp``).  Only tests/, the smoke check and
bench.py's cpu_baseline leg use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Iterable

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "dampm_oracle.cpp")
LIB = os.path.join(HERE, "_build", "libdampm_oracle.so")

_DP = C.POINTER(C.c_double)


class oracle_data(C.Structure):
    _fields_ = [("Nex", C.c_int), ("Ney", C.c_int), ("hx", C.c_double), ("hy", C.c_double),
                ("g", C.c_double), ("T", C.c_double), ("rho", C.c_double),
                ("xi", C.c_double), ("mu", C.c_double), ("phi", C.c_double),
                ("tauy", C.c_double), ("BINGHAM_ON", C.c_double),
                ("FRICTION_ON", C.c_double), ("CFL", C.c_double), ("BC_FLAG", C.c_int),
                ("MERGE_SPLIT_ON", C.c_int), ("eq_level", C.c_double),
                ("DT_FIXED", C.c_double), ("NSTEPS", C.c_int),
                ("ms_alpha", C.c_double), ("ms_beta", C.c_double),
                ("ms_split_hp_min", C.c_double), ("ms_shear_split", C.c_double),
                ("ms_hp_min", C.c_double), ("ms_max_dv", C.c_double),
                ("ms_min_level", C.c_int), ("ms_max_level", C.c_int),
                ("ms_min_particles_per_cell", C.c_int), ("ms_call_interval", C.c_int),
                ("ms_max_ops", C.c_double), ("ms_pair_dist", C.c_double),
                ("ms_variant", C.c_int), ("ms_stretch_thresh", C.c_double)]


def build(force: bool = False) -> str:
    """g++ -O2 -ffp-contract=off -fopenmp: no FMA contraction, so every
    operation rounds as the reference's expressions do."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC",
                    "-shared", "-o", LIB + ".tmp", SRC], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [C.POINTER(oracle_data), _DP, _DP, _DP, C.c_longlong] + \
            [_DP] * 10 + [C.c_int, C.c_int]
        L.oracle_destroy.argtypes = [P]
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [P, C.c_int]
        L.oracle_merge_split.argtypes = [P, C.c_double]
        L.oracle_num_particles.restype = C.c_longlong
        L.oracle_num_particles.argtypes = [P]
        L.oracle_iteration.restype = C.c_int
        L.oracle_iteration.argtypes = [P]
        L.oracle_time.restype = C.c_double
        L.oracle_time.argtypes = [P]
        L.oracle_last_dt.restype = C.c_double
        L.oracle_last_dt.argtypes = [P]
        L.oracle_ledger.argtypes = [P, _DP]
        L.oracle_ms_counts.argtypes = [P, C.POINTER(C.c_longlong)]
        L.oracle_get.restype = C.c_int
        L.oracle_get.argtypes = [P, C.c_char_p, _DP]
        L.oracle_set.restype = C.c_int
        L.oracle_set.argtypes = [P, C.c_char_p, _DP]
        L.oracle_get_nodal.restype = C.c_int
        L.oracle_get_nodal.argtypes = [P, C.c_char_p, _DP]
        L.oracle_binning.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _od(d) -> oracle_data:
    s = d.scalars
    return oracle_data(int(s["Nex"]), int(s["Ney"]), float(s["hx"]), float(s["hy"]),
                       float(s["g"]), float(s["T"]), float(s["rho"]), float(s["xi"]),
                       float(s["mu"]), float(s["phi"]), float(s["tauy"]),
                       float(s["BINGHAM_ON"]), float(s["FRICTION_ON"]), float(s["CFL"]),
                       int(s["BC_FLAG"]), int(s["MERGE_SPLIT_ON"]), float(s["eq_level"]),
                       float(s["DT_FIXED"]), int(s["NSTEPS"]), float(s["ms_alpha"]),
                       float(s["ms_beta"]), float(s["ms_split_hp_min"]),
                       float(s["ms_shear_split"]), float(s["ms_hp_min"]),
                       float(s["ms_max_dv"]), int(s["ms_min_level"]),
                       int(s["ms_max_level"]), int(s["ms_min_particles_per_cell"]),
                       int(s["ms_call_interval"]), float(s["ms_max_ops"]),
                       float(s.get("ms_pair_dist", 0.0)), int(s.get("ms_variant", 0)),
                       float(s.get("ms_stretch_thresh", 1e7)))


class Oracle:
    """The reference step on the CPU (serial when threads == 1)."""

    def __init__(self, d, threads: int = 1, merge_split: bool = False):
        self.L = lib()
        self.d = d
        A = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in d.arrays.items()}
        self._A = A
        self._od = _od(d)
        P = lambda k: A[k].ctypes.data_as(_DP)
        self.h = self.L.oracle_create(C.byref(self._od), P("Z"), P("dZdx"), P("dZdy"), d.np,
                                      P("x"), P("y"), P("Mp"), P("Ap"), P("vpx"), P("vpy"),
                                      P("hp"), P("mom_px"), P("mom_py"), P("Vp"),
                                      int(threads), 1 if merge_split else 0)
        self.nn = d.nnodes

    def close(self):
        if self.h:
            self.L.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps: int) -> int:
        return int(self.L.oracle_run(self.h, int(nsteps)))

    def merge_split(self, dt: float):
        self.L.oracle_merge_split(self.h, float(dt))
        c = (C.c_longlong * 4)()
        self.L.oracle_ms_counts(self.h, c)
        return [int(v) for v in c]

    @property
    def np(self) -> int:
        return int(self.L.oracle_num_particles(self.h))

    @property
    def it(self) -> int:
        return int(self.L.oracle_iteration(self.h))

    @property
    def t(self) -> float:
        return float(self.L.oracle_time(self.h))

    @property
    def dt(self) -> float:
        return float(self.L.oracle_last_dt(self.h))

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.np, dtype=np.float64)
        if self.L.oracle_get(self.h, name.encode(), out.ctypes.data_as(_DP)) != 0:
            raise KeyError(name)
        return out

    def set(self, name: str, v: np.ndarray):
        v = np.ascontiguousarray(v, dtype=np.float64)
        if self.L.oracle_set(self.h, name.encode(), v.ctypes.data_as(_DP)) != 0:
            raise KeyError(name)

    def fields(self, names: Iterable[str]) -> Dict[str, np.ndarray]:
        return {k: self.get(k) for k in names}

    def nodal(self, name: str) -> np.ndarray:
        out = np.empty(self.nn, dtype=np.float64)
        if self.L.oracle_get_nodal(self.h, name.encode(), out.ctypes.data_as(_DP)) != 0:
            raise KeyError(name)
        return out

    def ledger(self) -> np.ndarray:
        out = np.empty(9, dtype=np.float64)
        self.L.oracle_ledger(self.h, out.ctypes.data_as(_DP))
        return out

    def binning(self):
        n = self.np
        nc = int(self.d.scalars["Nex"]) * int(self.d.scalars["Ney"])
        p2c = np.empty(n, dtype=np.int32)
        cs = np.empty(nc + 1, dtype=np.int32)
        cp = np.empty(n, dtype=np.int32)
        IP = C.POINTER(C.c_int)
        self.L.oracle_binning(self.h, p2c.ctypes.data_as(IP), cs.ctypes.data_as(IP),
                              cp.ctypes.data_as(IP))
        return p2c, cs, cp
