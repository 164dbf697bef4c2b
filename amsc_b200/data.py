"""DATA: the solver input of dampm, mirroring ``struct DATA``.

Reference: main/mpm_data.h:6-122.  Required keys are read with ``j.at`` and
raise when missing (:64-97); optional keys fall back to the defaults of
:99-112.  DATA.json files hold only numbers and flat number arrays, written
with ``%.17g`` by the scenario generators (data/dambreak/dambreak.m:146-165),
so a round trip through :func:`to_json` / :func:`from_json` is exact.

Node arrays (Z, dZdx, dZdy) are in quadgrid order: node (r, c) at
r + c*(Ney+1), i.e. Octave's column-major ``Z(:)`` of a meshgrid with y
varying fastest.
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field, fields
from typing import Dict

import numpy as np

PARTICLE_KEYS = ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp", "mom_px", "mom_py", "Vp")
NODE_KEYS = ("Z", "dZdx", "dZdy")
# required scalar keys (main/mpm_data.h:70-97) and their types
REQUIRED_SCALARS = {
    "Nex": int, "Ney": int, "hx": float, "hy": float, "rho": float, "g": float,
    "T": float, "xi": float, "mu": float, "phi": float, "tauy": float,
    "BINGHAM_ON": float, "FRICTION_ON": float, "CFL": float, "BC_FLAG": int,
    "MERGE_SPLIT_ON": int, "eq_level": float,
}
# optional keys and defaults (main/mpm_data.h:99-112)
OPTIONAL_DEFAULTS = {
    "DT_FIXED": 0.0, "NSTEPS": 0,
    "ms_alpha": 0.9, "ms_beta": 0.30, "ms_split_hp_min": 0.0,
    "ms_shear_split": 1e30, "ms_hp_min": 0.05, "ms_max_dv": 0.01,
    "ms_min_level": -2, "ms_max_level": 2, "ms_min_particles_per_cell": 2,
    "ms_call_interval": 10, "ms_max_ops": 1e9,
    # no counterpart in the reference (which ignores the key): merge only
    # pairs closer than ms_pair_dist * min(hx, hy); 0 = no limit
    "ms_pair_dist": 0.0,
    # no counterpart among the reference's DATA keys: which merge/split runs
    # at the cadence -- 0 the one gpu_offload calls (main/merge_split_ops_cmes.h),
    # 1 the ELFS variant of main/merge_split_ops.h -- and the ELFS
    # divergence trigger (its ms_config::stretch_thresh default)
    "ms_variant": 0,
    "ms_stretch_thresh": 1e7,
}
_INT_KEYS = {"Nex", "Ney", "BC_FLAG", "MERGE_SPLIT_ON", "NSTEPS", "ms_min_level",
             "ms_max_level", "ms_min_particles_per_cell", "ms_call_interval", "ms_variant"}


class DataError(KeyError):
    pass


@dataclass
class DATA:
    """Flat scenario description; arrays are float64 numpy arrays."""

    arrays: Dict[str, np.ndarray] = field(default_factory=dict)
    scalars: Dict[str, float] = field(default_factory=dict)

    # -- convenience accessors ------------------------------------------------
    def __getattr__(self, name):
        if name in ("arrays", "scalars"):
            raise AttributeError(name)
        a = self.__dict__.get("arrays", {})
        s = self.__dict__.get("scalars", {})
        if name in a:
            return a[name]
        if name in s:
            return s[name]
        raise AttributeError(name)

    @property
    def np(self) -> int:
        return int(self.arrays["x"].shape[0])

    @property
    def nnodes(self) -> int:
        return (int(self.scalars["Nex"]) + 1) * (int(self.scalars["Ney"]) + 1)

    def copy(self) -> "DATA":
        return DATA({k: v.copy() for k, v in self.arrays.items()}, dict(self.scalars))

    def validate(self) -> None:
        for k in PARTICLE_KEYS:
            if k not in self.arrays:
                raise DataError(f"DATA: missing key '{k}'")
        for k in NODE_KEYS:
            if k not in self.arrays:
                raise DataError(f"DATA: missing key '{k}'")
        for k in REQUIRED_SCALARS:
            if k not in self.scalars:
                raise DataError(f"DATA: missing key '{k}'")
        n = self.np
        for k in PARTICLE_KEYS:
            if self.arrays[k].shape != (n,):
                raise DataError(f"DATA: '{k}' has {self.arrays[k].shape[0]} values, expected {n}")
        nn = self.nnodes
        for k in NODE_KEYS:
            if self.arrays[k].shape != (nn,):
                raise DataError(f"DATA: '{k}' has {self.arrays[k].shape[0]} values, expected {nn}")


def from_dict(j: dict) -> DATA:
    """``from_json`` of main/mpm_data.h:61-114."""
    arrays, scalars = {}, {}
    for k in PARTICLE_KEYS + NODE_KEYS:
        if k not in j:
            raise DataError(f"DATA: missing key '{k}'")
        arrays[k] = np.ascontiguousarray(np.asarray(j[k], dtype=np.float64).reshape(-1))
    for k, typ in REQUIRED_SCALARS.items():
        if k not in j:
            raise DataError(f"DATA: missing key '{k}'")
        scalars[k] = int(j[k]) if typ is int else float(j[k])
    for k, dflt in OPTIONAL_DEFAULTS.items():
        v = j.get(k, dflt)
        scalars[k] = int(v) if k in _INT_KEYS else float(v)
    d = DATA(arrays, scalars)
    d.validate()
    return d


def from_json(path: str) -> DATA:
    """``DATA::DATA(const char*)`` (main/mpm_data.h:116-122), through the
    library's streaming reader (dampm_json_read): each number is parsed
    straight into a float64 array, so DATA.json files of a gigabyte load
    without per-number Python objects."""
    import ctypes as C
    from .dampm import DampmError, load_library
    lib = load_library()
    h = C.c_void_p()
    rc = lib.dampm_json_read(path.encode(), C.byref(h))
    try:
        if rc != 0:
            msg = lib.dampm_json_error(h).decode() if h else f"cannot open {path}"
            raise DampmError(f"DATA: {msg}")
        j = {}
        for k in PARTICLE_KEYS + NODE_KEYS + tuple(REQUIRED_SCALARS) + tuple(OPTIONAL_DEFAULTS):
            n = C.c_longlong()
            lib.dampm_json_size(h, k.encode(), C.byref(n))
            if n.value < 0:
                continue
            a = np.empty(max(n.value, 1), dtype=np.float64)
            lib.dampm_json_get(h, k.encode(), a.ctypes.data_as(C.POINTER(C.c_double)))
            kind = C.c_int()
            lib.dampm_json_kind(h, k.encode(), C.byref(kind))
            j[k] = a[:n.value] if kind.value else float(a[0])
    finally:
        if h:
            lib.dampm_json_free(h)
    return from_dict(j)


def _fmt(v) -> str:
    return "%.17g" % float(v)


def _fmt_array(a: np.ndarray) -> str:
    # repr() of a Python float is the shortest string that parses back to
    # the same double, so the round trip stays exact
    return ",".join(map(repr, np.asarray(a, dtype=np.float64).tolist()))


def to_json(d: DATA, path: str) -> None:
    """Writes DATA.json the way the Octave generators' ``v2j`` does."""
    d.validate()
    with open(path, "w") as f:
        f.write("{\n")
        items = []
        for k in PARTICLE_KEYS + NODE_KEYS:
            a = d.arrays[k]
            items.append('"%s": [%s]' % (k, _fmt_array(a)))
        for k, v in d.scalars.items():
            items.append('"%s": %s' % (k, str(int(v)) if k in _INT_KEYS else _fmt(v)))
        f.write(",\n".join(items))
        f.write("\n}\n")
