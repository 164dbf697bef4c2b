"""TEST INFRASTRUCTURE ONLY -- drives the reference project's own programs
built by ``make ref`` in oracle/ (``_ref/optim_par``, ``_ref/ms_harness``,
``_ref/elfs_harness``).

``run_optim_par`` writes DATA.json into a scratch directory, runs the
reference's main/optim_par.cpp there and parses what it writes: the
``nc_particles_<it>.csv`` files (state at the start of step ``it``, i.e.
after it-1 steps, main/optim_par.cpp:311-337), ``conservation_errors.csv``
and the PERF line.  ``run_merge_split`` runs the reference's
adaptive_merge_split (main/merge_split_ops_cmes.h) on a given state, and
``run_merge_split_elfs`` its ELFS variant (main/merge_split_ops.h).
"""
from __future__ import annotations

import csv
import os
import struct
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
OPTIM_PAR = os.path.join(REF_DIR, "optim_par")
MS_HARNESS = os.path.join(REF_DIR, "ms_harness")
ELFS_HARNESS = os.path.join(REF_DIR, "elfs_harness")
BINDING = os.path.join(REF_DIR, "b200_offload")


def available() -> bool:
    return all(os.path.exists(p) for p in (OPTIM_PAR, MS_HARNESS, ELFS_HARNESS))


def reference_root() -> Optional[str]:
    """The reference checkout: $DAMPM_REFERENCE, else a checkout named
    ``reference`` beside this repository; None when neither holds main/."""
    cands = [os.environ.get("DAMPM_REFERENCE", ""),
             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "main")):
            return os.path.abspath(c)
    return None


def build(ref_root: Optional[str] = None) -> bool:
    """Builds _ref/ from the reference sources when they are present."""
    ref_root = ref_root or reference_root()
    if ref_root is None:
        return available()
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    lib = os.path.join(os.path.dirname(HERE), "amsc_b200", "libdampm_cuda.so")
    if os.path.exists(lib):  # the reference-side driver of the C ABI
        subprocess.run(["make", "-s", "-C", HERE, "binding", f"REF={ref_root}"], check=True)
    return available()


def read_csv(path: str) -> Dict[str, np.ndarray]:
    with open(path, newline="") as f:
        rows = list(csv.reader(f))
    header = [c.strip().strip('"').strip() for c in rows[0]]
    data = np.array([[float(v) for v in r] for r in rows[1:] if r], dtype=np.float64)
    return {name: data[:, k].copy() for k, name in enumerate(header)}


def run_optim_par(d, workdir: Optional[str] = None, timeout: float = 600.0):
    """Runs the reference CPU solver on DATA `d`; returns (csvs, errors, perf)
    where csvs maps it -> {column: array}."""
    from amsc_b200.data import to_json
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="dampm_ref_")
    to_json(d, os.path.join(wd, "DATA.json"))
    out = subprocess.run([OPTIM_PAR], cwd=wd, capture_output=True, text=True,
                         timeout=timeout, check=True)
    csvs = {}
    for fn in os.listdir(wd):
        if fn.startswith("nc_particles_") and fn.endswith(".csv"):
            csvs[int(fn[len("nc_particles_"):-4])] = read_csv(os.path.join(wd, fn))
    errs = np.loadtxt(os.path.join(wd, "conservation_errors.csv"), delimiter=",",
                      skiprows=1, ndmin=2)
    perf = [l for l in out.stdout.splitlines() if l.startswith("PERF")]
    if own:
        for fn in os.listdir(wd):
            os.unlink(os.path.join(wd, fn))
        os.rmdir(wd)
    return csvs, errs, (perf[0] if perf else "")


def _write_state(f, dprops, x, y, level, label):
    f.write(struct.pack("<ii", x.shape[0], len(dprops)))
    for k, v in dprops.items():
        kb = k.encode()
        f.write(struct.pack("<i", len(kb)))
        f.write(kb)
        f.write(np.ascontiguousarray(v, dtype="<f8").tobytes())
    f.write(np.ascontiguousarray(x, dtype="<f8").tobytes())
    f.write(np.ascontiguousarray(y, dtype="<f8").tobytes())
    f.write(np.ascontiguousarray(level, dtype="<i4").tobytes())
    f.write(np.ascontiguousarray(label, dtype="<i4").tobytes())


def _read_state(raw: bytes, nd: int) -> Dict[str, np.ndarray]:
    pos = 0
    (n,) = struct.unpack_from("<i", raw, pos)
    pos += 4
    out = {}
    for _ in range(nd):
        (ln,) = struct.unpack_from("<i", raw, pos)
        pos += 4
        name = raw[pos:pos + ln].decode()
        pos += ln
        out[name] = np.frombuffer(raw, dtype="<f8", count=n, offset=pos).copy()
        pos += 8 * n
    out["x"] = np.frombuffer(raw, dtype="<f8", count=n, offset=pos).copy()
    pos += 8 * n
    out["y"] = np.frombuffer(raw, dtype="<f8", count=n, offset=pos).copy()
    pos += 8 * n
    out["level"] = np.frombuffer(raw, dtype="<i4", count=n, offset=pos).astype(np.float64)
    pos += 4 * n
    out["label"] = np.frombuffer(raw, dtype="<i4", count=n, offset=pos).astype(np.float64)
    return out


def _run_harness(exe: str, header: bytes, dprops, x, y, level, label):
    with tempfile.TemporaryDirectory(prefix="dampm_ms_") as wd:
        fin = os.path.join(wd, "in.bin")
        fout = os.path.join(wd, "out.bin")
        with open(fin, "wb") as f:
            f.write(header)
            _write_state(f, dprops, x, y, level, label)
        subprocess.run([exe, fin, fout], check=True, capture_output=True)
        raw = open(fout, "rb").read()
    return _read_state(raw, len(dprops))


def run_merge_split(grid: dict, ms: dict, dt: float, dprops: Dict[str, np.ndarray],
                    x: np.ndarray, y: np.ndarray, level: np.ndarray, label: np.ndarray):
    """Runs the reference's adaptive_merge_split (main/merge_split_ops_cmes.h)
    on the given state."""
    header = (struct.pack("<ii", grid["Nex"], grid["Ney"]) +
              struct.pack("<ddd", grid["hx"], grid["hy"], dt) +
              struct.pack("<dddddd", ms["alpha"], ms["beta"], ms["split_hp_min"],
                          ms["shear_split"], ms["hp_min"], ms["max_dv"]) +
              struct.pack("<iiii", ms["min_level"], ms["max_level"],
                          ms["min_particles_per_cell"], ms["call_interval"]) +
              struct.pack("<d", ms["max_ops"]))
    return _run_harness(MS_HARNESS, header, dprops, x, y, level, label)


def run_merge_split_elfs(grid: dict, ms: dict, dprops: Dict[str, np.ndarray],
                         x: np.ndarray, y: np.ndarray, level: np.ndarray,
                         label: np.ndarray):
    """Runs the reference's ELFS adaptive_merge_split (main/merge_split_ops.h)
    on the given state."""
    header = (struct.pack("<ii", grid["Nex"], grid["Ney"]) +
              struct.pack("<dd", grid["hx"], grid["hy"]) +
              struct.pack("<ddddd", ms["alpha"], ms["beta"], ms["hp_min"], ms["max_dv"],
                          ms["stretch_thresh"]) +
              struct.pack("<iii", ms["min_level"], ms["max_level"], ms["call_interval"]) +
              struct.pack("<d", ms["max_ops"]))
    return _run_harness(ELFS_HARNESS, header, dprops, x, y, level, label)
