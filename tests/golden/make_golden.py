#!/usr/bin/env python3
"""Generates the golden fixtures in this directory from the reference
project's own programs (oracle/_ref, built by `make -C oracle ref` from the
reference sources; needs the reference checkout, so it runs only where that
exists).

  optim_par_bench1000.npz  reference main/optim_par.cpp on the shipped
                           DATA_bench_1000 fixture (regenerated bit for bit
                           by amsc_b200.scenarios.bench_slab), NSTEPS = 20:
                           every column of nc_particles_10/20.csv and the
                           conservation_errors.csv rows.
  optim_par_digests.json   the same runs for the flat dam break and the
                           conservation bump: SHA-256 of every CSV column
                           (float64 little-endian bytes) and the errors.
  ms_bench1000.json        reference adaptive_merge_split
                           (main/merge_split_ops_cmes.h) on a perturbed state
                           of the bench case (recipe: ms_case()): SHA-256 of
                           every input and output column, the particle counts.
  ms_elfs_bench1000.json   reference ELFS adaptive_merge_split
                           (main/merge_split_ops.h) on another perturbed state
                           of the bench case (recipe: elfs_case()), for each
                           configuration of ELFS_CONFIGS: the same digests.

Usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from amsc_b200 import scenarios  # noqa: E402
from oracle import refrun  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DPROPS = ["Mp", "Ap", "vpx", "vpy", "mom_px", "mom_py", "hp", "Vp", "F_ext_px", "F_ext_py",
          "apx", "apy", "F_11", "F_12", "F_21", "F_22", "vpx_dx", "vpx_dy", "vpy_dx",
          "vpy_dy", "Fb_x", "Fb_y", "hpZ", "dZxp", "dZyp", "Zp", "xp", "yp", "Fric_px",
          "Fric_py", "Fpx", "Fpy", "vpxL", "vpyL", "H"]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def golden_cases():
    d = scenarios.conservation_bump()
    d.scalars.update({"DT_FIXED": 1e-3, "NSTEPS": 20})
    return {"dam_break": scenarios.dam_break_flat(nsteps=20), "conservation_bump": d}


def ms_case():
    """A bench state after 30 steps with perturbed areas, velocities and
    levels so that splits, merges and undo all occur."""
    from oracle.oracle import Oracle
    d = scenarios.bench_slab(1000, nsteps=100)
    o = Oracle(d, threads=1)
    o.run(30)
    rng = np.random.default_rng(7)
    n = o.np
    state = {k: o.get(k) for k in DPROPS}
    state["Ap"] = state["Ap"] * rng.choice([0.05, 1.0, 1.0, 3.0], size=n)
    state["vpx"] = state["vpx"] + rng.normal(0, 0.002, n)
    level = rng.integers(-2, 3, n).astype(np.int32)
    ms = dict(alpha=0.7, beta=0.2, split_hp_min=0.0, shear_split=1e30, hp_min=0.05,
              max_dv=0.01, min_level=-2, max_level=2, min_particles_per_cell=2,
              call_interval=10, max_ops=1e9)
    return d, state, o.get("x"), o.get("y"), level, o.get("label").astype(np.int32), ms


# ELFS ms_config values (main/merge_split_ops.h:17-30): its defaults (a
# binding max_ops of 50), no cap, and a low divergence trigger
ELFS_CONFIGS = {
    "defaults": dict(alpha=2.0, beta=3.0, hp_min=0.05, max_dv=0.01, stretch_thresh=1e7,
                     min_level=-2, max_level=2, call_interval=10, max_ops=50.0),
    "uncapped": dict(alpha=2.0, beta=3.0, hp_min=0.05, max_dv=0.01, stretch_thresh=1e7,
                     min_level=-2, max_level=2, call_interval=10, max_ops=1e9),
    "stretch": dict(alpha=1.0, beta=2.0, hp_min=0.05, max_dv=0.05, stretch_thresh=0.5,
                    min_level=-2, max_level=2, call_interval=10, max_ops=1e9),
}


def elfs_case():
    """A bench state after 30 steps (a flow with a free surface inside the
    grid) with perturbed areas, velocities and levels."""
    from oracle.oracle import Oracle
    d = scenarios.bench_slab(1000, nsteps=100)
    o = Oracle(d, threads=1)
    o.run(30)
    rng = np.random.default_rng(11)
    n = o.np
    state = {k: o.get(k) for k in DPROPS}
    state["Ap"] = state["Ap"] * rng.choice([0.3, 1.0, 1.0, 2.0], size=n)
    state["vpx"] = state["vpx"] + rng.normal(0, 0.002, n)
    level = rng.integers(-2, 3, n).astype(np.int32)
    return d, state, o.get("x"), o.get("y"), level, o.get("label").astype(np.int32)


def main():
    if not refrun.build():
        sys.exit("reference build (oracle/_ref) unavailable")
    d = scenarios.bench_slab(1000, nsteps=20)
    csvs, errs, _ = refrun.run_optim_par(d)
    out = {"errors": errs}
    for it, cols in csvs.items():
        for k, v in cols.items():
            out[f"it{it}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "optim_par_bench1000.npz"), **out)

    dig = {}
    for name, dd in golden_cases().items():
        csvs, errs, _ = refrun.run_optim_par(dd)
        dig[name] = {"errors": errs.tolist(),
                     "columns": {f"it{it}/{k}": digest(v) for it, cols in csvs.items()
                                 for k, v in cols.items()}}
    with open(os.path.join(HERE, "optim_par_digests.json"), "w") as f:
        json.dump(dig, f, indent=1, sort_keys=True)

    d, state, x, y, level, label, ms = ms_case()
    grid = dict(Nex=int(d.scalars["Nex"]), Ney=int(d.scalars["Ney"]),
                hx=float(d.scalars["hx"]), hy=float(d.scalars["hy"]))
    res = refrun.run_merge_split(grid, ms, 1e-3, state, x, y, level, label)
    inputs = dict(state, x=x, y=y, level=level.astype(np.float64), label=label.astype(np.float64))
    with open(os.path.join(HERE, "ms_bench1000.json"), "w") as f:
        json.dump({"ms": ms, "dt": 1e-3, "np_in": int(x.shape[0]), "np_out": int(res["x"].shape[0]),
                   "in": {k: digest(v) for k, v in inputs.items()},
                   "out": {k: digest(v) for k, v in res.items()}}, f, indent=1, sort_keys=True)

    d, state, x, y, level, label = elfs_case()
    inputs = dict(state, x=x, y=y, level=level.astype(np.float64), label=label.astype(np.float64))
    out = {"in": {k: digest(v) for k, v in inputs.items()}, "np_in": int(x.shape[0]),
           "configs": {}}
    for name, ms in ELFS_CONFIGS.items():
        res = refrun.run_merge_split_elfs(grid, ms, state, x, y, level, label)
        out["configs"][name] = {"ms": ms, "np_out": int(res["x"].shape[0]),
                                "out": {k: digest(v) for k, v in res.items()}}
    with open(os.path.join(HERE, "ms_elfs_bench1000.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("written", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
