"""The optim_par program on the GPU: same input, loop and output files.

    python -m amsc_b200.driver [DATA.json] [--outdir DIR] [--no-output]

Reads DATA.json (main/mpm_data.h), runs the loop
``while (fixed ? it < NSTEPS : t < T)`` of main/optim_par.cpp:281-668 through
the C ABI and writes, as optim_par does:

  * GRID_forZ.vts before the first step (:269);
  * nc_particles_<it>.csv when it % 10 == 0, holding the particles as they
    are when step `it` begins (:311-337);
  * nc_grid_<it>.vts when it % 10 == 0, the nodal vars after step `it`
    (:655-665; the second vtk_export there overwrites the first);
  * conservation_errors.csv, one row per step (:274, 395-428).

The steps between outputs run on the device without host synchronisation;
output-only fields are materialised (dampm_record_outputs) only for the
steps whose results are written, and the conservation rows come back from
the device log in chunks.  The particle fields of an output step are copied
to page-locked buffers on a second stream while the next step runs
(dampm_stage_download), and the files are formatted and written by a writer
thread while the following steps run; two buffer sets alternate, so at most
one output is being written while the next is copied.  The last line printed is
``PERF np=<n> counted_steps=<k> tot_s=<s>`` over the steps after the
reference's 5 warm-up steps.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import outputs
from .data import from_json
from .dampm import Solver, pinned_array

_ZERO_VARS = ("div_v",)  # declared by optim_par, never computed


_UNWRITTEN = ("F_ext_px", "F_ext_py")  # declared, never written by optim_par


def particle_fields(s: Solver) -> dict:
    cols = {}
    for k in ("x", "y") + outputs.DPROPS + outputs.IPROPS:
        if k in _UNWRITTEN:
            cols[k] = np.zeros(s.num_particles)
        else:
            cols[k] = s.download(k)
    return cols


class _StagedParticles:
    """Two sets of page-locked buffers for the particle fields of an output
    step: one is copied into while the writer thread may still read the
    other."""

    NAMES = tuple(k for k in ("x", "y") + outputs.DPROPS + outputs.IPROPS if k not in _UNWRITTEN)

    def __init__(self):
        self.sets = [None, None]
        self.busy = [None, None]  # the writer's future reading each set
        self.turn = 0

    def stage(self, s: Solver):
        """Starts the copies of the particles as they are now; returns the
        set index and the particle count."""
        i = self.turn
        self.turn ^= 1
        if self.busy[i] is not None:
            self.busy[i].result()
            self.busy[i] = None
        n = s.num_particles
        if self.sets[i] is None or self.sets[i]["x"].size < n:
            cap = max(n, 1)
            self.sets[i] = {k: pinned_array(cap) for k in self.NAMES}
        return i, s.stage_download(self.sets[i])

    def columns(self, i: int, n: int) -> dict:
        cols = {k: self.sets[i][k][:n] for k in self.NAMES}
        for k in _UNWRITTEN:
            cols[k] = np.zeros(n)
        return cols


def nodal_vars(s: Solver, nn: int) -> dict:
    v = {}
    for k in ("Mv", "mom_vx", "mom_vy", "F_int_vx", "F_int_vy", "Fric_x", "Fric_y", "avx",
              "avy", "vvx", "vvy", "Z", "dZdx", "dZdy", "HV", "FPxv", "FPyv", "vvxL", "vvyL"):
        v[k] = s.download_nodal(k)
    # main/optim_par.cpp:467-482, the same IEEE sums on the host
    v["F_ext_vx"] = v["FPxv"] + v["Fric_x"]
    v["F_ext_vy"] = v["FPyv"] + v["Fric_y"]
    v["Ftot_vx"] = v["F_ext_vx"] - v["F_int_vx"]
    v["Ftot_vy"] = v["F_ext_vy"] - v["F_int_vy"]
    for k in _ZERO_VARS:
        v[k] = np.zeros(nn)
    return v


def run(data_path: str, outdir: str = ".", write: bool = True, max_steps: int = 1 << 40,
        out=sys.stdout) -> dict:
    d = from_json(data_path)
    sc = d.scalars
    nrows, ncols = int(sc["Ney"]), int(sc["Nex"])
    hx, hy = float(sc["hx"]), float(sc["hy"])
    fixed = float(sc.get("DT_FIXED", 0.0)) > 0.0
    nsteps, T = int(sc.get("NSTEPS", 0)), float(sc["T"])

    def cond(st):  # the loop condition of main/optim_par.cpp:281
        return (st["it"] < nsteps if fixed else st["t"] < T) and st["it"] < max_steps

    os.makedirs(outdir, exist_ok=True)
    path = lambda name: os.path.join(outdir, name)  # noqa: E731
    with Solver(d) as s:
        if not write:
            s.step(5)  # the reference's warm-up steps
            st = s.status()
            warm_it, t0 = st["it"], time.perf_counter()
            s.run(max_steps=max(max_steps - warm_it, 0))
            st = s.status()
            tot, it, np_ = time.perf_counter() - t0, st["it"], st["np"]
        else:
            grid0 = {k: np.zeros(d.nnodes) for k in outputs.VARS}
            grid0.update({"Z": d.arrays["Z"], "dZdx": d.arrays["dZdx"], "dZdy": d.arrays["dZdy"]})
            outputs.write_vts(path("GRID_forZ.vts"), nrows, ncols, hx, hy, grid0)
            errf = open(path("conservation_errors.csv"), "w")
            outputs.write_errors_header(errf)
            writer = ThreadPoolExecutor(max_workers=1)
            staged = _StagedParticles()
            pending = []
            logged, t0, warm_it = 0, None, 0
            st = s.status()
            while cond(st):
                it = st["it"]
                nxt = (it // 10 + 1) * 10  # the next step that writes output
                if nxt - 2 - it > 0:
                    s.step(nxt - 2 - it)
                if nxt - 2 - it >= 0:   # step nxt-1, whose fields the CSV shows
                    s.lib.dampm_record_outputs(s.h, 1)
                    s.step(1)
                    s.lib.dampm_record_outputs(s.h, 0)
                st = s.status()
                if cond(st) and st["it"] == nxt - 1:
                    # step nxt begins: the particles as they are now, copied
                    # while step nxt runs
                    i, n = staged.stage(s)
                    s.lib.dampm_record_outputs(s.h, 1)
                    s.step(1)
                    s.lib.dampm_record_outputs(s.h, 0)
                    st = s.status()
                    s.staged_wait()
                    staged.busy[i] = writer.submit(outputs.write_particles_csv,
                                                   path(f"nc_particles_{nxt}.csv"),
                                                   staged.columns(i, n))
                    pending.append(staged.busy[i])
                    if st["it"] == nxt:  # and its nodal vars once it has run
                        pending.append(writer.submit(outputs.write_vts,
                                                     path(f"nc_grid_{nxt}.vts"), nrows, ncols,
                                                     hx, hy, nodal_vars(s, d.nnodes)))
                    for f in [f for f in pending if f.done()]:
                        f.result()  # a writer's exception surfaces here
                    pending = [f for f in pending if not f.done()]
                if st["it"] > logged:
                    rows = s.ledger_history(logged + 1, st["it"] - logged)
                    outputs.write_error_rows(errf, rows)
                    logged = st["it"]
                if t0 is None and st["it"] >= 5:
                    t0, warm_it = time.perf_counter(), st["it"]
                if st["it"] == it:  # nothing ran: the loop has ended on the device
                    break
            for f in pending:
                f.result()  # a writer's exception surfaces here
            writer.shutdown()
            errf.close()
            tot = time.perf_counter() - t0 if t0 is not None else 0.0
            it, np_ = st["it"], st["np"]
    counted = max(it - warm_it, 0)
    print(f"PERF np={np_} counted_steps={counted} tot_s={tot:.6f}", file=out)
    return {"it": it, "np": np_, "counted_steps": counted, "tot_s": tot}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("data", nargs="?", default="DATA.json")
    ap.add_argument("--outdir", default=".")
    ap.add_argument("--no-output", action="store_true")
    ap.add_argument("--max-steps", type=int, default=1 << 40)
    a = ap.parse_args(argv)
    run(a.data, a.outdir, write=not a.no_output, max_steps=a.max_steps)


if __name__ == "__main__":
    main()
