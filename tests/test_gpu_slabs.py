"""One scenario split over slabs of cell columns, on one GPU: two and three
slab contexts exchanging ghosts, node columns and migrants by device
copies (amsc_b200/slabs.py, LocalLink) give the single-context run bit for
bit, and the ledger over all slabs matches it to round-off (its sums are
added in another order)."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import Solver
from amsc_b200.slabs import column_of, local_run

FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "Mp", "Vp", "H")


@pytest.mark.gpu
@pytest.mark.parametrize("case,nslabs,steps", [("bench_slab", 2, 40), ("mudflow", 2, 40),
                                              ("mudflow", 3, 25)])
def test_slabs_equal_single_context(cuda_lib, case, nslabs, steps):
    if case == "bench_slab":  # fixed dt, Bingham + Voellmy
        d = scenarios.bench_slab(10000, nsteps=steps)
    else:  # adaptive CFL on the bumpy slope
        d = scenarios.mudflow(N=256)
    with Solver(d) as s:
        s.step(steps)
        ref = {k: s.download(k) for k in FIELDS}
        st = s.status()
        led = s.ledgers()
    run = local_run(d, nslabs)
    try:
        run.step(steps)
        got = run.status()
        assert got["it"] == st["it"] and got["t"] == st["t"] and got["np"] == st["np"]
        for k in FIELDS:
            np.testing.assert_array_equal(run.gather(k), ref[k], err_msg=k)
        np.testing.assert_allclose(run.ledgers()[:6], led[:6], rtol=1e-12, atol=1e-9)
        if case == "bench_slab":
            return  # the fixed-dt slab moves too little to cross an edge in 40 steps
        # particles did cross the slab edges
        d2 = d.copy()
        d2.arrays["x"] = run.gather("x")
        moved = (np.searchsorted([b[0] for b in run.bounds], column_of(d2), side="right") !=
                 np.searchsorted([b[0] for b in run.bounds], column_of(d), side="right"))
        assert moved.any()
    finally:
        run.close()
