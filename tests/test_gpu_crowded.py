"""Cells crowded with hundreds to thousands of particles (as the unstable
members of a fixed-dt ensemble pile theirs against a wall): P2G's batches
that lie inside one cell hand that cell's node sums to one thread each, and
the per-cell order of the sort takes its path for crowded cells (sorted runs
merged).  Every sum keeps the reference's order, so the state stays bitwise
equal to the oracle's, on the plain path and in batches cut into units in
different ways."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.batch import Batch
from amsc_b200.dampm import Solver
from oracle.oracle import Oracle

FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "Mp", "Vp", "H")
STEPS = 20


def _cells(d):
    h = d.scalars["hx"]
    n = int(d.scalars["Ney"])
    return (d.arrays["x"] // h).astype(np.int64) * n + (d.arrays["y"] // h).astype(np.int64)


def test_scenario_has_crowded_cells():
    d = scenarios.crowded_cells()
    cnt = np.bincount(_cells(d))
    # one cell above a sorted run of the per-cell order (16384 entries)
    assert cnt.max() > 16384 and (cnt >= 512).sum() == 4


@pytest.mark.gpu
def test_crowded_cells_bitwise_against_oracle(cuda_lib):
    d = scenarios.crowded_cells()
    o = Oracle(d, threads=4)
    o.run(STEPS)
    with Solver(d) as s:
        s.step(STEPS)
        s.sync()
        st = s.status()
        assert st["it"] == o.it and st["t"] == o.t
        for k in FIELDS:
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)
        # the ledger totals are summed per P2G unit, then over the units (the
        # oracle sums particle by particle): round-off of the order, 2e-12
        # relative here, where 32,000 particles' masses span four decades
        led_g, led_o = s.ledgers(), o.ledger()
        np.testing.assert_allclose(led_g[:6], led_o[:6], rtol=1e-11, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("units,weight", [(2, 192), (8, 64), (1, 512)])
def test_crowded_cells_in_a_batch(cuda_lib, units, weight):
    d = scenarios.crowded_cells()
    other = scenarios.ensemble_member(3, side_range=(48, 64))
    with Solver(d) as s:
        s.step(STEPS)
        ref = {k: s.download(k) for k in FIELDS}
    with Batch(200_000, 200_000, 4) as b:
        ho = b.add(other)
        h = b.add(d)
        b.tune(units_per_cta=units, col_weight=weight)
        b.step(STEPS)
        b.sync()
        for k in FIELDS:
            np.testing.assert_array_equal(b.download(h, k), ref[k], err_msg=k)
        assert b.query(ho)["it"] == STEPS
