"""Properties of the CPU oracle that the reference's validation scripts
check (data/*/scripts): conservation, lake at rest, and equality of the
serial and OpenMP modes."""
import numpy as np

from amsc_b200 import scenarios
from oracle.oracle import Oracle


def test_serial_equals_openmp():
    d = scenarios.bench_slab(3000, nsteps=30)
    a, b = Oracle(d, threads=1), Oracle(d, threads=4)
    a.run(30)
    b.run(30)
    for k in ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "Ap"):
        np.testing.assert_array_equal(a.get(k), b.get(k))


def test_conservation_machine_precision():
    """conservation_check.py: err_mass, err_mom < 1e-10 at every step."""
    d = scenarios.conservation_bump(T=0.3)
    o = Oracle(d, threads=4)
    while o.run(1):
        led = o.ledger()
        assert led[6] < 1e-10 and led[7] < 1e-10


def test_lake_at_rest():
    """wb_error.py: |hp - (eq - Zp)|, |hp vpx|, |hp vpy| below 1e-10 at T = 1."""
    d = scenarios.well_balance()
    o = Oracle(d, threads=4)
    o.run(1 << 30)
    assert abs(o.t - 1.0) < 0.01
    hp, Zp = o.get("hp"), o.get("Zp")
    assert np.abs(hp - (10.0 - Zp)).max() < 1e-10
    assert np.abs(hp * o.get("vpx")).max() < 1e-10
    assert np.abs(hp * o.get("vpy")).max() < 1e-10


def test_momentum_conserved_without_forcing():
    """Flat bed, walls off, no rheology, material away from the walls: total
    particle momentum stays at its initial value (zero here) to round-off."""
    d = scenarios.dam_break_flat(nsteps=50)
    d.scalars["BC_FLAG"] = 0
    d.arrays["x"] = d.arrays["x"] + 6.0
    o = Oracle(d, threads=4)
    o.run(50)
    mx = (o.get("vpx") * o.get("Mp")).sum()
    mass = o.get("Mp").sum()
    assert abs(mx) / mass < 1e-12


def test_pair_distance_gate():
    """The optional merge gate (ms_pair_dist, no counterpart in the reference):
    0 keeps the reference's pairing; a limit below every pair's distance
    stops all merges; a wide limit merges as without one; merges never pair
    particles farther apart than the limit."""
    d = scenarios.bench_slab(1000, nsteps=20)
    d.scalars.update({"ms_alpha": 0.5, "ms_beta": 0.5, "ms_max_dv": 1.0, "MERGE_SPLIT_ON": 1})
    counts = {}
    for gate in (0.0, 1e-9, 100.0, 0.2):
        dd = d.copy()
        dd.scalars["ms_pair_dist"] = gate
        o = Oracle(dd, threads=2)
        o.run(12)
        counts[gate] = o.merge_split(1e-3)
    assert counts[0.0][1] > 0
    assert counts[1e-9][1] == 0
    assert counts[100.0] == counts[0.0]
    assert 0 <= counts[0.2][1] <= counts[0.0][1]
