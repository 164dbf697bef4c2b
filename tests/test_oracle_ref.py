"""Live comparison with the reference project's own programs, where they can
be built (oracle/_ref from the reference sources; absent on machines without
the reference checkout)."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from oracle import refrun
from oracle.oracle import Oracle

pytestmark = pytest.mark.skipif(not refrun.build(), reason="reference sources not present")


def test_optim_par_well_balance_prefix():
    """Lake at rest with BC off and eq_level > 0 (the well-balanced terms),
    fixed dt: every CSV column bitwise."""
    d = scenarios.well_balance()
    d.scalars.update({"DT_FIXED": 2e-3, "NSTEPS": 10})
    csvs, errs, perf = refrun.run_optim_par(d)
    assert perf.startswith("PERF")
    o = Oracle(d, threads=2)
    o.run(9)
    for k, v in csvs[10].items():
        np.testing.assert_array_equal(o.get(k), v, err_msg=k)


def test_optim_par_bench3000_fixture():
    d = scenarios.bench_slab(3000, nsteps=10)
    csvs, errs, _ = refrun.run_optim_par(d)
    o = Oracle(d, threads=2)
    o.run(9)
    for k, v in csvs[10].items():
        np.testing.assert_array_equal(o.get(k), v, err_msg=k)


def test_bench_generator_matches_shipped_fixtures():
    """scaling.m restated in numpy reproduces DATA_bench_<N>.json exactly."""
    import json
    import os
    for N in (1000, 3000, 10000, 30000):
        path = os.path.join(refrun.reference_root() or "", "data", "performance",
                            f"DATA_bench_{N}.json")
        if not os.path.exists(path):
            pytest.skip("fixtures absent")
        ref = json.load(open(path))
        d = scenarios.bench_slab(N)
        for k, v in ref.items():
            if isinstance(v, list):
                np.testing.assert_array_equal(d.arrays[k], np.asarray(v), err_msg=f"{N} {k}")
            else:
                assert d.scalars[k] == v, (N, k)
