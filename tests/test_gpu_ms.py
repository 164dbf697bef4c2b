"""Merge/split on the GPU against the oracle (which is pinned to the
reference's main/merge_split_ops_cmes.h): standalone calls and the
gpu_offload cadence inside the step loop.  Bitwise."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import Solver
from oracle.oracle import Oracle

FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_21", "F_22", "Mp", "Vp", "H",
          "Ap", "mom_px", "mom_py", "Fb_x", "Fb_y", "label", "level",
          "vpx_dx", "vpx_dy", "vpy_dx", "vpy_dy", "xp", "yp")


def ms_data(nsteps=100):
    d = scenarios.bench_slab(1000, nsteps=nsteps)
    # areas straddle both thresholds after a few steps: splits and merges
    d.scalars.update({"ms_alpha": 0.5, "ms_beta": 0.5, "ms_max_dv": 1.0,
                      "ms_hp_min": 0.05, "MERGE_SPLIT_ON": 1})
    return d


def compare(s, o, fields=FIELDS):
    assert s.num_particles == o.np
    for k in fields:
        a, b = s.download(k), o.get(k)
        np.testing.assert_array_equal(a, b, err_msg=k)


@pytest.mark.gpu
def test_standalone_merge_split(cuda_lib):
    d = ms_data()
    o = Oracle(d, threads=4)
    o.run(12)
    with Solver(d, record=True) as s:
        s.step(12)
        cg = s.merge_split(1e-3)
        co = o.merge_split(1e-3)
        assert cg == co, (cg, co)
        assert co[0] > 0 and co[1] > 0 and co[3] != co[2]
        compare(s, o)
        # the step after a merge/split reads the emitted Ap/mom/Fb
        s.step(3)
        o.run(3)
        compare(s, o, FIELDS[:12] + ("Ap", "mom_px", "Fb_x"))


@pytest.mark.gpu
def test_merge_split_cadence(cuda_lib):
    """MERGE_SPLIT_ON with ms_call_interval = 10: three calls in 35 steps."""
    d = ms_data()
    o = Oracle(d, threads=4, merge_split=True)
    o.run(35)
    with Solver(d, merge_split=True) as s:
        s.step(35)
        st = s.status()
        assert st["it"] == o.it and st["np"] == o.np
        compare(s, o, FIELDS[:19])


@pytest.mark.gpu
def test_merge_split_cap(cuda_lib):
    """max_ops binds: splits capped in (cell, index) order and the merge
    budget walked cell by cell."""
    d = ms_data()
    d.scalars["ms_max_ops"] = 7.0
    o = Oracle(d, threads=4)
    o.run(12)
    with Solver(d, record=True) as s:
        s.step(12)
        cg = s.merge_split(1e-3)
        co = o.merge_split(1e-3)
        assert cg == co and co[0] == 7 and co[1] <= 7
        compare(s, o)
