"""Batches of independent scenarios on the GPU: every scenario's state after
a batched run equals its state after the same passes run alone (bitwise),
whatever else shares the batch, through removals and compaction."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.batch import Batch
from amsc_b200.dampm import Solver

FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "mom_px")


def solo(d, steps):
    with Solver(d) as s:
        s.step(steps)
        return {k: s.download(k) for k in FIELDS}, s.status()


def adaptive_member(seed):
    d = scenarios.ensemble_member(seed, side_range=(48, 96))
    d.scalars.update({"DT_FIXED": 0.0, "NSTEPS": 0, "T": 1e30, "CFL": 0.4})
    return d


def mix():
    return [scenarios.ensemble_member(1, side_range=(48, 96)),
            adaptive_member(2),
            scenarios.dam_break_flat(nsteps=500),
            scenarios.ensemble_member(3, side_range=(100, 160))]


def check_same(b, h, d, steps):
    ref, st = solo(d, steps)
    for k in FIELDS:
        np.testing.assert_array_equal(b.download(h, k), ref[k], err_msg=k)
    q = b.query(h)
    assert q["it"] == st["it"] and q["t"] == st["t"] and q["dt"] == st["dt"]


@pytest.mark.gpu
def test_batch_equals_each_scenario_alone(cuda_lib):
    ds = mix()
    with Batch(200_000, 200_000, 16) as b:
        hs = [b.add(d) for d in ds]
        b.step(25)
        b.sync()
        for h, d in zip(hs, ds):
            check_same(b, h, d, 25)
        # per-scenario conservation ledger of the last pass, as alone
        with Solver(ds[0]) as s:
            s.step(25)
            np.testing.assert_allclose(b.ledgers(hs[0]), s.ledgers(), rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_batch_remove_compact_and_admit(cuda_lib):
    a, bb, c, d = mix()
    with Batch(200_000, 200_000, 8) as b:
        ha, hb, hc = b.add(a), b.add(bb), b.add(c)
        b.step(10)
        b.remove(hb)
        assert b.usage()["removed"] == 1
        b.compact()
        assert b.usage()["removed"] == 0 and b.usage()["live"] == 2
        hd = b.add(d)
        b.step(12)
        check_same(b, ha, a, 22)
        check_same(b, hc, c, 22)
        check_same(b, hd, d, 12)


@pytest.mark.gpu
def test_batch_scenario_stops_at_its_own_end(cuda_lib):
    short = scenarios.ensemble_member(5, side_range=(48, 64), nsteps=6)
    long_ = scenarios.ensemble_member(6, side_range=(48, 64), nsteps=1000)
    with Batch(100_000, 100_000, 4) as b:
        hs, hl = b.add(short), b.add(long_)
        b.step(15)
        assert not b.query(hs)["running"] and b.query(hs)["it"] == 6
        assert b.query(hl)["running"] and b.query(hl)["it"] == 15
        check_same(b, hs, short, 15)
        check_same(b, hl, long_, 15)


@pytest.mark.gpu
def test_batch_full_is_an_error(cuda_lib):
    from amsc_b200.dampm import DampmError
    d = scenarios.ensemble_member(7, side_range=(48, 64))
    with Batch(d.np + 10, 100_000, 4) as b:
        b.add(d)
        with pytest.raises(DampmError):
            b.add(d)


@pytest.mark.gpu
def test_graphs_and_tuning_change_no_result(cuda_lib):
    ds = mix()[:3]
    with Batch(200_000, 200_000, 8) as b:
        hs = [b.add(d) for d in ds]
        b.tune(units_per_cta=8, col_weight=64, graphs=False)
        b.step(6)
        # two replays of the 16-pass graph, then 5 passes one by one (the
        # next call starts from the other half)
        b.tune(units_per_cta=2, col_weight=512, graphs=True)
        b.step(37)
        info = b.autotune(passes=16, units=(2, 4), weights=(192,))
        assert info["units_per_cta"] in (2, 4) and info["passes"] > 0
        b.sync()
        total = 43 + info["passes"]
        for h, d in zip(hs, ds):
            check_same(b, h, d, total)
