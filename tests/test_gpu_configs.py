"""The benchmark configurations at their own sizes, against the oracle.

* C1 flat dam break: the whole 500-step run.
* C2 2048^2 mudflow (4,021,256 particles, adaptive CFL): the workload the
  benchmark times, for 10 steps.
* C3 mudflow with merge/split at the configuration's mapped thresholds
  (split at Ap > 2 A0, merge at Ap < 0.5 A0, levels -2..2, every 10 steps),
  on the 256^2 grid: three merge/split calls in 35 steps.
* C4 ensemble members of different sides inside one batch, and a C5 request
  served in a mix, each compared directly with the oracle run alone.

Tolerance 0 (bitwise) throughout; the parity bar is 1e-10 relative.
"""
import os

import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.batch import Batch
from amsc_b200.dampm import Solver
from amsc_b200.serving import Request, Server
from oracle.oracle import Oracle

STATE = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_21", "F_22", "Mp", "Vp", "H")
DERIVED = ("Ap", "mom_px", "mom_py", "Fb_x", "Fb_y")
MS_FIELDS = STATE + DERIVED + ("label", "level")
THREADS = os.cpu_count() or 4


def _equal(get_a, get_b, names):
    for k in names:
        a, b = get_a(k), get_b(k)
        assert a.shape == b.shape, k
        np.testing.assert_array_equal(a, b, err_msg=k)


@pytest.mark.gpu
def test_c1_dam_break_whole_run(cuda_lib):
    d = scenarios.dam_break_flat(nsteps=500)
    o = Oracle(d, threads=THREADS)
    n_o = o.run(1 << 20)
    with Solver(d) as s:
        n_g = s.run()
        assert n_g == n_o == 500
        st = s.status()
        assert st["it"] == o.it and st["t"] == o.t
        _equal(s.download, o.get, STATE + DERIVED)
        np.testing.assert_allclose(s.ledgers()[:6], o.ledger()[:6], rtol=1e-12, atol=1e-9)


@pytest.mark.gpu
def test_c2_mudflow_2048_benchmark_workload(cuda_lib):
    d = scenarios.mudflow(N=2048)
    assert d.np == 4_021_256
    o = Oracle(d, threads=THREADS)
    o.run(10)
    with Solver(d) as s:
        s.step(10)
        st = s.status()
        assert st["it"] == o.it == 10 and st["t"] == o.t and st["dt"] == o.dt
        _equal(s.download, o.get, ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22"))
        led = s.ledgers()
        assert led[6] < 1e-12 and led[7] < 1e-12


@pytest.mark.gpu
def test_c3_mudflow_merge_split_mapped_thresholds(cuda_lib):
    d = scenarios.mudflow(N=256, merge_split=True)
    A0 = (0.5 / 4) ** 2
    assert d.scalars["ms_alpha"] == np.sqrt(2 * A0) / 0.5
    o = Oracle(d, threads=THREADS, merge_split=True)
    o.run(35)
    assert o.np > d.np  # the calls at steps 10, 20 and 30 split particles
    with Solver(d, merge_split=True) as s:
        s.step(35)
        st = s.status()
        assert st["it"] == o.it and st["np"] == o.np and st["t"] == o.t
        _equal(s.download, o.get, MS_FIELDS)


@pytest.mark.gpu
def test_c4_members_in_one_batch_against_oracle(cuda_lib):
    members = []
    for seed in (3, 11, 29):
        d = scenarios.ensemble_member(seed, side_range=(64, 200), nsteps=150)
        members.append(d)
    assert len({m.scalars["Nex"] for m in members}) == 3  # different sides
    with Batch(sum(m.np for m in members) + 16,
               sum(m.nnodes for m in members) + 16, 8) as b:
        hs = [b.add(m) for m in members]
        b.step(150)
        b.sync()
        for h, m in zip(hs, members):
            assert b.query(h)["it"] == 150
            o = Oracle(m, threads=THREADS)
            o.run(150)
            _equal(lambda k: b.download(h, k), o.get,
                   ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "mom_px", "mom_py"))


class _Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3
        return self.t


@pytest.mark.gpu
def test_c5_request_in_a_served_mix_against_oracle(cuda_lib):
    reqs = []
    for k, seed in enumerate((101, 102, 103, 104)):
        d = scenarios.ensemble_member(seed, side_range=(64, 160))
        d.scalars.update({"DT_FIXED": 0.0, "NSTEPS": 0, "T": 0.6 + 0.2 * k, "CFL": 0.4})
        reqs.append(Request(k, d, arrival=0.004 * k))
    with Server(4e9, max_scenarios=16, tick=4) as srv:
        srv.run(reqs, clock=_Clock())
        assert max(srv.occupancy) >= 2
    for r in reqs:
        assert r.status == "done"
        o = Oracle(r.data, threads=THREADS)
        n = o.run(1 << 20)
        assert r.passes == n
        _equal(lambda k: r.result[k], o.get, ("x", "y", "hp"))
