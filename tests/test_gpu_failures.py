"""Failure detection on the GPU, with every failure made on the host.

A NaN or an infinity is written into a scenario's input arrays before
upload (into arrays the first step reads: the depth, or the momentum it
transfers -- an uploaded velocity is replaced by the first G2P before it is
used); no kernel is made to fault.  G2P raises the scenario's status word,
its later passes do nothing, and the host sees the status through
dampm_sync / dampm_status (single scenario), dampm_batch_states (a batch)
or the serving loop (the request is marked failed and removed).  The other
scenarios' results stay bitwise equal to their runs alone.
"""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.batch import Batch
from amsc_b200.dampm import DampmError, Solver
from amsc_b200.serving import Request, Server


def _alone(d, fields=("x", "y", "hp")):
    with Solver(d) as s:
        s.run()
        return {k: s.download(k) for k in fields}, s.status()["it"]


@pytest.mark.gpu
@pytest.mark.parametrize("field,value", [("hp", np.nan), ("mom_px", np.inf)])
def test_diverged_state_stops_the_run(cuda_lib, field, value):
    d = scenarios.bench_slab(1000, nsteps=20)
    d.arrays[field] = d.arrays[field].copy()
    d.arrays[field][123] = value
    with Solver(d) as s:
        s.step(5)
        with pytest.raises(DampmError, match="-5"):
            s.sync()
        assert s.failed
        rc, st = s._status()
        assert rc == -5 and st["it"] == 1  # the pass that diverged, then nothing
        hp = s.download("hp")  # the diverged state can still be read
        assert not np.isfinite(hp).all()
        with pytest.raises(DampmError):
            s.run()


@pytest.mark.gpu
def test_diverged_scenario_in_a_batch_stops_alone(cuda_lib):
    members = [scenarios.ensemble_member(s, side_range=(48, 96), nsteps=60)
               for s in (5, 6, 7)]
    members[1].arrays["hp"] = members[1].arrays["hp"].copy()
    members[1].arrays["hp"][7] = np.nan
    with Batch(sum(m.np for m in members) + 16, sum(m.nnodes for m in members) + 16,
               8) as b:
        hs = [b.add(m) for m in members]
        b.step(60)
        st = b.states()
        assert st[hs[1]]["failed"] and not st[hs[1]]["running"]
        assert st[hs[1]]["it"] == 1
        for k in (0, 2):
            assert not st[hs[k]]["failed"] and st[hs[k]]["it"] == 60
            ref, it = _alone(members[k])
            for f, v in ref.items():
                np.testing.assert_array_equal(b.download(hs[k], f), v, err_msg=f)
        with pytest.raises(DampmError):
            b.sync()


class _Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3
        return self.t


@pytest.mark.gpu
def test_serving_failed_timed_out_and_dropped_requests(cuda_lib):
    reqs = []
    for k in range(6):
        d = scenarios.ensemble_member(200 + k, side_range=(48, 112))
        d.scalars.update({"DT_FIXED": 0.0, "NSTEPS": 0, "T": 0.8, "CFL": 0.4})
        reqs.append(Request(k, d, arrival=0.003 * k))
    reqs[1].data.arrays["hp"] = reqs[1].data.arrays["hp"].copy()
    reqs[1].data.arrays["hp"][3] = np.nan          # diverges
    reqs[3].max_passes = 5                         # the watchdog stops it
    reqs[4].cancel_at = 0.02                       # the client drops it
    with Server(2e9, max_scenarios=16, tick=4) as srv:
        srv.run(reqs, clock=_Clock())
    assert reqs[1].status == "failed" and reqs[1].result == {}
    assert reqs[3].status == "timeout" and 5 <= reqs[3].passes < 9
    assert reqs[4].status == "cancelled" and reqs[4].result == {}
    for k in (0, 2, 5):
        assert reqs[k].status == "done"
        ref, it = _alone(reqs[k].data)
        assert reqs[k].passes == it
        for f, v in ref.items():
            np.testing.assert_array_equal(reqs[k].result[f], v, err_msg=f"{k} {f}")
