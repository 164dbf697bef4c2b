"""The serving loop's request handling on the CPU: failures, the watchdog,
cancellation and admission, against a stand-in batch.

The stand-in keeps the Batch interface and its contract -- a scenario runs
its own fixed number of passes, independently of the others, and a scenario
whose input depth holds a NaN is stopped by its status word after its first
pass -- so every failure here is made on the host; no GPU is involved.
"""
import numpy as np

from amsc_b200 import scenarios
from amsc_b200.serving import Request, Server


class StandInBatch:
    def __init__(self, particle_cap, node_cap, scenario_cap):
        self.cap = (particle_cap, node_cap, scenario_cap)
        self.scn = {}  # handle -> dict(data, it, dead)
        self.next = 0

    def tune(self, **kw):
        pass

    def usage(self):
        live = [s for s in self.scn.values() if not s["dead"]]
        dead = [s for s in self.scn.values() if s["dead"]]
        return {"live": len(live), "removed": len(dead),
                "particles": sum(s["data"].np for s in self.scn.values()),
                "particle_cap": self.cap[0],
                "nodes": sum(s["data"].nnodes for s in self.scn.values()),
                "node_cap": self.cap[1], "scenario_cap": self.cap[2], "launches": 0}

    def add(self, d):
        h = self.next
        self.next += 1
        self.scn[h] = {"data": d, "it": 0, "dead": False, "failed": False}
        return h

    def remove(self, h):
        self.scn[h]["dead"] = True

    def compact(self):
        self.scn = {h: s for h, s in self.scn.items() if not s["dead"]}

    def step(self, n):
        for s in self.scn.values():
            if s["dead"]:
                continue
            for _ in range(n):
                if s["failed"] or s["it"] >= s["data"].scalars["NSTEPS"]:
                    break
                s["it"] += 1
                if np.isnan(s["data"].arrays["hp"]).any():
                    s["failed"] = True

    def states(self):
        return {h: {"running": not s["failed"] and s["it"] < s["data"].scalars["NSTEPS"],
                    "failed": s["failed"], "it": s["it"], "t": 0.0}
                for h, s in self.scn.items() if not s["dead"]}

    def download(self, h, f):
        s = self.scn[h]
        return s["data"].arrays[f] + s["it"]


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3
        return self.t


def _req(k, nsteps, **kw):
    d = scenarios.dam_break_flat(nsteps=nsteps)
    return Request(k, d, arrival=0.002 * k, **kw)


def _server(**kw):
    return Server(1e12, max_scenarios=64, tick=4,
                  batch=StandInBatch(10**9, 10**9, 64), **kw)


def _expect_done(r, nsteps):
    assert r.status == "done" and r.passes == nsteps
    np.testing.assert_array_equal(r.result["hp"], r.data.arrays["hp"] + nsteps)


def test_diverged_request_fails_alone():
    reqs = [_req(k, 9 + k) for k in range(4)]
    reqs[2].data.arrays["hp"] = reqs[2].data.arrays["hp"].copy()
    reqs[2].data.arrays["hp"][17] = np.nan
    _server().run(reqs, clock=Clock())
    assert reqs[2].status == "failed" and reqs[2].result == {}
    for k in (0, 1, 3):
        _expect_done(reqs[k], 9 + k)


def test_watchdog_pass_cap_and_deadline():
    reqs = [_req(0, 10), _req(1, 10**6, max_passes=20), _req(2, 10**6, deadline_s=0.05),
            _req(3, 12)]
    srv = _server(max_passes=None)
    srv.run(reqs, clock=Clock())
    assert reqs[1].status == "timeout" and 20 <= reqs[1].passes < 20 + srv.tick
    assert reqs[2].status == "timeout" and reqs[2].finished - reqs[2].arrival >= 0.05
    _expect_done(reqs[0], 10)
    _expect_done(reqs[3], 12)
    # the server-wide cap applies to requests that set none
    r = [_req(0, 10**6)]
    _server(max_passes=8).run(r, clock=Clock())
    assert r[0].status == "timeout" and r[0].passes == 8


def test_dropped_requests_leave_queue_and_batch():
    reqs = [_req(0, 40), _req(1, 10**6, cancel_at=0.02), _req(2, 30, cancel_at=0.0),
            _req(3, 25)]
    _server().run(reqs, clock=Clock())
    assert reqs[1].status == "cancelled" and reqs[1].admitted is not None
    assert reqs[1].result == {}
    assert reqs[2].status == "cancelled" and reqs[2].admitted is None  # while queued
    _expect_done(reqs[0], 40)
    _expect_done(reqs[3], 25)


def test_admission_waits_for_room():
    d = scenarios.dam_break_flat(nsteps=6)
    reqs = [Request(k, scenarios.dam_break_flat(nsteps=6), arrival=0.0) for k in range(5)]
    srv = Server(1e12, max_scenarios=64, tick=4,
                 batch=StandInBatch(2 * d.np, 10**9, 64))
    srv.run(reqs, clock=Clock())
    assert max(srv.occupancy) == 2 and srv.compactions >= 1
    for r in reqs:
        _expect_done(r, 6)
    assert sum(1 for r in reqs if r.admitted > reqs[0].finished) >= 2
