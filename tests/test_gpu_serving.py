"""The serving loop on the GPU: requests arriving while others run are
admitted by footprint and batched with them, and every result equals the
same scenario run alone, bit for bit (tolerance 0)."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import Solver
from amsc_b200.serving import (BYTES_PER_NODE, BYTES_PER_PARTICLE, Request, Server,
                               latency_summary)


def request(seed, t_end):
    d = scenarios.ensemble_member(seed, side_range=(48, 112))
    d.scalars.update({"DT_FIXED": 0.0, "NSTEPS": 0, "T": t_end, "CFL": 0.4})
    return d


def alone(d):
    with Solver(d) as s:
        s.run()
        return {k: s.download(k) for k in ("x", "y", "hp")}, s.status()["it"]


def check(reqs):
    for r in reqs:
        ref, it = alone(r.data)
        assert r.passes == it
        for k in ref:
            np.testing.assert_array_equal(r.result[k], ref[k], err_msg=f"{r.rid} {k}")


class VirtualClock:
    """Advances 1 ms per reading, so arrivals interleave with ticks the same
    way on every run."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3
        return self.t


@pytest.mark.gpu
def test_staggered_arrivals_same_as_alone(cuda_lib):
    reqs = [Request(k, request(40 + k, 1.0 + 0.5 * (k % 3)), arrival=0.005 * k)
            for k in range(6)]
    with Server(2e9, max_scenarios=16, tick=4) as srv:
        srv.run(reqs, clock=VirtualClock())
        assert max(srv.occupancy) >= 2
    assert all(r.finished is not None for r in reqs)
    # some request joined while another was running
    assert any(a.admitted < b.admitted < a.finished for a in reqs for b in reqs)
    assert latency_summary(reqs)["p99_s"] > 0
    check(reqs)


@pytest.mark.gpu
def test_tight_budget_queues_and_compacts(cuda_lib):
    reqs = [Request(k, request(60, 0.4), arrival=0.0) for k in range(5)]
    big = reqs[0].data
    # room for two of these requests at once
    pbytes = 2.2 * big.np * BYTES_PER_PARTICLE
    nbytes = 2.2 * big.nnodes * BYTES_PER_NODE
    with Server(pbytes + nbytes, max_scenarios=8, tick=8,
                node_share=nbytes / (pbytes + nbytes)) as srv:
        srv.run(reqs, clock=VirtualClock())
        assert max(srv.occupancy) == 2 and srv.compactions >= 1
    assert sum(1 for r in reqs if r.admitted > reqs[0].finished) >= 2  # queued
    check(reqs)


@pytest.mark.gpu
def test_request_larger_than_budget_is_refused(cuda_lib):
    d = request(80, 0.1)
    with Server(1e6, max_scenarios=4) as srv:
        with pytest.raises(ValueError):
            srv.run([Request(0, d, 0.0)])
