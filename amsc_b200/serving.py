"""Serving: a continuous-batching request loop over one ``Batch``.

Landslide scenarios (terrain, release zone, rheology; each its own grid and
particle count) arrive over time.  The server keeps every admitted
scenario's particle and grid state resident in HBM and advances all of them
together, ``tick`` passes at a time; a request is admitted as soon as its
footprint (particles and nodes) fits in the room left, so requests that
arrive while others run join the same passes.  After each tick the loop
state of every scenario is read in one synchronisation; a scenario whose
loop condition (t < T, or it < NSTEPS) has failed is downloaded, removed,
and its room reclaimed by compaction.  Each result is the same, bit for bit,
as the scenario run alone: a scenario's passes never depend on its
neighbours.

Time-to-result is measured from a request's arrival to the moment its
result is on the host.

Failures are handled per request and never stop the server:
  * a scenario whose state diverges (NaN/inf or negative depth) is stopped on
    the device by its status word; the server marks the request "failed" and
    removes it;
  * a watchdog stops a request that has run more than its pass cap (a CFL dt
    that collapses would otherwise run forever) or is older than its
    deadline: "timeout";
  * a request the client drops (``cancel_at``) leaves the queue or the batch:
    "cancelled".
The other scenarios' passes do not depend on the removed one, so their
results are unchanged.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .batch import Batch
from .dampm import DampmError
from .data import DATA

# device bytes per particle and per node a batch holds (double-buffered
# persistent state, sort and P2G scratch)
BYTES_PER_PARTICLE = 390
BYTES_PER_NODE = 56
BYTES_PER_PARTICLE_F32 = 230
BYTES_PER_NODE_F32 = 48
_INT_MAX = 2**31 - 1


@dataclass
class Request:
    rid: int
    data: DATA
    arrival: float  # seconds after the server starts
    max_passes: Optional[int] = None  # watchdog: pass cap (None: the server's)
    deadline_s: Optional[float] = None  # watchdog: seconds after arrival
    cancel_at: Optional[float] = None  # the client drops the request then
    admitted: Optional[float] = None
    finished: Optional[float] = None
    passes: int = 0
    status: str = "pending"  # then queued, running, done, failed, timeout, cancelled
    result: Dict[str, np.ndarray] = field(default_factory=dict)

    @property
    def latency(self) -> Optional[float]:
        return None if self.finished is None else self.finished - self.arrival


class Server:
    """Admission by memory footprint, continuous batching, results on the host.

    ``budget_bytes`` is the device memory the batch may take; it is split
    between particle and node capacity by ``node_share``.
    """

    def __init__(self, budget_bytes: float, max_scenarios: int = 1024, tick: int = 16,
                 node_share: float = 0.45, result_fields: Sequence[str] = ("x", "y", "hp"),
                 stream: Optional[int] = None, precision: str = "fp64",
                 graphs: bool = True, max_passes: Optional[int] = None, batch=None):
        """max_passes: the watchdog's default pass cap per request (a request
        is stopped within one tick of reaching it).  batch: an object with
        the Batch interface to serve on (by default a new Batch)."""
        bpp, bpn = ((BYTES_PER_PARTICLE_F32, BYTES_PER_NODE_F32) if precision == "fp32"
                    else (BYTES_PER_PARTICLE, BYTES_PER_NODE))
        pc = int(budget_bytes * (1.0 - node_share) / bpp)
        nc = int(budget_bytes * node_share / bpn)
        self.particle_cap = min(pc, _INT_MAX)
        self.node_cap = min(nc, _INT_MAX)
        self.max_scenarios = max_scenarios
        self.tick = tick
        self.fields = tuple(result_fields)
        self.max_passes = max_passes
        if batch is None:
            batch = Batch(self.particle_cap, self.node_cap, max_scenarios, stream=stream,
                          precision=precision)
        self.b = batch
        self.b.tune(graphs=graphs)
        self.compactions = 0
        self.ticks = 0
        self.occupancy: List[int] = []

    def close(self):
        self.b.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def fits_alone(self, d: DATA) -> bool:
        return d.np <= self.particle_cap and d.nnodes <= self.node_cap

    def _try_admit(self, r: Request) -> Optional[int]:
        u = self.b.usage()
        if (u["particles"] + r.data.np > u["particle_cap"] or
                u["nodes"] + r.data.nnodes > u["node_cap"] or
                u["live"] + u["removed"] >= u["scenario_cap"]):
            return None
        try:
            return self.b.add(r.data)
        except DampmError:  # another table of the batch is full
            return None

    def run(self, requests: List[Request], clock: Callable[[], float] = time.perf_counter
            ) -> List[Request]:
        """Serves `requests` (sorted by arrival) until each is done, failed,
        timed out or cancelled."""
        for r in requests:
            if not self.fits_alone(r.data):
                raise ValueError(f"request {r.rid} is larger than the whole batch")
        t0 = clock()
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: collections.deque = collections.deque()
        live: Dict[int, Request] = {}
        self._removed = 0

        def leave(h: int, r: Request, status: str, now: float):
            live.pop(h)
            r.status = status
            r.finished = now
            self.b.remove(h)
            self._removed += 1

        def expired(r: Request, now: float) -> Optional[str]:
            if r.cancel_at is not None and now >= r.cancel_at:
                return "cancelled"
            if r.deadline_s is not None and now - r.arrival >= r.deadline_s:
                return "timeout"
            return None

        while pending or waiting or live:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                r.status = "queued"
                waiting.append(r)
            # the client side and the deadline watchdog, before any admission
            for r in list(waiting):
                st = expired(r, now)
                if st:
                    waiting.remove(r)
                    r.status, r.finished = st, now
            for h, r in list(live.items()):
                st = expired(r, now)
                if st:
                    leave(h, r, st, now)
            # admission, first come first served, by footprint
            while waiting:
                h = self._try_admit(waiting[0])
                if h is None and self._removed:
                    self.b.compact()
                    self.compactions += 1
                    self._removed = 0
                    h = self._try_admit(waiting[0])
                if h is None:
                    break
                r = waiting.popleft()
                r.admitted = clock() - t0
                r.status = "running"
                live[h] = r
            if not live:
                if waiting:  # the head does not fit even in an empty batch
                    raise RuntimeError(f"request {waiting[0].rid} cannot be admitted")
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                continue
            self.b.step(self.tick)
            self.ticks += 1
            self.occupancy.append(len(live))
            for h, s in self.b.states().items():
                if h not in live:
                    continue
                r = live[h]
                r.passes = s["it"]
                cap = r.max_passes if r.max_passes is not None else self.max_passes
                if s.get("failed"):
                    leave(h, r, "failed", clock() - t0)
                elif not s["running"]:
                    r.result = {f: self.b.download(h, f) for f in self.fields}
                    leave(h, r, "done", clock() - t0)
                elif cap is not None and s["it"] >= cap:
                    leave(h, r, "timeout", clock() - t0)
            # reclaim room once removed scenarios hold a quarter of it
            u = self.b.usage()
            if self._removed and (u["removed"] * 4 >= u["live"] + u["removed"]):
                self.b.compact()
                self.compactions += 1
                self._removed = 0
        return requests


def latency_summary(requests: Sequence[Request]) -> Dict[str, float]:
    """Time-to-result percentiles over the requests that completed."""
    lat = np.array([r.latency for r in requests
                    if r.latency is not None and r.status == "done"])
    if lat.size == 0:
        return {}
    return {"p50_s": float(np.percentile(lat, 50)), "p95_s": float(np.percentile(lat, 95)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "max_s": float(lat.max())}


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
