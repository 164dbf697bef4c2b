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
BYTES_PER_PARTICLE_F32 = 210
BYTES_PER_NODE_F32 = 48
_INT_MAX = 2**31 - 1


@dataclass
class Request:
    rid: int
    data: DATA
    arrival: float  # seconds after the server starts
    admitted: Optional[float] = None
    finished: Optional[float] = None
    passes: int = 0
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
                 graphs: bool = True):
        bpp, bpn = ((BYTES_PER_PARTICLE_F32, BYTES_PER_NODE_F32) if precision == "fp32"
                    else (BYTES_PER_PARTICLE, BYTES_PER_NODE))
        pc = int(budget_bytes * (1.0 - node_share) / bpp)
        nc = int(budget_bytes * node_share / bpn)
        self.particle_cap = min(pc, _INT_MAX)
        self.node_cap = min(nc, _INT_MAX)
        self.max_scenarios = max_scenarios
        self.tick = tick
        self.fields = tuple(result_fields)
        self.b = Batch(self.particle_cap, self.node_cap, max_scenarios, stream=stream,
                       precision=precision)
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
        """Serves `requests` (sorted by arrival) to completion."""
        for r in requests:
            if not self.fits_alone(r.data):
                raise ValueError(f"request {r.rid} is larger than the whole batch")
        t0 = clock()
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: collections.deque = collections.deque()
        live: Dict[int, Request] = {}
        removed = 0
        while pending or waiting or live:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            # admission, first come first served, by footprint
            while waiting:
                h = self._try_admit(waiting[0])
                if h is None and removed:
                    self.b.compact()
                    self.compactions += 1
                    removed = 0
                    h = self._try_admit(waiting[0])
                if h is None:
                    break
                r = waiting.popleft()
                r.admitted = clock() - t0
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
                if s["running"] or h not in live:
                    continue
                r = live.pop(h)
                r.result = {f: self.b.download(h, f) for f in self.fields}
                r.passes = s["it"]
                r.finished = clock() - t0
                self.b.remove(h)
                removed += 1
            # reclaim room once removed scenarios hold a quarter of it
            u = self.b.usage()
            if removed and (u["removed"] * 4 >= u["live"] + u["removed"]):
                self.b.compact()
                self.compactions += 1
                removed = 0
        return requests


def latency_summary(requests: Sequence[Request]) -> Dict[str, float]:
    lat = np.array([r.latency for r in requests if r.latency is not None])
    if lat.size == 0:
        return {}
    return {"p50_s": float(np.percentile(lat, 50)), "p95_s": float(np.percentile(lat, 95)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "max_s": float(lat.max())}


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
