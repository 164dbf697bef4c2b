"""The slab exchange protocol (amsc_b200/slabs.py) on the CPU.

A stand-in engine with simple column dynamics replaces the GPU context: the
particles of a column feel the node values of its two node columns, a node
value counts the particles of the two cell columns beside it, and a particle
moves by its velocity (dt from the CFL-like maximum of all slabs).  A node
value next to a slab edge therefore needs the neighbour's ghosts (before
"P2G") or the neighbour's node column (before "G2P"), and particles migrate
across the edges.  Run over slabs -- in one process (LocalLink) and as two
gloo ranks (DistLink) -- the gathered state must equal the single-domain run
exactly, particle for particle.
"""
import os

import numpy as np
import pytest
import torch

from amsc_b200.slabs import RECORD, DistLink, LocalLink, SlabRun

NCOLS = 24
L = float(NCOLS)


def initial(n=700, seed=4):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.2, L - 0.2, n)
    v = rng.normal(0.0, 0.7, n)
    return x, v


def reference(steps, x, v):
    x, v = x.copy(), v.copy()
    for _ in range(steps):
        dt = 0.5 / (1e-2 + np.abs(v).max())
        col = np.clip(np.floor(x), 0, NCOLS - 1).astype(int)
        cnt = np.bincount(col, minlength=NCOLS).astype(float)
        node = np.zeros(NCOLS + 1)
        node[1:] += cnt
        node[:-1] += cnt
        v = v + 1e-3 * (node[col + 1] - node[col])
        x = np.clip(x + dt * v, 1e-9, L - 1e-9)
    return x, v


class StandIn:
    """The engine interface of SlabEngine over numpy particles of columns
    [lo, hi)."""

    def __init__(self, x, v, lo, hi):
        col = np.floor(x).astype(int)
        mine = np.nonzero((col >= lo) & (col < hi))[0]
        self.x, self.v, self.idx = x[mine].copy(), v[mine].copy(), mine.copy()
        self.lo, self.hi = lo, hi
        self.gx = np.zeros(0)
        self.node = np.zeros(NCOLS + 1)
        self.maxv = np.zeros(3)
        self.it = 0

    def _rows(self, sel):
        t = torch.zeros((int(sel.sum()), RECORD), dtype=torch.float64)
        t[:, 0] = torch.from_numpy(self.x[sel])
        t[:, 1] = torch.from_numpy(self.v[sel])
        t[:, 2] = torch.from_numpy(self.idx[sel].astype(np.float64))
        return t

    def ghosts(self):
        return self._rows(np.floor(self.x).astype(int) == self.hi - 1)

    def import_(self, t, ghosts):
        a = t.numpy()
        if ghosts:
            assert (np.floor(a[:, 0]) == self.lo - 1).all()
            self.gx = a[:, 0].copy()
        else:
            assert ((np.floor(a[:, 0]) >= self.lo) & (np.floor(a[:, 0]) < self.hi)).all()
            self.x = np.concatenate([self.x, a[:, 0]])
            self.v = np.concatenate([self.v, a[:, 1]])
            self.idx = np.concatenate([self.idx, a[:, 2].astype(np.int64)])

    def pass_(self, phase):
        if phase == 0:  # node values of the columns this slab writes
            col = np.floor(np.concatenate([self.x, self.gx])).astype(int)
            cnt = np.bincount(col, minlength=NCOLS).astype(float)
            node = np.zeros(NCOLS + 1)
            node[1:] += cnt
            node[:-1] += cnt
            hi = self.hi if self.hi == NCOLS else self.hi - 1
            self.node[self.lo:hi + 1] = node[self.lo:hi + 1]
            self.gx = np.zeros(0)
        else:
            dt = 0.5 / (1e-2 + self.maxv[0])
            col = np.floor(self.x).astype(int)
            self.v = self.v + 1e-3 * (self.node[col + 1] - self.node[col])
            self.x = np.clip(self.x + dt * self.v, 1e-9, L - 1e-9)
            self.it += 1

    def node_column(self, c):
        return torch.tensor([[self.node[c], 0.0]], dtype=torch.float64)

    def set_node_column(self, c, t):
        self.node[c] = float(t[0, 0])

    def route(self):
        col = np.floor(self.x).astype(int)
        left, right = col < self.lo, col >= self.hi
        out = (self._rows(left), self._rows(right))
        keep = ~(left | right)
        self.x, self.v, self.idx = self.x[keep], self.v[keep], self.idx[keep]
        return out

    def cfl(self):
        return np.array([np.abs(self.v).max() if self.v.size else 0.0, 0.0, 0.0])

    def set_cfl(self, m):
        self.maxv = np.asarray(m, dtype=np.float64).copy()

    def download(self, field):
        return (self.x if field == "x" else self.v).copy(), self.idx.copy()

    def status(self):
        return {"it": self.it, "t": 0.0, "dt": 0.0, "np": int(self.x.size)}

    def ledgers(self):
        return np.array([self.x.size, self.v.sum(), 0.0, self.x.size, self.v.sum(), 0.0, 0, 0, 0])


BOUNDS3 = [(0, 7), (7, 15), (15, NCOLS)]


def test_slabs_in_one_process_equal_one_domain():
    x, v = initial()
    rx, rv = reference(40, x, v)
    run = SlabRun({r: StandIn(x, v, lo, hi) for r, (lo, hi) in enumerate(BOUNDS3)}, BOUNDS3,
                  LocalLink(3), fixed_dt=False)
    run.step(40)
    assert run.status()["np"] == x.size
    np.testing.assert_array_equal(run.gather("x"), rx)
    np.testing.assert_array_equal(run.gather("v"), rv)
    moved = [e.idx for e in run.E.values()]
    assert sum(m.size for m in moved) == x.size  # every particle on exactly one slab


def _rank(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, v = initial()
        bounds = [(0, 11), (11, NCOLS)]
        run = SlabRun({rank: StandIn(x, v, *bounds[rank])}, bounds, DistLink(), fixed_dt=False)
        run.step(40)
        gx, gv = run.gather("x"), run.gather("v")
        n = run.status()["np"]
        if rank == 0:
            rx, rv = reference(40, x, v)
            q.put((bool(np.array_equal(gx, rx)), bool(np.array_equal(gv, rv)), n, x.size))
    finally:
        dist.destroy_process_group()


def test_slabs_over_two_gloo_ranks_equal_one_domain():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    same_x, same_v, n, n0 = q.get(timeout=5)
    assert same_x and same_v and n == n0
