"""One scenario split over slabs of cell columns.

The 2048^2 mudflow fits one B200, so the single-GPU path is the one that
matters; this splits a scenario that would not (or that should run faster
on several GPUs) along x, one slab per context.  Every slab keeps the whole
grid's node arrays and terrain but only the particles of its own cell
columns [lo, hi).  A step moves three things between neighbours:

1. before P2G, copies ("ghosts") of the particles in the left slab's last
   column go to the right slab: its P2G starts the chains of its first node
   column from them, so every nodal sum runs over the same particles in the
   same cell-sweep order as on one domain (bit for bit);
2. after P2G, the right slab's first node column of (vvxL, vvyL) goes to
   the left slab, whose G2P interpolates it;
3. after G2P, particles whose new cell is in the neighbour's columns move
   there; then the CFL maxima are reduced over all slabs (max: exact).

The sort orders each cell's particles by their reference index wherever they
sit in storage, so moved particles need no ordering.  Merge/split and
recorded outputs are not available in slab mode.

Two transports carry the exchanges: :class:`LocalLink`, all slabs in one
process (on one GPU: device-to-device copies), and :class:`DistLink`, one
slab per rank over ``torch.distributed`` (NCCL between GPUs, gloo on CPU).
:class:`SlabRun` is the step loop over either; the slab engine is
:class:`SlabEngine` (a ``dampm_ctx`` in slab mode) or any object with its
methods.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .data import DATA
from .dampm import Solver, _DP

RECORD = 20  # doubles per travelling particle (dampm_slab_record_doubles)


def partition_columns(d: DATA, nslabs: int, min_width: int = 2) -> List[Tuple[int, int]]:
    """Cell-column ranges [lo, hi) holding about equal particle counts."""
    nex = int(d.scalars["Nex"])
    if nslabs < 1 or nslabs * min_width > nex:
        raise ValueError(f"cannot cut {nex} columns into {nslabs} slabs of {min_width}+")
    hx = float(d.scalars["hx"])
    col = np.clip(np.floor(d.arrays["x"] / hx), 0, nex - 1).astype(np.int64)
    cum = np.cumsum(np.bincount(col, minlength=nex))
    cuts = [0]
    for k in range(1, nslabs):
        c = int(np.searchsorted(cum, k * cum[-1] / nslabs, side="left")) + 1
        c = max(c, cuts[-1] + min_width)
        c = min(c, nex - (nslabs - k) * min_width)
        cuts.append(c)
    cuts.append(nex)
    return [(cuts[k], cuts[k + 1]) for k in range(nslabs)]


def column_of(d: DATA) -> np.ndarray:
    nex, hx = int(d.scalars["Nex"]), float(d.scalars["hx"])
    return np.clip(np.floor(d.arrays["x"] / hx), 0, nex - 1).astype(np.int64)


class SlabEngine:
    """One slab: a dampm_ctx in slab mode holding the particles of columns
    [lo, hi) of `d` (with their reference indices)."""

    def __init__(self, d: DATA, lo: int, hi: int, device: int = 0, capacity: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.lo, self.hi = lo, hi
        self.ny = int(d.scalars["Ney"])
        col = column_of(d)
        mine = np.nonzero((col >= lo) & (col < hi))[0]
        sub = d.copy()
        for k in ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp", "mom_px", "mom_py", "Vp"):
            sub.arrays[k] = np.ascontiguousarray(d.arrays[k][mine])
        cap = capacity or 2 * d.np + 1024
        self.s = Solver(sub, capacity=cap)
        self.lib, self.h = self.s.lib, self.s.h
        self.s._check(self.lib.dampm_slab_set(self.h, lo, hi))
        ix = np.ascontiguousarray(mine.astype(np.int32))
        self.s._check(self.lib.dampm_slab_set_index(self.h, ix.ctypes.data_as(C.POINTER(C.c_int))))
        self.xcap = max(4096, cap // 8)
        self._buf = [torch.empty((self.xcap, RECORD), dtype=torch.float64, device=self.dev)
                     for _ in range(3)]
        self.ncols = int(d.scalars["Nex"])

    def close(self):
        self.s.close()

    def _grow(self):
        self.xcap *= 2
        self._buf = [self.torch.empty((self.xcap, RECORD), dtype=self.torch.float64,
                                      device=self.dev) for _ in range(3)]

    def ghosts(self):
        n = C.c_longlong()
        while True:
            rc = self.lib.dampm_slab_ghosts(self.h, C.c_void_p(self._buf[0].data_ptr()),
                                            self.xcap, C.byref(n))
            if rc != -4:  # DAMPM_ERR_CAPACITY: a larger buffer and again
                break
            self._grow()
        self.s._check(rc)
        return self._buf[0][:n.value].clone()

    def import_(self, t, ghosts: bool):
        t = t.to(self.dev).contiguous()
        self.s._check(self.lib.dampm_slab_import(self.h, C.c_void_p(t.data_ptr() if t.numel() else 0),
                                                 t.shape[0], 1 if ghosts else 0))

    def pass_(self, phase: int):
        self.s._check(self.lib.dampm_slab_pass(self.h, phase))

    def node_column(self, col: int):
        t = self.torch.empty((self.ny + 1, 2), dtype=self.torch.float64, device=self.dev)
        self.s._check(self.lib.dampm_slab_node_column(self.h, col, C.c_void_p(t.data_ptr()), 0))
        return t

    def set_node_column(self, col: int, t):
        t = t.to(self.dev).contiguous()
        self.s._check(self.lib.dampm_slab_node_column(self.h, col, C.c_void_p(t.data_ptr()), 1))

    def route(self):
        nl, nr = C.c_longlong(), C.c_longlong()
        while True:
            rc = self.lib.dampm_slab_route(
                self.h, C.c_void_p(self._buf[1].data_ptr() if self.lo > 0 else 0),
                C.c_void_p(self._buf[2].data_ptr() if self.hi < self.ncols else 0),
                self.xcap, C.byref(nl), C.byref(nr))
            if rc != -4:
                break
            self._grow()
        self.s._check(rc)
        return self._buf[1][:nl.value].clone(), self._buf[2][:nr.value].clone()

    def cfl(self) -> np.ndarray:
        m = np.zeros(3)
        self.s._check(self.lib.dampm_slab_cfl(self.h, m.ctypes.data_as(_DP), 0))
        return m

    def set_cfl(self, m: np.ndarray):
        m = np.ascontiguousarray(m, dtype=np.float64)
        self.s._check(self.lib.dampm_slab_cfl(self.h, m.ctypes.data_as(_DP), 1))

    def download(self, field: str):
        n = self.s._status()[1]["np"]
        out = np.empty(n, dtype=np.float64)
        idx = np.empty(n, dtype=np.int64)
        self.s._check(self.lib.dampm_slab_download(self.h, field.encode(), out.ctypes.data_as(_DP),
                                                   idx.ctypes.data_as(C.POINTER(C.c_longlong))))
        return out, idx

    def status(self) -> Dict[str, float]:
        return self.s.status()

    def ledgers(self) -> np.ndarray:
        return self.s.ledgers()


class LocalLink:
    """All slabs in this process: a message is handed over as it is."""

    def __init__(self, nslabs: int):
        self.n = nslabs

    def shift_right(self, out: Dict[int, object], width: int) -> Dict[int, object]:
        return {r + 1: t for r, t in out.items() if r + 1 < self.n}

    def shift_left(self, out: Dict[int, object], width: int) -> Dict[int, object]:
        return {r - 1: t for r, t in out.items() if r >= 1}

    def allmax(self, vals: Dict[int, np.ndarray]) -> np.ndarray:
        return np.max(np.stack(list(vals.values())), axis=0)

    def allsum(self, vals: Dict[int, np.ndarray]) -> np.ndarray:
        return np.sum(np.stack(list(vals.values())), axis=0)

    def gather(self, vals: Dict[int, object]) -> List[object]:
        return [vals[r] for r in sorted(vals)]


class DistLink:
    """One slab per rank (slab r on rank r) over torch.distributed: a
    message to a neighbour is its length, then its rows."""

    def __init__(self, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank, self.n = dist.get_rank(), dist.get_world_size()
        self.device = device if device is not None else torch.device("cpu")

    def _exchange(self, out, to: int, frm: int, width: int):
        torch, dist = self.torch, self.dist
        t = out.get(self.rank)
        cnt_out = torch.tensor([0 if t is None else t.shape[0]], dtype=torch.int64,
                               device=self.device)
        cnt_in = torch.zeros(1, dtype=torch.int64, device=self.device)
        ops = []
        if 0 <= to < self.n:
            ops.append(dist.P2POp(dist.isend, cnt_out, to))
        if 0 <= frm < self.n:
            ops.append(dist.P2POp(dist.irecv, cnt_in, frm))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        recv = None
        ops = []
        if 0 <= to < self.n and int(cnt_out.item()) > 0:
            ops.append(dist.P2POp(dist.isend, t.to(self.device).contiguous(), to))
        if 0 <= frm < self.n:
            recv = torch.empty((int(cnt_in.item()), width), dtype=torch.float64,
                               device=self.device)
            if recv.shape[0] > 0:
                ops.append(dist.P2POp(dist.irecv, recv, frm))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        return {} if recv is None else {self.rank: recv}

    def shift_right(self, out, width: int):
        return self._exchange(out, self.rank + 1, self.rank - 1, width)

    def shift_left(self, out, width: int):
        return self._exchange(out, self.rank - 1, self.rank + 1, width)

    def allmax(self, vals):
        t = self.torch.tensor(np.asarray(vals[self.rank], dtype=np.float64), device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return t.cpu().numpy()

    def allsum(self, vals):
        t = self.torch.tensor(np.asarray(vals[self.rank], dtype=np.float64), device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def gather(self, vals):
        out = [None] * self.n
        self.dist.all_gather_object(out, vals[self.rank])
        return out


class SlabRun:
    """The step loop of one scenario over slabs.  `engines` maps the slab
    numbers this process drives to their engines (all of them with a
    LocalLink; its own one per rank with a DistLink); `bounds` are every
    slab's column ranges."""

    def __init__(self, engines: Dict[int, object], bounds: Sequence[Tuple[int, int]], link,
                 fixed_dt: bool):
        self.E = engines
        self.bounds = list(bounds)
        self.n = len(self.bounds)
        self.link = link
        self.fixed = fixed_dt
        self._sync_cfl()

    def _sync_cfl(self):
        m = self.link.allmax({r: e.cfl() for r, e in self.E.items()})
        for e in self.E.values():
            e.set_cfl(m)

    def step(self, nsteps: int = 1):
        E, link = self.E, self.link
        for _ in range(nsteps):
            # 1. the left neighbour's last column, for the leading column of P2G
            got = link.shift_right({r: e.ghosts() for r, e in E.items() if r < self.n - 1},
                                   RECORD)
            for r, t in got.items():
                E[r].import_(t, ghosts=True)
            for e in E.values():
                e.pass_(0)  # step start, sort, P2G
            # 2. each slab's first node column to its left neighbour
            cols = link.shift_left({r: e.node_column(self.bounds[r][0])
                                    for r, e in E.items() if r > 0}, 2)
            for r, t in cols.items():
                E[r].set_node_column(self.bounds[r + 1][0], t.reshape(-1, 2))
            for e in E.values():
                e.pass_(1)  # G2P, step end
            # 3. migrants, then the CFL maxima of all slabs
            routed = {r: e.route() for r, e in E.items()}
            to_right = link.shift_right({r: o[1] for r, o in routed.items()}, RECORD)
            to_left = link.shift_left({r: o[0] for r, o in routed.items()}, RECORD)
            for inbox in (to_right, to_left):
                for r, t in inbox.items():
                    E[r].import_(t, ghosts=False)
            self._sync_cfl()

    def status(self) -> Dict[str, float]:
        st = {r: e.status() for r, e in self.E.items()}
        one = next(iter(st.values()))
        n = self.link.allsum({r: np.array([s["np"]], dtype=np.float64) for r, s in st.items()})
        return {"it": one["it"], "t": one["t"], "dt": one["dt"], "np": int(n[0])}

    def running(self, d: DATA) -> bool:
        st = self.status()
        s = d.scalars
        return st["it"] < s["NSTEPS"] if self.fixed else st["t"] < s["T"]

    def gather(self, field: str) -> np.ndarray:
        """One particle field of the whole scenario in reference order."""
        parts = self.link.gather({r: e.download(field) for r, e in self.E.items()})
        n = sum(v.shape[0] for v, _ in parts)
        out = np.full(n, np.nan)
        for v, ix in parts:
            out[ix] = v
        return out

    def ledgers(self) -> np.ndarray:
        """The conservation ledger of the last step over all slabs: the sums
        of main/optim_par.cpp:395-425 and their errors."""
        t = self.link.allsum({r: e.ledgers()[:6] for r, e in self.E.items()})
        err_mass = abs(t[0] - t[3]) / t[0]
        norm = max(1.0, max(abs(t[1]), abs(t[2])))
        err_mom = max(abs(t[1] - t[4]), abs(t[2] - t[5])) / norm
        return np.concatenate([t, [err_mass, err_mom]])

    def close(self):
        for e in self.E.values():
            if hasattr(e, "close"):
                e.close()


def local_run(d: DATA, nslabs: int, device: int = 0) -> SlabRun:
    """All slabs of `d` in this process on one device."""
    bounds = partition_columns(d, nslabs)
    engines = {r: SlabEngine(d, lo, hi, device) for r, (lo, hi) in enumerate(bounds)}
    return SlabRun(engines, bounds, LocalLink(nslabs), fixed_dt=d.scalars["DT_FIXED"] > 0)


def dist_run(d: DATA, device: Optional[int] = None) -> SlabRun:
    """This rank's slab of `d` (slab r on rank r, on cuda:`device`), the
    exchanges over torch.distributed (NCCL)."""
    import torch
    import torch.distributed as dist
    r, n = dist.get_rank(), dist.get_world_size()
    dev = torch.cuda.current_device() if device is None else device
    bounds = partition_columns(d, n)
    eng = SlabEngine(d, *bounds[r], device=dev)
    return SlabRun({r: eng}, bounds, DistLink(torch.device("cuda", dev)),
                   fixed_dt=d.scalars["DT_FIXED"] > 0)
