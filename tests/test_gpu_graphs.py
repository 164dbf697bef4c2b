"""Passes replayed from a CUDA graph give the same state, bit for bit, as
passes launched one by one, and the graph is captured again when the
buffers change."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import Solver

FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22", "mom_px", "Vp")


def _run(d, graphs, n):
    with Solver(d) as s:
        s.set_graphs(graphs)
        s.step(n)
        st = s.status()
        return st, {k: s.download(k) for k in FIELDS}


@pytest.mark.gpu
def test_graph_replay_bitwise(cuda_lib):
    d = scenarios.mudflow(N=256)
    n = 16 * 3 + 5  # three replays and five plain passes
    st_g, f_g = _run(d, True, n)
    st_p, f_p = _run(d, False, n)
    assert st_g["it"] == st_p["it"] == n and st_g["t"] == st_p["t"]
    for k in FIELDS:
        np.testing.assert_array_equal(f_g[k], f_p[k], err_msg=k)


@pytest.mark.gpu
def test_graph_recaptured_when_buffers_change(cuda_lib):
    """Recording outputs allocates the output fields (new particle buffers),
    so the next run of passes captures its graph again."""
    d = scenarios.dam_break_flat(nsteps=200)
    out = []
    for graphs in (True, False):
        with Solver(d) as s:
            s.set_graphs(graphs)
            s.step(32)
            s.lib.dampm_record_outputs(s.h, 1)
            s.step(1)
            s.lib.dampm_record_outputs(s.h, 0)
            s.step(32)
            assert s.status()["it"] == 65
            out.append({k: s.download(k) for k in FIELDS})
    for k in FIELDS:
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)


@pytest.mark.gpu
def test_graph_merge_split_cycles_bitwise(cuda_lib):
    """With merge/split every 10 passes, whole cycles replay from a graph
    captured at the phase of the first call; calls that start at another
    phase run plainly up to it."""
    d = scenarios.mudflow(N=256, merge_split=True)
    out = []
    for graphs in (True, False):
        with Solver(d, merge_split=True) as s:
            s.set_graphs(graphs)
            for n in (5, 23, 3, 31):  # phases 0, 5, 8, 1 at the calls
                s.step(n)
            st = s.status()
            assert st["it"] == 62
            out.append((st, {k: s.download(k) for k in FIELDS + ("label",)}))
    assert out[0][0]["np"] == out[1][0]["np"] and out[0][0]["t"] == out[1][0]["t"]
    for k in FIELDS + ("label",):
        np.testing.assert_array_equal(out[0][1][k], out[1][1][k], err_msg=k)


@pytest.mark.gpu
def test_graph_falls_back_on_an_uncapturable_stream(cuda_lib):
    """On the legacy default stream (handle 1), which CUDA cannot capture, the
    context launches plainly and gives the same state."""
    d = scenarios.dam_break_flat(nsteps=200)
    out = []
    for stream in (None, 1):
        with Solver(d, stream=stream) as s:
            s.step(40)
            assert s.status()["it"] == 40
            out.append({k: s.download(k) for k in FIELDS})
    for k in FIELDS:
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)
