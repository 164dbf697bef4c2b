"""Recorded outputs, state round trips and edge cases on the GPU."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import STATE_FIELDS, Solver
from oracle.oracle import Oracle

OUT_FIELDS = ("apx", "apy", "Zp", "hpZ", "dZxp", "dZyp", "Fpx", "Fpy", "Fric_px",
              "Fric_py", "vpx_dx", "vpx_dy", "vpy_dx", "vpy_dy", "vpxL", "vpyL")
NODAL = ("Mv", "mom_vx", "mom_vy", "avx", "avy", "vvx", "vvy", "vvxL", "vvyL", "FPxv",
         "FPyv", "Fric_x", "Fric_y", "F_int_vx", "F_int_vy", "HV")


@pytest.mark.gpu
def test_recorded_fields_bitwise(cuda_lib):
    d = scenarios.bench_slab(1000)
    o = Oracle(d, threads=4)
    o.run(7)
    with Solver(d, record=True) as s:
        s.step(7)
        for k in OUT_FIELDS:
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)
        for k in NODAL:
            np.testing.assert_array_equal(s.download_nodal(k), o.nodal(k), err_msg=k)


@pytest.mark.gpu
def test_state_round_trip(cuda_lib):
    """get_state -> set_state -> step equals stepping through."""
    d = scenarios.bench_slab(3000)
    o = Oracle(d, threads=4)
    o.run(10)
    with Solver(d) as s:
        s.step(5)
        st = s.get_state()
        s.set_state(st)
        s.step(5)
        for k in STATE_FIELDS:
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)


@pytest.mark.gpu
def test_mudflow_small_adaptive(cuda_lib):
    """The mudflow workload scaled to 256x256 (Bingham + Voellmy, bumpy
    terrain, adaptive CFL): 40 steps bitwise."""
    d = scenarios.mudflow(N=256)
    o = Oracle(d, threads=8)
    o.run(40)
    with Solver(d) as s:
        s.step(40)
        st = s.status()
        assert st["it"] == o.it and st["t"] == o.t
        for k in ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_22"):
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)
        led = s.ledgers()
        assert led[6] < 1e-10 and led[7] < 1e-10


@pytest.mark.gpu
def test_edge_pileup_and_walls(cuda_lib):
    """Pile-ups (a cell with 60 particles takes the warp rank sort of the
    per-cell ordering, a cell with 300 the serial one; columns above the P2G
    batch size are split into batches), particles on the domain walls."""
    d = scenarios.dam_break_flat(nsteps=20)
    x, y = d.arrays["x"].copy(), d.arrays["y"].copy()
    x[:60] = 2.126 + 1e-3 * np.arange(60) / 60
    y[:60] = 7.9 + 1e-3 * np.arange(60) / 60
    x[60:700] = 3.9  # one column with ~640 particles
    y[60:700] = np.linspace(0.01, 15.99, 640)
    x[700], y[700] = 0.0, 0.0
    x[701], y[701] = 16.0, 16.0
    x[702:1002] = 1.1 + 1e-2 * np.arange(300) / 300
    y[702:1002] = 3.3 + 1e-2 * np.arange(300)[::-1] / 300
    d.arrays["x"], d.arrays["y"] = x, y
    o = Oracle(d, threads=4)
    o.run(20)
    with Solver(d) as s:
        s.step(20)
        for k in ("x", "y", "vpx", "vpy", "hp", "F_11", "F_22"):
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)


@pytest.mark.gpu
def test_cell_with_twenty_thousand_particles(cuda_lib):
    """One cell holding 20,000 particles: its index order comes from sorted
    runs of 8192 merged pairwise (k_segment_order_big)."""
    d = scenarios.bench_slab(30000, nsteps=3)
    x, y = d.arrays["x"].copy(), d.arrays["y"].copy()
    rng = np.random.default_rng(7)
    pick = rng.permutation(x.size)[:20000]
    hx = float(d.scalars["hx"])
    x[pick] = 40.3 * hx + 0.2 * hx * rng.random(20000)
    y[pick] = 5.3 * hx + 0.2 * hx * rng.random(20000)
    d.arrays["x"], d.arrays["y"] = x, y
    o = Oracle(d, threads=8)
    o.run(3)
    with Solver(d) as s:
        s.step(3)
        for k in ("x", "y", "vpx", "vpy", "hp", "F_11", "F_22"):
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)


@pytest.mark.gpu
def test_odd_grid_and_non_pow2_spacing(cuda_lib):
    """Lake at rest (hx = 0.2, not a power of two; BC off) on a 50x50 grid and
    a 37x23 rectangular grid."""
    d = scenarios.well_balance(T=0.05)
    o = Oracle(d, threads=4)
    o.run(1 << 20)
    with Solver(d) as s:
        s.run()
        for k in ("x", "y", "vpx", "vpy", "hp"):
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)
    d = scenarios.bench_slab(1000, nsteps=15)
    d.scalars.update({"Nex": 37, "Ney": 23})
    n = (37 + 1) * (23 + 1)
    for k in ("Z", "dZdx", "dZdy"):
        d.arrays[k] = np.linspace(0, 1, n) if k == "Z" else np.zeros(n)
    keep = (d.arrays["x"] < 36.5) & (d.arrays["y"] < 22.5)
    for k in ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp", "mom_px", "mom_py", "Vp"):
        d.arrays[k] = d.arrays[k][keep]
    o = Oracle(d, threads=4)
    o.run(15)
    with Solver(d) as s:
        s.step(15)
        for k in ("x", "y", "vpx", "vpy", "hp", "F_11", "F_22"):
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)


@pytest.mark.gpu
def test_empty_and_single_particle(cuda_lib):
    d = scenarios.dam_break_flat(nsteps=5)
    for k in ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp", "mom_px", "mom_py", "Vp"):
        d.arrays[k] = d.arrays[k][:1]
    o = Oracle(d, threads=1)
    o.run(5)
    with Solver(d) as s:
        s.step(5)
        for k in ("x", "y", "vpx", "hp"):
            np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)
    for k in ("x", "y", "Mp", "Ap", "vpx", "vpy", "hp", "mom_px", "mom_py", "Vp"):
        d.arrays[k] = d.arrays[k][:0]
    with Solver(d) as s:
        s.step(5)
        assert s.status()["np"] == 0


@pytest.mark.gpu
def test_staged_download_overlaps_later_steps(cuda_lib):
    """Fields staged before a step hold the particles as they were when the
    call was made, though later steps are enqueued before the copies are
    waited for; they equal the synchronous download of the same state."""
    from amsc_b200.dampm import pinned_array
    d = scenarios.mudflow(N=128)
    names = ("x", "y", "vpx", "hp", "Mp", "H", "mom_px", "label", "level")
    with Solver(d) as s:
        s.step(12)  # the particles are no longer in their initial order
        want = {k: s.download(k) for k in names}
        bufs = {k: pinned_array(s.num_particles + 5) for k in names}
        n = s.stage_download(bufs)
        assert n == s.num_particles
        s.step(6)
        s.staged_wait()
        for k in names:
            np.testing.assert_array_equal(bufs[k][:n], want[k], err_msg=k)
        # the next call reuses the staging buffer after the last copies ended
        want2 = {k: s.download(k) for k in names[:3]}
        n2 = s.stage_download({k: bufs[k] for k in names[:3]})
        s.staged_wait()
        for k in names[:3]:
            np.testing.assert_array_equal(bufs[k][:n2], want2[k], err_msg=k)
        with pytest.raises(Exception):
            s.stage_download({"no_such_field": bufs["x"]})
