"""The FP32 form (batches with precision="fp32") against the FP64 path.

Stated errors, from runs of these scenarios (FP32 vs FP64, same passes):
  * mass: the per-pass conservation error of the FP32 nodal sums stays below
    1e-8 and the particle mass totals agree to ~1e-9 (tolerance 1e-6);
  * depth hp, relative L2 over the particles: dam break without yield stress
    1.8e-5 after 500 passes, the low-yield-stress bench slab 4.3e-5 after
    200 (tolerance 1e-4);
  * yield-stress flows (tau_y of hundreds of Pa): the Bingham stress
    tau_y/sqrt(II) switches sharply where the flow plugs, so FP32 and FP64
    trajectories part after tens of passes: 5e-4 to 1.2e-3 after 50 passes,
    1e-2 after 200 (tolerance 1e-2 at 50 passes).
The FP32 form is deterministic: a scenario's FP32 numbers are the same alone
and in a batch (tolerance 0)."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.batch import Batch
from amsc_b200.serving import Request, Server


def run(ds, passes, precision):
    P = sum(d.np for d in ds) + 64
    N = sum(d.nnodes for d in ds) + 64
    with Batch(P, N, len(ds) + 1, precision=precision) as b:
        hs = [b.add(d) for d in ds]
        b.step(passes)
        b.sync()
        return [({k: b.download(h, k) for k in ("x", "y", "hp")}, b.ledgers(h)) for h in hs]


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
def test_fp32_smooth_flows_depth_and_mass(cuda_lib):
    for d, passes in ((scenarios.dam_break_flat(nsteps=500), 500),
                      (scenarios.bench_slab(10000, nsteps=1000), 200)):
        (f64, l64), = run([d], passes, "fp64")
        (f32, l32), = run([d], passes, "fp32")
        assert rel_l2(f32["hp"], f64["hp"]) <= 1e-4
        assert l32[6] <= 1e-6                           # err_mass of the last pass
        assert abs(l32[0] - l64[0]) <= 1e-6 * l64[0]    # particle mass total


@pytest.mark.gpu
def test_fp32_yield_stress_flow_stated_error(cuda_lib):
    d = scenarios.ensemble_member(1, side_range=(48, 160))
    (f64, l64), = run([d], 50, "fp64")
    (f32, l32), = run([d], 50, "fp32")
    assert rel_l2(f32["hp"], f64["hp"]) <= 1e-2
    assert l32[6] <= 1e-6 and abs(l32[0] - l64[0]) <= 1e-6 * l64[0]


@pytest.mark.gpu
def test_fp32_same_alone_and_in_batch(cuda_lib):
    a = scenarios.ensemble_member(2, side_range=(48, 96))
    others = [scenarios.ensemble_member(s, side_range=(48, 128)) for s in (3, 4)]
    (alone, _), = run([a], 40, "fp32")
    mixed = run(others + [a], 40, "fp32")[-1][0]
    for k in alone:
        np.testing.assert_array_equal(mixed[k], alone[k], err_msg=k)


@pytest.mark.gpu
def test_fp32_serving_same_as_alone(cuda_lib):
    ds = []
    for s in (5, 6, 7):
        d = scenarios.ensemble_member(s, side_range=(48, 96))
        d.scalars.update({"DT_FIXED": 0.0, "NSTEPS": 0, "T": 0.6, "CFL": 0.4})
        ds.append(d)
    reqs = [Request(k, d, arrival=0.0) for k, d in enumerate(ds)]
    with Server(1e9, max_scenarios=8, tick=4, precision="fp32") as srv:
        srv.run(reqs)
    for r in reqs:
        with Batch(r.data.np + 64, r.data.nnodes + 64, 2, precision="fp32") as b:
            h = b.add(r.data)
            while b.query(h)["running"]:
                b.step(8)
            for k in ("x", "y", "hp"):
                np.testing.assert_array_equal(r.result[k], b.download(h, k), err_msg=k)
