"""The reference-side C++ driver of the C ABI (tests/binding/b200_offload.cpp).

It reads DATA.json through the reference's own DATA struct
(main/mpm_data.h) and fills dampm_grid / dampm_params / dampm_ms_params from
it by position, as a maintainer of the reference would.  Built against the
reference checkout into oracle/_ref; where that build is absent the test is
skipped.  Its final state must equal the Python binding's, bit for bit: a
field-order slip between DATA and the C structs would change the run.
"""
import os
import subprocess

import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import Solver
from amsc_b200.data import to_json
from oracle import refrun


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["bench_slab", "mudflow_cfl"])
def test_reference_side_driver_matches_python_binding(cuda_lib, tmp_path, case):
    if not os.path.exists(refrun.BINDING):
        pytest.skip("the reference-side driver was not built (no reference checkout)")
    if case == "bench_slab":  # Bingham + Voellmy, fixed dt
        d = scenarios.bench_slab(3000, nsteps=40)
    else:  # adaptive CFL until T, bumpy terrain, merge/split on at its cadence
        d = scenarios.mudflow(N=128, merge_split=True)
        d.scalars.update({"T": 0.5, "DT_FIXED": 0.0, "NSTEPS": 0})
    to_json(d, str(tmp_path / "DATA.json"))
    out = subprocess.run([refrun.BINDING], cwd=tmp_path, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    line = out.stdout.strip().splitlines()[-1]
    kv = dict(f.split("=") for f in line.split())
    raw = np.fromfile(tmp_path / "state.bin", dtype=np.float64)
    n = int(kv["np"])
    got = dict(zip(("x", "y", "vpx", "vpy", "hp"), raw.reshape(5, n)))
    with Solver(d, merge_split=True) as s:
        s.run()
        st = s.status()
        assert int(kv["it"]) == st["it"] and float(kv["t"]) == st["t"] and n == st["np"]
        for k, v in got.items():
            np.testing.assert_array_equal(v, s.download(k), err_msg=k)
