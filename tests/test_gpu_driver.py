"""The optim_par-compatible driver on the GPU against the reference program's
own output files for the same DATA (the golden fixture: every column of
nc_particles_10/20.csv written by main/optim_par.cpp on DATA_bench_1000,
NSTEPS = 20) and against the oracle's nodal vars."""
import os

import numpy as np
import pytest

from amsc_b200 import driver, outputs, scenarios
from amsc_b200.data import to_json
from oracle.oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "optim_par_bench1000.npz")


@pytest.mark.gpu
def test_driver_writes_the_reference_files(cuda_lib, tmp_path):
    d = scenarios.bench_slab(1000, nsteps=20)
    to_json(d, str(tmp_path / "DATA.json"))
    res = driver.run(str(tmp_path / "DATA.json"), outdir=str(tmp_path / "out"))
    assert res["it"] == 20
    out = tmp_path / "out"
    names = sorted(os.listdir(out))
    assert names == ["GRID_forZ.vts", "conservation_errors.csv", "nc_grid_10.vts",
                     "nc_grid_20.vts", "nc_particles_10.csv", "nc_particles_20.csv"]
    g = np.load(GOLDEN)
    for it in (10, 20):
        cols = outputs.read_particles_csv(str(out / f"nc_particles_{it}.csv"))
        assert tuple(cols) == outputs.particle_columns()
        for k in cols:
            np.testing.assert_array_equal(cols[k], g[f"it{it}/{k}"], err_msg=f"{it} {k}")
    err = np.loadtxt(out / "conservation_errors.csv", delimiter=",", skiprows=1, ndmin=2)
    assert err.shape == g["errors"].shape
    np.testing.assert_array_equal(err[:, 0], g["errors"][:, 0])
    np.testing.assert_allclose(err[:, 1:], g["errors"][:, 1:], rtol=0, atol=1e-12)
    o = Oracle(d, threads=4)
    nrows, ncols = int(d.scalars["Ney"]), int(d.scalars["Nex"])
    for it in (10, 20):
        o.run(10)
        v = outputs.read_vts(str(out / f"nc_grid_{it}.vts"), nrows, ncols)
        assert sorted(v) == sorted(outputs.VARS)
        for k in ("Mv", "mom_vx", "vvx", "avy", "F_int_vx", "Fric_y", "HV", "vvxL", "Z"):
            np.testing.assert_array_equal(v[k], o.nodal(k), err_msg=f"{it} {k}")
        np.testing.assert_array_equal(v["F_ext_vx"], o.nodal("FPxv") + o.nodal("Fric_x"))
    z = outputs.read_vts(str(out / "GRID_forZ.vts"), nrows, ncols)
    np.testing.assert_array_equal(z["Z"], d.arrays["Z"])
