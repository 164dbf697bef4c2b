"""DATA.json input (main/mpm_data.h): keys, defaults, exact round trip."""
import json

import numpy as np
import pytest

from amsc_b200 import data, scenarios


def test_round_trip_exact(tmp_path):
    d = scenarios.dam_break_flat()
    p = tmp_path / "DATA.json"
    data.to_json(d, str(p))
    e = data.from_json(str(p))
    for k, v in d.arrays.items():
        np.testing.assert_array_equal(e.arrays[k], v)
    for k, v in d.scalars.items():
        assert e.scalars[k] == v


def test_defaults_and_required(tmp_path):
    d = scenarios.dam_break_flat()
    j = {k: v.tolist() for k, v in d.arrays.items()}
    j.update({k: v for k, v in d.scalars.items() if not k.startswith("ms_") and k not in ("DT_FIXED", "NSTEPS")})
    e = data.from_dict(j)
    # main/mpm_data.h:99-112
    assert e.scalars["DT_FIXED"] == 0.0 and e.scalars["NSTEPS"] == 0
    assert e.scalars["ms_alpha"] == 0.9 and e.scalars["ms_beta"] == 0.30
    assert e.scalars["ms_shear_split"] == 1e30 and e.scalars["ms_max_ops"] == 1e9
    assert e.scalars["ms_min_level"] == -2 and e.scalars["ms_call_interval"] == 10
    del j["tauy"]
    with pytest.raises(data.DataError):
        data.from_dict(j)


def test_size_validation():
    d = scenarios.dam_break_flat()
    d.arrays["hp"] = d.arrays["hp"][:-1]
    with pytest.raises(data.DataError):
        d.validate()


def test_scenario_shapes():
    d = scenarios.dam_break_flat()
    assert d.np == 4096 and d.nnodes == 65 * 65
    assert np.all(d.arrays["Z"] == 0)
    m = scenarios.mudflow(N=256)
    assert abs(m.np - 4021256 / 64) / (4021256 / 64) < 0.02  # same shapes scaled
    assert np.all(m.arrays["hp"] > 0) and m.scalars["BINGHAM_ON"] == 1.0
    e = scenarios.ensemble_member(3)
    assert 64 <= e.scalars["Nex"] <= 512 and e.scalars["DT_FIXED"] == 0.02
