"""The library's streaming DATA.json reader (dampm_json_*, used by
amsc_b200.data.from_json) against Python's json on the same text."""
import json

import numpy as np
import pytest

from amsc_b200 import data, scenarios
from amsc_b200.dampm import DampmError


def test_round_trip_of_a_generated_scenario_is_exact(tmp_path):
    d = scenarios.mudflow(N=96)
    p = str(tmp_path / "DATA.json")
    data.to_json(d, p)
    e = data.from_json(p)
    for k, a in d.arrays.items():
        np.testing.assert_array_equal(e.arrays[k], a, err_msg=k)
    assert e.scalars == d.scalars


def test_numbers_parse_as_python_float_does(tmp_path):
    vals = [0.0, -0.0, 1.0, -1.5, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
            0.1, 1e22, 123456789012345678, 3.141592653589793, -2.5e-7, 1e-300]
    rng = np.random.default_rng(0)
    vals += list(rng.standard_normal(500) * 10.0 ** rng.integers(-200, 200, 500))
    text = '{"x": [%s], "Nex": 3, "nested": [[1, 2], [3, [4.5e-3]]], "one": 7.25}' % (
        ", ".join(repr(float(v)) for v in vals))
    p = tmp_path / "t.json"
    p.write_text(text)
    import ctypes as C
    from amsc_b200.dampm import load_library
    lib = load_library()
    h = C.c_void_p()
    assert lib.dampm_json_read(str(p).encode(), C.byref(h)) == 0
    ref = json.loads(text)

    def get(k):
        n = C.c_longlong()
        lib.dampm_json_size(h, k.encode(), C.byref(n))
        out = np.empty(max(n.value, 1))
        assert lib.dampm_json_get(h, k.encode(), out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return out[:n.value]

    np.testing.assert_array_equal(get("x"), np.array(ref["x"], dtype=np.float64))
    assert np.signbit(get("x")[1])
    np.testing.assert_array_equal(get("nested"), [1.0, 2.0, 3.0, 4.5e-3])
    assert list(get("one")) == [7.25] and list(get("Nex")) == [3.0]
    n = C.c_longlong()
    lib.dampm_json_size(h, b"absent", C.byref(n))
    assert n.value == -1
    lib.dampm_json_free(h)


def test_one_particle_written_as_a_scalar(tmp_path):
    d = scenarios.dam_break_flat(nsteps=5)
    j = {k: v.tolist() for k, v in d.arrays.items()}
    for k in data.PARTICLE_KEYS:
        j[k] = float(d.arrays[k][0])  # a single value, as v2j writes a 1x1 matrix
    j.update(d.scalars)
    p = tmp_path / "DATA.json"
    p.write_text(json.dumps(j))
    e = data.from_json(str(p))
    assert e.np == 1 and e.arrays["x"][0] == d.arrays["x"][0]


def test_bad_values_and_missing_keys_are_errors(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{"x": [1, 2], "name": "slope"}')
    with pytest.raises(DampmError, match="name"):
        data.from_json(str(p))
    p.write_text('{"x": [1, 2]}')
    with pytest.raises(data.DataError):
        data.from_json(str(p))
    with pytest.raises(DampmError):
        data.from_json(str(tmp_path / "absent.json"))
