"""The output writers (no GPU): column order, number formats, round trips."""
import numpy as np

from amsc_b200 import outputs


def test_csv_columns_in_map_order_and_exact_round_trip(tmp_path):
    names = outputs.particle_columns()
    assert names[:2] == ("x", "y") and names[-1] == "label"
    assert list(names[2:-1]) == sorted(names[2:-1])  # std::map order
    assert names.index("F_11") < names.index("Mp") < names.index("apx")  # bytes, not case-folded
    rng = np.random.default_rng(3)
    cols = {k: rng.standard_normal(7) * 10.0 ** rng.integers(-20, 20) for k in names[:-1]}
    cols["x"][0] = -0.0
    cols["label"] = np.arange(7)
    p = tmp_path / "nc_particles_10.csv"
    outputs.write_particles_csv(str(p), cols)
    head = p.read_text().splitlines()[0]
    assert head.startswith('"x", "y", "Ap", "F_11"')
    back = outputs.read_particles_csv(str(p))
    for k in names:
        np.testing.assert_array_equal(back[k], np.asarray(cols[k], dtype=np.float64), err_msg=k)


def test_vts_round_trip_in_node_order(tmp_path):
    nrows, ncols = 3, 4
    nn = (nrows + 1) * (ncols + 1)
    rng = np.random.default_rng(5)
    f = {"Z": rng.standard_normal(nn), "HV": rng.standard_normal(nn) * 1e-7}
    p = tmp_path / "g.vts"
    outputs.write_vts(str(p), nrows, ncols, 0.5, 0.25, f)
    text = p.read_text()
    assert 'WholeExtent="0 4 0 3 0 0"' in text and text.index('Name="HV"') < text.index('Name="Z"')
    back = outputs.read_vts(str(p), nrows, ncols)
    for k in f:
        np.testing.assert_array_equal(back[k], f[k])


def test_error_rows_like_a_default_cpp_stream():
    import io
    s = io.StringIO()
    outputs.write_errors_header(s)
    outputs.write_error_rows(s, [(0.0, 0.0, 0.0), (0.001, 1.9798531e-16, 1.534712e-14)])
    assert s.getvalue() == "time,err_mass,err_mom\n0,0,0\n0.001,1.97985e-16,1.53471e-14\n"
