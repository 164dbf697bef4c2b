"""The terrain importer (amsc_b200/terrain.py) on the CPU.

* The reference's own real-terrain input: data/fena/input_fena.m turns the
  GeoTIFF dtm_liguria_2017.tif into the Z, dZdx, dZdy of the shipped
  data/fena/DATA.json (259 x 350 cells).  The importer reproduces those
  three arrays bit for bit (where the reference checkout is present).
* The codecs the reader supports, on small rasters written by Pillow.
"""
import json
import os

import numpy as np
import pytest

from amsc_b200 import terrain
from oracle import refrun


def test_fena_terrain_equals_shipped_data_json():
    root = refrun.reference_root()
    if root is None:
        pytest.skip("reference checkout absent")
    tif = os.path.join(root, "data", "fena", "dtm_liguria_2017.tif")
    shipped = json.load(open(os.path.join(root, "data", "fena", "DATA.json")))
    t = terrain.fena_terrain(tif)
    assert (t["Nex"], t["Ney"], t["hx"], t["hy"]) == (shipped["Nex"], shipped["Ney"],
                                                       shipped["hx"], shipped["hy"])
    for k in ("Z", "dZdx", "dZdy"):
        np.testing.assert_array_equal(t[k], np.asarray(shipped[k], dtype=np.float64),
                                      err_msg=k)


@pytest.mark.parametrize("compression", [None, "tiff_adobe_deflate", "tiff_lzw", "packbits"])
@pytest.mark.parametrize("mode", ["I;16", "I", "F"])
def test_geotiff_codecs(tmp_path, compression, mode):
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(3)
    if mode == "F":
        a = rng.normal(300.0, 80.0, size=(37, 53)).astype(np.float32)
        img = Image.fromarray(a, mode="F")
    elif mode == "I":
        a = rng.integers(-3000, 3000, size=(37, 53)).astype(np.int32)
        img = Image.fromarray(a, mode="I")
    else:
        a = rng.integers(0, 60000, size=(37, 53)).astype(np.uint16)
        img = Image.frombytes("I;16", (53, 37), a.astype("<u2").tobytes())
    path = str(tmp_path / "t.tif")
    try:
        img.save(path, compression=compression) if compression else img.save(path)
    except (OSError, ValueError, KeyError) as e:
        pytest.skip(f"Pillow cannot write {compression}/{mode}: {e}")
    np.testing.assert_array_equal(terrain.read_geotiff(path), a.astype(np.float64))


def test_gradient_and_node_order():
    rng = np.random.default_rng(5)
    g = rng.normal(size=(7, 11))
    gx, gy = terrain.octave_gradient(g, 2.0, 0.5)
    np.testing.assert_array_equal(gx, np.gradient(g, 2.0, axis=1, edge_order=1))
    np.testing.assert_array_equal(gy, np.gradient(g, 0.5, axis=0, edge_order=1))
    Z, _, _ = terrain.nodes_from_grid(g)
    Ney = g.shape[0] - 1
    for r, c in ((0, 0), (3, 4), (6, 10)):
        assert Z[r + c * (Ney + 1)] == g[r, c]  # node (r, c) at r + c*(Ney+1)
    with pytest.raises(terrain.TerrainError):
        terrain.window(g, (0, 3), (1, 2))
