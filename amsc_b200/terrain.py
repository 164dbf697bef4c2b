"""Terrain import: a digital terrain model (DTM) raster to the node arrays
Z, dZdx, dZdy of a DATA scenario.

The reference builds its real-terrain scenarios with Octave scripts:
data/fena/input_fena.m reads the GeoTIFF dtm_liguria_2017.tif (converted to
text by data/fena/convert.py), crops a window, flips it so that row 0 is the
southern edge (y grows upward), clamps the sea to -1 m and takes the
gradient; data/cortenova/cortenova_entire_dtm.m does the same from a
MATLAB .mat DEM.  This module restates those steps:

* :func:`read_geotiff` -- a single-band GeoTIFF (strips or tiles; no
  compression, Deflate, LZW or PackBits; horizontal predictor), returned as
  float64 with row 0 the raster's first (northern) row;
* :func:`read_mat` -- a numeric variable of a MATLAB .mat file;
* :func:`window` -- Octave's 1-based inclusive ``A(r0:r1, c0:c1)``;
* :func:`nodes_from_grid` -- a grid with row 0 at y = 0 into quadgrid node
  order (node (r, c) at r + c*(Ney+1), Octave's column-major ``Z(:)``) with
  Octave's ``gradient`` (central differences inside, one-sided at the edges);
* :func:`fena_terrain` -- the whole terrain step of input_fena.m.
"""
from __future__ import annotations

import struct
import zlib
from typing import Dict, Tuple

import numpy as np

_TYPES = {1: ("B", 1), 2: ("c", 1), 3: ("H", 2), 4: ("I", 4), 5: ("II", 8), 6: ("b", 1),
          7: ("B", 1), 8: ("h", 2), 9: ("i", 4), 10: ("ii", 8), 11: ("f", 4),
          12: ("d", 8), 16: ("Q", 8)}


class TerrainError(ValueError):
    pass


def _ifd(buf: bytes, bo: str, off: int) -> Dict[int, tuple]:
    n = struct.unpack(bo + "H", buf[off:off + 2])[0]
    tags = {}
    for k in range(n):
        e = off + 2 + 12 * k
        tag, typ, cnt = struct.unpack(bo + "HHI", buf[e:e + 8])
        if typ not in _TYPES:
            continue
        fmt, size = _TYPES[typ]
        nbytes = size * cnt
        data = buf[e + 8:e + 12] if nbytes <= 4 else \
            buf[struct.unpack(bo + "I", buf[e + 8:e + 12])[0]:][:nbytes]
        if typ == 2:
            tags[tag] = (data.rstrip(b"\0").decode("latin-1"),)
        elif typ in (5, 10):
            tags[tag] = struct.unpack(bo + fmt[0] * (2 * cnt), data)
        else:
            tags[tag] = struct.unpack(bo + fmt * cnt, data[:nbytes])
    return tags


def _lzw_decode(data: bytes) -> bytes:
    """TIFF LZW (MSB-first codes, 9 to 12 bits, Clear 256, EOI 257)."""
    out = bytearray()
    table = [bytes([i]) for i in range(256)] + [b"", b""]
    width, bitbuf, nbits, prev = 9, 0, 0, None
    for byte in data:
        bitbuf = (bitbuf << 8) | byte
        nbits += 8
        while nbits >= width:
            nbits -= width
            code = (bitbuf >> nbits) & ((1 << width) - 1)
            if code == 256:
                table = table[:258]
                width, prev = 9, None
                continue
            if code == 257:
                return bytes(out)
            if prev is None:
                entry = table[code]
            elif code < len(table):
                entry = table[code]
                table.append(prev + entry[:1])
            else:
                entry = prev + prev[:1]
                table.append(entry)
            out += entry
            prev = entry
            # the early change of TIFF's LZW: widen one code before the table fills
            if len(table) + 1 >= (1 << width) and width < 12:
                width += 1
    return bytes(out)


def _packbits_decode(data: bytes) -> bytes:
    out = bytearray()
    i = 0
    while i < len(data):
        n = data[i] if data[i] < 128 else data[i] - 256
        i += 1
        if n >= 0:
            out += data[i:i + n + 1]
            i += n + 1
        elif n != -128:
            out += data[i:i + 1] * (1 - n)
            i += 1
    return bytes(out)


def read_geotiff(path: str) -> np.ndarray:
    """The first band of a GeoTIFF as float64, row 0 first in the file."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:4] not in (b"II*\0", b"MM\0*"):
        raise TerrainError(f"{path}: not a classic TIFF")
    bo = "<" if buf[:2] == b"II" else ">"
    t = _ifd(buf, bo, struct.unpack(bo + "I", buf[4:8])[0])
    width, height = t[256][0], t[257][0]
    bits = t.get(258, (1,))[0]
    comp = t.get(259, (1,))[0]
    spp = t.get(277, (1,))[0]
    pred = t.get(317, (1,))[0]
    fmt = t.get(339, (1,))[0]
    kind = {1: "u", 2: "i", 3: "f"}.get(fmt)
    if kind is None or bits not in (8, 16, 32, 64):
        raise TerrainError(f"{path}: sample format {fmt}/{bits} bits not supported")
    dt = np.dtype(f"{bo}{kind}{bits // 8}")
    if 322 in t:  # tiles
        tw, th = t[322][0], t[323][0]
        offs, counts = t[324], t[325]
        blocks = [(r, c) for r in range(0, height, th) for c in range(0, width, tw)]
        bw, bh = tw, th
    else:  # strips
        rps = t.get(278, (height,))[0]
        offs, counts = t[273], t[279]
        blocks = [(r, 0) for r in range(0, height, rps)]
        bw, bh = width, rps
    out = np.empty((height, width), dtype=np.float64)
    for (r0, c0), off, cnt in zip(blocks, offs, counts):
        raw = buf[off:off + cnt]
        if comp == 1:
            data = raw
        elif comp in (8, 32946):
            data = zlib.decompress(raw)
        elif comp == 5:
            data = _lzw_decode(raw)
        elif comp == 32773:
            data = _packbits_decode(raw)
        else:
            raise TerrainError(f"{path}: compression {comp} not supported")
        rows = bh if 322 in t else min(bh, height - r0)
        a = np.frombuffer(data, dtype=dt, count=rows * bw * spp).reshape(rows, bw, spp)[:, :, 0]
        if pred == 2:  # horizontal differencing, in the sample type
            a = np.cumsum(a, axis=1, dtype=dt)
        elif pred != 1:
            raise TerrainError(f"{path}: predictor {pred} not supported")
        h = min(rows, height - r0)
        w = min(bw, width - c0)
        out[r0:r0 + h, c0:c0 + w] = a[:h, :w]
    return out


def read_mat(path: str, name: str) -> np.ndarray:
    """A numeric variable of a MATLAB .mat file (v5), as float64."""
    from scipy.io import loadmat
    m = loadmat(path)
    if name not in m:
        raise TerrainError(f"{path}: no variable '{name}'")
    return np.asarray(m[name], dtype=np.float64)


def window(A: np.ndarray, rows: Tuple[int, int], cols: Tuple[int, int]) -> np.ndarray:
    """Octave's ``A(r0:r1, c0:c1)``: 1-based, both ends included."""
    (r0, r1), (c0, c1) = rows, cols
    if not (1 <= r0 <= r1 <= A.shape[0] and 1 <= c0 <= c1 <= A.shape[1]):
        raise TerrainError(f"window {rows} x {cols} outside a {A.shape} raster")
    return A[r0 - 1:r1, c0 - 1:c1].copy()


def octave_gradient(Z: np.ndarray, dx: float = 1.0, dy: float = 1.0):
    """Octave's ``[gx, gy] = gradient(Z, dx, dy)`` for Z indexed (row = y,
    column = x): (Z[:, i+1] - Z[:, i-1]) / (2 dx) inside, one-sided
    differences at the edges."""
    gx = np.empty_like(Z)
    gy = np.empty_like(Z)
    for g, A, h, axis in ((gx, Z, dx, 1), (gy, Z, dy, 0)):
        n = A.shape[axis]
        sl = lambda a, b: (slice(None), slice(a, b)) if axis == 1 else (slice(a, b), slice(None))
        if n < 2:
            g[...] = 0.0
            continue
        g[sl(0, 1)] = (A[sl(1, 2)] - A[sl(0, 1)]) / h
        g[sl(n - 1, n)] = (A[sl(n - 1, n)] - A[sl(n - 2, n - 1)]) / h
        if n > 2:
            g[sl(1, n - 1)] = (A[sl(2, n)] - A[sl(0, n - 2)]) / (2.0 * h)
    return gx, gy


def nodes_from_grid(Zg: np.ndarray, gradient_spacing: Tuple[float, float] = (1.0, 1.0)):
    """Z, dZdx, dZdy in quadgrid node order from a grid with row 0 at y = 0
    (shape (Ney+1, Nex+1)).  The gradient spacing defaults to 1, as the
    reference's importers call ``gradient(Z)`` without spacings (the step
    recomputes the terrain gradient from Z at the particles, so dZdx/dZdy
    feed only the initial recorded fields)."""
    gx, gy = octave_gradient(Zg, *gradient_spacing)
    col = lambda a: np.ascontiguousarray(a.reshape(-1, order="F"))
    return col(Zg), col(gx), col(gy)


FENA_ROWS = (550, 900)  # data/fena/input_fena.m:6-10
FENA_COLS = (171, 430)
FENA_H = 5.0


def fena_terrain(tif_path: str) -> Dict[str, object]:
    """The terrain step of data/fena/input_fena.m:6-60 from the GeoTIFF:
    rows 550..900 and columns 171..430 of the raster, flipped so that row 0
    is the southern edge, heights below 0 set to -1 (then the zero and
    negative heights to -1 as well), at hx = hy = 5 m."""
    raster = read_geotiff(tif_path)
    g = window(raster, FENA_ROWS, FENA_COLS)[::-1, :]
    g[g < 0] = -1.0
    g[g <= 0] = -1.0
    Z, dZdx, dZdy = nodes_from_grid(g)
    return {"Z": Z, "dZdx": dZdx, "dZdy": dZdy, "Nex": g.shape[1] - 1,
            "Ney": g.shape[0] - 1, "hx": FENA_H, "hy": FENA_H}
