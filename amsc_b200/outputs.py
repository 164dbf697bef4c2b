"""The reference's output files, written from fields brought back from the GPU.

  nc_particles_<it>.csv   particles_t::print<csv> (main/optim_par.cpp:311-337):
                          a header of quoted names -- "x", "y", the dprops in
                          map order, the iprops in map order -- then one row
                          per particle, %.17g values (integers for iprops),
                          ", " between columns.
  GRID_forZ.vts,          quadgrid_t::vtk_export (main/optim_par.cpp:269,
  nc_grid_<it>.vts        655-665): an ASCII VTK StructuredGrid, one
                          Float64 DataArray per nodal field in map order
                          (node (r, c) listed row by row), then the node
                          coordinates (c*hx, r*hy, 0).
  conservation_errors.csv "time,err_mass,err_mom" then one row per step, the
                          numbers as a default C++ stream prints them (six
                          significant digits, %g) (main/optim_par.cpp:274,421).

The quadgrid submodule that holds print<csv> and vtk_export is absent from
the reference checkout; these layouts are those of the stand-in the
reference's own programs are built with here (oracle/ref_shim), so the files
the two write for the same run compare equal.
"""
from __future__ import annotations

from typing import Dict, Iterable, Mapping, Sequence

import numpy as np

# dprops of main/optim_par.cpp:139-145 and the iprops of :139
DPROPS = ("Mp", "Ap", "vpx", "vpy", "mom_px", "mom_py", "hp", "Vp", "F_ext_px", "F_ext_py",
          "apx", "apy", "F_11", "F_12", "F_21", "F_22", "vpx_dx", "vpx_dy", "vpy_dx",
          "vpy_dy", "Fb_x", "Fb_y", "hpZ", "dZxp", "dZyp", "Zp", "xp", "yp", "Fric_px",
          "Fric_py", "Fpx", "Fpy", "vpxL", "vpyL", "H")
IPROPS = ("label",)
# vars of main/optim_par.cpp:200-225
VARS = ("Mv", "mom_vx", "mom_vy", "F_ext_vx", "F_ext_vy", "F_int_vx", "F_int_vy", "Fric_x",
        "Fric_y", "div_v", "avx", "avy", "vvx", "vvy", "Z", "dZdx", "dZdy", "Ftot_vx",
        "Ftot_vy", "HV", "FPxv", "FPyv", "vvxL", "vvyL")


def particle_columns() -> Sequence[str]:
    """CSV column order: x, y, dprops and iprops each in std::map order."""
    return ("x", "y") + tuple(sorted(DPROPS)) + tuple(sorted(IPROPS))


def write_particles_csv(path: str, cols: Mapping[str, np.ndarray]) -> None:
    names = particle_columns()
    dnames = names[:-len(IPROPS)]
    n = len(cols["x"])
    arrays = [np.asarray(cols[k], dtype=np.float64) for k in dnames]
    ints = [np.asarray(cols[k]).astype(np.int64) for k in IPROPS]
    with open(path, "w") as f:
        f.write(", ".join(f'"{k}"' for k in names) + "\n")
        fmt = ", ".join(["%.17g"] * len(dnames) + ["%d"] * len(IPROPS)) + "\n"
        rows = [tuple(a[i] for a in arrays) + tuple(int(a[i]) for a in ints) for i in range(n)]
        f.write("".join(fmt % r for r in rows))


def read_particles_csv(path: str) -> Dict[str, np.ndarray]:
    with open(path) as f:
        header = [c.strip().strip('"') for c in f.readline().split(",")]
        data = np.loadtxt(f, delimiter=",", ndmin=2)
    return {k: data[:, j].copy() for j, k in enumerate(header)}


def _shortest(v: float) -> str:
    # shortest text that reads back as the same double (std::to_chars' choice)
    s = repr(float(v))
    return s[:-2] if s.endswith(".0") else s


def write_vts(path: str, nrows: int, ncols: int, hx: float, hy: float,
              fields: Mapping[str, np.ndarray]) -> None:
    NR, NC = nrows + 1, ncols + 1
    out = ['<?xml version="1.0"?>\n<VTKFile type="StructuredGrid" version="0.1" '
           'byte_order="LittleEndian">\n'
           f'<StructuredGrid WholeExtent="0 {ncols} 0 {nrows} 0 0">\n'
           f'<Piece Extent="0 {ncols} 0 {nrows} 0 0">\n<PointData>\n']
    for k in sorted(fields):
        a = np.asarray(fields[k], dtype=np.float64).reshape(NC, NR)  # node r + c*NR
        out.append(f'<DataArray type="Float64" Name="{k}" format="ascii">\n')
        out.append("\n".join(_shortest(v) for v in a.T.reshape(-1)) + "\n")
        out.append("</DataArray>\n")
    out.append('</PointData>\n<Points>\n<DataArray type="Float64" NumberOfComponents="3" '
               'format="ascii">\n')
    out.append("".join("%.17g %.17g 0\n" % (c * hx, r * hy)
                       for r in range(NR) for c in range(NC)))
    out.append("</DataArray>\n</Points>\n</Piece>\n</StructuredGrid>\n</VTKFile>\n")
    with open(path, "w") as f:
        f.write("".join(out))


def read_vts(path: str, nrows: int, ncols: int) -> Dict[str, np.ndarray]:
    """Nodal fields of a VTS file, back in quadgrid node order."""
    NR, NC = nrows + 1, ncols + 1
    fields, name, vals = {}, None, []
    with open(path) as f:
        for line in f:
            if line.startswith('<DataArray type="Float64" Name="'):
                name, vals = line.split('Name="')[1].split('"')[0], []
            elif line.startswith("</DataArray>") and name is not None:
                fields[name] = np.array(vals, dtype=np.float64).reshape(NR, NC).T.reshape(-1)
                name = None
            elif name is not None:
                vals.append(float(line))
    return fields


def write_errors_header(f) -> None:
    f.write("time,err_mass,err_mom\n")


def write_error_rows(f, rows: Iterable[Sequence[float]]) -> None:
    f.write("".join("%g,%g,%g\n" % (t, em, ep) for t, em, ep in rows))
