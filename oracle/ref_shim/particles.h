// TEST INFRASTRUCTURE ONLY -- stand-in for particles_t of the absent
// `quadgrid` submodule (.gitmodules:1-4 of the reference project), restating
// the interface the reference's main/*.cpp and main/merge_split_ops_cmes.h
// use.  Its transfer operators are the same restatement as the CPU oracle
// (oracle/dampm_oracle.cpp):
//   * init_particle_mesh: cell (floor(y/hy), floor(x/hx)) clamped; grd_to_ptcl
//     and the CSR cell_start/cell_ptcls in (cell, particle index) order; four
//     colours (r%2) + 2*(c%2) for the colour lists gpu_offload launches over;
//   * p2g / p2gd: the quadgrid cell sweep -- cells by id, particles by index,
//     local nodes 0..3, vars[out] += contribution;
//   * g2p / g2pd: per particle, local nodes 0..3, dprops[out] += N * var;
//   * shape functions of main/gpu_kernels.cpp:21-59;
//   * print<csv>: a header of quoted names ("x", "y", the dprops in map order,
//     the iprops in map order) and one row per particle, %.17g.
// build_mass() has no visible effect in the reference's callers and is a
// no-op here.
#pragma once
#include <algorithm>
#include <cmath>
#include <fstream>
#include <iostream>
#include <map>
#include <numeric>
#include <ostream>
#include <string>
#include <vector>

#include "quadgrid_cpp.h"

class particles_t {
 public:
  using idx_t = int;
  using grid_t = quadgrid_t<std::vector<double>>;
  enum class output_format { csv };

  idx_t num_particles;
  std::vector<double> x, y;
  std::map<std::string, std::vector<double>> dprops;
  std::map<std::string, std::vector<idx_t>> iprops;
  const grid_t& grid;

  std::map<idx_t, std::vector<idx_t>> grd_to_ptcl;
  std::vector<int> ptcl_to_grd, cell_start, cell_ptcls, color_cell_idx;
  int color_offsets[5] = {0, 0, 0, 0, 0};

  particles_t(idx_t n, const std::vector<std::string>& inames,
              const std::vector<std::string>& dnames, const grid_t& g,
              const std::vector<double>& xx, const std::vector<double>& yy)
      : num_particles(n), x(xx), y(yy), grid(g) {
    for (auto const& k : dnames) dprops[k].assign(n, 0.0);
    for (auto const& k : inames) iprops[k].assign(n, 0);
    init_particle_mesh();
  }

  void build_mass() {}

  void init_particle_mesh() {
    const idx_t nr = grid.num_rows(), nc = grid.num_cols(), ncell = nr * nc;
    ptcl_to_grd.assign(num_particles, 0);
    cell_start.assign(ncell + 1, 0);
    grd_to_ptcl.clear();
    for (idx_t i = 0; i < num_particles; ++i) {
      double fr = std::floor(y[i] / grid.hy()), fc = std::floor(x[i] / grid.hx());
      idx_t r = !(fr >= 0.0) ? 0 : (fr > double(nr - 1) ? nr - 1 : idx_t(fr));
      idx_t c = !(fc >= 0.0) ? 0 : (fc > double(nc - 1) ? nc - 1 : idx_t(fc));
      ptcl_to_grd[i] = r + c * nr;
      cell_start[ptcl_to_grd[i] + 1]++;
      grd_to_ptcl[ptcl_to_grd[i]].push_back(i);
    }
    for (idx_t k = 0; k < ncell; ++k) cell_start[k + 1] += cell_start[k];
    std::vector<int> fill(cell_start.begin(), cell_start.end() - 1);
    cell_ptcls.assign(num_particles, 0);
    for (idx_t i = 0; i < num_particles; ++i) cell_ptcls[fill[ptcl_to_grd[i]]++] = i;
    color_cell_idx.assign(ncell, 0);
    int pos = 0;
    for (int col = 0; col < 4; ++col) {
      color_offsets[col] = pos;
      for (idx_t cell = 0; cell < ncell; ++cell) {
        const idx_t r = cell % nr, c = cell / nr;
        if ((r % 2) + 2 * (c % 2) == col) color_cell_idx[pos++] = cell;
      }
    }
    color_offsets[4] = pos;
  }

  // shape functions (main/gpu_kernels.cpp:33-59) in local coordinates
  static double shp(double xi, double eta, int inode) {
    switch (inode) {
      case 3: return xi * eta;
      case 2: return xi * (1.0 - eta);
      case 1: return (1.0 - xi) * eta;
      default: return (1.0 - xi) * (1.0 - eta);
    }
  }
  static double shg(double xi, double eta, int idir, int inode, double hx, double hy) {
    switch (inode) {
      case 3: return idir == 0 ? (1.0 / hx) * eta : xi * (1.0 / hy);
      case 2: return idir == 0 ? (1.0 / hx) * (1.0 - eta) : xi * (-1.0 / hy);
      case 1: return idir == 0 ? (-1.0 / hx) * eta : (1.0 - xi) * (1.0 / hy);
      default: return idir == 0 ? (-1.0 / hx) * (1.0 - eta) : (1.0 - xi) * (-1.0 / hy);
    }
  }
  void local(idx_t ip, idx_t cell, double& xi, double& eta, idx_t& r, idx_t& c) const {
    r = cell % grid.num_rows();
    c = cell / grid.num_rows();
    xi = (x[ip] - c * grid.hx()) / grid.hx();
    eta = (y[ip] - r * grid.hy()) / grid.hy();
  }
  idx_t gt(int inode, idx_t r, idx_t c) const {
    const idx_t bl = r + c * (grid.num_rows() + 1);
    switch (inode) {
      case 0: return bl;
      case 1: return bl + 1;
      case 2: return bl + (grid.num_rows() + 1);
      default: return bl + (grid.num_rows() + 2);
    }
  }

  void p2g(std::map<std::string, std::vector<double>>& vars,
           const std::vector<std::string>& pnames,
           const std::vector<std::string>& gnames) const {
    const size_t nv = pnames.size();
    std::vector<const double*> src(nv);
    std::vector<double*> dst(nv);
    for (size_t v = 0; v < nv; ++v) {
      src[v] = dprops.at(pnames[v]).data();
      dst[v] = vars[gnames[v]].data();
    }
    for (auto const& kv : grd_to_ptcl)
      for (idx_t ip : kv.second) {
        double xi, eta;
        idx_t r, c;
        local(ip, kv.first, xi, eta, r, c);
        for (int inode = 0; inode < 4; ++inode) {
          const double N = shp(xi, eta, inode);
          const idx_t n = gt(inode, r, c);
          for (size_t v = 0; v < nv; ++v) dst[v][n] += N * src[v][ip];
        }
      }
  }

  // out[k] += (Nx * xnames[k] + Ny * ynames[k]) * w
  void p2gd(std::map<std::string, std::vector<double>>& vars,
            const std::vector<std::string>& xnames,
            const std::vector<std::string>& ynames, const std::string& wname,
            const std::vector<std::string>& gnames) const {
    const double* w = dprops.at(wname).data();
    const size_t nv = gnames.size();
    std::vector<const double*> sx(nv), sy(nv);
    std::vector<double*> dst(nv);
    for (size_t v = 0; v < nv; ++v) {
      sx[v] = dprops.at(xnames[v]).data();
      sy[v] = dprops.at(ynames[v]).data();
      dst[v] = vars[gnames[v]].data();
    }
    for (auto const& kv : grd_to_ptcl)
      for (idx_t ip : kv.second) {
        double xi, eta;
        idx_t r, c;
        local(ip, kv.first, xi, eta, r, c);
        for (int inode = 0; inode < 4; ++inode) {
          const double Nx = shg(xi, eta, 0, inode, grid.hx(), grid.hy());
          const double Ny = shg(xi, eta, 1, inode, grid.hx(), grid.hy());
          const idx_t n = gt(inode, r, c);
          for (size_t v = 0; v < nv; ++v)
            dst[v][n] += (Nx * sx[v][ip] + Ny * sy[v][ip]) * w[ip];
        }
      }
  }

  void g2p(std::map<std::string, std::vector<double>>& vars,
           const std::vector<std::string>& gnames,
           const std::vector<std::string>& pnames) {
    const size_t nv = gnames.size();
    std::vector<const double*> src(nv);
    std::vector<double*> dst(nv);
    for (size_t v = 0; v < nv; ++v) {
      src[v] = vars[gnames[v]].data();
      dst[v] = dprops[pnames[v]].data();
    }
    for (idx_t ip = 0; ip < num_particles; ++ip) {
      double xi, eta;
      idx_t r, c;
      local(ip, ptcl_to_grd[ip], xi, eta, r, c);
      for (int inode = 0; inode < 4; ++inode) {
        const double N = shp(xi, eta, inode);
        const idx_t n = gt(inode, r, c);
        for (size_t v = 0; v < nv; ++v) dst[v][ip] += N * src[v][n];
      }
    }
  }

  void g2pd(std::map<std::string, std::vector<double>>& vars,
            const std::vector<std::string>& gnames,
            const std::vector<std::string>& dxnames,
            const std::vector<std::string>& dynames) {
    const size_t nv = gnames.size();
    std::vector<const double*> src(nv);
    std::vector<double*> ddx(nv), ddy(nv);
    for (size_t v = 0; v < nv; ++v) {
      src[v] = vars[gnames[v]].data();
      ddx[v] = dprops[dxnames[v]].data();
      ddy[v] = dprops[dynames[v]].data();
    }
    for (idx_t ip = 0; ip < num_particles; ++ip) {
      double xi, eta;
      idx_t r, c;
      local(ip, ptcl_to_grd[ip], xi, eta, r, c);
      for (int inode = 0; inode < 4; ++inode) {
        const double Nx = shg(xi, eta, 0, inode, grid.hx(), grid.hy());
        const double Ny = shg(xi, eta, 1, inode, grid.hx(), grid.hy());
        const idx_t n = gt(inode, r, c);
        for (size_t v = 0; v < nv; ++v) {
          ddx[v][ip] += Nx * src[v][n];
          ddy[v][ip] += Ny * src[v][n];
        }
      }
    }
  }

  template <output_format F>
  void print(std::ostream& os) const {
    os << "\"x\", \"y\"";
    for (auto const& kv : dprops) os << ", \"" << kv.first << "\"";
    for (auto const& kv : iprops) os << ", \"" << kv.first << "\"";
    os << "\n";
    char buf[64];
    for (idx_t i = 0; i < num_particles; ++i) {
      std::snprintf(buf, sizeof buf, "%.17g", x[i]);
      os << buf;
      std::snprintf(buf, sizeof buf, ", %.17g", y[i]);
      os << buf;
      for (auto const& kv : dprops) {
        std::snprintf(buf, sizeof buf, ", %.17g", kv.second[i]);
        os << buf;
      }
      for (auto const& kv : iprops) os << ", " << kv.second[i];
      os << "\n";
    }
  }
};
