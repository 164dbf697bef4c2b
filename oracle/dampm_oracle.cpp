// ============================================================================
//  dampm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the parity oracle).
//
//  A plain C++17 restatement, on the CPU, of the depth-averaged MPM time step
//  of dampm (lucadiprofio/AMSC).  Only tests/, __graft_entry__.smoke() and the
//  cpu_baseline leg of bench.py may load this library, and only as the
//  checker or the timed CPU baseline.  The product (amsc_b200/) never links,
//  imports or calls it.
//
//  What it restates (file:line in the reference project):
//    * the step loop of main/optim_par.cpp:281-668 (order, guards, floors),
//      initialisation main/optim_par.cpp:133-270;
//    * quadgrid's transfer operators p2g / g2p / g2pd / p2gd and
//      init_particle_mesh, which live in the absent `quadgrid` submodule
//      (.gitmodules:1-4, lucadiprofio fork, no pinned commit).  Their shape
//      functions and index conventions follow main/gpu_kernels.cpp:7-59;
//      the accumulation order is the quadgrid cell sweep (cells ascending by
//      id r + c*nrows, particles ascending by index, local nodes 0..3) that
//      main/gpu_kernels.cpp:104-127 also walks per colour;
//    * adaptive merge/split of main/merge_split_ops_cmes.h:93-447, invoked at
//      the main/gpu_offload.cpp:321 cadence (after it++, before the step);
//    * the DATA keys/defaults of main/mpm_data.h:61-114 (taken as arguments).
//
//  Documented choices where the reference is undefined or absent:
//    * first adaptive dt (optim_par.cpp:284,303 reads an uninitialised
//      variable) = 1e-3, the value gpu_offload.cpp:255 defines;
//    * cell of a particle = (floor(y/hy), floor(x/hx)), clamped into the grid;
//    * build_mass() (optim_par.cpp:268) has no visible effect and is skipped.
//
//  Two execution modes give bit-identical results: serial (reference order)
//  and OpenMP (per-particle loops in parallel, P2G as a per-node gather that
//  visits the same contributions in the same order).
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Mirrors the scalar members of struct DATA (main/mpm_data.h:6-57).
typedef struct {
  int Nex, Ney;
  double hx, hy;
  double g, T, rho, xi, mu, phi, tauy;
  double BINGHAM_ON, FRICTION_ON, CFL;
  int BC_FLAG;
  int MERGE_SPLIT_ON;
  double eq_level;
  double DT_FIXED;
  int NSTEPS;
  double ms_alpha, ms_beta, ms_split_hp_min, ms_shear_split, ms_hp_min,
      ms_max_dv;
  int ms_min_level, ms_max_level, ms_min_particles_per_cell, ms_call_interval;
  double ms_max_ops;
  double ms_pair_dist;  // pair-distance gate (0: none, the reference's pairing)
  int ms_variant;            // 0: merge_split_ops_cmes.h, 1: merge_split_ops.h (ELFS)
  double ms_stretch_thresh;  // ELFS ms_config::stretch_thresh
} oracle_data;

}  // extern "C"

namespace {

using idx_t = int;

// names of the 35 particle dprops (main/optim_par.cpp:140-144,
// main/gpu_offload.cpp:35-40).
const char* kDprops[] = {"Mp",     "Ap",      "vpx",     "vpy",     "mom_px",
                         "mom_py", "hp",      "Vp",      "F_ext_px", "F_ext_py",
                         "apx",    "apy",     "F_11",    "F_12",    "F_21",
                         "F_22",   "vpx_dx",  "vpx_dy",  "vpy_dx",  "vpy_dy",
                         "Fb_x",   "Fb_y",    "hpZ",     "dZxp",    "dZyp",
                         "Zp",     "xp",      "yp",      "Fric_px", "Fric_py",
                         "Fpx",    "Fpy",     "vpxL",    "vpyL",    "H"};

// nodal vars of main/optim_par.cpp:199-225
const char* kVars[] = {"Mv",      "mom_vx",  "mom_vy",  "F_ext_vx", "F_ext_vy",
                       "F_int_vx", "F_int_vy", "Fric_x", "Fric_y",   "div_v",
                       "avx",     "avy",     "vvx",     "vvy",      "Z",
                       "dZdx",    "dZdy",    "Ftot_vx", "Ftot_vy",  "HV",
                       "FPxv",    "FPyv",    "vvxL",    "vvyL"};

struct Oracle {
  oracle_data d;
  idx_t nrows, ncols;  // grid.set_sizes (Ney, Nex, ...): rows = Ney
  double hx, hy;
  std::vector<double> Z0, dZdx0, dZdy0;

  idx_t np = 0;
  std::vector<double> x, y;
  std::map<std::string, std::vector<double>> dprops;
  std::map<std::string, std::vector<idx_t>> iprops;  // label, level
  std::map<std::string, std::vector<double>> vars;

  // init_particle_mesh products
  std::vector<idx_t> p2c;         // cell of each particle
  std::vector<idx_t> cell_start;  // CSR by cell, ncells+1
  std::vector<idx_t> cell_ptcls;  // particles sorted by (cell, index)

  double t = 0.0;
  int it = 0;
  double dt_last = 0.0;
  bool ms_enabled = false;
  int nthreads = 1;

  // ledger of the last step (main/optim_par.cpp:395-425)
  double led[9] = {0};
  // merge/split counters of the last call
  long long ms_counts[4] = {0};

  idx_t nnodes() const { return (nrows + 1) * (ncols + 1); }
  idx_t ncells() const { return nrows * ncols; }
};

// ---------------------------------------------------------------------------
// index and shape helpers: main/gpu_kernels.cpp:7-59
// ---------------------------------------------------------------------------
inline idx_t gt(int inode, idx_t c, idx_t r, idx_t nrows) {
  const idx_t bl = r + c * (nrows + 1);
  switch (inode) {
    case 0: return bl;
    case 1: return bl + 1;
    case 2: return bl + (nrows + 1);
    default: return bl + (nrows + 2);
  }
}

// local coordinates relative to the bottom-left node of cell (r, c):
// pnode(0,0,c,r) = c*hx, pnode(1,0,c,r) = r*hy (gpu_kernels.cpp:21-31)
inline void local_xy(double x, double y, idx_t c, idx_t r, double hx,
                     double hy, double& xi, double& eta) {
  xi = (x - c * hx) / hx;
  eta = (y - r * hy) / hy;
}

// shp (gpu_kernels.cpp:33-41)
inline double shp(double xi, double eta, int inode) {
  switch (inode) {
    case 3: return xi * eta;
    case 2: return xi * (1.0 - eta);
    case 1: return (1.0 - xi) * eta;
    default: return (1.0 - xi) * (1.0 - eta);
  }
}

// shg (gpu_kernels.cpp:43-59)
inline double shg(double xi, double eta, int idir, int inode, double hx,
                  double hy) {
  switch (inode) {
    case 3:
      if (idir == 0) return (1.0 / hx) * eta;
      return xi * (1.0 / hy);
    case 2:
      if (idir == 0) return (1.0 / hx) * (1.0 - eta);
      return xi * (-1.0 / hy);
    case 1:
      if (idir == 0) return (-1.0 / hx) * eta;
      return (1.0 - xi) * (1.0 / hy);
    default:
      if (idir == 0) return (-1.0 / hx) * (1.0 - eta);
      return (1.0 - xi) * (-1.0 / hy);
  }
}

inline idx_t cell_row(double y, double hy, idx_t nrows) {
  double f = std::floor(y / hy);
  if (!(f >= 0.0)) return 0;  // also maps NaN to 0
  if (f > double(nrows - 1)) return nrows - 1;
  return idx_t(f);
}
inline idx_t cell_col(double x, double hx, idx_t ncols) {
  double f = std::floor(x / hx);
  if (!(f >= 0.0)) return 0;
  if (f > double(ncols - 1)) return ncols - 1;
  return idx_t(f);
}

// ---------------------------------------------------------------------------
// quadgrid restatements
// ---------------------------------------------------------------------------

// init_particle_mesh: bin particles to cells; CSR in (cell, index) order.
void init_particle_mesh(Oracle& o) {
  const idx_t nc = o.ncells();
  o.p2c.assign(o.np, 0);
  o.cell_start.assign(nc + 1, 0);
  for (idx_t i = 0; i < o.np; ++i) {
    const idx_t r = cell_row(o.y[i], o.hy, o.nrows);
    const idx_t c = cell_col(o.x[i], o.hx, o.ncols);
    o.p2c[i] = r + c * o.nrows;
    o.cell_start[o.p2c[i] + 1]++;
  }
  for (idx_t k = 0; k < nc; ++k) o.cell_start[k + 1] += o.cell_start[k];
  std::vector<idx_t> fill(o.cell_start.begin(), o.cell_start.end() - 1);
  o.cell_ptcls.assign(o.np, 0);
  for (idx_t i = 0; i < o.np; ++i) o.cell_ptcls[fill[o.p2c[i]]++] = i;
}

// Visit, for every node, the particle contributions in cell-sweep order.
// Node (r,c) is local node 3 of cell (r-1,c-1), 2 of (r,c-1), 1 of (r-1,c)
// and 0 of (r,c); ascending cell id r + c*nrows puts them in that order.
template <class F>
inline void node_gather(const Oracle& o, idx_t nr, idx_t nc_, F&& f) {
  const idx_t cr[4] = {nr - 1, nr, nr - 1, nr};
  const idx_t cc[4] = {nc_ - 1, nc_ - 1, nc_, nc_};
  const int ln[4] = {3, 2, 1, 0};
  for (int k = 0; k < 4; ++k) {
    if (cr[k] < 0 || cr[k] >= o.nrows || cc[k] < 0 || cc[k] >= o.ncols)
      continue;
    const idx_t cell = cr[k] + cc[k] * o.nrows;
    for (idx_t j = o.cell_start[cell]; j < o.cell_start[cell + 1]; ++j)
      f(o.cell_ptcls[j], cr[k], cc[k], ln[k]);
  }
}

// p2g: vars[out] += N * dprops[in], cell sweep order.
void p2g(Oracle& o, const std::vector<std::string>& in,
         const std::vector<std::string>& out) {
  const size_t nv = in.size();
  std::vector<const double*> src(nv);
  std::vector<double*> dst(nv);
  for (size_t v = 0; v < nv; ++v) {
    src[v] = o.dprops.at(in[v]).data();
    dst[v] = o.vars.at(out[v]).data();
  }
  if (o.nthreads <= 1) {
    for (idx_t cell = 0; cell < o.ncells(); ++cell) {
      const idx_t r = cell % o.nrows, c = cell / o.nrows;
      for (idx_t j = o.cell_start[cell]; j < o.cell_start[cell + 1]; ++j) {
        const idx_t ip = o.cell_ptcls[j];
        double xi, eta;
        local_xy(o.x[ip], o.y[ip], c, r, o.hx, o.hy, xi, eta);
        for (int inode = 0; inode < 4; ++inode) {
          const double N = shp(xi, eta, inode);
          const idx_t n = gt(inode, c, r, o.nrows);
          for (size_t v = 0; v < nv; ++v) dst[v][n] += N * src[v][ip];
        }
      }
    }
    return;
  }
  const idx_t NR = o.nrows + 1, NC = o.ncols + 1;
#pragma omp parallel for schedule(dynamic, 16) num_threads(o.nthreads)
  for (idx_t n = 0; n < NR * NC; ++n) {
    const idx_t nr = n % NR, nc_ = n / NR;
    node_gather(o, nr, nc_, [&](idx_t ip, idx_t r, idx_t c, int inode) {
      double xi, eta;
      local_xy(o.x[ip], o.y[ip], c, r, o.hx, o.hy, xi, eta);
      const double N = shp(xi, eta, inode);
      for (size_t v = 0; v < nv; ++v) dst[v][n] += N * src[v][ip];
    });
  }
}

// p2gd (vars, {xa,xb}, {ya,yb}, w, {o1,o2}):
//   o1 += (Nx*xa + Ny*ya)*w ;  o2 += (Nx*xb + Ny*yb)*w
// restated from main/gpu_kernels.cpp:287-291 for the call at
// main/optim_par.cpp:476 (xa=F_11, xb=F_21, ya=F_12, yb=F_22; the stress is
// symmetric, F_12 == F_21, so both pairings give the same numbers).
void p2gd_forces(Oracle& o) {
  const double* F11 = o.dprops.at("F_11").data();
  const double* F12 = o.dprops.at("F_12").data();
  const double* F21 = o.dprops.at("F_21").data();
  const double* F22 = o.dprops.at("F_22").data();
  const double* Vp = o.dprops.at("Vp").data();
  double* fx = o.vars.at("F_int_vx").data();
  double* fy = o.vars.at("F_int_vy").data();
  auto contrib = [&](idx_t ip, idx_t r, idx_t c, int inode, idx_t n) {
    double xi, eta;
    local_xy(o.x[ip], o.y[ip], c, r, o.hx, o.hy, xi, eta);
    const double Nx = shg(xi, eta, 0, inode, o.hx, o.hy);
    const double Ny = shg(xi, eta, 1, inode, o.hx, o.hy);
    fx[n] += (Nx * F11[ip] + Ny * F21[ip]) * Vp[ip];
    fy[n] += (Nx * F12[ip] + Ny * F22[ip]) * Vp[ip];
  };
  if (o.nthreads <= 1) {
    for (idx_t cell = 0; cell < o.ncells(); ++cell) {
      const idx_t r = cell % o.nrows, c = cell / o.nrows;
      for (idx_t j = o.cell_start[cell]; j < o.cell_start[cell + 1]; ++j)
        for (int inode = 0; inode < 4; ++inode)
          contrib(o.cell_ptcls[j], r, c, inode, gt(inode, c, r, o.nrows));
    }
    return;
  }
  const idx_t NR = o.nrows + 1, NC = o.ncols + 1;
#pragma omp parallel for schedule(dynamic, 16) num_threads(o.nthreads)
  for (idx_t n = 0; n < NR * NC; ++n) {
    node_gather(o, n % NR, n / NR,
                [&](idx_t ip, idx_t r, idx_t c, int inode) {
                  contrib(ip, r, c, inode, n);
                });
  }
}

// g2p: dprops[out] += N * vars[in] for local nodes 0..3 (particle's cell).
void g2p(Oracle& o, const std::vector<std::string>& in,
         const std::vector<std::string>& out) {
  const size_t nv = in.size();
  std::vector<const double*> src(nv);
  std::vector<double*> dst(nv);
  for (size_t v = 0; v < nv; ++v) {
    src[v] = o.vars.at(in[v]).data();
    dst[v] = o.dprops.at(out[v]).data();
  }
#pragma omp parallel for schedule(static) num_threads(o.nthreads) if (o.nthreads > 1)
  for (idx_t ip = 0; ip < o.np; ++ip) {
    const idx_t cell = o.p2c[ip];
    const idx_t r = cell % o.nrows, c = cell / o.nrows;
    double xi, eta;
    local_xy(o.x[ip], o.y[ip], c, r, o.hx, o.hy, xi, eta);
    for (int inode = 0; inode < 4; ++inode) {
      const double N = shp(xi, eta, inode);
      const idx_t n = gt(inode, c, r, o.nrows);
      for (size_t v = 0; v < nv; ++v) dst[v][ip] += N * src[v][n];
    }
  }
}

// g2pd (vars, in, dx_out, dy_out): dx_out += Nx*in, dy_out += Ny*in
void g2pd(Oracle& o, const std::vector<std::string>& in,
          const std::vector<std::string>& dxo,
          const std::vector<std::string>& dyo) {
  const size_t nv = in.size();
  std::vector<const double*> src(nv);
  std::vector<double*> ddx(nv), ddy(nv);
  for (size_t v = 0; v < nv; ++v) {
    src[v] = o.vars.at(in[v]).data();
    ddx[v] = o.dprops.at(dxo[v]).data();
    ddy[v] = o.dprops.at(dyo[v]).data();
  }
#pragma omp parallel for schedule(static) num_threads(o.nthreads) if (o.nthreads > 1)
  for (idx_t ip = 0; ip < o.np; ++ip) {
    const idx_t cell = o.p2c[ip];
    const idx_t r = cell % o.nrows, c = cell / o.nrows;
    double xi, eta;
    local_xy(o.x[ip], o.y[ip], c, r, o.hx, o.hy, xi, eta);
    for (int inode = 0; inode < 4; ++inode) {
      const double Nx = shg(xi, eta, 0, inode, o.hx, o.hy);
      const double Ny = shg(xi, eta, 1, inode, o.hx, o.hy);
      const idx_t n = gt(inode, c, r, o.nrows);
      for (size_t v = 0; v < nv; ++v) {
        ddx[v][ip] += Nx * src[v][n];
        ddy[v][ip] += Ny * src[v][n];
      }
    }
  }
}

template <class F>
inline void par_for(const Oracle& o, idx_t n, F&& f) {
#pragma omp parallel for schedule(static) num_threads(o.nthreads) if (o.nthreads > 1)
  for (idx_t i = 0; i < n; ++i) f(i);
}

// ---------------------------------------------------------------------------
// Bingham stress: the stress_tensor_t functor, main/optim_par.cpp:68-120
// ---------------------------------------------------------------------------
struct StressArgs {
  const double *vpx, *vpy, *hp, *H, *vpx_dx, *vpy_dy, *vpx_dy, *vpy_dx;
  double *F_11, *F_12, *F_21, *F_22;
};

inline StressArgs stress_args(Oracle& o) {
  auto& dp = o.dprops;
  return StressArgs{dp["vpx"].data(),    dp["vpy"].data(),    dp["hp"].data(),
                    dp["H"].data(),      dp["vpx_dx"].data(), dp["vpy_dy"].data(),
                    dp["vpx_dy"].data(), dp["vpy_dx"].data(), dp["F_11"].data(),
                    dp["F_12"].data(),   dp["F_21"].data(),   dp["F_22"].data()};
}

inline void stress_one(const oracle_data& data, const StressArgs& s, idx_t ip) {
  double A{3. / 2.}, B{-114. / 32.}, C{65. / 32.};
  const double BING = data.BINGHAM_ON;
  const double hp = s.hp[ip];
  const double nrm = std::sqrt(s.vpx[ip] * s.vpx[ip] + s.vpy[ip] * s.vpy[ip]);
  const double mu = data.mu;
  const double tau_Y = data.tauy;
  const double ALF = hp > 1.e-3 ? (6. * mu * nrm) / ((hp + 0.001) * tau_Y) : 0.0;
  B = -114. / 32. - ALF;
  const double Z1 = (-B + std::sqrt(B * B - 4. * A * C)) / (2. * A);
  const double Z2 = (-B - std::sqrt(B * B - 4. * A * C)) / (2. * A);
  const double ZZ = std::abs(Z1 - .5) <= .5 ? Z1 : Z2;
  const double s_xx = s.vpx_dx[ip];
  const double s_xy = 0.5 * (s.vpx_dy[ip] + s.vpy_dx[ip]);
  const double s_yy = s.vpy_dy[ip];
  const double D_xx = s_xx, D_xy = s_xy, D_yy = s_yy;
  const double D_zx =
      hp > 1.e-3 ? 0.5 * (3. / (2. + ZZ)) * (s.vpx[ip] / (hp + 0.001)) : 0.0;
  const double D_zy =
      hp > 1.e-3 ? 0.5 * (3. / (2. + ZZ)) * (s.vpy[ip] / (hp + 0.001)) : 0.0;
  const double D_zz = -(s.vpx_dx[ip] + s.vpy_dy[ip]);
  const double invII = 0.5 * (D_xx * D_xx + D_yy * D_yy + D_zz * D_zz) +
                       D_zx * D_zx + D_zy * D_zy + D_xy * D_xy;
  const double sig_xx =
      invII != 0 ? (tau_Y / std::sqrt(invII) + 2. * mu) * D_xx : 0.0;
  const double sig_xy =
      invII != 0 ? (tau_Y / std::sqrt(invII) + 2. * mu) * D_xy : 0.0;
  const double sig_yy =
      invII != 0 ? (tau_Y / std::sqrt(invII) + 2. * mu) * D_yy : 0.0;
  const double H = s.H[ip];
  const double h_corr = hp > 1e-10 ? hp - (H * H) / hp : 0.0;
  s.F_11[ip] = BING * sig_xx - .5 * data.rho * data.g * h_corr;
  s.F_12[ip] = BING * sig_xy;
  s.F_21[ip] = BING * sig_xy;
  s.F_22[ip] = BING * sig_yy - .5 * data.rho * data.g * h_corr;
}

// ---------------------------------------------------------------------------
// merge/split: main/merge_split_ops_cmes.h
// ---------------------------------------------------------------------------
enum action_t : int { KEEP = 0, SPLIT = 1, MERGE_PRIMARY = 2, MERGE_SECONDARY = 3 };

inline bool is_extensive(const std::string& n) {
  return n == "Mp" || n == "Vp" || n == "Ap" || n == "mom_px" || n == "mom_py";
}

// principal_stretch_dir: merge_split_ops_cmes.h:93-110
inline void principal_stretch_dir(double exx, double eyy, double exy,
                                  double& ux, double& uy) {
  const double tr = exx + eyy;
  const double diff = 0.5 * (exx - eyy);
  const double disc = std::sqrt(diff * diff + exy * exy);
  const double l1 = 0.5 * tr + disc;
  double vx = l1 - eyy;
  double vy = exy;
  double n = std::sqrt(vx * vx + vy * vy);
  if (n < 1e-12) {
    ux = 1.0;
    uy = 0.0;
  } else {
    ux = vx / n;
    uy = vy / n;
  }
}

// The per-cell part of decide_actions, cells in order with their particles
// in index order (grd_to_ptcl = CSR order): the split cap, the greedy
// pairing of co-moving merge candidates and the undo of merges while a cell
// would hold fewer than min_ppc particles.  merge_split_ops_cmes.h:174-249
// (split_w 2, min_ppc = min_particles_per_cell, the optional gate) and
// merge_split_ops.h:406-497 (split_w 4, min_ppc 2, no gate) differ only in
// those three.  Writes the counts to ms_counts[0..1].
void pair_in_cells(Oracle& o, std::vector<int>& act, std::vector<int>& partner, int max_ops,
                   double max_dv2, double gate2, int split_w, int min_ppc) {
  const double* vpx = o.dprops.at("vpx").data();
  const double* vpy = o.dprops.at("vpy").data();
  long long n_split = 0, n_merge = 0;
  for (idx_t cell = 0; cell < o.ncells(); ++cell) {
    const idx_t b = o.cell_start[cell], e = o.cell_start[cell + 1];
    if (b == e) continue;
    for (idx_t j = b; j < e; ++j) {
      const idx_t p = o.cell_ptcls[j];
      if (act[p] == SPLIT) {
        if (n_split < max_ops) ++n_split;
        else act[p] = KEEP;
      }
    }
    std::vector<idx_t> cand;
    for (idx_t j = b; j < e; ++j)
      if (act[o.cell_ptcls[j]] == MERGE_PRIMARY) cand.push_back(o.cell_ptcls[j]);
    std::vector<char> paired(cand.size(), 0);
    for (size_t i = 0; i < cand.size() && n_merge < max_ops; ++i) {
      if (paired[i]) continue;
      const idx_t i1 = cand[i];
      double best = std::numeric_limits<double>::max();
      size_t bj = cand.size();
      for (size_t j = i + 1; j < cand.size(); ++j) {
        if (paired[j]) continue;
        const idx_t i2 = cand[j];
        const double dx = o.x[i1] - o.x[i2];
        const double dy = o.y[i1] - o.y[i2];
        const double d2 = dx * dx + dy * dy;
        const double dvx = vpx[i1] - vpx[i2];
        const double dvy = vpy[i1] - vpy[i2];
        if (d2 < best && (dvx * dvx + dvy * dvy) < max_dv2 && (gate2 == 0.0 || d2 < gate2)) {
          best = d2;
          bj = j;
        }
      }
      if (bj < cand.size()) {
        act[i1] = MERGE_PRIMARY;
        act[cand[bj]] = MERGE_SECONDARY;
        partner[i1] = int(cand[bj]);
        paired[i] = 1;
        paired[bj] = 1;
        ++n_merge;
      } else {
        act[i1] = KEEP;
      }
    }
    for (size_t i = 0; i < cand.size(); ++i)
      if (!paired[i]) act[cand[i]] = KEEP;
    int projected = 0;
    for (idx_t j = b; j < e; ++j) {
      const int a = act[o.cell_ptcls[j]];
      if (a == KEEP) projected += 1;
      else if (a == SPLIT) projected += split_w;
      else if (a == MERGE_PRIMARY) projected += 1;
    }
    while (projected < min_ppc) {
      bool undone = false;
      for (idx_t j = b; j < e; ++j) {
        const idx_t p = o.cell_ptcls[j];
        if (act[p] == MERGE_PRIMARY) {
          const int q = partner[p];
          if (q >= 0) act[q] = KEEP;
          partner[p] = -1;
          act[p] = KEEP;
          --n_merge;
          projected += 1;
          undone = true;
          break;
        }
      }
      if (!undone) break;
    }
  }
  o.ms_counts[0] = n_split;
  o.ms_counts[1] = n_merge;
}

// decide_actions: merge_split_ops_cmes.h:116-253 (grd_to_ptcl = CSR order)
void decide_actions(Oracle& o, double dt, std::vector<int>& act,
                    std::vector<int>& partner) {
  const idx_t N = o.np;
  act.assign(N, KEEP);
  partner.assign(N, -1);
  const double min_h = std::min(o.hx, o.hy);
  const double r_split = o.d.ms_alpha * min_h;
  const double r_merge = o.d.ms_beta * min_h;
  const double shear_split = o.d.ms_shear_split;
  const double split_hp_min = o.d.ms_split_hp_min;
  const double hp_min = o.d.ms_hp_min;
  const int min_level = o.d.ms_min_level, max_level = o.d.ms_max_level;
  const int max_ops = (int)o.d.ms_max_ops;  // gpu_offload.cpp:317
  const int min_ppc = o.d.ms_min_particles_per_cell;
  const double* Ap = o.dprops.at("Ap").data();
  const double* hp = o.dprops.at("hp").data();
  const double* exx_ = o.dprops.at("vpx_dx").data();
  const double* eyy_ = o.dprops.at("vpy_dy").data();
  const double* exy1 = o.dprops.at("vpx_dy").data();
  const double* exy2 = o.dprops.at("vpy_dx").data();
  const idx_t* lvl = o.iprops.at("level").data();
  for (idx_t ip = 0; ip < N; ++ip) {
    const double r_i = std::sqrt(Ap[ip]);
    const double exx = exx_[ip], eyy = eyy_[ip];
    const double exy = 0.5 * (exy1[ip] + exy2[ip]);
    const double gdot = std::sqrt(2.0 * (exx * exx + eyy * eyy + 2.0 * exy * exy));
    const bool stretched = (r_i > r_split);
    const bool sheared = (gdot * dt > shear_split);
    const bool thick = (r_i < r_merge);
    const bool thin_skip = (hp[ip] < split_hp_min);
    if ((stretched || sheared) && !thin_skip && (int(lvl[ip]) > min_level))
      act[ip] = SPLIT;
    else if (thick && hp[ip] > hp_min && int(lvl[ip]) < max_level)
      act[ip] = MERGE_PRIMARY;
  }
  const double max_dv2 = o.d.ms_max_dv * o.d.ms_max_dv;
  // the optional pair-distance gate (no counterpart in the reference)
  const double gmin_h = (o.d.hy < o.d.hx) ? o.d.hy : o.d.hx;
  const double gr = o.d.ms_pair_dist * gmin_h;
  const double gate2 = o.d.ms_pair_dist > 0.0 ? gr * gr : 0.0;
  pair_in_cells(o, act, partner, max_ops, max_dv2, gate2, 2, min_ppc);
}

// execute_merge_split: merge_split_ops_cmes.h:258-427
void execute_merge_split(Oracle& o, const std::vector<int>& act,
                         const std::vector<int>& partner) {
  const idx_t N = o.np;
  const int weights[] = {1, 2, 1, 0};
  std::vector<idx_t> offset(N, 0);
  idx_t Nnew = 0;
  for (idx_t i = 0; i < N; ++i) {
    offset[i] = Nnew;
    Nnew += weights[act[i]];
  }
  std::vector<double> nx(Nnew), ny(Nnew);
  std::vector<std::string> dpk, ipk;
  for (auto const& kv : o.dprops) dpk.push_back(kv.first);
  for (auto const& kv : o.iprops) ipk.push_back(kv.first);
  const int ndp = int(dpk.size()), nip = int(ipk.size());
  std::vector<std::vector<double>> ndp_v(ndp, std::vector<double>(Nnew));
  std::vector<std::vector<idx_t>> nip_v(nip, std::vector<idx_t>(Nnew));
  std::vector<const double*> in_dp(ndp);
  std::vector<double*> out_dp(ndp);
  std::vector<int> ext(ndp, 0);
  std::vector<const idx_t*> in_ip(nip);
  std::vector<idx_t*> out_ip(nip);
  int iMp = -1, ivpx = -1, ivpy = -1, ixp = -1, iyp = -1, impx = -1, impy = -1,
      iAp = -1, iVp = -1, ihp = -1, iexx = -1, ieyy = -1, iexy1 = -1, iexy2 = -1;
  for (int k = 0; k < ndp; ++k) {
    in_dp[k] = o.dprops.at(dpk[k]).data();
    out_dp[k] = ndp_v[k].data();
    ext[k] = is_extensive(dpk[k]) ? 1 : 0;
    const std::string& n = dpk[k];
    if (n == "Mp") iMp = k;
    else if (n == "vpx") ivpx = k;
    else if (n == "vpy") ivpy = k;
    else if (n == "xp") ixp = k;
    else if (n == "yp") iyp = k;
    else if (n == "mom_px") impx = k;
    else if (n == "mom_py") impy = k;
    else if (n == "Ap") iAp = k;
    else if (n == "Vp") iVp = k;
    else if (n == "hp") ihp = k;
    else if (n == "vpx_dx") iexx = k;
    else if (n == "vpy_dy") ieyy = k;
    else if (n == "vpx_dy") iexy1 = k;
    else if (n == "vpy_dx") iexy2 = k;
  }
  int ilevel = -1, ilabel = -1;
  for (int k = 0; k < nip; ++k) {
    in_ip[k] = o.iprops.at(ipk[k]).data();
    out_ip[k] = nip_v[k].data();
    if (ipk[k] == "level") ilevel = k;
    else if (ipk[k] == "label") ilabel = k;
  }
  const double hx = o.hx, hy = o.hy;
  const double Lx = o.ncols * hx, Ly = o.nrows * hy;
  const double eps = 1e-10;
  auto clampx = [&](double v) { return v < eps ? eps : (v > Lx - eps ? Lx - eps : v); };
  auto clampy = [&](double v) { return v < eps ? eps : (v > Ly - eps ? Ly - eps : v); };
  par_for(o, N, [&](idx_t i) {
    const int a = act[i];
    if (a == KEEP) {
      const idx_t oo = offset[i];
      nx[oo] = o.x[i];
      ny[oo] = o.y[i];
      for (int k = 0; k < ndp; ++k) out_dp[k][oo] = in_dp[k][i];
      for (int k = 0; k < nip; ++k) out_ip[k][oo] = in_ip[k][i];
    } else if (a == SPLIT) {
      const idx_t o1 = offset[i], o2 = offset[i] + 1;
      const idx_t level = (ilevel >= 0) ? in_ip[ilevel][i] : 0;
      double ux, uy;
      const double exx = (iexx >= 0) ? in_dp[iexx][i] : 0.0;
      const double eyy = (ieyy >= 0) ? in_dp[ieyy][i] : 0.0;
      const double exy = 0.5 * (((iexy1 >= 0) ? in_dp[iexy1][i] : 0.0) +
                                ((iexy2 >= 0) ? in_dp[iexy2][i] : 0.0));
      principal_stretch_dir(exx, eyy, exy, ux, uy);
      const double r_i = (iAp >= 0) ? std::sqrt(in_dp[iAp][i]) : 0.0;
      const double off = 0.25 * r_i;
      const double cx = o.x[i], cy = o.y[i];
      nx[o1] = clampx(cx + off * ux);
      ny[o1] = clampy(cy + off * uy);
      nx[o2] = clampx(cx - off * ux);
      ny[o2] = clampy(cy - off * uy);
      for (int k = 0; k < ndp; ++k) {
        const double val = in_dp[k][i] / (ext[k] ? 2.0 : 1.0);
        out_dp[k][o1] = val;
        out_dp[k][o2] = val;
      }
      for (int k = 0; k < nip; ++k) {
        out_ip[k][o1] = in_ip[k][i];
        out_ip[k][o2] = in_ip[k][i];
      }
      if (iAp >= 0 && iVp >= 0 && ihp >= 0) {
        const double h = out_dp[ihp][o1];
        out_dp[iAp][o1] = out_dp[iVp][o1] / h;
        out_dp[iAp][o2] = out_dp[iVp][o2] / h;
      }
      if (ixp >= 0) { out_dp[ixp][o1] = nx[o1]; out_dp[ixp][o2] = nx[o2]; }
      if (iyp >= 0) { out_dp[iyp][o1] = ny[o1]; out_dp[iyp][o2] = ny[o2]; }
      if (impx >= 0 && iMp >= 0 && ivpx >= 0) {
        out_dp[impx][o1] = out_dp[iMp][o1] * out_dp[ivpx][o1];
        out_dp[impx][o2] = out_dp[iMp][o2] * out_dp[ivpx][o2];
      }
      if (impy >= 0 && iMp >= 0 && ivpy >= 0) {
        out_dp[impy][o1] = out_dp[iMp][o1] * out_dp[ivpy][o1];
        out_dp[impy][o2] = out_dp[iMp][o2] * out_dp[ivpy][o2];
      }
      if (ilevel >= 0) { out_ip[ilevel][o1] = level - 1; out_ip[ilevel][o2] = level - 1; }
      if (ilabel >= 0) { out_ip[ilabel][o1] = -1; out_ip[ilabel][o2] = -1; }
    } else if (a == MERGE_PRIMARY) {
      const int j = partner[i];
      const idx_t oo = offset[i];
      const idx_t level = (ilevel >= 0) ? in_ip[ilevel][i] : 0;
      const double M1 = (iMp >= 0) ? in_dp[iMp][i] : 1.0;
      const double M2 = (iMp >= 0) ? in_dp[iMp][j] : 1.0;
      const double Mt = M1 + M2;
      nx[oo] = (M1 * o.x[i] + M2 * o.x[j]) / Mt;
      ny[oo] = (M1 * o.y[i] + M2 * o.y[j]) / Mt;
      for (int k = 0; k < ndp; ++k)
        out_dp[k][oo] = ext[k] ? (in_dp[k][i] + in_dp[k][j])
                               : (M1 * in_dp[k][i] + M2 * in_dp[k][j]) / Mt;
      for (int k = 0; k < nip; ++k) out_ip[k][oo] = in_ip[k][i];
      if (ihp >= 0 && iVp >= 0 && iAp >= 0)
        out_dp[ihp][oo] = out_dp[iVp][oo] / out_dp[iAp][oo];
      if (ixp >= 0) out_dp[ixp][oo] = nx[oo];
      if (iyp >= 0) out_dp[iyp][oo] = ny[oo];
      if (impx >= 0 && iMp >= 0 && ivpx >= 0)
        out_dp[impx][oo] = out_dp[iMp][oo] * out_dp[ivpx][oo];
      if (impy >= 0 && iMp >= 0 && ivpy >= 0)
        out_dp[impy][oo] = out_dp[iMp][oo] * out_dp[ivpy][oo];
      if (ilevel >= 0) out_ip[ilevel][oo] = level + 1;
      if (ilabel >= 0) out_ip[ilabel][oo] = -1;
    }
  });
  o.x = std::move(nx);
  o.y = std::move(ny);
  for (int k = 0; k < ndp; ++k) o.dprops[dpk[k]] = std::move(ndp_v[k]);
  for (int k = 0; k < nip; ++k) o.iprops[ipk[k]] = std::move(nip_v[k]);
  o.np = Nnew;
}

// adaptive_merge_split: merge_split_ops_cmes.h:432-447
void adaptive_merge_split(Oracle& o, double dt) {
  std::vector<int> act, partner;
  decide_actions(o, dt, act, partner);
  o.ms_counts[2] = o.np;
  bool any = false;
  for (int a : act)
    if (a != KEEP) { any = true; break; }
  if (any) execute_merge_split(o, act, partner);
  o.ms_counts[3] = o.np;
}

// ---------------------------------------------------------------------------
// ELFS merge/split: main/merge_split_ops.h (refine near the free surface,
// coarsen far from it; splits 1 -> 4)
// ---------------------------------------------------------------------------
// Cells with particles (grd_to_ptcl's non-empty lists).
std::vector<char> wet_cells(const Oracle& o) {
  std::vector<char> wet(o.ncells(), 0);
  for (idx_t c = 0; c < o.ncells(); ++c) wet[c] = o.cell_start[c + 1] > o.cell_start[c];
  return wet;
}

// mark_exterior_cells, merge_split_ops.h:86-164: the empty cells connected
// to an empty cell on the grid's edge through empty cells (4-neighbours).
// The set does not depend on the visiting order; this walks it depth first.
std::vector<char> exterior_cells(const Oracle& o, const std::vector<char>& wet) {
  const idx_t nr = o.nrows, nc = o.ncols;
  std::vector<char> ext(o.ncells(), 0);
  std::vector<idx_t> stack;
  auto seed = [&](idx_t r, idx_t c) {
    const idx_t k = r + nr * c;
    if (!wet[k] && !ext[k]) {
      ext[k] = 1;
      stack.push_back(k);
    }
  };
  for (idx_t c = 0; c < nc; ++c) {
    seed(0, c);
    seed(nr - 1, c);
  }
  for (idx_t r = 0; r < nr; ++r) {
    seed(r, 0);
    seed(r, nc - 1);
  }
  while (!stack.empty()) {
    const idx_t k = stack.back();
    stack.pop_back();
    const idx_t r = k % nr, c = k / nr;
    if (r > 0) seed(r - 1, c);
    if (r + 1 < nr) seed(r + 1, c);
    if (c > 0) seed(r, c - 1);
    if (c + 1 < nc) seed(r, c + 1);
  }
  return ext;
}

// compute_boundary_distance, merge_split_ops.h:170-260: hops through wet
// cells (4-neighbours) from the wet cells off the grid's edge that have an
// exterior cell left or right of them (the seeds, 0), times min(hx, hy);
// cells no hop reaches keep DBL_MAX.  A breadth-first search by levels: the
// hop count of a cell is unique, whatever the order inside a level.
std::vector<double> boundary_distance(const Oracle& o, const std::vector<char>& wet,
                                      const std::vector<char>& ext) {
  const idx_t nr = o.nrows, nc = o.ncols;
  const double h = std::min(o.hx, o.hy);
  std::vector<double> dist(o.ncells(), std::numeric_limits<double>::max());
  std::vector<int> hops(o.ncells(), -1);
  std::vector<idx_t> level, next;
  for (idx_t c = 0; c < nc; ++c)
    for (idx_t r = 0; r < nr; ++r) {
      const idx_t k = r + nr * c;
      if (!wet[k]) continue;
      if (r == 0 || r == nr - 1 || c == 0 || c == nc - 1) continue;
      if (ext[r + nr * (c - 1)] || ext[r + nr * (c + 1)]) {
        hops[k] = 0;
        dist[k] = 0.0;
        level.push_back(k);
      }
    }
  for (int d = 0; !level.empty(); ++d) {
    next.clear();
    for (idx_t k : level) {
      const idx_t r = k % nr, c = k / nr;
      const idx_t nb[4] = {r > 0 ? k - 1 : -1, r + 1 < nr ? k + 1 : -1,
                           c > 0 ? k - nr : -1, c + 1 < nc ? k + nr : -1};
      for (idx_t q : nb) {
        if (q < 0 || !wet[q] || hops[q] >= 0) continue;
        hops[q] = d + 1;
        dist[q] = (d + 1) * h;
        next.push_back(q);
      }
    }
    level.swap(next);
  }
  return dist;
}

// compute_elfs, merge_split_ops.h:266-343: the cell distance, refined for
// particles within max(hx, hy) of the surface by the distance to the
// nearest exterior cell box among the two cells left and right in the row.
std::vector<double> elfs_values(const Oracle& o, const std::vector<double>& dist,
                                const std::vector<char>& ext) {
  const idx_t nr = o.nrows, nc = o.ncols;
  const double hx = o.hx, hy = o.hy;
  const double refine = std::max(hx, hy);
  std::vector<double> e(o.np);
  for (idx_t ip = 0; ip < o.np; ++ip) {
    const idx_t cell = o.p2c[ip];
    const double base = dist[cell];
    if (base > refine) {
      e[ip] = base;
      continue;
    }
    const double px = o.x[ip], py = o.y[ip];
    double md = base;
    const idx_t r = cell % nr, c0 = cell / nr;
    for (int dc = -2; dc <= 2; ++dc) {
      const idx_t c = c0 + dc;
      if (c < 0 || c >= nc) continue;
      if (!ext[r + nr * c]) continue;
      const double cx_lo = c * hx, cx_hi = (c + 1) * hx;
      const double cy_lo = r * hy, cy_hi = (r + 1) * hy;
      const double qx = px < cx_lo ? cx_lo : (px > cx_hi ? cx_hi : px);
      const double qy = py < cy_lo ? cy_lo : (py > cy_hi ? cy_hi : py);
      const double dx = px - qx, dy = py - qy;
      const double d = std::sqrt(dx * dx + dy * dy);
      if (d < md) md = d;
    }
    e[ip] = md;
  }
  return e;
}

// decide_actions, merge_split_ops.h:349-510: split near the surface (elfs <
// alpha * sqrt(Ap)) or where the divergence exceeds stretch_thresh, merge
// far from it (elfs > beta * sqrt(Ap), hp > hp_min), then the cells.
void decide_actions_elfs(Oracle& o, std::vector<int>& act, std::vector<int>& partner) {
  const idx_t N = o.np;
  act.assign(N, KEEP);
  partner.assign(N, -1);
  const std::vector<char> wet = wet_cells(o);
  const std::vector<char> ext = exterior_cells(o, wet);
  const std::vector<double> dist = boundary_distance(o, wet, ext);
  const std::vector<double> elfs = elfs_values(o, dist, ext);
  const double alpha = o.d.ms_alpha, beta = o.d.ms_beta;
  const int min_level = o.d.ms_min_level, max_level = o.d.ms_max_level;
  const double* Ap = o.dprops.at("Ap").data();
  const double* hp = o.dprops.at("hp").data();
  const double* exx = o.dprops.at("vpx_dx").data();
  const double* eyy = o.dprops.at("vpy_dy").data();
  const idx_t* lvl = o.iprops.at("level").data();
  for (idx_t ip = 0; ip < N; ++ip) {
    const double r_i = std::sqrt(Ap[ip]);
    const double div = exx[ip] + eyy[ip];
    if ((elfs[ip] < alpha * r_i) || (div > o.d.ms_stretch_thresh)) {
      if (lvl[ip] > min_level) act[ip] = SPLIT;
    } else if (elfs[ip] > beta * r_i && hp[ip] > o.d.ms_hp_min) {
      if (lvl[ip] < max_level) act[ip] = MERGE_PRIMARY;
    }
  }
  pair_in_cells(o, act, partner, (int)o.d.ms_max_ops, o.d.ms_max_dv * o.d.ms_max_dv, 0.0, 4,
                2);
}

// execute_merge_split, merge_split_ops.h:513-717: weights {1, 4, 1, 0};
// a split puts four children at (+-r/2, +-r/2) around the parent (r =
// sqrt(Ap), clamped into the domain) with the extensive fields divided by
// 4; a merge puts the pair's centre of mass with the extensive fields
// summed, the rest mass-averaged and the primary's label kept.
void execute_merge_split_elfs(Oracle& o, const std::vector<int>& act,
                              const std::vector<int>& partner) {
  const idx_t N = o.np;
  const int weights[] = {1, 4, 1, 0};
  std::vector<idx_t> offset(N, 0);
  idx_t Nnew = 0;
  for (idx_t i = 0; i < N; ++i) {
    offset[i] = Nnew;
    Nnew += weights[act[i]];
  }
  std::vector<double> nx(Nnew), ny(Nnew);
  std::vector<std::string> dpk, ipk;
  for (auto const& kv : o.dprops) dpk.push_back(kv.first);
  for (auto const& kv : o.iprops) ipk.push_back(kv.first);
  const int ndp = int(dpk.size()), nip = int(ipk.size());
  std::vector<std::vector<double>> ndp_v(ndp, std::vector<double>(Nnew));
  std::vector<std::vector<idx_t>> nip_v(nip, std::vector<idx_t>(Nnew));
  std::vector<int> ext(ndp, 0);
  int iMp = -1, ivpx = -1, ivpy = -1, ixp = -1, iyp = -1, impx = -1, impy = -1, iAp = -1;
  for (int k = 0; k < ndp; ++k) {
    const std::string& n = dpk[k];
    ext[k] = is_extensive(n) ? 1 : 0;
    if (n == "Mp") iMp = k;
    else if (n == "vpx") ivpx = k;
    else if (n == "vpy") ivpy = k;
    else if (n == "xp") ixp = k;
    else if (n == "yp") iyp = k;
    else if (n == "mom_px") impx = k;
    else if (n == "mom_py") impy = k;
    else if (n == "Ap") iAp = k;
  }
  int ilevel = -1, ilabel = -1;
  for (int k = 0; k < nip; ++k) {
    if (ipk[k] == "level") ilevel = k;
    else if (ipk[k] == "label") ilabel = k;
  }
  std::vector<const double*> in_dp(ndp);
  for (int k = 0; k < ndp; ++k) in_dp[k] = o.dprops.at(dpk[k]).data();
  std::vector<const idx_t*> in_ip(nip);
  for (int k = 0; k < nip; ++k) in_ip[k] = o.iprops.at(ipk[k]).data();
  const double Lx = o.ncols * o.hx, Ly = o.nrows * o.hy;
  const double eps = 1e-10;
  auto clampx = [&](double v) { return v < eps ? eps : (v > Lx - eps ? Lx - eps : v); };
  auto clampy = [&](double v) { return v < eps ? eps : (v > Ly - eps ? Ly - eps : v); };
  par_for(o, N, [&](idx_t i) {
    const int a = act[i];
    const idx_t oo = offset[i];
    if (a == KEEP) {
      nx[oo] = o.x[i];
      ny[oo] = o.y[i];
      for (int k = 0; k < ndp; ++k) ndp_v[k][oo] = in_dp[k][i];
      for (int k = 0; k < nip; ++k) nip_v[k][oo] = in_ip[k][i];
    } else if (a == SPLIT) {
      const double r_i = std::sqrt(in_dp[iAp][i]);
      const double off = r_i / 2.0;
      const double px = o.x[i], py = o.y[i];
      const double cx[4] = {clampx(px + off), clampx(px + off), clampx(px - off),
                            clampx(px - off)};
      const double cy[4] = {clampy(py + off), clampy(py - off), clampy(py + off),
                            clampy(py - off)};
      for (int q = 0; q < 4; ++q) {
        const idx_t t = oo + q;
        nx[t] = cx[q];
        ny[t] = cy[q];
        for (int k = 0; k < ndp; ++k) ndp_v[k][t] = in_dp[k][i] / (ext[k] ? 4.0 : 1.0);
        for (int k = 0; k < nip; ++k) nip_v[k][t] = in_ip[k][i];
        if (ixp >= 0) ndp_v[ixp][t] = cx[q];
        if (iyp >= 0) ndp_v[iyp][t] = cy[q];
        if (impx >= 0) ndp_v[impx][t] = ndp_v[iMp][t] * ndp_v[ivpx][t];
        if (impy >= 0) ndp_v[impy][t] = ndp_v[iMp][t] * ndp_v[ivpy][t];
        if (ilevel >= 0) nip_v[ilevel][t] = in_ip[ilevel][i] - 1;
        if (ilabel >= 0) nip_v[ilabel][t] = -1;
      }
    } else if (a == MERGE_PRIMARY) {
      const int j = partner[i];
      const double M1 = in_dp[iMp][i], M2 = in_dp[iMp][j];
      const double Mt = M1 + M2;
      nx[oo] = (M1 * o.x[i] + M2 * o.x[j]) / Mt;
      ny[oo] = (M1 * o.y[i] + M2 * o.y[j]) / Mt;
      for (int k = 0; k < ndp; ++k)
        ndp_v[k][oo] = ext[k] ? (in_dp[k][i] + in_dp[k][j])
                              : (M1 * in_dp[k][i] + M2 * in_dp[k][j]) / Mt;
      for (int k = 0; k < nip; ++k) nip_v[k][oo] = in_ip[k][i];
      if (ixp >= 0) ndp_v[ixp][oo] = nx[oo];
      if (iyp >= 0) ndp_v[iyp][oo] = ny[oo];
      if (impx >= 0) ndp_v[impx][oo] = ndp_v[iMp][oo] * ndp_v[ivpx][oo];
      if (impy >= 0) ndp_v[impy][oo] = ndp_v[iMp][oo] * ndp_v[ivpy][oo];
      if (ilevel >= 0) nip_v[ilevel][oo] = in_ip[ilevel][i] + 1;
    }
  });
  o.x = std::move(nx);
  o.y = std::move(ny);
  for (int k = 0; k < ndp; ++k) o.dprops[dpk[k]] = std::move(ndp_v[k]);
  for (int k = 0; k < nip; ++k) o.iprops[ipk[k]] = std::move(nip_v[k]);
  o.np = Nnew;
}

// adaptive_merge_split, merge_split_ops.h:720-755
void adaptive_merge_split_elfs(Oracle& o) {
  std::vector<int> act, partner;
  decide_actions_elfs(o, act, partner);
  o.ms_counts[2] = o.np;
  bool any = false;
  for (int a : act)
    if (a != KEEP) { any = true; break; }
  if (any) execute_merge_split_elfs(o, act, partner);
  o.ms_counts[3] = o.np;
}

// The merge/split the scenario selects: the gpu_offload one
// (merge_split_ops_cmes.h) or the ELFS variant (merge_split_ops.h).
void merge_split_call(Oracle& o, double dt) {
  if (o.d.ms_variant == 1)
    adaptive_merge_split_elfs(o);
  else
    adaptive_merge_split(o, dt);
}

// ---------------------------------------------------------------------------
// one pass of the while-loop body of main/optim_par.cpp:281-668
// ---------------------------------------------------------------------------
bool loop_condition(const Oracle& o) {
  const bool fixed = (o.d.DT_FIXED > 0.0);
  return fixed ? (o.it < o.d.NSTEPS) : (o.t < o.d.T);
}

double compute_dt(Oracle& o) {
  const bool fixed = (o.d.DT_FIXED > 0.0);
  double dt = 1.0e-3;  // first adaptive step: gpu_offload.cpp:255
  if (fixed) return o.d.DT_FIXED;
  const auto& vpx = o.dprops.at("vpx");
  const auto& vpy = o.dprops.at("vpy");
  const auto& hp = o.dprops.at("hp");
  if (o.np == 0) return dt;
  double max_vel_x = *std::max_element(vpx.begin(), vpx.end());
  double min_vel_x = *std::min_element(vpx.begin(), vpx.end());
  max_vel_x = std::max(std::abs(max_vel_x), std::abs(min_vel_x));
  double max_vel_y = *std::max_element(vpy.begin(), vpy.end());
  double min_vel_y = *std::min_element(vpy.begin(), vpy.end());
  max_vel_y = std::max(std::abs(max_vel_y), std::abs(min_vel_y));
  double hmean = *std::max_element(hp.begin(), hp.end());
  double max_vel = std::max(std::sqrt(o.d.g * hmean) + max_vel_x,
                            std::sqrt(o.d.g * hmean) + max_vel_y);
  double cel = std::abs(max_vel);
  if (o.it > 0) dt = o.d.CFL * std::min(o.d.hx, o.d.hy) / (1e-2 + cel);
  return dt;
}

void step_body(Oracle& o, double dt) {
  auto& dp = o.dprops;
  auto& V = o.vars;
  // (0) connectivity
  init_particle_mesh(o);
  for (auto& v : V) std::fill(v.second.begin(), v.second.end(), 0.0);
  V["Z"] = o.Z0;
  V["dZdx"] = o.dZdx0;
  V["dZdy"] = o.dZdy0;
  std::fill(dp["dZxp"].begin(), dp["dZxp"].end(), 0.0);
  std::fill(dp["dZyp"].begin(), dp["dZyp"].end(), 0.0);

  // (1) P2G mass / momentum, grad Z to particles
  p2g(o, {"Mp", "mom_px", "mom_py"}, {"Mv", "mom_vx", "mom_vy"});
  g2pd(o, {"Z"}, {"dZxp"}, {"dZyp"});

  // conservation ledger (optim_par.cpp:395-425)
  {
    double tmp = 0, tmx = 0, tmy = 0, tnm = 0, tnx = 0, tny = 0;
    const auto& Mp = dp["Mp"];
    const auto& mpx = dp["mom_px"];
    const auto& mpy = dp["mom_py"];
    for (idx_t ip = 0; ip < o.np; ++ip) {
      tmp += Mp[ip];
      tmx += mpx[ip];
      tmy += mpy[ip];
    }
    const auto& Mv = V["Mv"];
    const auto& mvx = V["mom_vx"];
    const auto& mvy = V["mom_vy"];
    for (idx_t n = 0; n < o.nnodes(); ++n) {
      tnm += Mv[n];
      tnx += mvx[n];
      tny += mvy[n];
    }
    const double err_mass = std::abs(tmp - tnm) / tmp;
    const double norm_mom = std::max(1.0, std::max(std::abs(tmx), std::abs(tmy)));
    const double err_mom =
        std::max(std::abs(tmx - tnx) / norm_mom, std::abs(tmy - tny) / norm_mom);
    o.led[0] = tmp; o.led[1] = tmx; o.led[2] = tmy;
    o.led[3] = tnm; o.led[4] = tnx; o.led[5] = tny;
    o.led[6] = err_mass; o.led[7] = err_mom; o.led[8] = o.t;
  }

  // (2) external forces
  {
    const double* Vp = dp["Vp"].data();
    const double* dZxp = dp["dZxp"].data();
    const double* dZyp = dp["dZyp"].data();
    const double* hp = dp["hp"].data();
    const double* H = dp["H"].data();
    double* Fpx = dp["Fpx"].data();
    double* Fpy = dp["Fpy"].data();
    const double g = o.d.g, rho = o.d.rho;
    par_for(o, o.np, [&](idx_t ip) {
      double wb_factor = hp[ip] > 1e-10 ? 1.0 - (H[ip] / hp[ip]) : 1.0;
      Fpx[ip] = -g * Vp[ip] * rho * dZxp[ip] * wb_factor;
      Fpy[ip] = -g * Vp[ip] * rho * dZyp[ip] * wb_factor;
    });
    const double* Ap = dp["Ap"].data();
    const double* Fbx = dp["Fb_x"].data();
    const double* Fby = dp["Fb_y"].data();
    double* Frx = dp["Fric_px"].data();
    double* Fry = dp["Fric_py"].data();
    par_for(o, o.np, [&](idx_t ip) {
      Frx[ip] = Ap[ip] * Fbx[ip];
      Fry[ip] = Ap[ip] * Fby[ip];
    });
  }
  p2g(o, {"Fpx", "Fpy", "Fric_px", "Fric_py"}, {"FPxv", "FPyv", "Fric_x", "Fric_y"});
  {
    const idx_t nn = o.nnodes();
    for (idx_t n = 0; n < nn; ++n) {
      V["F_ext_vx"][n] = V["FPxv"][n] + V["Fric_x"][n];
      V["F_ext_vy"][n] = V["FPyv"][n] + V["Fric_y"][n];
    }
  }
  // (3) internal forces and momentum balance
  p2gd_forces(o);
  {
    const idx_t nn = o.nnodes();
    double* Fex = V["F_ext_vx"].data(); double* Fey = V["F_ext_vy"].data();
    double* Fix = V["F_int_vx"].data(); double* Fiy = V["F_int_vy"].data();
    double* Ftx = V["Ftot_vx"].data(); double* Fty = V["Ftot_vy"].data();
    double* mvx = V["mom_vx"].data(); double* mvy = V["mom_vy"].data();
    double* Mv = V["Mv"].data();
    double* avx = V["avx"].data(); double* avy = V["avy"].data();
    double* vvx = V["vvx"].data(); double* vvy = V["vvy"].data();
    double* vvxL = V["vvxL"].data(); double* vvyL = V["vvyL"].data();
    for (idx_t n = 0; n < nn; ++n) {
      Ftx[n] = Fex[n] - Fix[n];
      Fty[n] = Fey[n] - Fiy[n];
    }
    for (idx_t n = 0; n < nn; ++n) {
      mvx[n] = dt * Ftx[n] + mvx[n];
      mvy[n] = dt * Fty[n] + mvy[n];
    }
    // (4) nodal accelerations and velocities
    for (idx_t n = 0; n < nn; ++n) {
      avx[n] = Mv[n] > 1.e-2 ? Ftx[n] / Mv[n] : 0.0;
      avy[n] = Mv[n] > 1.e-2 ? Fty[n] / Mv[n] : 0.0;
      vvx[n] = Mv[n] > 1.e-2 ? mvx[n] / Mv[n] : 0.0;
      vvy[n] = Mv[n] > 1.e-2 ? mvy[n] / Mv[n] : 0.0;
      vvxL[n] = dt * avx[n] + vvx[n];
      vvyL[n] = dt * avy[n] + vvy[n];
    }
    // (5) boundary conditions: cells on the x walls (e(2), e(3)) zero the
    // x components of their 4 nodes, cells on the y walls the y components
    if (o.d.BC_FLAG) {
      for (idx_t cell = 0; cell < o.ncells(); ++cell) {
        const idx_t r = cell % o.nrows, c = cell / o.nrows;
        if (c == 0 || c == o.ncols - 1)
          for (int k = 0; k < 4; ++k) {
            const idx_t n = gt(k, c, r, o.nrows);
            avx[n] = 0.0; vvx[n] = 0.0; vvxL[n] = 0.0; mvx[n] = 0.0;
          }
        if (r == 0 || r == o.nrows - 1)
          for (int k = 0; k < 4; ++k) {
            const idx_t n = gt(k, c, r, o.nrows);
            avy[n] = 0.0; vvy[n] = 0.0; vvyL[n] = 0.0; mvy[n] = 0.0;
          }
      }
    }
  }
  // (6) G2P and advection (PIC)
  for (const char* k : {"vpxL", "vpyL", "apx", "apy"})
    std::fill(dp[k].begin(), dp[k].end(), 0.0);
  g2p(o, {"vvxL", "vvyL", "avx", "avy"}, {"vpxL", "vpyL", "apx", "apy"});
  {
    double* vpx = dp["vpx"].data(); double* vpy = dp["vpy"].data();
    const double* vpxL = dp["vpxL"].data(); const double* vpyL = dp["vpyL"].data();
    const double eps = 1e-10;
    const double Lx = o.d.Nex * o.d.hx, Ly = o.d.Ney * o.d.hy;
    par_for(o, o.np, [&](idx_t ip) {
      vpx[ip] = vpxL[ip];
      vpy[ip] = vpyL[ip];
      o.x[ip] = o.x[ip] + dt * vpx[ip];
      o.y[ip] = o.y[ip] + dt * vpy[ip];
      if (o.x[ip] < eps) o.x[ip] = eps;
      if (o.x[ip] > Lx - eps) o.x[ip] = Lx - eps;
      if (o.y[ip] < eps) o.y[ip] = eps;
      if (o.y[ip] > Ly - eps) o.y[ip] = Ly - eps;
    });
  }
  // (7) height update from the strain rate (gradients at the new position,
  // with the cell of the step start)
  for (const char* k : {"vpx_dx", "vpy_dy", "vpx_dy", "vpy_dx"})
    std::fill(dp[k].begin(), dp[k].end(), 0.0);
  g2pd(o, {"vvxL", "vvyL"}, {"vpx_dx", "vpy_dx"}, {"vpx_dy", "vpy_dy"});
  {
    double* hp = dp["hp"].data();
    const double* exx = dp["vpx_dx"].data();
    const double* eyy = dp["vpy_dy"].data();
    const double* vpx = dp["vpx"].data(); const double* vpy = dp["vpy"].data();
    const double* Mp = dp["Mp"].data(); const double* Vp = dp["Vp"].data();
    double* mpx = dp["mom_px"].data(); double* mpy = dp["mom_py"].data();
    double* Ap = dp["Ap"].data();
    par_for(o, o.np, [&](idx_t ip) {
      const double div = exx[ip] + eyy[ip];
      hp[ip] = hp[ip] / (1 + dt * div);
      hp[ip] = hp[ip] < 1e-2 ? 1e-2 : hp[ip];
      mpx[ip] = vpx[ip] * Mp[ip];
      mpy[ip] = vpy[ip] * Mp[ip];
      Ap[ip] = hp[ip] > 1.e-2 ? Vp[ip] / hp[ip] : 0.0;
    });
  }
  // (7b) Voellmy friction (optim_par.cpp:613-626)
  {
    const double fric_ang = o.d.phi * M_PI / 180.;
    const double* vpx = dp["vpx"].data(); const double* vpy = dp["vpy"].data();
    const double* hp = dp["hp"].data();
    double* Fbx = dp["Fb_x"].data(); double* Fby = dp["Fb_y"].data();
    const auto& D = o.d;
    par_for(o, o.np, [&](idx_t ip) {
      const double vx = vpx[ip], vy = vpy[ip], h = hp[ip];
      const double nv = std::sqrt(vx * vx + vy * vy);
      if (D.FRICTION_ON > 0 && nv > 1e-10 && D.xi > 0) {
        const double v2 = vx * vx + vy * vy;
        Fbx[ip] = -D.FRICTION_ON *
                  (D.rho * D.g * h * std::tan(fric_ang) + D.rho * D.g * v2 / D.xi) *
                  vx / nv;
        Fby[ip] = -D.FRICTION_ON *
                  (D.rho * D.g * h * std::tan(fric_ang) + D.rho * D.g * v2 / D.xi) *
                  vy / nv;
      } else {
        Fbx[ip] = 0.0;
        Fby[ip] = 0.0;
      }
    });
  }
  // (8) stress update and output-only fields
  {
    const StressArgs sa = stress_args(o);
    par_for(o, o.np, [&](idx_t ip) { stress_one(o.d, sa, ip); });
  }
  std::fill(dp["hpZ"].begin(), dp["hpZ"].end(), 0.0);
  std::fill(dp["Zp"].begin(), dp["Zp"].end(), 0.0);
  g2p(o, {"Z"}, {"Zp"});
  {
    const double* hp = dp["hp"].data(); const double* Zp = dp["Zp"].data();
    double* hpZ = dp["hpZ"].data();
    par_for(o, o.np, [&](idx_t ip) { hpZ[ip] = hp[ip] + Zp[ip]; });
  }
  p2g(o, {"hp"}, {"HV"});
}

}  // namespace

// ===========================================================================
// C ABI used by the tests (ctypes) and by bench.py's CPU baseline
// ===========================================================================
extern "C" {

void* oracle_create(const oracle_data* d, const double* Z, const double* dZdx,
                    const double* dZdy, long long np, const double* x,
                    const double* y, const double* Mp, const double* Ap,
                    const double* vpx, const double* vpy, const double* hp,
                    const double* mom_px, const double* mom_py,
                    const double* Vp, int nthreads, int ms_enabled) {
  Oracle* o = new Oracle();
  o->d = *d;
  o->nrows = d->Ney;
  o->ncols = d->Nex;
  o->hx = d->hx;
  o->hy = d->hy;
  o->nthreads = nthreads < 1 ? 1 : nthreads;
  o->ms_enabled = ms_enabled != 0;
  const idx_t nn = o->nnodes();
  o->Z0.assign(Z, Z + nn);
  o->dZdx0.assign(dZdx, dZdx + nn);
  o->dZdy0.assign(dZdy, dZdy + nn);
  o->np = idx_t(np);
  o->x.assign(x, x + np);
  o->y.assign(y, y + np);
  for (const char* k : kDprops) o->dprops[k].assign(np, 0.0);
  o->dprops["Mp"].assign(Mp, Mp + np);
  o->dprops["Ap"].assign(Ap, Ap + np);
  o->dprops["vpx"].assign(vpx, vpx + np);
  o->dprops["vpy"].assign(vpy, vpy + np);
  o->dprops["mom_px"].assign(mom_px, mom_px + np);
  o->dprops["mom_py"].assign(mom_py, mom_py + np);
  o->dprops["hp"].assign(hp, hp + np);
  o->dprops["Vp"].assign(Vp, Vp + np);
  o->dprops["xp"].assign(x, x + np);
  o->dprops["yp"].assign(y, y + np);
  o->iprops["label"].resize(np);
  std::iota(o->iprops["label"].begin(), o->iprops["label"].end(), 0);
  o->iprops["level"].assign(np, 0);
  for (const char* k : kVars) o->vars[k].assign(nn, 0.0);
  o->vars["Z"] = o->Z0;
  o->vars["dZdx"] = o->dZdx0;
  o->vars["dZdy"] = o->dZdy0;
  // initialisation: optim_par.cpp:239-264
  init_particle_mesh(*o);
  g2p(*o, {"Z"}, {"Zp"});
  std::fill(o->dprops["dZxp"].begin(), o->dprops["dZxp"].end(), 0.0);
  std::fill(o->dprops["dZyp"].begin(), o->dprops["dZyp"].end(), 0.0);
  g2p(*o, {"dZdx", "dZdy"}, {"dZxp", "dZyp"});
  auto& dp = o->dprops;
  for (idx_t ip = 0; ip < o->np; ++ip) {
    dp["hpZ"][ip] = dp["hp"][ip] + dp["Zp"][ip];
    double diff = d->eq_level - dp["Zp"][ip];
    dp["H"][ip] = (d->eq_level > 0 && diff > 0) ? diff : 0.0;
  }
  for (idx_t ip = 0; ip < o->np; ++ip) {
    double h_corr = dp["hp"][ip] > 1e-10
                        ? dp["hp"][ip] - (dp["H"][ip] * dp["H"][ip]) / dp["hp"][ip]
                        : 0.0;
    dp["F_11"][ip] = -.5 * d->rho * d->g * h_corr;
    dp["F_12"][ip] = 0.0;
    dp["F_21"][ip] = 0.0;
    dp["F_22"][ip] = -.5 * d->rho * d->g * h_corr;
  }
  o->it = 0;
  o->t = 0.0;
  return o;
}

void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }

// Runs up to `nsteps` passes of the loop body while the loop condition
// holds.  Returns the number of steps taken.
int oracle_run(void* h, int nsteps) {
  Oracle& o = *static_cast<Oracle*>(h);
  int done = 0;
  while (done < nsteps && loop_condition(o)) {
    const double dt = compute_dt(o);
    o.it++;
    if (o.ms_enabled && o.d.ms_call_interval > 0 &&
        o.it % o.d.ms_call_interval == 0 && o.it > 0) {
      init_particle_mesh(o);
      merge_split_call(o, dt);
    }
    step_body(o, dt);
    o.t += dt;
    o.dt_last = dt;
    ++done;
  }
  return done;
}

// Standalone merge/split on the current state (no step), as invoked by
// gpu_offload.cpp:341 after a fresh binning.
void oracle_merge_split(void* h, double dt) {
  Oracle& o = *static_cast<Oracle*>(h);
  init_particle_mesh(o);
  merge_split_call(o, dt);
}

long long oracle_num_particles(void* h) { return static_cast<Oracle*>(h)->np; }
int oracle_iteration(void* h) { return static_cast<Oracle*>(h)->it; }
double oracle_time(void* h) { return static_cast<Oracle*>(h)->t; }
double oracle_last_dt(void* h) { return static_cast<Oracle*>(h)->dt_last; }
void oracle_ledger(void* h, double* out9) {
  std::memcpy(out9, static_cast<Oracle*>(h)->led, sizeof(double) * 9);
}
void oracle_ms_counts(void* h, long long* out4) {
  std::memcpy(out4, static_cast<Oracle*>(h)->ms_counts, sizeof(long long) * 4);
}

// Copies a particle field: "x", "y", any of the 35 dprops, or the iprops
// "label"/"level" (as doubles).  Returns 0 on success, -1 if unknown.
int oracle_get(void* h, const char* name, double* out) {
  Oracle& o = *static_cast<Oracle*>(h);
  const std::string n(name);
  if (n == "x") { std::copy(o.x.begin(), o.x.end(), out); return 0; }
  if (n == "y") { std::copy(o.y.begin(), o.y.end(), out); return 0; }
  auto it = o.dprops.find(n);
  if (it != o.dprops.end()) { std::copy(it->second.begin(), it->second.end(), out); return 0; }
  auto jt = o.iprops.find(n);
  if (jt != o.iprops.end()) {
    for (size_t i = 0; i < jt->second.size(); ++i) out[i] = double(jt->second[i]);
    return 0;
  }
  return -1;
}

// Overwrites a particle field (same names as oracle_get).
int oracle_set(void* h, const char* name, const double* in) {
  Oracle& o = *static_cast<Oracle*>(h);
  const std::string n(name);
  if (n == "x") { std::copy(in, in + o.np, o.x.begin()); return 0; }
  if (n == "y") { std::copy(in, in + o.np, o.y.begin()); return 0; }
  auto it = o.dprops.find(n);
  if (it != o.dprops.end()) { std::copy(in, in + o.np, it->second.begin()); return 0; }
  auto jt = o.iprops.find(n);
  if (jt != o.iprops.end()) {
    for (idx_t i = 0; i < o.np; ++i) jt->second[i] = idx_t(in[i]);
    return 0;
  }
  return -1;
}

// Copies a nodal var of the last step (the 24 names of optim_par.cpp:199-225).
int oracle_get_nodal(void* h, const char* name, double* out) {
  Oracle& o = *static_cast<Oracle*>(h);
  auto it = o.vars.find(name);
  if (it == o.vars.end()) return -1;
  std::copy(it->second.begin(), it->second.end(), out);
  return 0;
}

// Cell of every particle from the last binning and the CSR arrays.
void oracle_binning(void* h, int* p2c, int* cell_start, int* cell_ptcls) {
  Oracle& o = *static_cast<Oracle*>(h);
  init_particle_mesh(o);
  if (p2c) std::copy(o.p2c.begin(), o.p2c.end(), p2c);
  if (cell_start) std::copy(o.cell_start.begin(), o.cell_start.end(), cell_start);
  if (cell_ptcls) std::copy(o.cell_ptcls.begin(), o.cell_ptcls.end(), cell_ptcls);
}

}  // extern "C"
