// dampm_device.cuh -- device-side definitions shared by the step kernels.
//
// Every FP64 expression below keeps the operand order of the reference
// (main/optim_par.cpp, main/gpu_kernels.cpp) and the translation units are
// built with --fmad=false, so each operation rounds exactly as the
// reference's C++ does: the FP64 path is bitwise reproducible against the
// CPU restatement, not merely close.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dampm {

// Geometry (grid.set_sizes(Ney, Nex, hx, hy), main/optim_par.cpp:136).
struct Geom {
  int nrows;   // Ney
  int ncols;   // Nex
  double hx, hy;
  double Lx, Ly;  // Nex*hx, Ney*hy (main/optim_par.cpp:557-558)
  int hx_pow2, hy_pow2;  // h is a power of two: v/h == v*(1/h) exactly
};

// Scalars of struct DATA used inside the step (main/mpm_data.h:21-44).
struct Phys {
  double g, rho, mu, tauy, xi;
  double tan_fa;  // tan(phi*pi/180), evaluated on the host with libm
  double BING, FON, CFL, eq_level, DT_FIXED, T;
  int BC, NSTEPS, fixed;
};

// Loop state kept on the device so that whole runs need no host sync.
struct Scalars {
  double t;
  double dt;
  int it;
  int active;   // this pass of the loop body executes
  int fresh;    // next P2G reads Ap/mom/Fb from the stored arrays
  int status;   // error bits (kStatus*)
  int np;       // current particle count
  int np_next;  // particle count after a merge/split emit
  unsigned long long red_cur[3];   // ordered keys of max|vpx|, max|vpy|, max hp
  unsigned long long red_next[3];  // ... produced by this step's G2P
  double ledger[9];
  long long ms_counts[4];
};

constexpr int kStatusCapacity = 1;
constexpr int kStatusNonFinite = 2;

// --- order-preserving double <-> u64 map for atomicMax reductions --------
__device__ __forceinline__ unsigned long long ordered_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ordered_value(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// --- quadgrid index helpers (main/gpu_kernels.cpp:7-16) -------------------
__device__ __forceinline__ int node_of(int inode, int c, int r, int nrows) {
  const int bl = r + c * (nrows + 1);
  switch (inode) {
    case 0: return bl;
    case 1: return bl + 1;
    case 2: return bl + (nrows + 1);
    default: return bl + (nrows + 2);
  }
}

// Cell (row, col) of a position: floor(y/hy), floor(x/hx), clamped.
__device__ __forceinline__ int cell_row(double y, double hy, int nrows) {
  double f = floor(y / hy);
  if (!(f >= 0.0)) return 0;
  if (f > double(nrows - 1)) return nrows - 1;
  return int(f);
}
__device__ __forceinline__ int cell_col(double x, double hx, int ncols) {
  double f = floor(x / hx);
  if (!(f >= 0.0)) return 0;
  if (f > double(ncols - 1)) return ncols - 1;
  return int(f);
}

// Local coordinates in cell (r, c): (x - c*hx)/hx, (y - r*hy)/hy
// (pnode, main/gpu_kernels.cpp:21-31).
__device__ __forceinline__ void local_xy(double x, double y, int c, int r,
                                         double hx, double hy, double& xi,
                                         double& eta) {
  xi = (x - c * hx) / hx;
  eta = (y - r * hy) / hy;
}

// Same values as local_xy; when h is a power of two the quotient by h equals
// the product with 1/h exactly, and the division is skipped.
__device__ __forceinline__ void local_xy_g(double x, double y, int c, int r,
                                           const Geom& G, double ihx,
                                           double ihy, double& xi,
                                           double& eta) {
  const double dx = x - c * G.hx, dy = y - r * G.hy;
  xi = G.hx_pow2 ? dx * ihx : dx / G.hx;
  eta = G.hy_pow2 ? dy * ihy : dy / G.hy;
}

// shp (main/gpu_kernels.cpp:33-41)
__device__ __forceinline__ double shp(double xi, double eta, int inode) {
  switch (inode) {
    case 3: return xi * eta;
    case 2: return xi * (1.0 - eta);
    case 1: return (1.0 - xi) * eta;
    default: return (1.0 - xi) * (1.0 - eta);
  }
}

// shg (main/gpu_kernels.cpp:43-59); ihx = 1.0/hx, mihx = -1.0/hx, etc.
__device__ __forceinline__ double shg_x(double eta, int inode, double ihx,
                                        double mihx) {
  switch (inode) {
    case 3: return ihx * eta;
    case 2: return ihx * (1.0 - eta);
    case 1: return mihx * eta;
    default: return mihx * (1.0 - eta);
  }
}
__device__ __forceinline__ double shg_y(double xi, int inode, double ihy,
                                        double mihy) {
  switch (inode) {
    case 3: return xi * ihy;
    case 2: return xi * mihy;
    case 1: return (1.0 - xi) * ihy;
    default: return (1.0 - xi) * mihy;
  }
}

// Voellmy basal friction (main/optim_par.cpp:613-626).
__device__ __forceinline__ void voellmy(const Phys& P, double vx, double vy,
                                        double h, double& fbx, double& fby) {
  const double nv = sqrt(vx * vx + vy * vy);
  if (P.FON > 0 && nv > 1e-10 && P.xi > 0) {
    const double v2 = vx * vx + vy * vy;
    const double s = P.rho * P.g * h * P.tan_fa + P.rho * P.g * v2 / P.xi;
    fbx = -P.FON * s * vx / nv;
    fby = -P.FON * s * vy / nv;
  } else {
    fbx = 0.0;
    fby = 0.0;
  }
}

// Bingham stress + well-balanced pressure: the stress_tensor_t functor of
// main/optim_par.cpp:68-120.  F_21 == F_12.
__device__ __forceinline__ void bingham_stress(const Phys& P, double vpx,
                                               double vpy, double hp, double H,
                                               double vpx_dx, double vpy_dy,
                                               double vpx_dy, double vpy_dx,
                                               double& F11, double& F12,
                                               double& F22) {
  const double A = 3. / 2., C = 65. / 32.;
  const double nrm = sqrt(vpx * vpx + vpy * vpy);
  const double mu = P.mu, tau_Y = P.tauy;
  const double ALF = hp > 1.e-3 ? (6. * mu * nrm) / ((hp + 0.001) * tau_Y) : 0.0;
  const double B = -114. / 32. - ALF;
  const double Z1 = (-B + sqrt(B * B - 4. * A * C)) / (2. * A);
  const double Z2 = (-B - sqrt(B * B - 4. * A * C)) / (2. * A);
  const double ZZ = fabs(Z1 - .5) <= .5 ? Z1 : Z2;
  const double D_xx = vpx_dx;
  const double D_xy = 0.5 * (vpx_dy + vpy_dx);
  const double D_yy = vpy_dy;
  const double D_zx =
      hp > 1.e-3 ? 0.5 * (3. / (2. + ZZ)) * (vpx / (hp + 0.001)) : 0.0;
  const double D_zy =
      hp > 1.e-3 ? 0.5 * (3. / (2. + ZZ)) * (vpy / (hp + 0.001)) : 0.0;
  const double D_zz = -(vpx_dx + vpy_dy);
  const double invII = 0.5 * (D_xx * D_xx + D_yy * D_yy + D_zz * D_zz) +
                       D_zx * D_zx + D_zy * D_zy + D_xy * D_xy;
  double sig_xx = 0.0, sig_xy = 0.0, sig_yy = 0.0;
  if (invII != 0) {
    const double k = tau_Y / sqrt(invII) + 2. * mu;
    sig_xx = k * D_xx;
    sig_xy = k * D_xy;
    sig_yy = k * D_yy;
  }
  const double h_corr = hp > 1e-10 ? hp - (H * H) / hp : 0.0;
  const double pres = .5 * P.rho * P.g * h_corr;
  F11 = P.BING * sig_xx - pres;
  F12 = P.BING * sig_xy;
  F22 = P.BING * sig_yy - pres;
}

}  // namespace dampm
