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
  double ihx, ihy;       // 1/hx, 1/hy (used where h is a power of two)
  // The part of the grid a slab owns (the whole grid outside slab mode):
  // particles of cell columns [pc_lo, pc_hi), node columns [nc_lo, nc_hi]
  // written by P2G.
  int pc_lo, pc_hi, nc_lo, nc_hi;
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
  int nghost;   // slab mode: copies of the neighbour's last column, sorted first
  int nleave;   // slab mode: particles G2P moved out of the slab's columns
  unsigned long long red_cur[3];   // ordered keys of max|vpx|, max|vpy|, max hp
  unsigned long long red_next[3];  // ... produced by this step's G2P
  // cell-key ranges for the counting sort's scan: krange = the keys the cell
  // starts describe, knext = the keys G2P produced since (lo > hi: none)
  int krange[2];
  int knext[2];
  double ledger[9];
  long long ms_counts[4];
};

constexpr int kStatusCapacity = 1;
constexpr int kStatusNonFinite = 2;
constexpr int kStatusSlab = 4;  // a particle arrived outside the slab's columns
constexpr int kStatusMsLimit = 8;  // a merge/split loop ran past its bound

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

// Cell (row, col) of a position: floor(y/hy), floor(x/hx), clamped.  Where
// h is a power of two the quotient equals the product with 1/h exactly
// (both are the correctly rounded value of the same real number), and the
// division is skipped.
__device__ __forceinline__ int cell_index(double f, int n) {
  if (!(f >= 0.0)) return 0;
  if (f > double(n - 1)) return n - 1;
  return int(f);
}
__device__ __forceinline__ int cell_row(double y, const Geom& G) {
  if (G.hy_pow2) return cell_index(floor(y * G.ihy), G.nrows);
  return cell_index(floor(y / G.hy), G.nrows);
}
__device__ __forceinline__ int cell_col(double x, const Geom& G) {
  if (G.hx_pow2) return cell_index(floor(x * G.ihx), G.ncols);
  return cell_index(floor(x / G.hx), G.ncols);
}

// The functions below are templates on the real type R of the particle
// arithmetic: R = double is the FP64 path (the expressions are the
// reference's, operand for operand); R = float is the FP32 form, whose
// well-balanced depth terms are still evaluated in FP64.

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
template <class R>
__device__ __forceinline__ void local_xy_g(R x, R y, int c, int r, const Geom& G,
                                           R ihx, R ihy, R& xi, R& eta) {
  const R dx = x - c * R(G.hx), dy = y - r * R(G.hy);
  xi = G.hx_pow2 ? dx * ihx : dx / R(G.hx);
  eta = G.hy_pow2 ? dy * ihy : dy / R(G.hy);
}

// shp (main/gpu_kernels.cpp:33-41)
template <class R>
__device__ __forceinline__ R shp(R xi, R eta, int inode) {
  switch (inode) {
    case 3: return xi * eta;
    case 2: return xi * (R(1) - eta);
    case 1: return (R(1) - xi) * eta;
    default: return (R(1) - xi) * (R(1) - eta);
  }
}

// shg (main/gpu_kernels.cpp:43-59); ihx = 1.0/hx, mihx = -1.0/hx, etc.
template <class R>
__device__ __forceinline__ R shg_x(R eta, int inode, R ihx, R mihx) {
  switch (inode) {
    case 3: return ihx * eta;
    case 2: return ihx * (R(1) - eta);
    case 1: return mihx * eta;
    default: return mihx * (R(1) - eta);
  }
}
template <class R>
__device__ __forceinline__ R shg_y(R xi, int inode, R ihy, R mihy) {
  switch (inode) {
    case 3: return xi * ihy;
    case 2: return xi * mihy;
    case 1: return (R(1) - xi) * ihy;
    default: return (R(1) - xi) * mihy;
  }
}

// Voellmy basal friction (main/optim_par.cpp:613-626).
template <class R>
__device__ __forceinline__ void voellmy(const Phys& P, R vx, R vy, R h, R& fbx,
                                        R& fby) {
  const R nv = sqrt(vx * vx + vy * vy);
  if (P.FON > 0 && nv > R(1e-10) && P.xi > 0) {
    const R rho = R(P.rho), g = R(P.g);
    const R v2 = vx * vx + vy * vy;
    const R s = rho * g * h * R(P.tan_fa) + rho * g * v2 / R(P.xi);
    fbx = -R(P.FON) * s * vx / nv;
    fby = -R(P.FON) * s * vy / nv;
  } else {
    fbx = R(0);
    fby = R(0);
  }
}

// Bingham stress + well-balanced pressure: the stress_tensor_t functor of
// main/optim_par.cpp:68-120.  F_21 == F_12.  The pressure term
// 0.5*rho*g*(hp - H^2/hp), which nearly cancels over a lake at rest, is
// evaluated in FP64 whatever R is.
template <class R>
__device__ __forceinline__ void bingham_stress(const Phys& P, R vpx, R vpy, R hp,
                                               R H, R vpx_dx, R vpy_dy, R vpx_dy,
                                               R vpy_dx, R& F11, R& F12, R& F22) {
  const R A = R(3.) / R(2.), C = R(65.) / R(32.);
  const R nrm = sqrt(vpx * vpx + vpy * vpy);
  const R mu = R(P.mu), tau_Y = R(P.tauy);
  const R ALF = hp > R(1.e-3) ? (R(6.) * mu * nrm) / ((hp + R(0.001)) * tau_Y) : R(0);
  const R B = -R(114.) / R(32.) - ALF;
  const R sq = sqrt(B * B - R(4.) * A * C);
  const R Z2 = (-B - sq) / (R(2.) * A);
  // The reference takes Z1 when |Z1 - 0.5| <= 0.5.  With B <= -3 (every
  // ALF >= 0) Z1 = (-B + sq)/3 >= 1 rounds to at least 1.1875 whenever sq
  // is a number (and is NaN otherwise), so Z2 is taken: Z1 is only
  // evaluated where it can be chosen.  The result is the same in every case.
  R ZZ = Z2;
  if (!(B <= R(-3.))) {
    const R Z1 = (-B + sq) / (R(2.) * A);
    ZZ = fabs(Z1 - R(.5)) <= R(.5) ? Z1 : Z2;
  }
  const R D_xx = vpx_dx;
  const R D_xy = R(0.5) * (vpx_dy + vpy_dx);
  const R D_yy = vpy_dy;
  const R D_zx =
      hp > R(1.e-3) ? R(0.5) * (R(3.) / (R(2.) + ZZ)) * (vpx / (hp + R(0.001))) : R(0);
  const R D_zy =
      hp > R(1.e-3) ? R(0.5) * (R(3.) / (R(2.) + ZZ)) * (vpy / (hp + R(0.001))) : R(0);
  const R D_zz = -(vpx_dx + vpy_dy);
  const R invII = R(0.5) * (D_xx * D_xx + D_yy * D_yy + D_zz * D_zz) +
                  D_zx * D_zx + D_zy * D_zy + D_xy * D_xy;
  R sig_xx = R(0), sig_xy = R(0), sig_yy = R(0);
  if (invII != R(0)) {
    const R k = tau_Y / sqrt(invII) + R(2.) * mu;
    sig_xx = k * D_xx;
    sig_xy = k * D_xy;
    sig_yy = k * D_yy;
  }
  const double hpd = hp, Hd = H;
  // (H*H)/hp is +0 when H == 0 (no still-water level): hp - 0 is hp
  const double h_corr = hpd > 1e-10 ? (Hd == 0.0 ? hpd : hpd - (Hd * Hd) / hpd) : 0.0;
  const double pres = .5 * P.rho * P.g * h_corr;
  F11 = R(P.BING * double(sig_xx) - pres);
  F12 = R(P.BING * double(sig_xy));
  F22 = R(P.BING * double(sig_yy) - pres);
}

// The rheology of the FP32 form (the Bingham stress with its plug switch,
// the Voellmy friction) is evaluated in FP32.  Building with
// DAMPM_FP32_RHEOLOGY=64 evaluates it in FP64 on the FP32 values instead;
// measured against the FP64 path, that changes the depth error of neither
// smooth flows (1.8e-5 after 500 passes either way) nor yield-stress flows
// (8.2e-2 against 8.8e-2 after 1000 passes, the flow's own sensitivity
// dominating) and costs a fifth of the FP32 mudflow's step time.
#ifndef DAMPM_FP32_RHEOLOGY
#define DAMPM_FP32_RHEOLOGY 32
#endif
template <class R>
__device__ __forceinline__ void rheology_stress(const Phys& P, R vpx, R vpy, R hp, R H,
                                                R vpx_dx, R vpy_dy, R vpx_dy, R vpy_dx,
                                                R& F11, R& F12, R& F22) {
  if constexpr (sizeof(R) == 4 && DAMPM_FP32_RHEOLOGY == 64) {
    double f11, f12, f22;
    bingham_stress<double>(P, vpx, vpy, hp, H, vpx_dx, vpy_dy, vpx_dy, vpy_dx, f11, f12,
                           f22);
    F11 = R(f11);
    F12 = R(f12);
    F22 = R(f22);
  } else {
    bingham_stress<R>(P, vpx, vpy, hp, H, vpx_dx, vpy_dy, vpx_dy, vpy_dx, F11, F12, F22);
  }
}

template <class R>
__device__ __forceinline__ void rheology_friction(const Phys& P, R vx, R vy, R h, R& fbx,
                                                  R& fby) {
  if constexpr (sizeof(R) == 4 && DAMPM_FP32_RHEOLOGY == 64) {
    double fx, fy;
    voellmy<double>(P, vx, vy, h, fx, fy);
    fbx = R(fx);
    fby = R(fy);
  } else {
    voellmy<R>(P, vx, vy, h, fbx, fby);
  }
}

}  // namespace dampm
