// host_util.h -- host-side helpers shared by the single-scenario and batch
// boundaries: device geometry and physics from the C-ABI structs.
#pragma once
#include <cmath>

#include "../../include/dampm_cuda.h"
#include "dampm_kernels.h"

namespace dampm {

// grid.set_sizes(Ney, Nex, hx, hy) (main/optim_par.cpp:136): rows = Ney.
inline Geom make_geom(const dampm_grid& g) {
  Geom G{};
  G.nrows = g.Ney;
  G.ncols = g.Nex;
  G.hx = g.hx;
  G.hy = g.hy;
  G.Lx = g.Nex * g.hx;
  G.Ly = g.Ney * g.hy;
  int e;
  G.hx_pow2 = std::frexp(g.hx, &e) == 0.5 ? 1 : 0;
  G.hy_pow2 = std::frexp(g.hy, &e) == 0.5 ? 1 : 0;
  G.ihx = 1.0 / g.hx;
  G.ihy = 1.0 / g.hy;
  G.pc_lo = 0;
  G.pc_hi = g.Nex;
  G.nc_lo = 0;
  G.nc_hi = g.Nex;
  return G;
}

inline Phys make_phys(const dampm_params& d) {
  Phys P{};
  P.g = d.g;
  P.rho = d.rho;
  P.mu = d.mu;
  P.tauy = d.tauy;
  P.xi = d.xi;
  const double fric_ang = d.phi * M_PI / 180.;  // main/optim_par.cpp:193
  P.tan_fa = std::tan(fric_ang);
  P.BING = d.BINGHAM_ON;
  P.FON = d.FRICTION_ON;
  P.CFL = d.CFL;
  P.eq_level = d.eq_level;
  P.DT_FIXED = d.DT_FIXED;
  P.T = d.T;
  P.BC = d.BC_FLAG;
  P.NSTEPS = d.NSTEPS;
  P.fixed = d.DT_FIXED > 0.0 ? 1 : 0;
  return P;
}

// Host halves (a, b) of n pairs into a pair array: two strided copies.
template <class T, class V>
cudaError_t upload_pair(V* dst, const T* a, const T* b, long long n, cudaStream_t st) {
  static_assert(sizeof(V) == 2 * sizeof(T), "pair of T");
  if (n <= 0) return cudaSuccess;
  cudaError_t e = cudaMemcpy2DAsync(dst, sizeof(V), a, sizeof(T), sizeof(T), size_t(n),
                                    cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  return cudaMemcpy2DAsync(reinterpret_cast<T*>(dst) + 1, sizeof(V), b, sizeof(T),
                           sizeof(T), size_t(n), cudaMemcpyHostToDevice, st);
}

// Half `half` (0: first, 1: second) of n pairs to the host.
template <class T, class V>
cudaError_t download_pair_half(T* out, const V* src, int half, long long n,
                               cudaStream_t st) {
  static_assert(sizeof(V) == 2 * sizeof(T), "pair of T");
  if (n <= 0) return cudaSuccess;
  return cudaMemcpy2DAsync(out, sizeof(T), reinterpret_cast<const T*>(src) + half, sizeof(V),
                           sizeof(T), size_t(n), cudaMemcpyDeviceToHost, st);
}

inline int grid_blocks(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return int(b);
}

}  // namespace dampm
