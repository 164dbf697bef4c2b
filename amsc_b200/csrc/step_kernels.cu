// step_kernels.cu -- the FP64 MPM time step on sm_100a.
//
// One pass of the loop body of main/optim_par.cpp:281-668 is
//   step_begin  : dt (fixed or CFL from the previous G2P's max-reductions),
//                 it++, loop condition -- one thread, no host sync
//   SORT        : count -> scan -> scatter -> per-cell order  (a1)
//   P2G+NODAL   : per-node sequential chains over the sorted particles of the
//                 node's 4 cells, nodal momentum/velocity/BC  (a2-a7, a10, a14)
//   G2P         : velocity, advection, gradients, height, Bingham stress,
//                 next cell key, CFL max-reductions  (a8, a9, a11, a13)
//   step_end    : t += dt
#include <cstdio>

#include "dampm_device.cuh"
#include "dampm_kernels.h"

namespace dampm {

// ---------------------------------------------------------------------------
// loop control
// ---------------------------------------------------------------------------
__global__ void k_step_begin(Scalars* S, Geom G, Phys P) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool cond = P.fixed ? (S->it < P.NSTEPS) : (S->t < P.T);
  if (!cond || S->status != 0) {
    S->active = 0;
    return;
  }
  S->active = 1;
  double dt;
  if (P.fixed) {
    dt = P.DT_FIXED;
  } else {
    // main/optim_par.cpp:289-304; first pass: 1e-3 (main/gpu_offload.cpp:255)
    dt = 1.0e-3;
    if (S->it > 0) {
      const double mvx = ordered_value(S->red_cur[0]);
      const double mvy = ordered_value(S->red_cur[1]);
      const double hmean = ordered_value(S->red_cur[2]);
      const double a = sqrt(P.g * hmean) + mvx;
      const double b = sqrt(P.g * hmean) + mvy;
      const double max_vel = (a < b) ? b : a;  // std::max
      const double cel = fabs(max_vel);
      const double hmin = (G.hy < G.hx) ? G.hy : G.hx;  // std::min
      dt = P.CFL * hmin / (1e-2 + cel);
    }
  }
  S->dt = dt;
  S->it += 1;
  S->red_next[0] = S->red_next[1] = S->red_next[2] = 0ull;
}

__global__ void k_step_end(Scalars* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (!S->active) return;
  S->t += S->dt;
  S->fresh = 0;
  S->red_cur[0] = S->red_next[0];
  S->red_cur[1] = S->red_next[1];
  S->red_cur[2] = S->red_next[2];
}

// ---------------------------------------------------------------------------
// initialisation after upload: main/optim_par.cpp:239-264
// ---------------------------------------------------------------------------
__global__ void k_init_particles(Particles p, const double* __restrict__ Z,
                                 const double* __restrict__ dZdx,
                                 const double* __restrict__ dZdy, Geom G,
                                 Phys P, Scalars* S, int np) {
  __shared__ unsigned long long red[3];
  if (threadIdx.x < 3) red[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const double x = p.x[i], y = p.y[i];
    const int r = cell_row(y, G.hy, G.nrows), c = cell_col(x, G.hx, G.ncols);
    p.key[i] = r + c * G.nrows;
    p.label[i] = i;
    p.level[i] = 0;
    double xi, eta;
    local_xy(x, y, c, r, G.hx, G.hy, xi, eta);
    double zp = 0.0, dzx = 0.0, dzy = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double N = shp(xi, eta, k);
      const int n = node_of(k, c, r, G.nrows);
      zp += N * Z[n];
      dzx += N * dZdx[n];
      dzy += N * dZdy[n];
    }
    const double hp = p.hp[i];
    const double diff = P.eq_level - zp;
    const double H = (P.eq_level > 0 && diff > 0) ? diff : 0.0;
    p.H[i] = H;
    const double h_corr = hp > 1e-10 ? hp - (H * H) / hp : 0.0;
    const double f = -.5 * P.rho * P.g * h_corr;
    p.F11[i] = f;
    p.F12[i] = 0.0;
    p.F22[i] = f;
    p.Fbx[i] = 0.0;
    p.Fby[i] = 0.0;
    if (p.Zp) {
      p.Zp[i] = zp;
      p.hpZ[i] = hp + zp;
      p.dZxp[i] = dzx;
      p.dZyp[i] = dzy;
    }
    m0 = max(m0, ordered_key(fabs(p.vpx[i])));
    m1 = max(m1, ordered_key(fabs(p.vpy[i])));
    m2 = max(m2, ordered_key(hp));
  }
  atomicMax(&red[0], m0);
  atomicMax(&red[1], m1);
  atomicMax(&red[2], m2);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&S->red_cur[0], red[0]);
    atomicMax(&S->red_cur[1], red[1]);
    atomicMax(&S->red_cur[2], red[2]);
  }
}

// Recomputes the cell key of every particle (after a merge/split emit or a
// state upload).
__global__ void k_keys(const double* __restrict__ x,
                       const double* __restrict__ y, int* __restrict__ key,
                       Geom G, const Scalars* S) {
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int r = cell_row(y[i], G.hy, G.nrows);
    const int c = cell_col(x[i], G.hx, G.ncols);
    key[i] = r + c * G.nrows;
  }
}

// Max-reductions of the current state (for the next CFL dt).
__global__ void k_reduce_state(Particles p, Scalars* S) {
  __shared__ unsigned long long red[3];
  if (threadIdx.x < 3) red[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    m0 = max(m0, ordered_key(fabs(p.vpx[i])));
    m1 = max(m1, ordered_key(fabs(p.vpy[i])));
    m2 = max(m2, ordered_key(p.hp[i]));
  }
  atomicMax(&red[0], m0);
  atomicMax(&red[1], m1);
  atomicMax(&red[2], m2);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&S->red_cur[0], red[0]);
    atomicMax(&S->red_cur[1], red[1]);
    atomicMax(&S->red_cur[2], red[2]);
  }
}

// ---------------------------------------------------------------------------
// SORT: stable counting sort by cell, (cell, particle index) order
// (init_particle_mesh + cell_start/cell_ptcls, main/gpu_offload.cpp:243-249)
// ---------------------------------------------------------------------------
__global__ void k_count(const int* __restrict__ key, int* __restrict__ count,
                        int* __restrict__ slot, const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x)
    slot[i] = atomicAdd(&count[key[i]], 1);
}

// exclusive scan of count[0..n) into start[0..n]; count is zeroed on the way
// (ready for the next step).  Three phases over tiles of kScanTile items.
__global__ void k_scan_tiles(const int* __restrict__ count, int n,
                             int* __restrict__ tile_sum, const Scalars* S) {
  if (!S->active) return;
  __shared__ int wsum[32];
  const int base = blockIdx.x * kScanTile;
  int s = 0;
  for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
    const int i = base + k;
    if (i < n) s += count[i];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = (threadIdx.x < (blockDim.x >> 5)) ? wsum[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = v;
  }
}

// single block: exclusive scan of the tile sums in place; total at [ntiles]
__global__ void k_scan_tile_sums(int* __restrict__ tile_sum, int ntiles,
                                 const Scalars* S) {
  if (!S->active) return;
  __shared__ int wsum[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int base = 0; base < ntiles; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = (i < ntiles) ? tile_sum[i] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      int ws = (lane < nw) ? wsum[lane] : 0;
      int wi = ws;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      if (lane < nw) wsum[lane] = wi - ws;  // exclusive warp offsets
    }
    __syncthreads();
    const int excl = carry + wsum[w] + incl - v;
    if (i < ntiles) tile_sum[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sum[ntiles] = carry;
}

__global__ void k_scan_apply(int* __restrict__ count, int n,
                             const int* __restrict__ tile_sum,
                             int* __restrict__ start, const Scalars* S) {
  if (!S->active) return;
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int base = blockIdx.x * kScanTile;
  if (threadIdx.x == 0) carry = tile_sum[blockIdx.x];
  __syncthreads();
  for (int off = 0; off < kScanTile; off += blockDim.x) {
    const int i = base + off + threadIdx.x;
    int v = 0;
    if (i < n) {
      v = count[i];
      count[i] = 0;
    }
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      int ws = (lane < nw) ? wsum[lane] : 0;
      int wi = ws;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      if (lane < nw) wsum[lane] = wi - ws;
    }
    __syncthreads();
    const int excl = carry + wsum[w] + incl - v;
    if (i < n) start[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    start[n] = tile_sum[gridDim.x];
}

__global__ void k_scatter(const int* __restrict__ key,
                          const int* __restrict__ slot,
                          const int* __restrict__ start, int* __restrict__ perm,
                          const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x)
    perm[start[key[i]] + slot[i]] = i;
}

// Orders each cell's segment by ascending particle index (the atomics of
// k_count hand out slots in arbitrary order).  One thread per cell.
__global__ void k_segment_order(const int* __restrict__ start, int ncells,
                                int* __restrict__ perm, const Scalars* S) {
  if (!S->active) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += gridDim.x * blockDim.x) {
    const int b = start[c], e = start[c + 1];
    if (e - b < 2) continue;
    for (int j = b + 1; j < e; ++j) {
      const int v = perm[j];
      int k = j - 1;
      while (k >= b && perm[k] > v) {
        perm[k + 1] = perm[k];
        --k;
      }
      perm[k + 1] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// P2G + NODAL
//
// A CTA owns the node rows [r0, r0+kTR) of one strip and the node columns
// [cA, cB) of one chunk.  It walks the cell columns cA-1 .. cB-1.  For cell
// column cc the particles of cells (rlo..rhi, cc) are one contiguous range of
// the sorted order; records are computed once per particle into shared memory
// in batches of kCap.  Thread (row r, side):
//   side 0 finishes node (r, cc): it carries the chain over cells
//          (r-1, cc-1), (r, cc-1) handed over from the previous column and
//          adds cells (r-1, cc) [local node 1] then (r, cc) [local node 0];
//   side 1 starts node (r, cc+1) with cells (r-1, cc) [local node 3] then
//          (r, cc) [local node 2].
// These are exactly the node's contributions in quadgrid's cell-sweep order,
// so every nodal sum is the reference's sequential sum, bit for bit.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNQ = 9;  // Mv, mom_x, mom_y, FPx, FPy, Fric_x, Fric_y, Fint_x, Fint_y

struct P2GSmem {
  double xi[kCap], eta[kCap], Mp[kCap], mpx[kCap], mpy[kCap], Fpx[kCap],
      Fpy[kCap], Frx[kCap], Fry[kCap], F11[kCap], F12[kCap], F22[kCap],
      Vp[kCap];
  int rowstart[kTR + 2];
  double hand[kNQ][kTR];
  double led[6][kP2GThreads / 32];
};

__device__ __forceinline__ void add_contrib(double (&acc)[kNQ],
                                            const P2GSmem& s, int j, int k,
                                            double ihx, double mihx,
                                            double ihy, double mihy) {
  const double xi = s.xi[j], eta = s.eta[j];
  const double N = shp(xi, eta, k);
  const double Nx = shg_x(eta, k, ihx, mihx);
  const double Ny = shg_y(xi, k, ihy, mihy);
  acc[0] += N * s.Mp[j];
  acc[1] += N * s.mpx[j];
  acc[2] += N * s.mpy[j];
  acc[3] += N * s.Fpx[j];
  acc[4] += N * s.Fpy[j];
  acc[5] += N * s.Frx[j];
  acc[6] += N * s.Fry[j];
  const double f12 = s.F12[j], vp = s.Vp[j];
  acc[7] += (Nx * s.F11[j] + Ny * f12) * vp;
  acc[8] += (Nx * f12 + Ny * s.F22[j]) * vp;
}
}  // namespace

__global__ void __launch_bounds__(kP2GThreads)
    k_p2g(Particles p, const int* __restrict__ perm,
          const int* __restrict__ cstart, const double* __restrict__ Z,
          Nodes nodes, double* __restrict__ led_part, Geom G, Phys P,
          const Scalars* S, int record) {
  if (!S->active) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  P2GSmem& s = *reinterpret_cast<P2GSmem*>(smem_raw);

  const int nrows = G.nrows, ncols = G.ncols;
  const int r0 = blockIdx.x * kTR;
  const int cA = blockIdx.y * kLC;
  const int cB = min(cA + kLC, ncols + 1);
  const int rlo = max(r0 - 1, 0);
  const int rhi = min(r0 + kTR - 1, nrows - 1);
  const int ccFirst = max(cA - 1, 0);
  const int ccLast = min(cB - 1, ncols - 1);
  const int tid = threadIdx.x;
  const int row = tid % kTR, side = tid / kTR;
  const int r = r0 + row;
  const double dt = S->dt;
  const bool fresh = S->fresh != 0;
  const double hx = G.hx, hy = G.hy;
  const double ihx = 1.0 / hx, mihx = -1.0 / hx;
  const double ihy = 1.0 / hy, mihy = -1.0 / hy;

  // any particle in the cell block this CTA touches?
  int any = 0;
  if (tid == 0) {
    for (int cc = ccFirst; cc <= ccLast; ++cc)
      any |= (cstart[rhi + cc * nrows + 1] - cstart[rlo + cc * nrows]) != 0;
  }
  any = __syncthreads_or(any);
  double lp0 = 0, lp1 = 0, lp2 = 0, ln0 = 0, ln1 = 0, ln2 = 0;
  if (any || record) {
    for (int q = tid; q < kNQ * kTR; q += kP2GThreads)
      (&s.hand[0][0])[q] = 0.0;
    __syncthreads();

    for (int cc = ccFirst; cc <= ccLast; ++cc) {
      const int cbase = cc * nrows;
      for (int q = tid; q < kTR + 2; q += kP2GThreads) {
        const int rr = rlo + q;
        s.rowstart[q] = cstart[min(rr, rhi + 1) + cbase];
      }
      __syncthreads();
      const int seg0 = s.rowstart[0];
      const int seg1 = s.rowstart[rhi - rlo + 1];
      // per-thread ranges (global sorted positions) of cells r-1 and r
      int a0 = 0, a1 = 0, b0 = 0, b1 = 0;  // cell r-1: [a0,a1), cell r: [b0,b1)
      if (r - 1 >= rlo && r - 1 <= rhi) {
        a0 = s.rowstart[r - 1 - rlo];
        a1 = s.rowstart[r - rlo];
      }
      if (r >= rlo && r <= rhi) {
        b0 = s.rowstart[r - rlo];
        b1 = s.rowstart[r - rlo + 1];
      }
      const bool fin_active = (side == 0) && (cc >= cA) && (r <= nrows);
      const bool start_active = (side == 1) && (cc + 1 < cB) && (r <= nrows);
      double acc[kNQ];
#pragma unroll
      for (int q = 0; q < kNQ; ++q) acc[q] = (side == 0) ? s.hand[q][row] : 0.0;
      __syncthreads();  // hand[] consumed before it is rewritten

      for (int bb = seg0; bb < seg1; bb += kCap) {
        const int be = min(bb + kCap, seg1);
        // ---- particle records -------------------------------------------
        for (int j = bb + tid; j < be; j += kP2GThreads) {
          const int i = perm[j];
          const int lj = j - bb;
          const int pr = p.key[i] - cbase;  // cell row
          const double x = p.x[i], y = p.y[i];
          double xi, eta;
          local_xy(x, y, cc, pr, hx, hy, xi, eta);
          const double Mp = p.Mp[i], Vp = p.Vp[i], H = p.H[i], hp = p.hp[i];
          const double vx = p.vpx[i], vy = p.vpy[i];
          // g2pd Z -> dZxp, dZyp (main/optim_par.cpp:387)
          double dzx = 0.0, dzy = 0.0;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double zn = Z[node_of(k, cc, pr, nrows)];
            dzx += shg_x(eta, k, ihx, mihx) * zn;
            dzy += shg_y(xi, k, ihy, mihy) * zn;
          }
          // gravity along the bed, well balanced (main/optim_par.cpp:447-454)
          const double wb = hp > 1e-10 ? 1.0 - (H / hp) : 1.0;
          const double Fpx = -P.g * Vp * P.rho * dzx * wb;
          const double Fpy = -P.g * Vp * P.rho * dzy * wb;
          double Ap, fbx, fby, mpx, mpy;
          if (fresh) {
            Ap = p.Ap[i];
            fbx = p.Fbx[i];
            fby = p.Fby[i];
            mpx = p.mpx[i];
            mpy = p.mpy[i];
          } else {
            // values the reference stored at the end of the previous step
            // (main/optim_par.cpp:600-626)
            Ap = hp > 1.e-2 ? Vp / hp : 0.0;
            voellmy(P, vx, vy, hp, fbx, fby);
            mpx = vx * Mp;
            mpy = vy * Mp;
          }
          s.xi[lj] = xi;
          s.eta[lj] = eta;
          s.Mp[lj] = Mp;
          s.mpx[lj] = mpx;
          s.mpy[lj] = mpy;
          s.Fpx[lj] = Fpx;
          s.Fpy[lj] = Fpy;
          s.Frx[lj] = Ap * fbx;
          s.Fry[lj] = Ap * fby;
          s.F11[lj] = p.F11[i];
          s.F12[lj] = p.F12[i];
          s.F22[lj] = p.F22[i];
          s.Vp[lj] = Vp;
          if (record) {
            p.dZxp[i] = dzx;
            p.dZyp[i] = dzy;
            p.Fpx[i] = Fpx;
            p.Fpy[i] = Fpy;
            p.Frx[i] = Ap * fbx;
            p.Fry[i] = Ap * fby;
          }
          // particle ledger, once per particle (owning CTA only)
          if (pr >= r0 && pr < r0 + kTR && cc >= cA) {
            lp0 += Mp;
            lp1 += mpx;
            lp2 += mpy;
          }
        }
        __syncthreads();
        // ---- node chains --------------------------------------------------
        if (fin_active || start_active) {
          const int kA = fin_active ? 1 : 3;  // local node as seen from cell r-1
          const int kB = fin_active ? 0 : 2;  // ... from cell r
          for (int j = max(a0, bb); j < min(a1, be); ++j)
            add_contrib(acc, s, j - bb, kA, ihx, mihx, ihy, mihy);
          for (int j = max(b0, bb); j < min(b1, be); ++j)
            add_contrib(acc, s, j - bb, kB, ihx, mihx, ihy, mihy);
        }
        __syncthreads();
      }

      // ---- finished node (r, cc) [side 0] or (r, ncols) [side 1, last] ----
      const bool last_col = (side == 1) && (cc == ncols - 1) && (cB == ncols + 1) &&
                            (r <= nrows);
      if (fin_active || last_col) {
        const int nc = fin_active ? cc : ncols;
        const int n = r + nc * (nrows + 1);
        const double Mv = acc[0];
        double momx = acc[1], momy = acc[2];
        const double Fextx = acc[3] + acc[5];
        const double Fexty = acc[4] + acc[6];
        const double Ftx = Fextx - acc[7];
        const double Fty = Fexty - acc[8];
        ln0 += Mv;
        ln1 += momx;
        ln2 += momy;
        momx = dt * Ftx + momx;
        momy = dt * Fty + momy;
        const bool act = Mv > 1.e-2;
        double avx = act ? Ftx / Mv : 0.0;
        double avy = act ? Fty / Mv : 0.0;
        double vvx = act ? momx / Mv : 0.0;
        double vvy = act ? momy / Mv : 0.0;
        double vvxL = dt * avx + vvx;
        double vvyL = dt * avy + vvy;
        if (P.BC) {
          if (nc == 0 || nc == 1 || nc == ncols - 1 || nc == ncols) {
            avx = 0.0; vvx = 0.0; vvxL = 0.0; momx = 0.0;
          }
          if (r == 0 || r == 1 || r == nrows - 1 || r == nrows) {
            avy = 0.0; vvy = 0.0; vvyL = 0.0; momy = 0.0;
          }
        }
        nodes.vvxL[n] = vvxL;
        nodes.vvyL[n] = vvyL;
        if (record) {
          nodes.Mv[n] = Mv;
          nodes.mvx[n] = momx;
          nodes.mvy[n] = momy;
          nodes.avx[n] = avx;
          nodes.avy[n] = avy;
          nodes.vvx[n] = vvx;
          nodes.vvy[n] = vvy;
          nodes.FPxv[n] = acc[3];
          nodes.FPyv[n] = acc[4];
          nodes.Fricx[n] = acc[5];
          nodes.Fricy[n] = acc[6];
          nodes.Fintx[n] = acc[7];
          nodes.Finty[n] = acc[8];
        }
      }
      if (start_active) {
#pragma unroll
        for (int q = 0; q < kNQ; ++q) s.hand[q][row] = acc[q];
      }
      __syncthreads();
    }
  }
  // ---- ledger partials: fixed-order block reduction ----------------------
  {
    double v[6] = {lp0, lp1, lp2, ln0, ln1, ln2};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double x = v[q];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((tid & 31) == 0) s.led[q][tid >> 5] = x;
    }
    __syncthreads();
    if (tid < 6) {
      double x = 0.0;
      for (int w = 0; w < kP2GThreads / 32; ++w) x += s.led[tid][w];
      led_part[(size_t)(blockIdx.y * gridDim.x + blockIdx.x) * 6 + tid] = x;
    }
  }
}

__global__ void k_ledger_final(const double* __restrict__ led_part, int nparts,
                               Scalars* S) {
  if (!S->active) return;
  __shared__ double sm[6][32];
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] += led_part[(size_t)b * 6 + q];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[6];
    for (int q = 0; q < 6; ++q) {
      t[q] = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t[q] += sm[q][w];
      S->ledger[q] = t[q];
    }
    // main/optim_par.cpp:416-425
    const double err_mass = fabs(t[0] - t[3]) / t[0];
    const double a = fabs(t[1]), b = fabs(t[2]);
    const double m = (a < b) ? b : a;
    const double norm_mom = (1.0 < m) ? m : 1.0;
    const double ex = fabs(t[1] - t[4]) / norm_mom;
    const double ey = fabs(t[2] - t[5]) / norm_mom;
    S->ledger[6] = err_mass;
    S->ledger[7] = (ex < ey) ? ey : ex;
    S->ledger[8] = S->t;
  }
}

// ---------------------------------------------------------------------------
// G2P: velocity, advection, velocity gradients at the new position with the
// cell of the step start, height update, Bingham stress, next cell key and
// the CFL max-reductions (main/optim_par.cpp:532-651).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kG2PThreads)
    k_g2p(Particles p, Nodes nodes, const double* __restrict__ Z, Geom G,
          Phys P, Scalars* S, int record, int want_grad) {
  if (!S->active) return;
  __shared__ unsigned long long red[3];
  if (threadIdx.x < 3) red[threadIdx.x] = 0ull;
  __syncthreads();
  const int np = S->np;
  const double dt = S->dt;
  const int nrows = G.nrows, ncols = G.ncols;
  const double hx = G.hx, hy = G.hy;
  const double ihx = 1.0 / hx, mihx = -1.0 / hx;
  const double ihy = 1.0 / hy, mihy = -1.0 / hy;
  const double eps = 1e-10;
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int key = p.key[i];
    const int r = key % nrows, c = key / nrows;
    int nd[4];
    double vxn[4], vyn[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      nd[k] = node_of(k, c, r, nrows);
      vxn[k] = nodes.vvxL[nd[k]];
      vyn[k] = nodes.vvyL[nd[k]];
    }
    double x = p.x[i], y = p.y[i];
    double xi, eta;
    local_xy(x, y, c, r, hx, hy, xi, eta);
    double vxL = 0.0, vyL = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double N = shp(xi, eta, k);
      vxL += N * vxn[k];
      vyL += N * vyn[k];
    }
    if (record) {
      double ax = 0.0, ay = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double N = shp(xi, eta, k);
        ax += N * nodes.avx[nd[k]];
        ay += N * nodes.avy[nd[k]];
      }
      p.apx[i] = ax;
      p.apy[i] = ay;
    }
    const double vpx = vxL, vpy = vyL;
    x = x + dt * vpx;
    y = y + dt * vpy;
    if (x < eps) x = eps;
    if (x > G.Lx - eps) x = G.Lx - eps;
    if (y < eps) y = eps;
    if (y > G.Ly - eps) y = G.Ly - eps;
    // g2pd {vvxL, vvyL} at the new position, old cell (main/optim_par.cpp:578)
    local_xy(x, y, c, r, hx, hy, xi, eta);
    double vxdx = 0.0, vydx = 0.0, vxdy = 0.0, vydy = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double Nx = shg_x(eta, k, ihx, mihx);
      const double Ny = shg_y(xi, k, ihy, mihy);
      vxdx += Nx * vxn[k];
      vxdy += Ny * vxn[k];
      vydx += Nx * vyn[k];
      vydy += Ny * vyn[k];
    }
    // height from the strain rate (main/optim_par.cpp:595-599)
    const double div = vxdx + vydy;
    double hp = p.hp[i];
    hp = hp / (1 + dt * div);
    hp = hp < 1e-2 ? 1e-2 : hp;
    double F11, F12, F22;
    bingham_stress(P, vpx, vpy, hp, p.H[i], vxdx, vydy, vxdy, vydx, F11, F12,
                   F22);
    p.x[i] = x;
    p.y[i] = y;
    p.vpx[i] = vpx;
    p.vpy[i] = vpy;
    p.hp[i] = hp;
    p.F11[i] = F11;
    p.F12[i] = F12;
    p.F22[i] = F22;
    const int nr = cell_row(y, hy, nrows), ncl = cell_col(x, hx, ncols);
    p.key[i] = nr + ncl * nrows;
    if (want_grad) {
      p.vpx_dx[i] = vxdx;
      p.vpx_dy[i] = vxdy;
      p.vpy_dx[i] = vydx;
      p.vpy_dy[i] = vydy;
    }
    if (record) {
      // g2p Z -> Zp at the new position, old cell (main/optim_par.cpp:642)
      double zp = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) zp += shp(xi, eta, k) * Z[nd[k]];
      p.Zp[i] = zp;
      p.hpZ[i] = hp + zp;
      p.mpx[i] = vpx * p.Mp[i];
      p.mpy[i] = vpy * p.Mp[i];
      const double Vp = p.Vp[i];
      p.Ap[i] = hp > 1.e-2 ? Vp / hp : 0.0;
      double fbx, fby;
      voellmy(P, vpx, vpy, hp, fbx, fby);
      p.Fbx[i] = fbx;
      p.Fby[i] = fby;
      // HV: p2g hp with the same (stale) cell, atomics are fine here since
      // the field is output-only (main/optim_par.cpp:650)
    }
    m0 = max(m0, ordered_key(fabs(vpx)));
    m1 = max(m1, ordered_key(fabs(vpy)));
    m2 = max(m2, ordered_key(hp));
  }
  for (int o = 16; o > 0; o >>= 1) {
    m0 = max(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&red[0], m0);
    atomicMax(&red[1], m1);
    atomicMax(&red[2], m2);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&S->red_next[0], red[0]);
    atomicMax(&S->red_next[1], red[1]);
    atomicMax(&S->red_next[2], red[2]);
  }
}

size_t p2g_smem_bytes() { return sizeof(P2GSmem); }

}  // namespace dampm
