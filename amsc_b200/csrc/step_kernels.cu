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
// One scenario's pass start: the loop condition, dt, it++ (device side).
__device__ __forceinline__ void step_begin_one(Scalars* S, const Geom& G,
                                               const Phys& P) {
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

__device__ __forceinline__ void step_end_one(Scalars* S) {
  // slab mode: the neighbour's column copies were read by P2G only; G2P
  // wrote the slab's own particles
  S->np -= S->nghost;
  S->nghost = 0;
  if (!S->active) return;
  S->t += S->dt;
  S->fresh = 0;
  S->red_cur[0] = S->red_next[0];
  S->red_cur[1] = S->red_next[1];
  S->red_cur[2] = S->red_next[2];
}

__global__ void k_step_begin(Scalars* S, Geom G, Phys P) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  step_begin_one(S, G, P);
}

__global__ void k_step_end(Scalars* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  step_end_one(S);
}

// ---------------------------------------------------------------------------
// initialisation after upload: main/optim_par.cpp:239-264
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_init_particles(ParticlesT<R> p, const double* __restrict__ Z,
                                 const double* __restrict__ dZdx,
                                 const double* __restrict__ dZdy, Geom G,
                                 Phys P, Scalars* S, int np, int key_off) {
  __shared__ unsigned long long red[3];
  if (threadIdx.x < 3) red[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const double x = p.x[i], y = p.y[i];
    const int r = cell_row(y, G), c = cell_col(x, G);
    p.key[i] = r + c * G.nrows + key_off;
    p.idx[i] = i;
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

// Recomputes the cell key of every particle after a merge/split emit (which
// wrote idx) or a state upload (slots in reference order: set_idx sets
// idx = slot); the next sort scans every cell.
__global__ void k_keys(Particles p, Geom G, Scalars* S, int set_idx) {
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int r = cell_row(p.y[i], G);
    const int c = cell_col(p.x[i], G);
    p.key[i] = r + c * G.nrows;
    if (set_idx) p.idx[i] = i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->knext[0] = 0;
    S->knext[1] = G.nrows * G.ncols - 1;
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

// Record of the next P2G for every particle (see Particles): from the stored
// Ap/Fb/mom (derive == 0: after an upload or a merge/split) or from the state
// alone (derive != 0), exactly as the reference computes these values
// (main/optim_par.cpp:387,447-459,600-626).
// The terrain gradient and the well-balanced factor 1 - H/hp are evaluated
// in FP64 whatever R is (the bed slope and the near-cancelling free-surface
// difference).
template <class R>
__device__ __forceinline__ void next_record(const Geom& G, const Phys& P,
                                            const double* __restrict__ Z, R x,
                                            R y, R hp, R H, R Vp, R& xi, R& eta,
                                            R& gx, R& gy) {
  const int r = cell_row(double(y), G);
  const int c = cell_col(double(x), G);
  const R ihx = R(1) / R(G.hx), ihy = R(1) / R(G.hy);
  local_xy_g(x, y, c, r, G, ihx, ihy, xi, eta);
  // g2pd Z -> dZxp, dZyp (main/optim_par.cpp:387)
  const double dihx = 1.0 / G.hx, dmihx = -1.0 / G.hx;
  const double dihy = 1.0 / G.hy, dmihy = -1.0 / G.hy;
  const double dxi = xi, deta = eta;
  double dzx = 0.0, dzy = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double zn = Z[node_of(k, c, r, G.nrows)];
    dzx += shg_x(deta, k, dihx, dmihx) * zn;
    dzy += shg_y(dxi, k, dihy, dmihy) * zn;
  }
  // gravity along the bed, well balanced (main/optim_par.cpp:447-454)
  const double hpd = hp, Hd = H, Vpd = Vp;
  // H/hp is +0 when H == 0 (no still-water level): 1 - 0 is 1
  const double wb = (hpd > 1e-10 && Hd != 0.0) ? 1.0 - (Hd / hpd) : 1.0;
  gx = R(-P.g * Vpd * P.rho * dzx * wb);
  gy = R(-P.g * Vpd * P.rho * dzy * wb);
}

template <class R>
__global__ void k_prep(ParticlesT<R> p, const double* __restrict__ Z, Geom G,
                       Phys P, const Scalars* S, int derive) {
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const R hp = p.hp[i];
    R Ap, fbx, fby;
    if (derive) {
      Ap = hp > R(1.e-2) ? p.Vp[i] / hp : R(0);
      rheology_friction<R>(P, p.vpx[i], p.vpy[i], hp, fbx, fby);
      p.mp[i] = V2<R>{p.vpx[i] * p.Mp[i], p.vpy[i] * p.Mp[i]};
    } else {  // the stored values, in reference order
      const int r = p.idx[i];
      Ap = p.Ap[r];
      fbx = p.Fbx[r];
      fby = p.Fby[r];
    }
    p.qf[i] = V2<R>{Ap * fbx, Ap * fby};
    R xi, eta, gx, gy;
    next_record<R>(G, P, Z, p.x[i], p.y[i], hp, p.H[i], p.Vp[i], xi, eta, gx, gy);
    p.xe[i] = V2<R>{xi, eta};
    p.qg[i] = V2<R>{gx, gy};
  }
}

// ---------------------------------------------------------------------------
// SORT: stable counting sort by cell, (cell, particle index) order
// (init_particle_mesh + cell_start/cell_ptcls, main/gpu_offload.cpp:243-249)
// ---------------------------------------------------------------------------
// Particle i takes slot[i] among its cell's particles: one atomic per cell
// and warp (the lanes of a warp that share a cell take consecutive slots in
// index order).
__global__ void k_count(const int* __restrict__ key, int* __restrict__ count,
                        int* __restrict__ slot, const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); i0 < np; i0 += stride) {
    const int i = i0 + lane;
    const bool ok = i < np;
    const int k = ok ? key[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (ok && lane == leader) base = atomicAdd(&count[k], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (ok) slot[i] = base + __popc(peers & ((1u << lane) - 1u));
  }
}

// Exclusive scan of count[0..n) into start[0..n], restricted to the tiles of
// kScanTile = 4 x kScanThreads cells (each thread one int4) that meet the key
// range [L, H] = krange U knext: the keys the starts describe and the keys
// G2P produced since.  Outside that range no cell's count changed and every
// start is either 0 (below every key) or np (above), as before, so the old
// values stand.  k_scan_sums writes the tile totals; k_scan_apply adds, per
// tile, the totals of the preceding tiles in the range to a block scan.
// count is zeroed on the way (ready for the next step's atomics).  With
// tile flags (batches) only the flagged tiles are scanned: the others hold
// no particle of any scenario, now or at the last sort, so their totals are
// zero and their starts stand.  When
// `list` is given, cells holding two or more particles are appended to it
// (the cells whose order k_segment_order has to establish).
__device__ __forceinline__ int block_incl_scan(int v, int* wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    int ws = (lane < nw) ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += t;
    }
    if (lane < nw) wsum[lane] = ws;  // inclusive warp totals
  }
  __syncthreads();
  return incl + (w > 0 ? wsum[w - 1] : 0);
}

__device__ __forceinline__ int block_sum(int v, int* wsum) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wsum[w];
  __syncthreads();
  return t;
}

__device__ __forceinline__ int4 load_count4(const int* count, int i0, int n) {
  if (i0 + 3 < n && (i0 & 3) == 0) return *reinterpret_cast<const int4*>(count + i0);
  int4 c;
  c.x = (i0 < n) ? count[i0] : 0;
  c.y = (i0 + 1 < n) ? count[i0 + 1] : 0;
  c.z = (i0 + 2 < n) ? count[i0 + 2] : 0;
  c.w = (i0 + 3 < n) ? count[i0 + 3] : 0;
  return c;
}

// tiles [t0, t1] meet the scan range (t0 > t1: none); ranged == 0: all
__device__ __forceinline__ void scan_tiles_of(const Scalars* S, int n, int ranged, int& t0,
                                              int& t1) {
  if (!ranged) {
    t0 = 0;
    t1 = (n - 1) / kScanTile;
    return;
  }
  int L = min(S->krange[0], S->knext[0]);
  int H = max(S->krange[1], S->knext[1]);
  L = max(L, 0);
  H = min(H, n - 1);
  if (H < L) {
    t0 = 1;
    t1 = 0;
    return;
  }
  t0 = L / kScanTile;
  t1 = H / kScanTile;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_sums(const int* __restrict__ count, int n, int* __restrict__ tile_sum,
                int* __restrict__ list_n, const Scalars* S, int ranged,
                const unsigned char* __restrict__ tflag) {
  if (!S->active) return;
  if (list_n && blockIdx.x == 0 && threadIdx.x < 3) list_n[threadIdx.x] = 0;
  int t0, t1;
  scan_tiles_of(S, n, ranged, t0, t1);
  const int t = blockIdx.x;
  if (t < t0 || t > t1) return;  // block-uniform
  if (tflag && !tflag[t]) {  // a tile no scenario's keys meet: no particles
    if (threadIdx.x == 0) tile_sum[t] = 0;
    return;
  }
  __shared__ int wsum[32];
  const int4 c = load_count4(count, t * kScanTile + threadIdx.x * 4, n);
  const int tot = block_sum(c.x + c.y + c.z + c.w, wsum);
  if (threadIdx.x == 0) tile_sum[t] = tot;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_apply(int* __restrict__ count, int n, const int* __restrict__ tile_sum,
                 int* __restrict__ start, int* __restrict__ list,
                 int* __restrict__ list_n, const Scalars* S, int ranged,
                 const unsigned char* __restrict__ tflag) {
  if (!S->active) return;
  int t0, t1;
  scan_tiles_of(S, n, ranged, t0, t1);
  const int t = blockIdx.x;
  if (t < t0 || t > t1) return;  // block-uniform
  if (tflag && !tflag[t]) return;  // its starts stand (see k_b_tile_flags)
  __shared__ int wsum[32];
  // particles in the range's tiles before this one
  int pre = 0;
  for (int q = t0 + threadIdx.x; q < t; q += blockDim.x) pre += tile_sum[q];
  pre = block_sum(pre, wsum);
  const int i0 = t * kScanTile + threadIdx.x * 4;
  const int4 c = load_count4(count, i0, n);
  const int v = c.x + c.y + c.z + c.w;
  const int incl = block_incl_scan(v, wsum);
  const int e0 = pre + incl - v;
  int4 o;
  o.x = e0;
  o.y = e0 + c.x;
  o.z = o.y + c.y;
  o.w = o.z + c.z;
  if (i0 + 3 < n && (i0 & 3) == 0) {
    *reinterpret_cast<int4*>(start + i0) = o;
    *reinterpret_cast<int4*>(count + i0) = make_int4(0, 0, 0, 0);
  } else {
    const int ov[4] = {o.x, o.y, o.z, o.w};
    for (int k = 0; k < 4; ++k)
      if (i0 + k < n) {
        start[i0 + k] = ov[k];
        count[i0 + k] = 0;
      }
  }
  if (list) {
    // one atomic per warp: the warp's listed cells go to consecutive slots
    const int cv[4] = {c.x, c.y, c.z, c.w};
    int mine = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) mine += cv[k] >= 2 ? 1 : 0;
    const int lane = threadIdx.x & 31;
    int incl2 = mine;
#pragma unroll
    for (int o2 = 1; o2 < 32; o2 <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl2, o2);
      if (lane >= o2) incl2 += u;
    }
    const int wtot = __shfl_sync(0xffffffffu, incl2, 31);
    int base = 0;
    if (lane == 31 && wtot > 0) base = atomicAdd(list_n, wtot);
    base = __shfl_sync(0xffffffffu, base, 31);
    int q = base + incl2 - mine;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (cv[k] >= 2) list[q++] = i0 + k;
  }
  // start[n]: the total (with a key range: every particle, unchanged by a
  // step; written whenever the range reaches the last tile)
  if (t == (n - 1) / kScanTile && threadIdx.x == blockDim.x - 1) start[n] = pre + incl;
}

// perm[start[key] + slot] = the storage slot, skey there the key (the
// cell of each sorted position, which G2P reads without waiting for perm)
// and pk the entry idx << 32 | slot that the per-cell ordering sorts; block
// 0 then rolls the key ranges over: the starts now describe knext, and the
// next G2P starts an empty knext.
__global__ void k_scatter(const int* __restrict__ key,
                          const int* __restrict__ slot, const int* __restrict__ idx,
                          const int* __restrict__ start, int* __restrict__ perm,
                          int* __restrict__ skey, unsigned long long* __restrict__ pk,
                          Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int k = key[i];
    const int pos = start[k] + slot[i];
    perm[pos] = i;
    skey[pos] = k;
    pk[pos] = ((unsigned long long)(unsigned)idx[i] << 32) | (unsigned)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->krange[0] = S->knext[0];
    S->krange[1] = S->knext[1];
    S->knext[0] = 0x7fffffff;
    S->knext[1] = -1;
  }
}

// Orders each listed cell's segment of perm (storage slots) by the
// particles' reference index idx[slot] (the atomics of the count hand out
// slots in arbitrary order).  A segment entry is the 64-bit value
// idx << 32 | slot that the scatter wrote to pk at the same position, so
// sorting those values orders by reference index (unique) and carries the
// slot along; a cell whose entries are already in order is left as it is.  k_segment_order: each lane sorts a
// cell of up to kThreadSort particles in registers (a bitonic network over
// static indices) and hands larger cells on to `mid`.  k_segment_order_mid,
// one warp per cell: a register bitonic sort across the lanes for up to 32
// particles, a rank sort for up to 32 * kRankPer (each lane holds kRankPer
// values and counts, over all the cell's values broadcast lane by lane,
// those below each of its own; the values are unique, so the ranks are a
// permutation of [0, m)); larger cells go on to `big` for
// k_segment_order_big.
constexpr int kThreadSort = 16;
constexpr int kRankPer = 8;
constexpr int kBigRun = 8192;  // entries of a sorted run (two buffers: 128 KB of shared memory)
constexpr unsigned long long kNoEntry = ~0ull;

__device__ __forceinline__ void thread_sort_segment(int* __restrict__ seg, int m,
                                                    const unsigned long long* __restrict__ pk) {
  unsigned long long v[kThreadSort];
#pragma unroll
  for (int k = 0; k < kThreadSort; ++k) v[k] = k < m ? pk[k] : kNoEntry;
  bool in_order = true;
#pragma unroll
  for (int k = 1; k < kThreadSort; ++k) in_order &= (k >= m) || v[k - 1] < v[k];
  if (in_order) return;  // perm already holds this order
#pragma unroll
  for (int k = 2; k <= kThreadSort; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < kThreadSort; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned long long a = v[i], b = v[l];
          const bool up = (i & k) == 0;
          const bool sw = up ? (a > b) : (a < b);
          v[i] = sw ? b : a;
          v[l] = sw ? a : b;
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kThreadSort; ++k)
    if (k < m) seg[k] = int(unsigned(v[k]));
}

// the 32 values of a warp (one per lane) in ascending order across the lanes
__device__ __forceinline__ unsigned long long warp_bitonic32(unsigned long long v, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, j);
      const bool up = ((lane & k) == 0);
      const bool lower = ((lane & j) == 0);
      // keep the min in the lower lane of an ascending pair
      v = (lower == up) ? min(v, o) : max(v, o);
    }
  }
  return v;
}

// One level of a merge sort along the merge path: src holds sorted runs of w
// entries over [0, len) (the last one shorter), dst receives runs of 2w.
// Each thread writes a contiguous piece of the output: it finds where the
// piece starts in the two runs by a binary search, then merges sequentially
// (again after a search where the piece enters the next pair of runs).
__device__ __forceinline__ void merge_level(const unsigned long long* src,
                                            unsigned long long* dst, int len, int w) {
  const int per = (len + int(blockDim.x) - 1) / int(blockDim.x);
  int k = min(int(threadIdx.x) * per, len);
  const int k1 = min(k + per, len);
  while (k < k1) {
    const int lo = (k / (2 * w)) * (2 * w);
    const int la = min(w, len - lo), lb = max(0, min(w, len - lo - la));
    const unsigned long long* A = src + lo;
    const unsigned long long* B = A + la;
    const int kk = k - lo;
    int i0 = max(0, kk - lb), i1 = min(kk, la);  // output kk takes i of A, kk - i of B
    while (i0 < i1) {
      const int mid = (i0 + i1) >> 1;
      if (A[mid] < B[kk - mid - 1]) i0 = mid + 1; else i1 = mid;
    }
    int i = i0, j = kk - i0;
    const int kend = min(k1, lo + la + lb);
    for (; k < kend; ++k) {
      // i + j < la + lb, so j >= lb leaves i < la
      const bool take_a = j >= lb || (i < la && A[i] < B[j]);
      dst[k] = take_a ? A[i++] : B[j++];
    }
  }
}

__device__ __forceinline__ void warp_sort_segment(int* __restrict__ perm, int b, int m,
                                                  int c, int lane,
                                                  const unsigned long long* __restrict__ pk,
                                                  int* __restrict__ big,
                                                  int* __restrict__ list_n) {
  if (m <= 32) {
    const unsigned long long v = warp_bitonic32((lane < m) ? pk[b + lane] : kNoEntry, lane);
    if (lane < m) perm[b + lane] = int(unsigned(v));
  } else if (m <= 32 * kRankPer) {
    unsigned long long v[kRankPer];
    int rank[kRankPer];
#pragma unroll
    for (int t = 0; t < kRankPer; ++t) {
      const int q = lane + 32 * t;
      v[t] = (q < m) ? pk[b + q] : kNoEntry;
      rank[t] = 0;
    }
#pragma unroll
    for (int t2 = 0; t2 < kRankPer; ++t2) {
      if (32 * t2 >= m) break;  // warp-uniform
      for (int src = 0; src < 32; ++src) {
        const unsigned long long o = __shfl_sync(0xffffffffu, v[t2], src);
#pragma unroll
        for (int t = 0; t < kRankPer; ++t) rank[t] += (o < v[t]) ? 1 : 0;
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kRankPer; ++t)
      if (lane + 32 * t < m) perm[b + rank[t]] = int(unsigned(v[t]));
  } else if (lane == 0) {
    big[atomicAdd(&list_n[1], 1)] = c;
  }
}

// (four resident blocks per SM: registers for a lane's whole cell)
__global__ void __launch_bounds__(256, 4) k_segment_order(const int* __restrict__ start,
                                const int* __restrict__ list,
                                int* __restrict__ list_n,
                                int* __restrict__ perm,
                                const unsigned long long* __restrict__ pk,
                                int* __restrict__ mid, const Scalars* S) {
  if (!S->active) return;
  const int lane = threadIdx.x & 31;
  const int nl = list_n[0];
  for (int w0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; w0 < nl;
       w0 += ((gridDim.x * blockDim.x) >> 5) * 32) {
    const int q = w0 + lane;
    int c = 0, b = 0, m = 0;
    if (q < nl) {
      c = list[q];
      b = start[c];
      m = start[c + 1] - b;
    }
    if (m <= kThreadSort) {
      if (m >= 2) thread_sort_segment(perm + b, m, pk + b);
    }
    // larger cells: one atomic per warp
    const unsigned larger = __ballot_sync(0xffffffffu, m > kThreadSort);
    if (larger) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&list_n[2], __popc(larger));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (m > kThreadSort) mid[base + __popc(larger & ((1u << lane) - 1u))] = c;
    }
  }
}

__global__ void __launch_bounds__(256, 4) k_segment_order_mid(const int* __restrict__ start,
                                    const int* __restrict__ mid,
                                    int* __restrict__ list_n,
                                    int* __restrict__ perm,
                                    const unsigned long long* __restrict__ pk,
                                    int* __restrict__ big, const Scalars* S) {
  if (!S->active) return;
  const int lane = threadIdx.x & 31;
  const int nm = list_n[2];
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nm;
       w += (gridDim.x * blockDim.x) >> 5) {
    const int c = mid[w];
    const int b = start[c];
    warp_sort_segment(perm, b, start[c + 1] - b, c, lane, pk, big, list_n);
  }
}

// Crowded cells (more than 32 * kRankPer particles), one block of 1024
// threads each: runs of up to kBigRun entries of tmp[b, b+m) (the pk the
// scatter wrote) are sorted in shared memory -- groups of 32 by a bitonic
// network in each warp's registers, then merged level by level along the
// merge path between two buffers -- and written back; longer cells then
// merge the sorted runs pairwise, ping-ponging between tmp[b, b+m) and
// tmp[cap + b, cap + b + m): each thread finds where its piece of the output
// starts by a binary search along the merge path, then merges the piece
// sequentially.  The slots go back to perm.
__global__ void __launch_bounds__(1024)
    k_segment_order_big(const int* __restrict__ start, const int* __restrict__ big,
                        const int* __restrict__ list_n, int* __restrict__ perm,
                        unsigned long long* __restrict__ tmp, long long cap,
                        const Scalars* S) {
  if (!S->active) return;
  extern __shared__ unsigned long long sv[];  // two buffers of kBigRun entries
  const int nb = list_n[1];
  for (int q = blockIdx.x; q < nb; q += gridDim.x) {
    const int c = big[q];
    const int b = start[c], m = start[c + 1] - b;
    for (int r0 = 0; r0 < m; r0 += kBigRun) {
      const int len = min(kBigRun, m - r0);
      unsigned long long* A = sv;
      unsigned long long* B = sv + kBigRun;
      // groups of 32 sorted in registers, one warp each, then merged level
      // by level between the two buffers
      const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
      for (int g = threadIdx.x >> 5; g * 32 < len; g += nw) {
        const int q = g * 32 + lane;
        const unsigned long long v = warp_bitonic32(q < len ? tmp[b + r0 + q] : kNoEntry, lane);
        if (q < len) A[q] = v;
      }
      __syncthreads();
      for (int w = 32; w < len; w <<= 1) {
        merge_level(A, B, len, w);
        __syncthreads();
        unsigned long long* t = A;
        A = B;
        B = t;
      }
      for (int i = threadIdx.x; i < len; i += blockDim.x) tmp[b + r0 + i] = A[i];
      __syncthreads();
    }
    unsigned long long* src = tmp + b;
    unsigned long long* dst = tmp + cap + b;
    for (int w = kBigRun; w < m; w <<= 1) {
      for (int lo = 0; lo < m; lo += 2 * w) {  // runs [lo, lo+w) and [lo+w, lo+2w)
        const int la = min(w, m - lo), lb = max(0, min(w, m - lo - la));
        const int tot = la + lb;
        const unsigned long long* A = src + lo;
        const unsigned long long* B = A + la;
        const int per = (tot + int(blockDim.x) - 1) / int(blockDim.x);
        const int k0 = min(int(threadIdx.x) * per, tot), k1 = min(k0 + per, tot);
        if (k0 >= k1) continue;
        // output k0 takes i of A and k0 - i of B
        int i0 = max(0, k0 - lb), i1 = min(k0, la);
        while (i0 < i1) {
          const int mid = (i0 + i1) >> 1;
          if (A[mid] < B[k0 - mid - 1]) i0 = mid + 1; else i1 = mid;
        }
        int i = i0, j = k0 - i0;
        for (int k = k0; k < k1; ++k) {
          // i + j == k < tot, so j >= lb leaves i < la
          const bool take_a = j >= lb || (i < la && A[i] < B[j]);
          dst[lo + k] = take_a ? A[i++] : B[j++];
        }
      }
      __syncthreads();
      unsigned long long* t = src;
      src = dst;
      dst = t;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) perm[b + i] = int(unsigned(src[i]));
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// P2G + NODAL
//
// Work unit: node rows [r0, r0+kTR) of one strip x node columns [cA, cB); the
// unit walks the cell columns cA-1 .. cB-1.  For cell column cc the particles
// of cells (rlo..rhi, cc) are one contiguous range of the sorted order,
// processed in batches of at most kCap particles.  Each particle's record
// (local coordinates and the nine transferred quantities, built by the
// previous step's G2P) is copied with cp.async into shared memory: the four
// record pairs (xi, eta), (mom_x, mom_y), gravity and friction force with
// one 16-byte copy each, Mp, F11, F12, F22 and Vp with one 8-byte copy each.
// The sorted indices of the next batch are loaded while the copies fly.
// Four CTAs share an SM, so one CTA's copies overlap the others' transfers.
//
// Node row r is served by lane r of four warps, one per quantity group
// (warp-uniform code) g0 {Mv, mom_x, mom_y}, g1 {FPx, FPy, Fric_x, Fric_y},
// g2 {Fint_x}, g3 {Fint_y}; each lane carries two chains per quantity:
//   fin   node (r, cc)   -- local node 1 of cell (r-1,cc), then 0 of (r,cc);
//         it already holds cells (r-1,cc-1), (r,cc-1);
//   start node (r, cc+1) -- local node 3 of cell (r-1,cc), then 2 of (r,cc).
// That is each node's contributions in quadgrid's cell-sweep order, so every
// nodal sum equals the reference's sequential sum bit for bit.  At the end of
// a column the finished sums go through shared memory to warp kNodalWarp,
// which applies the nodal update to node column cc, and each lane's started
// chains become its finishing ones.  Records are stored SoA with an XOR
// swizzle of the low index bits so that lanes of consecutive rows (records
// ~ppc apart) hit distinct banks.
// ---------------------------------------------------------------------------
namespace {

constexpr int kPf = (kCap + kP2GThreads - 1) / kP2GThreads;

// The staged records of one batch: the four record pairs and five single
// values of each particle (13 values of R).
template <class R>
struct P2GSmemT {
  V2<R> pr[4][kCap];  // xe, mp, qg, qf
  R sg[5][kCap];      // Mp, F11, F12, F22, Vp
  R xch[9][kTR];      // finished sums per quantity
  double led[6][kP2GThreads / 32];
  int rowstart[3][kTR + 2];
};
using P2GSmem = P2GSmemT<double>;

// Slot of batch position j: an XOR of the bank-selecting low bits by the
// next ones, so that lanes reading cells 16 records apart hit distinct banks
// (8 sixteen-byte, 16 eight-byte or 32 four-byte slots span the 32 banks).
template <class R>
__device__ __forceinline__ int swz_pair(int j) {
  return sizeof(R) == 8 ? (j ^ ((j >> 4) & 7)) : (j ^ ((j >> 4) & 15));
}
template <class R>
__device__ __forceinline__ int swz_one(int j) {
  return sizeof(R) == 8 ? (j ^ ((j >> 4) & 15)) : (j ^ ((j >> 5) & 31));
}

template <int kBytes>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (kBytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else if (kBytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

struct Batch {
  int cc, bb, be;
  bool valid;
};

// the batch after b: the rest of its column, else the start of the next one
template <class R>
__device__ __forceinline__ Batch next_batch(const Batch& b, const P2GSmemT<R>& s,
                                            int nrs, int ccLast) {
  Batch n{0, 0, 0, false};
  if (!b.valid) return n;
  const int seg1 = s.rowstart[b.cc % 3][nrs - 1];
  if (b.be < seg1) return Batch{b.cc, b.be, min(b.be + kCap, seg1), true};
  if (b.cc + 1 > ccLast) return n;
  const int s0 = s.rowstart[(b.cc + 1) % 3][0];
  const int s1 = s.rowstart[(b.cc + 1) % 3][nrs - 1];
  return Batch{b.cc + 1, s0, min(s0 + kCap, s1), true};
}

__device__ __forceinline__ void load_perm(int (&pf)[kPf],
                                          const int* __restrict__ perm,
                                          const Batch& b) {
#pragma unroll
  for (int u = 0; u < kPf; ++u) {
    const int j = b.bb + threadIdx.x + u * kP2GThreads;
    pf[u] = (b.valid && j < b.be) ? perm[j] : 0;
  }
}

template <class R>
__device__ __forceinline__ void issue_gather(P2GSmemT<R>& s, const ParticlesT<R>& p,
                                             const int (&pf)[kPf],
                                             const Batch& b) {
  constexpr int kB = sizeof(R), kB2 = sizeof(V2<R>);
#pragma unroll
  for (int u = 0; u < kPf; ++u) {
    const int j = b.bb + threadIdx.x + u * kP2GThreads;
    if (j >= b.be) break;
    const int i = pf[u];
    const int l2 = swz_pair<R>(j - b.bb), l1 = swz_one<R>(j - b.bb);
    cp_async<kB2>(&s.pr[0][l2], p.xe + i);
    cp_async<kB2>(&s.pr[1][l2], p.mp + i);
    cp_async<kB2>(&s.pr[2][l2], p.qg + i);
    cp_async<kB2>(&s.pr[3][l2], p.qf + i);
    cp_async<kB>(&s.sg[0][l1], p.Mp + i);
    cp_async<kB>(&s.sg[1][l1], p.F11 + i);
    cp_async<kB>(&s.sg[2][l1], p.F12 + i);
    cp_async<kB>(&s.sg[3][l1], p.F22 + i);
    cp_async<kB>(&s.sg[4][l1], p.Vp + i);
  }
  cp_async_commit();
}

// Nodal momentum, velocity and wall conditions of node (r, nc) from its nine
// P2G sums (main/optim_par.cpp:467-529); also accumulates the node ledger.
template <class R>
__device__ __forceinline__ void nodal_update(
    R Mv, R momx, R momy, R FPx, R FPy, R Frx, R Fry, R Fix, R Fiy, int r, int nc,
    const Geom& G, const Phys& P, double dtd, const NodesT<R>& nodes, int record,
    double& ln0, double& ln1, double& ln2) {
  if (nc < G.nc_lo || nc > G.nc_hi) return;  // a slab's neighbour writes this column
  const int nrows = G.nrows, ncols = G.ncols;
  const int n = r + nc * (nrows + 1);
  const R dt = R(dtd);
  const R Fextx = FPx + Frx;
  const R Fexty = FPy + Fry;
  const R Ftx = Fextx - Fix;
  const R Fty = Fexty - Fiy;
  ln0 += Mv;
  ln1 += momx;
  ln2 += momy;
  momx = dt * Ftx + momx;
  momy = dt * Fty + momy;
  const bool act = Mv > R(1.e-2);
  R avx = act ? Ftx / Mv : R(0);
  R avy = act ? Fty / Mv : R(0);
  R vvx = act ? momx / Mv : R(0);
  R vvy = act ? momy / Mv : R(0);
  R vvxL = dt * avx + vvx;
  R vvyL = dt * avy + vvy;
  if (P.BC) {  // cells on the walls zero their 4 nodes (main/optim_par.cpp:503-529)
    if (nc == 0 || nc == 1 || nc == ncols - 1 || nc == ncols) {
      avx = R(0); vvx = R(0); vvxL = R(0); momx = R(0);
    }
    if (r == 0 || r == 1 || r == nrows - 1 || r == nrows) {
      avy = R(0); vvy = R(0); vvyL = R(0); momy = R(0);
    }
  }
  nodes.vvL[n] = V2<R>{vvxL, vvyL};
  if (record) {
    nodes.Mv[n] = Mv;
    nodes.mvx[n] = momx;
    nodes.mvy[n] = momy;
    nodes.avx[n] = avx;
    nodes.avy[n] = avy;
    nodes.vvx[n] = vvx;
    nodes.vvy[n] = vvy;
    nodes.FPxv[n] = FPx;
    nodes.FPyv[n] = FPy;
    nodes.Fricx[n] = Frx;
    nodes.Fricy[n] = Fry;
    nodes.Fintx[n] = Fix;
    nodes.Finty[n] = Fiy;
  }
}

template <class R>
struct ShapeT {
  R ihx, mihx, ihy, mihy;
};
using Shape = ShapeT<double>;

// s += v.  The FP32 chains are compensated (Kahan): c carries the part of
// the running sum that the last rounding lost, so a chain of thousands of
// contributions keeps FP32 precision.  The FP64 chains are the reference's
// plain sums.
template <class R>
__device__ __forceinline__ void acc_add(R& s, R& c, R v) {
  if constexpr (sizeof(R) == 4) {
    const R y = v - c;
    const R t = s + y;
    c = (t - s) - y;
    s = t;
  } else {
    s += v;
  }
}

// a chain's value: the FP32 sum with its carried correction
template <class R>
__device__ __forceinline__ R acc_value(R s, R c) {
  if constexpr (sizeof(R) == 4) return s - c;
  return s;
}

// Running sums of one lane: finishing (f) and starting (s) chains, with
// their compensations (FP32 only).  Quantity groups (one warp each):
//   0: Mv, mom_x, mom_y         1: FPx, FPy, Fric_x, Fric_y
//   2: F_int_x                   3: F_int_y
// about the same FP64 work per particle in each; the lightest (3) also runs
// the nodal update.
constexpr int kMaxQ = 4;
constexpr int kNodalWarp = 3;
template <class R>
struct Chains {
  R f[kMaxQ], fc[kMaxQ], s[kMaxQ], sc[kMaxQ];
};

// One particle's contributions to the chains of quantity group kG: kUpper
// selects the cell (r-1: local nodes 1 (fin) and 3 (start); r: local nodes 0
// and 2).  With fb = eta or (1-eta):
//   fin   N = (1-xi)*fb, Nx = mihx*fb, Ny = (1-xi)*(ihy or mihy)
//   start N = xi*fb,     Nx = ihx*fb,  Ny = xi*(ihy or mihy)
// -- shp/shg of main/gpu_kernels.cpp:33-59 for those local nodes.  kFin off
// runs the started chains alone (a unit's leading column).  Group 0 also
// adds Mp and the momentum to the particle ledger (`led`, once per particle).
template <class R, int kG, bool kFin, bool kUpper>
__device__ __forceinline__ void chain_step(Chains<R>& a, const P2GSmemT<R>& s, int j,
                                           const ShapeT<R>& sh, bool led,
                                           double& lp0, double& lp1, double& lp2) {
  const int l2 = swz_pair<R>(j), l1 = swz_one<R>(j);
  const V2<R> xe = s.pr[0][l2];
  const R xi = xe.x, eta = xe.y;
  const R fa = R(1) - xi;
  const R fb = kUpper ? eta : (R(1) - eta);
  if constexpr (kG == 0 || kG == 1) {
    constexpr int nq = kG == 0 ? 3 : 4;
    const R Nf = fa * fb;
    const R Ns = xi * fb;
    R q[nq];
    if constexpr (kG == 0) {
      const V2<R> m = s.pr[1][l2];
      q[0] = s.sg[0][l1];
      q[1] = m.x;
      q[2] = m.y;
      if (led) {
        lp0 += q[0];
        lp1 += q[1];
        lp2 += q[2];
      }
    } else {
      const V2<R> g = s.pr[2][l2], f = s.pr[3][l2];
      q[0] = g.x;
      q[1] = g.y;
      q[2] = f.x;
      q[3] = f.y;
    }
    if (kFin) {
#pragma unroll
      for (int k = 0; k < nq; ++k) acc_add(a.f[k], a.fc[k], Nf * q[k]);
    }
#pragma unroll
    for (int k = 0; k < nq; ++k) acc_add(a.s[k], a.sc[k], Ns * q[k]);
  } else {
    const R hy = kUpper ? sh.ihy : sh.mihy;
    const R Nxs = sh.ihx * fb, Nys = xi * hy;
    const R f12 = s.sg[2][l1], vp = s.sg[4][l1];
    const R fo = kG == 2 ? s.sg[1][l1] : s.sg[3][l1];  // F11 or F22
    // F_int_x: (Nx*F11 + Ny*F12)*Vp;  F_int_y: (Nx*F12 + Ny*F22)*Vp
    if (kFin) {
      const R Nxf = sh.mihx * fb, Nyf = fa * hy;
      const R v = kG == 2 ? (Nxf * fo + Nyf * f12) : (Nxf * f12 + Nyf * fo);
      acc_add(a.f[0], a.fc[0], v * vp);
    }
    const R v = kG == 2 ? (Nxs * fo + Nys * f12) : (Nxs * f12 + Nys * fo);
    acc_add(a.s[0], a.sc[0], v * vp);
  }
}

// The particles of cells (r-1, cc) and (r, cc) are the adjacent ranges
// [a0, a1) and [a1, b1) of the sorted order, walked in order: the first
// with the upper cell's shape factors, the second with the lower cell's
// (whose particles the lane's own row counts into the particle ledger).
template <class R, int kG, bool kFin>
__device__ __forceinline__ void chain_range(Chains<R>& a, const P2GSmemT<R>& s, int a0,
                                            int a1, int b1, int bb, int be,
                                            const ShapeT<R>& sh, bool own,
                                            double& lp0, double& lp1, double& lp2) {
  const int u1 = min(a1, be);
  int j = max(a0, bb);
#pragma unroll kChainUnroll
  for (; j < u1; ++j) chain_step<R, kG, kFin, true>(a, s, j - bb, sh, false, lp0, lp1, lp2);
  const int j1 = min(b1, be);
  const bool led = kG == 0 && own;
  j = max(a1, bb);
#pragma unroll kChainUnroll
  for (; j < j1; ++j) chain_step<R, kG, kFin, false>(a, s, j - bb, sh, led, lp0, lp1, lp2);
}

template <class R, int kG>
__device__ __forceinline__ void chain_group(Chains<R>& a, const P2GSmemT<R>& s, bool lead,
                                            int a0, int a1, int b1, int bb, int be,
                                            const ShapeT<R>& sh, bool own, double& lp0,
                                            double& lp1, double& lp2) {
  if (lead)
    chain_range<R, kG, false>(a, s, a0, a1, b1, bb, be, sh, own, lp0, lp1, lp2);
  else
    chain_range<R, kG, true>(a, s, a0, a1, b1, bb, be, sh, own, lp0, lp1, lp2);
}

// ---- a batch inside one crowded cell ---------------------------------------
// When a whole batch lies in one cell (rc, cc), only two lanes of each warp
// have work in it: lane rc+1 (the cell is its cell r-1: local nodes 1 and 3)
// and lane rc (its cell r: local nodes 0 and 2), each walking the batch's
// records one after another for its 2 to 8 chains.  Those chains -- 9
// quantities at each of the 4 nodes, the fin chains only outside a lead
// column -- and the cell's 3 ledger sums go through shared memory to one
// thread each, which walks the records with the operations of chain_step in
// the same order (so every sum is the same, bit for bit), and come back.
// A thread's chains are one kind per warp (warp 0: N * value, warp 1: the
// internal forces, warp 2: the ledger), so a warp's threads run the same
// instructions on different operands.
constexpr int kSoloMin = 32;  // records of a batch worth handing over

// The row of the cell that holds all of [bb, be), or -1, from the lanes'
// ranges of their two cells ([a0, a1): cell r-1, [a1, b1): cell r): every
// warp holds the same ranges, so each finds the same row without a barrier.
__device__ __forceinline__ int solo_row(int a0, int a1, int b1, int bb, int be, int r0) {
  if (be - bb < kSoloMin) return -1;
  const unsigned lo = __ballot_sync(0xffffffffu, b1 > a1 && a1 <= bb && be <= b1);
  if (lo) return r0 + __ffs(lo) - 1;
  const unsigned up = __ballot_sync(0xffffffffu, a1 > a0 && a0 <= bb && be <= a1);
  if (up) return r0 + __ffs(up) - 2;
  return -1;
}

// All threads of the block call it.  rc: the cell's row; chain (role, fs, q)
// sits at X[2 id] with its compensation at X[2 id + 1], id = (2 role + fs) 9 + q,
// role 0 for lane rc+1 and 1 for lane rc, fs 0 for the fin chains, 1 for the
// started ones, q the quantity (0-2 group 0, 3-6 group 1, 7 and 8 groups 2, 3).
template <class R>
__device__ __forceinline__ void solo_batch(Chains<R>& a, P2GSmemT<R>& s, int rc, int r0,
                                           int nrows, int grp, int slot0, int nq, bool lead,
                                           bool own, int n, const ShapeT<R>& sh,
                                           double& lp0, double& lp1, double& lp2) {
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int lup = rc + 1 - r0, llo = rc - r0;
  const bool pup = lup >= 0 && lup < kTR && rc + 1 <= nrows;
  const bool plo = llo >= 0 && llo < kTR && rc <= nrows;
  R* X = &s.xch[0][0];
  const int mine = (pup && lane == lup) ? 0 : ((plo && lane == llo) ? 1 : -1);
  if (mine >= 0) {
#pragma unroll
    for (int k = 0; k < kMaxQ; ++k) {
      if (k < nq) {
        const int idf = (2 * mine) * 9 + slot0 + k, ids = idf + 9;
        X[2 * idf] = a.f[k];
        X[2 * idf + 1] = a.fc[k];
        X[2 * ids] = a.s[k];
        X[2 * ids + 1] = a.sc[k];
      }
    }
    if (grp == 0 && mine == 1) {
      s.led[0][0] = lp0;
      s.led[1][0] = lp1;
      s.led[2][0] = lp2;
    }
  }
  __syncthreads();
  if (w == 0 && lane < 28) {  // Mv, mom_x, mom_y, FPx, FPy, Fric_x, Fric_y
    const int q = lane % 7, rf = lane / 7;
    const int role = rf >> 1, fs = rf & 1;
    if ((role == 0 ? pup : plo) && (fs == 1 || !lead)) {
      const int id = rf * 9 + q;
      R v = X[2 * id], c = X[2 * id + 1];
      const bool single = q == 0;
      const R* pb = reinterpret_cast<const R*>(s.pr[single ? 1 : (q + 1) >> 1]);
      const int half = (q + 1) & 1;
      for (int j = 0; j < n; ++j) {
        const int l2 = swz_pair<R>(j), l1 = swz_one<R>(j);
        const V2<R> xe = s.pr[0][l2];
        const R xi = xe.x, eta = xe.y;
        const R fa = R(1) - xi;
        const R fb = role == 0 ? eta : (R(1) - eta);
        const R N = (fs == 0 ? fa : xi) * fb;
        const R val = single ? s.sg[0][l1] : pb[2 * l2 + half];
        acc_add(v, c, N * val);
      }
      X[2 * id] = v;
      X[2 * id + 1] = c;
    }
  } else if (w == 1 && lane < 8) {  // F_int_x, F_int_y
    const int qb = lane & 1, rf = lane >> 1;
    const int role = rf >> 1, fs = rf & 1;
    if ((role == 0 ? pup : plo) && (fs == 1 || !lead)) {
      const int id = rf * 9 + 7 + qb;
      R v = X[2 * id], c = X[2 * id + 1];
      const R hy = role == 0 ? sh.ihy : sh.mihy;
      const R hxs = fs == 0 ? sh.mihx : sh.ihx;
      const R* P1 = s.sg[qb == 0 ? 1 : 2];  // F11 or F12
      const R* P2 = s.sg[qb == 0 ? 2 : 3];  // F12 or F22
      for (int j = 0; j < n; ++j) {
        const int l2 = swz_pair<R>(j), l1 = swz_one<R>(j);
        const V2<R> xe = s.pr[0][l2];
        const R xi = xe.x, eta = xe.y;
        const R fa = R(1) - xi;
        const R fb = role == 0 ? eta : (R(1) - eta);
        const R Nx = hxs * fb;
        const R Ny = (fs == 0 ? fa : xi) * hy;
        const R vv = Nx * P1[l1] + Ny * P2[l1];
        acc_add(v, c, vv * s.sg[4][l1]);
      }
      X[2 * id] = v;
      X[2 * id + 1] = c;
    }
  } else if (w == 2 && lane < 3) {  // the particle ledger of lane rc (Mp, mom)
    if (plo && own) {
      double lp = s.led[lane][0];
      const R* pb = reinterpret_cast<const R*>(s.pr[1]);
      for (int j = 0; j < n; ++j) {
        const int l2 = swz_pair<R>(j), l1 = swz_one<R>(j);
        lp += lane == 0 ? s.sg[0][l1] : pb[2 * l2 + (lane - 1)];
      }
      s.led[lane][0] = lp;
    }
  }
  __syncthreads();
  if (mine >= 0) {
#pragma unroll
    for (int k = 0; k < kMaxQ; ++k) {
      if (k < nq) {
        const int idf = (2 * mine) * 9 + slot0 + k, ids = idf + 9;
        a.f[k] = X[2 * idf];
        a.fc[k] = X[2 * idf + 1];
        a.s[k] = X[2 * ids];
        a.sc[k] = X[2 * ids + 1];
      }
    }
    if (grp == 0 && mine == 1) {
      lp0 = s.led[0][0];
      lp1 = s.led[1][0];
      lp2 = s.led[2][0];
    }
  }
  __syncthreads();  // the exchange space is free again
}

}  // namespace

// ---- P2G work units -------------------------------------------------------
// A unit is node rows [r0, r0+kTR) of one strip x node columns [cA, cB); it
// walks cell columns cA-1 .. cB-1.  Units are cut per strip so that each
// carries about the same weight -- its particles plus kColWeight per column
// -- whatever the local particle density: P2G takes them from a shared
// cursor, so its time is the average load rather than the heaviest fixed
// block.  The list is in (strip, column) order and the ledger partial of
// list entry u sits in slot u, so the ledger reduction order is fixed.
namespace {

template <typename T>
__device__ __forceinline__ T block_incl_scan(T v, T* warp_tot, T& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) warp_tot[w] = v;
  __syncthreads();
  if (w == 0) {
    T t = lane < nw ? warp_tot[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += u;
    }
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  if (w > 0) v += warp_tot[w - 1];
  total = warp_tot[nw - 1];
  __syncthreads();  // warp_tot is free again
  return v;
}

__device__ __forceinline__ int column_count(const int* __restrict__ cstart,
                                            int rlo, int rhi, int cc, int nrows) {
  return cstart[rhi + cc * nrows + 1] - cstart[rlo + cc * nrows];
}

}  // namespace

// One block per strip.  Pass A: node column nc (< ncols) weighs the
// particles of cell column nc in the strip's cell rows plus kColWeight; nc
// starts a unit where floor(exclusive prefix / T) changes.  Pass B keeps the
// units with particles (including those of the leading column cA-1, which
// feed node column cA).
// Cuts strip `strip` of one grid (cstart of that grid's cells) into units
// of weight about T; st/px are the strip's scratch, plan its output.  All
// threads of the block call it; it returns the number of units kept.
__device__ __forceinline__ int plan_strip(const int* __restrict__ cstart,
                                          const Geom& G, long long T, int strip,
                                          int* __restrict__ st,
                                          long long* __restrict__ px,
                                          int4* __restrict__ plan, int col_weight,
                                          int c_lo, int c_hi, int* __restrict__ heavy_n) {
  __shared__ long long wt_ll[32];
  __shared__ int wt_i[32];
  __shared__ long long last_id;
  const int nrows = G.nrows, ncols = G.ncols;
  const int r0 = strip * kTR;
  const int rlo = max(r0 - 1, 0), rhi = min(r0 + kTR - 1, nrows - 1);
  long long carry = 0, prev_id = -1;
  int K = 0;
  for (int base = c_lo; base <= c_hi; base += blockDim.x) {
    const int nc = base + threadIdx.x;
    long long w = 0;
    if (nc <= c_hi && nc < ncols) w = column_count(cstart, rlo, rhi, nc, nrows) + col_weight;
    long long tot;
    const long long incl = block_incl_scan<long long>(w, wt_ll, tot);
    const long long pex = carry + incl - w;
    const long long id = pex / T;
    // id of the column before: the neighbour thread's, or the previous tile's
    long long idp = __shfl_up_sync(0xffffffffu, id, 1);
    if ((threadIdx.x & 31) == 31) wt_ll[threadIdx.x >> 5] = id;
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
      idp = threadIdx.x == 0 ? prev_id : wt_ll[(threadIdx.x >> 5) - 1];
    if (threadIdx.x == blockDim.x - 1) last_id = id;
    __syncthreads();
    const int flag = (nc == c_lo) || (nc <= c_hi && nc < ncols && id != idp);
    int ktot;
    const int kin = block_incl_scan<int>(flag, wt_i, ktot);
    if (flag) {
      st[K + kin - 1] = nc;
      px[K + kin - 1] = pex;
    }
    carry += tot;
    prev_id = last_id;
    K += ktot;
    __syncthreads();
  }
  const long long ptotal = carry;
  int J = 0;
  for (int base = 0; base < K; base += blockDim.x) {
    const int k = base + threadIdx.x;
    int flag = 0, cA = 0, cB = 0, heavy = 0;
    if (k < K) {
      cA = st[k];
      const bool more = k + 1 < K;
      cB = more ? st[k + 1] : c_hi + 1;
      const long long sumw = (more ? px[k + 1] : ptotal) - px[k];
      const long long n = sumw - (long long)col_weight * (min(cB, ncols) - cA) +
                          (cA > 0 ? column_count(cstart, rlo, rhi, cA - 1, nrows) : 0);
      flag = n > 0;
      // more than twice the target weight (a crowded column): heavy
      heavy = n > 2 * T ? 1 : 0;
    }
    int jtot;
    const int jin = block_incl_scan<int>(flag, wt_i, jtot);
    if (flag) plan[J + jin - 1] = make_int4(cA, cB, heavy, 0);  // P2G takes heavy units first
    if (flag && heavy) atomicAdd(heavy_n, 1);
    J += jtot;
  }
  return J;
}

__device__ __forceinline__ long long unit_weight(const Scalars* S,
                                                 int target_units) {
  long long T = (long long)S->np / max(target_units, 1);
  return T < kUnitMinWeight ? kUnitMinWeight : T;
}

__global__ void __launch_bounds__(kPlanThreads)
    k_units_plan(const int* __restrict__ cstart, Geom G, const Scalars* S,
                 int target_units, int seg, int* __restrict__ ustart,
                 long long* __restrict__ upex, int4* __restrict__ plan,
                 int* __restrict__ strip_n, int* __restrict__ heavy_n) {
  if (!S->active) return;
  const int strip = blockIdx.x;
  const size_t b = (size_t)strip * seg;
  // node columns of the cells the particles are binned to (the key range the
  // scatter just rolled over), plus the column right of them
  const int L = S->krange[0], H = S->krange[1];
  if (L > H) {  // no particle
    if (threadIdx.x == 0) strip_n[strip] = 0;
    return;
  }
  const int c_lo = L / G.nrows, c_hi = min(H / G.nrows + 1, G.ncols);
  const int J = plan_strip(cstart, G, unit_weight(S, target_units), strip,
                           ustart + b, upex + b, plan + b, kColWeight, c_lo, c_hi, heavy_n);
  if (threadIdx.x == 0) strip_n[strip] = J;
}

// The order P2G hands the units out in: the heavy ones first, then the
// others, each group in list order (a stable partition; heavy(f) is 0 or 1).
// A unit's ledger slot stays its list position, so the order changes no sum.
// All threads of the block call it.
template <class F>
__device__ __forceinline__ void heavy_first(int total, F heavy, int* __restrict__ uorder,
                                            int* wt) {
  int hc = 0;
  for (int f = threadIdx.x; f < total; f += blockDim.x) hc += heavy(f);
  int H;
  block_incl_scan<int>(hc, wt, H);
  int carry = 0;
  for (int base = 0; base < total; base += blockDim.x) {
    const int f = base + threadIdx.x;
    const int h = f < total ? heavy(f) : 0;
    int tot;
    const int incl = block_incl_scan<int>(h, wt, tot);
    if (f < total) uorder[h ? carry + incl - 1 : H + f - (carry + incl)] = f;
    carry += tot;
  }
}

// One block: strip offsets by a scan of strip_n, then the flat unit list
// {strip, cA, cB} in (strip, column) order.  ucount[0] = units,
// ucount[1] = P2G's work cursor, ucount[2] = heavy units (P2G reads uorder
// when there are any, else takes the list in order), ucount[3] = the heavy
// units the plan counts for the next list.
__global__ void __launch_bounds__(kPlanThreads)
    k_units_flat(const int* __restrict__ strip_n, int strips, int seg,
                 const int4* __restrict__ plan, int4* __restrict__ ulist,
                 int* __restrict__ uorder, int* __restrict__ ucount, const Scalars* S) {
  if (!S->active) return;
  const int H = ucount[3];  // heavy units, counted by the plan
  extern __shared__ int uoff[];  // strips + 1
  __shared__ int wt_i[32];
  int carry = 0;
  for (int base = 0; base < strips; base += blockDim.x) {
    const int s = base + threadIdx.x;
    const int n = s < strips ? strip_n[s] : 0;
    int tot;
    const int incl = block_incl_scan<int>(n, wt_i, tot);
    if (s < strips) uoff[s] = carry + incl - n;
    carry += tot;
  }
  if (threadIdx.x == 0) uoff[strips] = carry;
  __syncthreads();
  const int total = carry;
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    int lo = 0, hi = strips;  // uoff[lo] <= f < uoff[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (uoff[mid] <= f) lo = mid; else hi = mid;
    }
    const int4 u = plan[(size_t)lo * seg + (f - uoff[lo])];
    ulist[f] = make_int4(lo, u.x, u.y, u.z);  // w: heavy
  }
  if (H > 0) {
    __syncthreads();
    heavy_first(total, [&](int f) { return ulist[f].w; }, uorder, wt_i);
  }
  if (threadIdx.x == 0) {
    ucount[0] = total;
    ucount[1] = 0;
    ucount[2] = H;  // P2G: list order when 0
    ucount[3] = 0;
  }
}

template <class R>
__device__ __forceinline__ void p2g_unit(
    const ParticlesT<R>& p, const int* __restrict__ perm,
    const int* __restrict__ cstart, const NodesT<R>& nodes,
    double* __restrict__ led_part, const Geom& G, const Phys& P,
    const Scalars* S, int record, P2GSmemT<R>& s, int slot, int4 unit) {
  const int nrows = G.nrows, ncols = G.ncols;
  const int r0 = unit.x * kTR;
  const int cA = unit.y;
  const int cB = unit.z;
  const int rlo = max(r0 - 1, 0);
  const int rhi = min(r0 + kTR - 1, nrows - 1);
  const int ccFirst = max(cA - 1, 0);
  const int ccLast = min(cB - 1, ncols - 1);
  const int nrs = rhi - rlo + 2;  // row starts per column
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int grp = warp;  // quantity group (warp-uniform)
  const int row = lane;
  const int r = r0 + row;
  const bool lane_ok = row < kTR;  // lanes kTR..31 idle
  const bool row_ok = lane_ok && (r <= nrows);
  const double dt = S->dt;
  const ShapeT<R> sh{R(1) / R(G.hx), -R(1) / R(G.hx), R(1) / R(G.hy), -R(1) / R(G.hy)};
  // exchange slots of each group's quantities: g0 0-2, g1 3-6, g2 7, g3 8
  const int slot0 = grp == 0 ? 0 : grp == 1 ? 3 : grp == 2 ? 7 : 8;
  const int nq = grp == 0 ? 3 : grp == 1 ? 4 : 1;
  const bool last_unit_col = (cB == ncols + 1);  // this unit closes node column ncols

  double lp0 = 0, lp1 = 0, lp2 = 0, ln0 = 0, ln1 = 0, ln2 = 0;
  Chains<R> a;
#pragma unroll
  for (int q = 0; q < kMaxQ; ++q) a.f[q] = a.fc[q] = a.s[q] = a.sc[q] = R(0);

  // prologue: row starts of the first two columns, sorted indices of batch 0
  for (int q = tid; q < 2 * nrs; q += kP2GThreads) {
    const int k = q / nrs, rr = q - k * nrs;
    const int cc = ccFirst + k;
    if (cc <= ccLast) s.rowstart[cc % 3][rr] = cstart[rlo + rr + cc * nrows];
  }
  __syncthreads();
  int pf[kPf];
  Batch cur;
  cur.cc = ccFirst;
  cur.bb = s.rowstart[ccFirst % 3][0];
  cur.be = min(cur.bb + kCap, s.rowstart[ccFirst % 3][nrs - 1]);
  cur.valid = true;
  load_perm(pf, perm, cur);
  int a0 = 0, a1 = 0, b1 = 0;  // my rows' ranges in the current column

  while (true) {
    issue_gather(s, p, pf, cur);
    // while the copies fly: this batch's bookkeeping and the next batch's
    // sorted indices
    const int* RS = s.rowstart[cur.cc % 3];
    const bool first_of_col = (cur.bb == RS[0]);
    const bool last_of_col = (cur.be == RS[nrs - 1]);
    int rs2 = 0;
    const bool has_rs2 = last_of_col && cur.cc + 2 <= ccLast && tid < nrs;
    if (has_rs2) rs2 = cstart[rlo + tid + (cur.cc + 2) * nrows];
    if (first_of_col) {
      // cell r-1: [a0, a1), cell r: [a1, b1) (empty where the cell is absent)
      a0 = a1 = b1 = 0;
      if (row_ok && r >= rlo && r <= rhi + 1) {
        const int k = r - rlo;  // row start of cell r (= end of cell r-1)
        a1 = RS[k];
        a0 = (r - 1 >= rlo) ? RS[k - 1] : a1;
        b1 = (r <= rhi) ? RS[k + 1] : a1;
      }
    }
    const Batch nxt = next_batch(cur, s, nrs, ccLast);
    load_perm(pf, perm, nxt);
    cp_async_wait_all();
    __syncthreads();  // batch `cur` is in shared memory
    const bool own = r >= r0 && r < r0 + kTR && cur.cc >= cA && cur.cc >= G.pc_lo &&
                     cur.cc < G.pc_hi;
    const bool lead = cur.cc < cA;  // started chains only
    const int rc = solo_row(a0, a1, b1, cur.bb, cur.be, r0);  // the same in every warp
    if (rc >= 0) {
      // own as the cell's lower lane sees it (its row lies in the unit)
      const bool own_c = cur.cc >= cA && cur.cc >= G.pc_lo && cur.cc < G.pc_hi;
      solo_batch<R>(a, s, rc, r0, nrows, grp, slot0, nq, lead, own_c, cur.be - cur.bb, sh,
                    lp0, lp1, lp2);
    } else {
      switch (grp) {
        case 0: chain_group<R, 0>(a, s, lead, a0, a1, b1, cur.bb, cur.be, sh, own, lp0, lp1, lp2); break;
        case 1: chain_group<R, 1>(a, s, lead, a0, a1, b1, cur.bb, cur.be, sh, own, lp0, lp1, lp2); break;
        case 2: chain_group<R, 2>(a, s, lead, a0, a1, b1, cur.bb, cur.be, sh, own, lp0, lp1, lp2); break;
        default: chain_group<R, 3>(a, s, lead, a0, a1, b1, cur.bb, cur.be, sh, own, lp0, lp1, lp2); break;
      }
    }
    if (last_of_col) {
      if (lane_ok)
        for (int q = 0; q < nq; ++q) s.xch[slot0 + q][row] = acc_value(a.f[q], a.fc[q]);
      if (has_rs2) s.rowstart[(cur.cc + 2) % 3][tid] = rs2;
    }
    __syncthreads();  // shared records free; finished sums exchanged
    if (last_of_col) {
      // ---- nodal update of node column cc ------------------------------
      if (warp == kNodalWarp && row_ok && cur.cc >= cA) {
        const R (*X)[kTR] = s.xch;
        nodal_update<R>(X[0][row], X[1][row], X[2][row], X[3][row], X[4][row],
                        X[5][row], X[6][row], X[7][row], X[8][row], r, cur.cc, G, P,
                        dt, nodes, record, ln0, ln1, ln2);
      }
      if (cur.cc == ncols - 1 && last_unit_col) {
        // node column ncols: its chains end with this column
        __syncthreads();  // warp 0 is done reading the exchange
        if (lane_ok)
          for (int q = 0; q < nq; ++q) s.xch[slot0 + q][row] = acc_value(a.s[q], a.sc[q]);
        __syncthreads();
        if (warp == kNodalWarp && row_ok) {
          const R (*X)[kTR] = s.xch;
          nodal_update<R>(X[0][row], X[1][row], X[2][row], X[3][row], X[4][row],
                          X[5][row], X[6][row], X[7][row], X[8][row], r, ncols, G, P,
                          dt, nodes, record, ln0, ln1, ln2);
        }
      }
#pragma unroll
      for (int q = 0; q < kMaxQ; ++q) {
        a.f[q] = a.s[q];
        a.fc[q] = a.sc[q];
        a.s[q] = R(0);
        a.sc[q] = R(0);
      }
    }
    if (!nxt.valid) break;
    cur = nxt;
  }
  // ---- ledger partials: fixed-order block reduction ----------------------
  {
    double v[6] = {lp0, lp1, lp2, ln0, ln1, ln2};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double x = v[q];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) s.led[q][warp] = x;
    }
    __syncthreads();
    if (tid < 6) {
      double x = 0.0;
      for (int w = 0; w < kP2GThreads / 32; ++w) x += s.led[tid][w];
      led_part[(size_t)slot * 6 + tid] = x;
    }
    __syncthreads();
  }
}

// kRecord: the nodal output fields are written (compiled out of the plain
// step)
template <bool kRecord>
__global__ void __launch_bounds__(kP2GThreads, kP2GMinBlocks)
    k_p2g(Particles p, const int* __restrict__ perm,
          const int* __restrict__ cstart, Nodes nodes,
          double* __restrict__ led_part, Geom G, Phys P, const Scalars* S,
          const int4* __restrict__ ulist, const int* __restrict__ uorder,
          const int* __restrict__ ucount) {
  constexpr int record = kRecord ? 1 : 0;
  if (!S->active) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  P2GSmem& s = *reinterpret_cast<P2GSmem*>(smem_raw);
  const int nunits = ucount[0], nheavy = ucount[2];
  __shared__ int next_unit;
  while (true) {
    // units are taken in the order of uorder (heavy ones first) from a
    // shared cursor: CTAs that drew light units take more (the per-SM load
    // stays even)
    if (threadIdx.x == 0) next_unit = atomicAdd(const_cast<int*>(ucount) + 1, 1);
    __syncthreads();
    const int k = next_unit;
    __syncthreads();
    if (k >= nunits) break;
    const int ui = nheavy ? uorder[k] : k;
    p2g_unit(p, perm, cstart, nodes, led_part, G, P, S, record, s, ui, ulist[ui]);
  }
}

size_t sort_big_smem_bytes() { return 2 * sizeof(unsigned long long) * kBigRun; }

int setup_sort() {
  return cudaFuncSetAttribute(k_segment_order_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(sort_big_smem_bytes())) == cudaSuccess;
}

int setup_p2g() {
  const size_t smem = p2g_smem_bytes();
  for (const void* f : {(const void*)k_p2g<false>, (const void*)k_p2g<true>}) {
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
        cudaSuccess)
      return 0;
    cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                         int(cudaSharedmemCarveoutMaxShared));
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_p2g<false>, kP2GThreads, smem);
  return per_sm < 1 ? 1 : per_sm;
}

void launch_p2g(int grid, cudaStream_t st, Particles p, const int* perm, const int* cstart,
                Nodes nodes, double* led_part, Geom G, Phys P, const Scalars* S, int record,
                const int4* ulist, const int* uorder, const int* ucount) {
  if (record)
    k_p2g<true><<<grid, kP2GThreads, p2g_smem_bytes(), st>>>(p, perm, cstart, nodes, led_part,
                                                             G, P, S, ulist, uorder, ucount);
  else
    k_p2g<false><<<grid, kP2GThreads, p2g_smem_bytes(), st>>>(p, perm, cstart, nodes, led_part,
                                                              G, P, S, ulist, uorder, ucount);
}

// Block reduction, in a fixed order, of the ledger partials of units
// [u0, u1) into S->ledger, and the conservation errors.
__device__ __forceinline__ void ledger_reduce(const double* __restrict__ led_part,
                                              int u0, int u1, Scalars* S) {
  __shared__ double sm[6][32];
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int b = u0 + threadIdx.x; b < u1; b += blockDim.x)
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

// log: a ring of kLedgerLog rows {t, err_mass, err_mom}, row (it-1) % kLedgerLog
__global__ void k_ledger_final(const double* __restrict__ led_part,
                               const int* __restrict__ ucount, Scalars* S,
                               double* __restrict__ log) {
  if (!S->active) return;
  ledger_reduce(led_part, 0, ucount[0], S);
  if (threadIdx.x == 0 && log) {
    double* row = log + 3 * ((S->it - 1) % kLedgerLog);
    row[0] = S->ledger[8];
    row[1] = S->ledger[6];
    row[2] = S->ledger[7];
  }
}

// ---------------------------------------------------------------------------
// G2P: velocity, advection, velocity gradients at the new position with the
// cell of the step start, height update, Bingham stress, next cell key and
// the CFL max-reductions (main/optim_par.cpp:532-651).
// ---------------------------------------------------------------------------
// The step-start values G2P reads of a particle.
template <class R>
struct G2PIn {
  R x, y, hp, H, Mp, Vp;
  int idx;
};
template <class R>
__device__ __forceinline__ G2PIn<R> g2p_in(const ParticlesT<R>& src, int s) {
  return G2PIn<R>{src.x[s], src.y[s], src.hp[s], src.H[s], src.Mp[s], src.Vp[s], src.idx[s]};
}

// One particle of G2P (the body of k_g2p and of the batched G2P): the
// particle in slot `s` of the step-start buffer `src` -- its values `in` --
// binned to cell `key`, written to slot `j` of `dst` (its position in this
// step's sorted order).  key_off is the scenario's first cell in a batch (its
// cell keys are offset by it); the new key is returned in `nkey`.
template <class R>
__device__ __forceinline__ void g2p_particle(
    const ParticlesT<R>& src, int s, const G2PIn<R>& in, int key_in,
    const ParticlesT<R>& dst, int j,
    const NodesT<R>& nodes, const double* __restrict__ Z, const Geom& G, const Phys& P,
    const ShapeT<R>& sh, double dtd, int record, int want_grad, int key_off,
    unsigned long long& m0, unsigned long long& m1, unsigned long long& m2, int& bad,
    int& nkey) {
  const int nrows = G.nrows;
  const R ihx = sh.ihx, mihx = sh.mihx;
  const R ihy = sh.ihy, mihy = sh.mihy;
  const R eps = R(1e-10);
  const R dt = R(dtd);
  const int key = key_in - key_off;
  const int r = key % nrows, c = key / nrows;
  int nd[4];
  R vxn[4], vyn[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    nd[k] = node_of(k, c, r, nrows);
    const V2<R> v = nodes.vvL[nd[k]];
    vxn[k] = v.x;
    vyn[k] = v.y;
  }
  R x = in.x, y = in.y;
  R xi, eta;
  local_xy_g(x, y, c, r, G, ihx, ihy, xi, eta);
  R vxL = R(0), vyL = R(0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const R N = shp(xi, eta, k);
    vxL += N * vxn[k];
    vyL += N * vyn[k];
  }
  if (record) {
    // this step's intermediates as the reference's dprops hold them after
    // the step (main/optim_par.cpp:387-459,542): apx/apy, grad Z and the
    // gravity and friction forces of this step's P2G
    R ax = R(0), ay = R(0);
    double dzx = 0.0, dzy = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const R N = shp(xi, eta, k);
      ax += N * nodes.avx[nd[k]];
      ay += N * nodes.avy[nd[k]];
      const double zn = Z[nd[k]];
      dzx += double(shg_x(eta, k, ihx, mihx)) * zn;
      dzy += double(shg_y(xi, k, ihy, mihy)) * zn;
    }
    dst.apx[j] = ax;
    dst.apy[j] = ay;
    dst.dZxp[j] = R(dzx);
    dst.dZyp[j] = R(dzy);
    const V2<R> qg = src.qg[s], qf = src.qf[s];
    dst.Fpx[j] = qg.x;
    dst.Fpy[j] = qg.y;
    dst.Frx[j] = qf.x;
    dst.Fry[j] = qf.y;
  }
  const R vpx = vxL, vpy = vyL;
  x = x + dt * vpx;
  y = y + dt * vpy;
  if (x < eps) x = eps;
  if (x > R(G.Lx) - eps) x = R(G.Lx) - eps;
  if (y < eps) y = eps;
  if (y > R(G.Ly) - eps) y = R(G.Ly) - eps;
  // g2pd {vvxL, vvyL} at the new position, old cell (main/optim_par.cpp:578)
  local_xy_g(x, y, c, r, G, ihx, ihy, xi, eta);
  R vxdx = R(0), vydx = R(0), vxdy = R(0), vydy = R(0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const R Nx = shg_x(eta, k, ihx, mihx);
    const R Ny = shg_y(xi, k, ihy, mihy);
    vxdx += Nx * vxn[k];
    vxdy += Ny * vxn[k];
    vydx += Nx * vyn[k];
    vydy += Ny * vyn[k];
  }
  // height from the strain rate (main/optim_par.cpp:595-599)
  const R div = vxdx + vydy;
  R hp = in.hp;
  hp = hp / (R(1) + dt * div);
  hp = hp < R(1e-2) ? R(1e-2) : hp;
  R F11, F12, F22;
  const R H = in.H;
  const R Mp = in.Mp, Vp = in.Vp;
  rheology_stress(P, vpx, vpy, hp, H, vxdx, vydy, vxdy, vydx, F11, F12, F22);
  dst.x[j] = x;
  dst.y[j] = y;
  dst.vpx[j] = vpx;
  dst.vpy[j] = vpy;
  dst.hp[j] = hp;
  dst.F11[j] = F11;
  dst.F12[j] = F12;
  dst.F22[j] = F22;
  dst.Mp[j] = Mp;
  dst.Vp[j] = Vp;
  dst.H[j] = H;
  dst.idx[j] = in.idx;
  const int nr = cell_row(double(y), G), ncl = cell_col(double(x), G);
  nkey = nr + ncl * nrows + key_off;
  dst.key[j] = nkey;
  if (want_grad) {
    dst.vpx_dx[j] = vxdx;
    dst.vpx_dy[j] = vxdy;
    dst.vpy_dx[j] = vydx;
    dst.vpy_dy[j] = vydy;
  }
  // the record of the next P2G: what the reference stores at the end of
  // the step (main/optim_par.cpp:600-626: momentum, Ap, basal friction) and
  // the local coordinates and gravity force in the cell of the next
  // binning (:387,447-454)
  {
    dst.mp[j] = V2<R>{vpx * Mp, vpy * Mp};
    const R Ap = hp > R(1.e-2) ? Vp / hp : R(0);
    R fbx, fby;
    rheology_friction(P, vpx, vpy, hp, fbx, fby);
    dst.qf[j] = V2<R>{Ap * fbx, Ap * fby};
    R qxi, qeta, qgx, qgy;
    next_record(G, P, Z, x, y, hp, H, Vp, qxi, qeta, qgx, qgy);
    dst.xe[j] = V2<R>{qxi, qeta};
    dst.qg[j] = V2<R>{qgx, qgy};
  }
  if (record) {
    // g2p Z -> Zp at the new position, old cell (main/optim_par.cpp:642)
    double zp = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) zp += double(shp(xi, eta, k)) * Z[nd[k]];
    dst.Zp[j] = R(zp);
    dst.hpZ[j] = R(double(hp) + zp);
  }
  m0 = max(m0, ordered_key(double(fabs(vpx))));
  m1 = max(m1, ordered_key(double(fabs(vpy))));
  m2 = max(m2, ordered_key(double(hp)));
  // a diverged particle (NaN/inf anywhere in the state a step carries, or a
  // negative depth) stops its scenario through the status word
  bad |= !(isfinite(x) && isfinite(y) && isfinite(vpx) && isfinite(vpy) &&
           isfinite(hp) && hp >= R(0));
}

// Copies the moving fields of slot s of src to slot j of dst (a particle
// that does not step in this pass, or the reordering into reference order).
template <class R>
__device__ __forceinline__ void copy_moving(const ParticlesT<R>& src, int s,
                                            const ParticlesT<R>& dst, int j) {
  dst.x[j] = src.x[s];
  dst.y[j] = src.y[s];
  dst.vpx[j] = src.vpx[s];
  dst.vpy[j] = src.vpy[s];
  dst.hp[j] = src.hp[s];
  dst.F11[j] = src.F11[s];
  dst.F12[j] = src.F12[s];
  dst.F22[j] = src.F22[s];
  dst.Mp[j] = src.Mp[s];
  dst.Vp[j] = src.Vp[s];
  dst.H[j] = src.H[s];
  dst.key[j] = src.key[s];
  dst.idx[j] = src.idx[s];
  dst.slot[j] = src.slot[s];
  dst.mp[j] = src.mp[s];
  dst.qf[j] = src.qf[s];
  dst.xe[j] = src.xe[s];
  dst.qg[j] = src.qg[s];
  if (src.vpx_dx) {
    dst.vpx_dx[j] = src.vpx_dx[s];
    dst.vpx_dy[j] = src.vpx_dy[s];
    dst.vpy_dx[j] = src.vpy_dx[s];
    dst.vpy_dy[j] = src.vpy_dy[s];
  }
}

// Raises kStatusNonFinite in S when any thread of the block saw a diverged
// particle (all threads of the block call it).
__device__ __forceinline__ void flag_non_finite(int bad, Scalars* S) {
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&S->status, kStatusNonFinite);
}

// The counting sort's first step for the next binning, done where the keys
// are made: particle j of a warp takes slot[j] among its cell's particles,
// one atomic per cell and warp (the lanes that share a cell take
// consecutive slots).  All 32 lanes call it; ok == false lanes take part
// without a particle.
__device__ __forceinline__ void count_key(int k, bool ok, int* __restrict__ count,
                                          int* __restrict__ slot_out) {
  const int lane = threadIdx.x & 31;
  const int kk = ok ? k : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, kk);
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (ok && lane == leader) base = atomicAdd(&count[kk], __popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (ok) *slot_out = base + __popc(peers & ((1u << lane) - 1u));
}

// Block min/max of the new keys into knext (the scan range of the next
// sort); all threads of the block call it.
__device__ __forceinline__ void key_range(int kmin, int kmax, int* sred, Scalars* S) {
  for (int o = 16; o > 0; o >>= 1) {
    kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
    kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&sred[0], kmin);
    atomicMax(&sred[1], kmax);
  }
  __syncthreads();
  if (threadIdx.x == 0 && sred[1] >= 0) {
    atomicMin(&S->knext[0], sred[0]);
    atomicMax(&S->knext[1], sred[1]);
  }
}

// Block reduction of the CFL maxima into one scenario's next-step slots.
__device__ __forceinline__ void cfl_block_max(unsigned long long m0,
                                              unsigned long long m1,
                                              unsigned long long m2,
                                              unsigned long long* red,
                                              Scalars* S) {
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

// kRecord / kGrad: the output fields and the velocity gradients are
// written (compiled out of the plain step).  Thread t takes the particle
// at position ng + t of this step's sorted order: slot perm[ng + t] of
// `cur`, written to slot t of `nxt`.  ng = 0 outside slab mode; in slab
// mode the first ng positions are the copies of the neighbour's last column
// (they sort first), which only P2G reads, and a particle whose new cell
// lies outside the slab's columns is listed in `leave` (and not counted:
// it moves to the neighbour).  A pass whose loop condition failed copies
// `cur` to `nxt` unchanged (the host exchanges the buffers after every
// pass).
template <bool kRecord, bool kGrad>
__global__ void __launch_bounds__(kG2PThreads, kG2PMinBlocks)
    k_g2p_t(Particles cur, Particles nxt, const int* __restrict__ perm,
            const int* __restrict__ skey, Nodes nodes, const double* __restrict__ Z, Geom G,
            Phys P, Scalars* S, int* __restrict__ count, int* __restrict__ leave) {
  const int ng = S->nghost;
  const int n = S->np - ng;  // the slab's own particles
  const int stride = gridDim.x * blockDim.x;
  if (!S->active) {  // (ghosts, imported last, sit in the slots after n)
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
      copy_moving(cur, j, nxt, j);
    return;
  }
  __shared__ unsigned long long red[3];
  __shared__ int kred[2];
  if (threadIdx.x < 3) red[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) {
    kred[0] = 0x7fffffff;
    kred[1] = -1;
  }
  __syncthreads();
  const double dt = S->dt;
  const Shape sh{1.0 / G.hx, -1.0 / G.hx, 1.0 / G.hy, -1.0 / G.hy};
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  int bad = 0, kmin = 0x7fffffff, kmax = -1;
  const int lane = threadIdx.x & 31;
  for (int t0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); t0 < n; t0 += stride) {
    const int t = t0 + lane;
    const bool ok = t < n;
    int nkey = -1;
    bool stay = ok;
    if (ok) {
      const int j = ng + t;
      const int s = perm[j];
      g2p_particle(cur, s, g2p_in(cur, s), skey[j], nxt, t, nodes, Z, G, P, sh, dt,
                   kRecord ? 1 : 0, kGrad ? 1 : 0, 0, m0, m1, m2, bad, nkey);
      kmin = min(kmin, nkey);
      kmax = max(kmax, nkey);
      if (leave) {
        const int col = nkey / G.nrows;
        if (col < G.pc_lo || col >= G.pc_hi) {
          stay = false;
          leave[atomicAdd(&S->nleave, 1)] = t;
        }
      }
    }
    count_key(nkey, stay, count, nxt.slot + (ok ? t : 0));
  }
  cfl_block_max(m0, m1, m2, red, S);
  key_range(kmin, kmax, kred, S);
  flag_non_finite(bad, S);
}

void launch_g2p(int grid, cudaStream_t st, Particles cur, Particles nxt, const int* perm,
                const int* skey, Nodes nodes, const double* Z, Geom G, Phys P, Scalars* S,
                int* count, int* leave, int record, int want_grad) {
  if (record)
    k_g2p_t<true, true><<<grid, kG2PThreads, 0, st>>>(cur, nxt, perm, skey, nodes, Z, G, P,
                                                       S, count, leave);
  else if (want_grad)
    k_g2p_t<false, true><<<grid, kG2PThreads, 0, st>>>(cur, nxt, perm, skey, nodes, Z, G, P,
                                                        S, count, leave);
  else
    k_g2p_t<false, false><<<grid, kG2PThreads, 0, st>>>(cur, nxt, perm, skey, nodes, Z, G,
                                                         P, S, count, leave);
}

size_t p2g_smem_bytes() { return sizeof(P2GSmemT<double>); }

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b,
                         long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = float(a[i]);
}

__global__ void k_to_f64(const float* __restrict__ a, double* __restrict__ b,
                         long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = double(a[i]);
}

// ---------------------------------------------------------------------------
// BATCH: the same step over many independent scenarios packed back to back.
// Each scenario keeps its own loop state (Scalars), geometry and physics; the
// sort runs over the cells of all of them at once (keys are offset by each
// scenario's first cell), P2G takes units of every scenario from one list,
// and G2P runs one block per 256 particles of one scenario.  A scenario's
// numbers are the same alone and in a batch: its sums run in the same
// per-node order whatever the unit cuts.
// ---------------------------------------------------------------------------
__global__ void k_b_step_begin(const Scn* __restrict__ scn, Scalars* S, int nscn,
                               Scalars* Sg) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < nscn; s += blockDim.x) {
    if (scn[s].live) {
      step_begin_one(&S[s], scn[s].G, scn[s].P);
      if (S[s].active) atomicOr(&any, 1);
    } else {
      S[s].active = 0;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) Sg->active = any;
}

__global__ void k_b_step_end(const Scn* __restrict__ scn, Scalars* S, int nscn) {
  for (int s = threadIdx.x; s < nscn; s += blockDim.x)
    if (scn[s].live) step_end_one(&S[s]);
}

// one block per strip of the batch
__global__ void __launch_bounds__(kPlanThreads)
    k_b_units_plan(const int* __restrict__ cstart, const Scn* __restrict__ scn,
                   const Scalars* S, const int* __restrict__ strip_scn,
                   const Scalars* Sg, int target_units, int col_weight,
                   int* __restrict__ ustart,
                   long long* __restrict__ upex, int4* __restrict__ plan,
                   int* __restrict__ strip_n, int* __restrict__ heavy_n) {
  const int b = blockIdx.x;
  const int s = strip_scn[b];
  if (!Sg->active || !S[s].active) {
    if (threadIdx.x == 0) strip_n[b] = 0;
    return;
  }
  const Geom G = scn[s].G;
  const int local = b - scn[s].strip_off;
  const size_t base = (size_t)scn[s].useg_off + (size_t)local * (G.ncols + 1);
  // node columns of the cells the scenario's particles are binned to (the
  // keys its last G2P made), plus the column right of them; every column
  // after a layout change
  int c_lo = 0, c_hi = G.ncols;
  if (!(Sg->krange[0] <= Sg->krange[1])) {
    const int L = S[s].knext[0], H = S[s].knext[1];
    if (L > H) {  // no particle
      if (threadIdx.x == 0) strip_n[b] = 0;
      return;
    }
    c_lo = (L - scn[s].c_off) / G.nrows;
    c_hi = min((H - scn[s].c_off) / G.nrows + 1, G.ncols);
  }
  const int J = plan_strip(cstart + scn[s].c_off, G, unit_weight(Sg, target_units),
                           local, ustart + base, upex + base, plan + base, col_weight,
                           c_lo, c_hi, heavy_n);
  if (threadIdx.x == 0) strip_n[b] = J;
}

// The scan tiles of a batch pass: those that meet the batch-wide range
// (every cell after a layout change) or a scenario's keys -- the keys its
// cell starts describe (krange) or the keys its last G2P made (knext).  A
// tile that meets neither holds no particle now or at the last sort, and
// its cells' starts (the particles of the scenarios before them) stand
// while the layout does.  One thread per tile; the scenarios' cells are
// consecutive, so a binary search finds the first that meets the tile.
__global__ void k_b_tile_flags(const Scn* __restrict__ scn, const Scalars* S, int nscn,
                               const Scalars* Sg, unsigned char* __restrict__ tflag,
                               int ntiles) {
  if (!Sg->active) return;
  const int gL = min(Sg->krange[0], Sg->knext[0]), gH = max(Sg->krange[1], Sg->knext[1]);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles;
       t += gridDim.x * blockDim.x) {
    const int c0 = t * kScanTile, c1 = c0 + kScanTile - 1;
    bool f = gL <= gH && gL <= c1 && gH >= c0;
    int lo = 0, hi = nscn;  // the first scenario whose cells end after c0
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (scn[mid].c_off + scn[mid].G.nrows * scn[mid].G.ncols <= c0) lo = mid + 1;
      else hi = mid;
    }
    for (int s = lo; !f && s < nscn && scn[s].c_off <= c1; ++s) {
      const int L = min(S[s].krange[0], S[s].knext[0]);
      const int H = max(S[s].krange[1], S[s].knext[1]);
      f = L <= H && L <= c1 && H >= c0;
    }
    tflag[t] = f ? 1 : 0;
  }
}

// one block: the flat list {scenario, strip, cA, cB} in strip order, and each
// scenario's range of list positions (its ledger slots)
__global__ void __launch_bounds__(kPlanThreads)
    k_b_units_flat(const int* __restrict__ strip_n, int strips,
                   const int* __restrict__ strip_scn, const Scn* __restrict__ scn,
                   int nscn, const int4* __restrict__ plan, int4* __restrict__ ulist,
                   int* __restrict__ uorder, int* __restrict__ ucount,
                   int2* __restrict__ scn_units,
                   Scalars* S, const Scalars* Sg) {
  if (!Sg->active) return;
  const int H = ucount[3];  // heavy units, counted by the plan
  extern __shared__ int uoff[];  // strips + 1
  __shared__ int wt_i[32];
  int carry = 0;
  for (int base = 0; base < strips; base += blockDim.x) {
    const int b = base + threadIdx.x;
    const int n = b < strips ? strip_n[b] : 0;
    int tot;
    const int incl = block_incl_scan<int>(n, wt_i, tot);
    if (b < strips) uoff[b] = carry + incl - n;
    carry += tot;
  }
  if (threadIdx.x == 0) uoff[strips] = carry;
  __syncthreads();
  const int total = carry;
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    int lo = 0, hi = strips;  // uoff[lo] <= f < uoff[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (uoff[mid] <= f) lo = mid; else hi = mid;
    }
    const int s = strip_scn[lo];
    const int local = lo - scn[s].strip_off;
    const size_t base =
        (size_t)scn[s].useg_off + (size_t)local * (scn[s].G.ncols + 1);
    const int4 u = plan[base + (f - uoff[lo])];
    ulist[f] = make_int4(s, local, u.x, u.y);
  }
  if (H > 0) {
    __syncthreads();
    heavy_first(
      total,
      [&](int f) {
        const int4 L = ulist[f];
        const int st = scn[L.x].strip_off + L.y;
        const size_t base = (size_t)scn[L.x].useg_off + (size_t)L.y * (scn[L.x].G.ncols + 1);
        return plan[base + (f - uoff[st])].z;
      },
      uorder, wt_i);
  }
  for (int s = threadIdx.x; s < nscn; s += blockDim.x) {
    const int b0 = scn[s].strip_off, b1 = b0 + scn[s].nstrips;
    scn_units[s] = make_int2(uoff[b0], uoff[b1]);
    // each scenario's key ranges roll over: the starts now describe the
    // keys its last G2P made, and the next G2P starts an empty range
    S[s].krange[0] = S[s].knext[0];
    S[s].krange[1] = S[s].knext[1];
    S[s].knext[0] = 0x7fffffff;
    S[s].knext[1] = -1;
  }
  if (threadIdx.x == 0) {
    ucount[0] = total;
    ucount[1] = 0;
    ucount[2] = H;  // P2G: list order when 0
    ucount[3] = 0;
  }
}

template <class R>
__global__ void __launch_bounds__(kP2GThreads, kP2GMinBlocks)
    k_b_p2g(ParticlesT<R> p, const int* __restrict__ perm, const int* __restrict__ cstart,
            V2<R>* __restrict__ vvL,
            double* __restrict__ led_part, const Scn* __restrict__ scn, Scalars* S,
            const int4* __restrict__ ulist, const int* __restrict__ uorder,
            const int* __restrict__ ucount, const Scalars* Sg) {
  if (!Sg->active) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  P2GSmemT<R>& sm = *reinterpret_cast<P2GSmemT<R>*>(smem_raw);
  const int nunits = ucount[0], nheavy = ucount[2];
  __shared__ int next_unit;
  while (true) {
    if (threadIdx.x == 0) next_unit = atomicAdd(const_cast<int*>(ucount) + 1, 1);
    __syncthreads();
    const int k = next_unit;
    __syncthreads();
    if (k >= nunits) break;
    const int ui = nheavy ? uorder[k] : k;  // heavy units first
    const int4 u = ulist[ui];
    const Geom G = scn[u.x].G;
    const Phys P = scn[u.x].P;
    const int n_off = scn[u.x].n_off, c_off = scn[u.x].c_off;
    NodesT<R> nd{};
    nd.vvL = vvL + n_off;
    p2g_unit<R>(p, perm, cstart + c_off, nd, led_part, G, P, &S[u.x], 0, sm, ui,
             make_int4(u.y, u.z, u.w, 0));
  }
}

// one block per scenario
__global__ void k_b_ledger(const double* __restrict__ led_part,
                           const int2* __restrict__ scn_units,
                           const Scn* __restrict__ scn, Scalars* S, int nscn,
                           const Scalars* Sg) {
  const int s = blockIdx.x;
  if (!Sg->active || s >= nscn || !scn[s].live || !S[s].active) return;
  ledger_reduce(led_part, scn_units[s].x, scn_units[s].y, &S[s]);
}

// gblk[b] = {scenario, its first particle handled by block b}.  A
// scenario's particles are positions [p_off, p_off + np) of the sorted order
// (its cell keys lie between those of the scenarios before and after it).
// Thread j takes position j: slot perm[j] of `cur`, written to slot j of
// `nxt`; a scenario that does not step in this pass (finished, stopped or
// removed) is copied through in sorted order and counted for the next sort;
// a pass in which no scenario steps copies `cur` to `nxt` unchanged.
template <class R>
__global__ void __launch_bounds__(kG2PThreads, kG2PMinBlocks)
    k_b_g2p(ParticlesT<R> cur, ParticlesT<R> nxt, const int* __restrict__ perm,
            const int* __restrict__ skey, const V2<R>* __restrict__ vvL,
            const double* __restrict__ Z,
            const Scn* __restrict__ scn, Scalars* S, const int2* __restrict__ gblk,
            Scalars* Sg, int* __restrict__ count) {
  const int2 e = gblk[blockIdx.x];
  const int s = e.x;
  const int p_off = scn[s].p_off, np = scn[s].np;
  const int li = e.y + threadIdx.x;
  const int j = p_off + li;
  const bool ok = li < np;
  if (!Sg->active) {
    if (ok) copy_moving(cur, j, nxt, j);
    return;
  }
  __shared__ unsigned long long red[3];
  __shared__ int kred[2];
  if (threadIdx.x < 3) red[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) {
    kred[0] = 0x7fffffff;
    kred[1] = -1;
  }
  __syncthreads();
  int nkey = -1;
  if (!S[s].active) {  // block-uniform
    if (ok) {
      copy_moving(cur, perm[j], nxt, j);
      nkey = nxt.key[j];
    }
    count_key(nkey, ok, count, nxt.slot + (ok ? j : 0));
    key_range(ok ? nkey : 0x7fffffff, ok ? nkey : -1, kred, &S[s]);
    return;
  }
  const Geom G = scn[s].G;
  const Phys P = scn[s].P;
  const int n_off = scn[s].n_off, c_off = scn[s].c_off;
  NodesT<R> nd{};
  nd.vvL = const_cast<V2<R>*>(vvL) + n_off;
  const ShapeT<R> sh{R(1) / R(G.hx), -R(1) / R(G.hx), R(1) / R(G.hy), -R(1) / R(G.hy)};
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  int bad = 0;
  if (ok)
    g2p_particle(cur, perm[j], g2p_in(cur, perm[j]), skey[j], nxt, j, nd, Z + n_off, G, P,
                 sh, S[s].dt, 0, 0,
                 c_off, m0, m1, m2, bad, nkey);
  count_key(nkey, ok, count, nxt.slot + (ok ? j : 0));
  cfl_block_max(m0, m1, m2, red, &S[s]);
  key_range(ok ? nkey : 0x7fffffff, ok ? nkey : -1, kred, &S[s]);
  flag_non_finite(bad, &S[s]);
}

// Compaction of a batch into the other half of its double buffer:
// mblk[b] = {destination first particle, source first particle, count <= 256,
// cell-key shift}.
template <class R>
__global__ void k_b_move(ParticlesT<R> dst, ParticlesT<R> src, const int4* __restrict__ mblk) {
  const int4 m = mblk[blockIdx.x];
  if ((int)threadIdx.x >= m.z) return;
  const int i = m.y + threadIdx.x, o = m.x + threadIdx.x;
  copy_moving(src, i, dst, o);
  dst.key[o] = src.key[i] + m.w;
}

// Slots and counts of the keys [0, n) (after an upload or a compaction).
__global__ void k_count_n(const int* __restrict__ key, int* __restrict__ count,
                          int* __restrict__ slot, int n) {
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); i0 < n; i0 += stride) {
    const int i = i0 + lane;
    const bool ok = i < n;
    count_key(ok ? key[i] : -1, ok, count, slot + (ok ? i : 0));
  }
}

// nblk[b] = {destination first node, source first node, count <= 256, 0}
__global__ void k_b_move_nodes(double* __restrict__ dst, const double* __restrict__ src,
                               const int4* __restrict__ nblk) {
  const int4 m = nblk[blockIdx.x];
  if ((int)threadIdx.x < m.z) dst[m.x + threadIdx.x] = src[m.y + threadIdx.x];
}

// HV: p2g of the updated depth hp at the updated positions, each particle
// still in the cell it was binned to at the start of the step
// (main/optim_par.cpp:650, after the vars were zeroed at :362-364).  `p` is
// the buffer this step's G2P wrote, in this step's sorted order, so the
// particles of a cell are the slots [cstart[cell], cstart[cell+1]) in
// reference index order.  One thread per node walks its four cells in id
// order -- (r-1,c-1) local 3, (r,c-1) local 2, (r-1,c) local 1, (r,c) local
// 0 -- the quadgrid cell-sweep order.  Output-only: launched when outputs
// are recorded.
__global__ void k_hv(const Particles p, const int* __restrict__ cstart,
                     double* __restrict__ HV, Geom G, const Scalars* S) {
  if (!S->active) return;
  const int nrows = G.nrows, ncols = G.ncols;
  const int nn = (nrows + 1) * (ncols + 1);
  const double ihx = 1.0 / G.hx, ihy = 1.0 / G.hy;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nn;
       n += gridDim.x * blockDim.x) {
    const int r = n % (nrows + 1), c = n / (nrows + 1);
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      // q: 0 -> cell (r-1,c-1) local 3, 1 -> (r,c-1) local 2,
      //    2 -> (r-1,c) local 1,   3 -> (r,c) local 0
      const int cr = (q & 1) ? r : r - 1;
      const int cc = (q & 2) ? c : c - 1;
      const int inode = 3 - q;
      if (cr < 0 || cr >= nrows || cc < 0 || cc >= ncols) continue;
      const int cell = cr + cc * nrows;
      for (int j = cstart[cell]; j < cstart[cell + 1]; ++j) {
        double xi, eta;
        local_xy_g(p.x[j], p.y[j], cc, cr, G, ihx, ihy, xi, eta);
        acc += shp(xi, eta, inode) * p.hp[j];
      }
    }
    HV[n] = acc;
  }
}

// ---- host launchers: the FP64 path and the FP32 form -----------------------
template <class R>
void launch_init_particles(int grid, int block, cudaStream_t st, ParticlesT<R> p,
                           const double* Z, const double* dZdx, const double* dZdy,
                           Geom G, Phys P, Scalars* S, int np, int key_off) {
  k_init_particles<R><<<grid, block, 0, st>>>(p, Z, dZdx, dZdy, G, P, S, np, key_off);
}

template <class R>
void launch_prep(int grid, int block, cudaStream_t st, ParticlesT<R> p, const double* Z,
                 Geom G, Phys P, const Scalars* S, int derive) {
  k_prep<R><<<grid, block, 0, st>>>(p, Z, G, P, S, derive);
}

template <class R>
void launch_b_p2g(int grid, cudaStream_t st, ParticlesT<R> p, const int* perm,
                  const int* cstart, V2<R>* vvL, double* led_part, const Scn* scn,
                  Scalars* S, const int4* ulist, const int* uorder, const int* ucount,
                  const Scalars* Sg) {
  k_b_p2g<R><<<grid, kP2GThreads, sizeof(P2GSmemT<R>), st>>>(
      p, perm, cstart, vvL, led_part, scn, S, ulist, uorder, ucount, Sg);
}

template <class R>
int setup_b_p2g() {
  const int smem = int(sizeof(P2GSmemT<R>));
  if (cudaFuncSetAttribute(k_b_p2g<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem) != cudaSuccess)
    return 0;
  cudaFuncSetAttribute(k_b_p2g<R>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       int(cudaSharedmemCarveoutMaxShared));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_b_p2g<R>, kP2GThreads,
                                                    smem) != cudaSuccess)
    return 0;
  return per_sm < 1 ? 1 : per_sm;
}

template <class R>
void launch_b_g2p(int grid, cudaStream_t st, ParticlesT<R> cur, ParticlesT<R> nxt,
                  const int* perm, const int* skey, const V2<R>* vvL, const double* Z,
                  const Scn* scn, Scalars* S, const int2* gblk, Scalars* Sg, int* count) {
  k_b_g2p<R><<<grid, kG2PThreads, 0, st>>>(cur, nxt, perm, skey, vvL, Z, scn, S, gblk, Sg,
                                           count);
}

template <class R>
void launch_b_move(int grid, cudaStream_t st, ParticlesT<R> dst, ParticlesT<R> src,
                   const int4* mblk) {
  k_b_move<R><<<grid, kG2PThreads, 0, st>>>(dst, src, mblk);
}

#define DAMPM_INSTANTIATE(R)                                                          \
  template void launch_init_particles<R>(int, int, cudaStream_t, ParticlesT<R>,       \
                                         const double*, const double*, const double*, \
                                         Geom, Phys, Scalars*, int, int);             \
  template void launch_prep<R>(int, int, cudaStream_t, ParticlesT<R>, const double*,  \
                               Geom, Phys, const Scalars*, int);                      \
  template void launch_b_p2g<R>(int, cudaStream_t, ParticlesT<R>, const int*,         \
                                const int*, V2<R>*, double*, const Scn*, Scalars*,    \
                                const int4*, const int*, const int*, const Scalars*); \
  template int setup_b_p2g<R>();                                                      \
  template void launch_b_g2p<R>(int, cudaStream_t, ParticlesT<R>, ParticlesT<R>,      \
                                const int*, const int*, const V2<R>*, const double*,  \
                                const Scn*, Scalars*, const int2*, Scalars*, int*);   \
  template void launch_b_move<R>(int, cudaStream_t, ParticlesT<R>, ParticlesT<R>,     \
                                 const int4*);
DAMPM_INSTANTIATE(double)
DAMPM_INSTANTIATE(float)
#undef DAMPM_INSTANTIATE

}  // namespace dampm
