// slab_kernels.cu -- one scenario split over slabs of cell columns.
//
// A slab (a context in slab mode) owns the particles of cell columns
// [pc_lo, pc_hi) of the global grid and writes node columns [nc_lo, nc_hi].
// Around each step the host moves three things between neighbouring slabs:
//   * before P2G, copies of the particles of the left slab's last column
//     ("ghosts"): P2G of the right slab starts the chains of its first node
//     column from them, in the cell-sweep order of the whole grid, so every
//     nodal sum is the single-domain sum bit for bit;
//   * after P2G, the right slab's first node column of (vvxL, vvyL), which
//     the left slab's G2P interpolates (a contiguous run of the node array);
//   * after G2P, the particles whose new cell lies in the neighbour's
//     columns ("migrants").
// A particle travels as one record of kSlabRecord doubles: the eleven state
// fields, the four pairs of the P2G record, and its cell key and reference
// index packed into the bits of the last double.
#include "dampm_kernels.h"

namespace dampm {

__device__ __forceinline__ double pack_ints(int a, int b) {
  const unsigned long long u =
      ((unsigned long long)(unsigned)b << 32) | (unsigned long long)(unsigned)a;
  return __longlong_as_double((long long)u);
}
__device__ __forceinline__ void unpack_ints(double d, int& a, int& b) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(d);
  a = int(unsigned(u & 0xffffffffull));
  b = int(unsigned(u >> 32));
}

// the particle in slot `a` of p into slot `b`
__device__ __forceinline__ void copy_moving_slots(const Particles& p, int a, int b) {
  p.x[b] = p.x[a];
  p.y[b] = p.y[a];
  p.vpx[b] = p.vpx[a];
  p.vpy[b] = p.vpy[a];
  p.hp[b] = p.hp[a];
  p.F11[b] = p.F11[a];
  p.F12[b] = p.F12[a];
  p.F22[b] = p.F22[a];
  p.Mp[b] = p.Mp[a];
  p.Vp[b] = p.Vp[a];
  p.H[b] = p.H[a];
  p.key[b] = p.key[a];
  p.idx[b] = p.idx[a];
  p.slot[b] = p.slot[a];
  p.mp[b] = p.mp[a];
  p.qf[b] = p.qf[a];
  p.xe[b] = p.xe[a];
  p.qg[b] = p.qg[a];
  if (p.vpx_dx) {
    p.vpx_dx[b] = p.vpx_dx[a];
    p.vpx_dy[b] = p.vpx_dy[a];
    p.vpy_dx[b] = p.vpy_dx[a];
    p.vpy_dy[b] = p.vpy_dy[a];
  }
}

// buf[k] <- the particle in slot slots[k] of p
__global__ void k_slab_pack(Particles p, const int* __restrict__ slots, int n,
                            double* __restrict__ buf) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int s = slots[k];
    double* r = buf + (size_t)k * kSlabRecord;
    r[0] = p.x[s];
    r[1] = p.y[s];
    r[2] = p.vpx[s];
    r[3] = p.vpy[s];
    r[4] = p.hp[s];
    r[5] = p.F11[s];
    r[6] = p.F12[s];
    r[7] = p.F22[s];
    r[8] = p.Mp[s];
    r[9] = p.Vp[s];
    r[10] = p.H[s];
    const double2 xe = p.xe[s], mp = p.mp[s], qg = p.qg[s], qf = p.qf[s];
    r[11] = xe.x;
    r[12] = xe.y;
    r[13] = mp.x;
    r[14] = mp.y;
    r[15] = qg.x;
    r[16] = qg.y;
    r[17] = qf.x;
    r[18] = qf.y;
    r[19] = pack_ints(p.key[s], p.idx[s]);
  }
}

// slot `base + k` of p <- buf[k] (appended particles; their sort slots
// come from the count that follows)
__global__ void k_slab_unpack(Particles p, const double* __restrict__ buf, int n, int base) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int s = base + k;
    const double* r = buf + (size_t)k * kSlabRecord;
    p.x[s] = r[0];
    p.y[s] = r[1];
    p.vpx[s] = r[2];
    p.vpy[s] = r[3];
    p.hp[s] = r[4];
    p.F11[s] = r[5];
    p.F12[s] = r[6];
    p.F22[s] = r[7];
    p.Mp[s] = r[8];
    p.Vp[s] = r[9];
    p.H[s] = r[10];
    p.xe[s] = make_double2(r[11], r[12]);
    p.mp[s] = make_double2(r[13], r[14]);
    p.qg[s] = make_double2(r[15], r[16]);
    p.qf[s] = make_double2(r[17], r[18]);
    int key, idx;
    unpack_ints(r[19], key, idx);
    p.key[s] = key;
    p.idx[s] = idx;
  }
}

// slots (in any order) of the first n particles whose cell lies in column
// `col`; *count receives how many
__global__ void k_slab_select(const int* __restrict__ key, int n, int col, int nrows,
                              int* __restrict__ slots, int* __restrict__ count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (key[i] / nrows == col) slots[atomicAdd(count, 1)] = i;
}

// Raises kStatusSlab when a key of the n imported particles lies outside
// cell columns [col_lo, col_hi) (a particle that moved more than one slab).
__global__ void k_slab_check(const int* __restrict__ key, int n, int col_lo, int col_hi,
                             int nrows, Scalars* S) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int c = key[k] / nrows;
    if (c < col_lo || c >= col_hi) atomicOr(&S->status, kStatusSlab);
  }
}

// out[k] = key[slots[k]]
__global__ void k_slab_keys(const int* __restrict__ key, const int* __restrict__ slots, int n,
                            int* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = key[slots[k]];
}

// moves[k] = {from, to}: the particle in slot `from` fills the hole at `to`
// (sources and holes are disjoint)
__global__ void k_slab_move(Particles p, const int2* __restrict__ moves, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    copy_moving_slots(p, moves[k].x, moves[k].y);
}

// The slab's loop scalars after a route or an import: the particle count,
// ghosts added, the next sort over every cell, the leaver list emptied.
__global__ void k_slab_scalars(Scalars* S, int np, int ghosts_added, int ncells) {
  if (threadIdx.x || blockIdx.x) return;
  S->np = np;
  S->nghost += ghosts_added;
  S->nleave = 0;
  S->knext[0] = 0;
  S->knext[1] = ncells - 1;
}

// The CFL maxima of the previous step (ordered keys), the same on every slab.
__global__ void k_slab_set_red(Scalars* S, unsigned long long a, unsigned long long b,
                               unsigned long long c) {
  if (threadIdx.x || blockIdx.x) return;
  S->red_cur[0] = a;
  S->red_cur[1] = b;
  S->red_cur[2] = c;
}

}  // namespace dampm
