// ms_kernels.cu -- adaptive merge/split (main/merge_split_ops_cmes.h) as
// prefix-scan stream compaction on sm_100a.
//
//   materialise : Ap/mom/Fb as stored by the reference (when not fresh)
//   mark        : per particle SPLIT / MERGE_PRIMARY candidates  (:143-168)
//   split cap   : rank of each split in (cell, index) order, keep < max_ops
//                 (:179-184)
//   pairing     : one thread per cell, greedy nearest co-moving partner in
//                 index order, then undo merges while the cell would drop
//                 below min_particles_per_cell (:186-248).  When the global
//                 merge budget could bind, one thread walks the cells holding
//                 a candidate in order instead (exact n_merge semantics),
//                 until the budget is spent.
//   scan        : exclusive scan of the weights {1,2,1,0} in index order
//                 (:268-274)
//   emit        : split 1->2 along the principal stretch, merge 2->1 at the
//                 centre of mass (:321-418); copy back; np := Nnew
//
// The ELFS variant (main/merge_split_ops.h) replaces the marks and the emit:
//   exterior    : empty cells joined by a union-find over 4-neighbours; the
//                 sets that reach the grid edge are the exterior (:86-164)
//   distance    : hops through cells with particles from the surface cells
//                 (exterior left or right), one block, level by level
//                 (:170-260)
//   mark        : ELFS value per particle (:266-343), split near the
//                 surface or on divergence, merge far from it (:385-402)
//   pairing     : as above with a split counting 4 and at least 2 per cell
//                 (:406-497)
//   emit        : split 1->4 at (+-r/2, +-r/2), merge 2->1 keeping the
//                 primary's label (:513-717)
#include <cfloat>

#include "dampm_device.cuh"
#include "ms_kernels.h"

namespace dampm {
namespace {

constexpr int KEEP = 0, SPLIT = 1, MERGE_PRIMARY = 2, MERGE_SECONDARY = 3;

struct MsCfg {
  double alpha, beta, split_hp_min, shear_split, hp_min, max_dv;
  int min_level, max_level, min_ppc;
  long long max_ops;  // (int)data.ms_max_ops, main/gpu_offload.cpp:317
  double pair_gate2;  // squared pair-distance limit; 0: none
  double dt_host;
  int use_step_dt;
  int split_w;        // particles a split leaves (2; ELFS 4)
  double stretch;     // ELFS divergence trigger
};

// Per storage slot: Ap, momentum and Fb as the reference stores them (the
// uploaded or emitted values while `fresh`, else derived from the state),
// and the reference-order fields xp, yp, label, level gathered through idx.
__global__ void k_ms_materialize(Particles p, Phys P, const Scalars* S, MsBuffers m) {
  if (!S->active) return;
  const bool fresh = S->fresh != 0;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int r = p.idx[i];
    m.xps[i] = p.xp[r];
    m.yps[i] = p.yp[r];
    m.labs[i] = p.label[r];
    m.levs[i] = p.level[r];
    if (fresh) {  // uploaded or emitted Ap, momentum and Fb stand as they are
      const double2 mm = p.mp[i];
      m.mx[i] = mm.x;
      m.my[i] = mm.y;
      m.aps[i] = p.Ap[r];
      m.fbxs[i] = p.Fbx[r];
      m.fbys[i] = p.Fby[r];
      continue;
    }
    const double hp = p.hp[i];
    m.aps[i] = hp > 1.e-2 ? p.Vp[i] / hp : 0.0;
    m.mx[i] = p.vpx[i] * p.Mp[i];
    m.my[i] = p.vpy[i] * p.Mp[i];
    double fx, fy;
    voellmy(P, p.vpx[i], p.vpy[i], hp, fx, fy);
    m.fbxs[i] = fx;
    m.fbys[i] = fy;
  }
}

// the momentum of the particles after the emit, back into its pair
__global__ void k_ms_pair_mom(const double* __restrict__ mx, const double* __restrict__ my,
                              Particles p, const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x)
    p.mp[i] = make_double2(mx[i], my[i]);
}

__global__ void k_ms_mark(Particles p, Geom G, MsCfg c, int* act, int cap,
                          Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  const double dt = c.use_step_dt ? S->dt : c.dt_host;
  const double min_h = (G.hy < G.hx) ? G.hy : G.hx;
  const double r_split = c.alpha * min_h;
  const double r_merge = c.beta * min_h;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap;
       i += gridDim.x * blockDim.x) {
    int a = KEEP;
    if (i < np) {
      const double r_i = sqrt(p.Ap[i]);
      const double exx = p.vpx_dx[i], eyy = p.vpy_dy[i];
      const double exy = 0.5 * (p.vpx_dy[i] + p.vpy_dx[i]);
      const double gdot = sqrt(2.0 * (exx * exx + eyy * eyy + 2.0 * exy * exy));
      const bool stretched = (r_i > r_split);
      const bool sheared = (gdot * dt > c.shear_split);
      const bool thick = (r_i < r_merge);
      const double hp = p.hp[i];
      const bool thin_skip = (hp < c.split_hp_min);
      const int lvl = p.level[i];
      if ((stretched || sheared) && !thin_skip && (lvl > c.min_level))
        a = SPLIT;
      else if (thick && hp > c.hp_min && lvl < c.max_level)
        a = MERGE_PRIMARY;
    }
    act[i] = a;
  }
}

// flag[j] = (particle at sorted position j is marked SPLIT)
__global__ void k_ms_split_flags(const int* perm, const int* act, int* flag,
                                 int cap, const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cap;
       j += gridDim.x * blockDim.x)
    flag[j] = (j < np && act[perm[j]] == SPLIT) ? 1 : 0;
}

// rank[j] = number of splits before sorted position j; demote beyond max_ops
__global__ void k_ms_split_cap(const int* perm, const int* rank, int* act,
                               MsCfg c, const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np;
       j += gridDim.x * blockDim.x) {
    const int i = perm[j];
    if (act[i] == SPLIT && (long long)rank[j] >= c.max_ops) act[i] = KEEP;
  }
}

// Pairing of one cell, merge_split_ops_cmes.h:186-248.  `budget` is the
// number of merges still allowed (n_merge < max_ops).  Returns the merges
// kept after the undo loop.
__device__ long long pair_cell(int b, int e, const int* perm, int* act,
                               int* partner, int* paired, const Particles& p,
                               double max_dv2, double gate2, int min_ppc,
                               int split_w, long long budget) {
  long long n = 0;
  for (int j = b; j < e; ++j) paired[j] = 0;
  for (int ji = b; ji < e && n < budget; ++ji) {
    const int i1 = perm[ji];
    if (act[i1] != MERGE_PRIMARY || paired[ji]) continue;
    double best = DBL_MAX;
    int bj = -1;
    const double x1 = p.x[i1], y1 = p.y[i1], u1 = p.vpx[i1], v1 = p.vpy[i1];
    for (int jj = ji + 1; jj < e; ++jj) {
      const int i2 = perm[jj];
      if (act[i2] != MERGE_PRIMARY || paired[jj]) continue;
      const double dx = x1 - p.x[i2];
      const double dy = y1 - p.y[i2];
      const double d2 = dx * dx + dy * dy;
      const double dvx = u1 - p.vpx[i2];
      const double dvy = v1 - p.vpy[i2];
      if (d2 < best && (dvx * dvx + dvy * dvy) < max_dv2 && (gate2 == 0.0 || d2 < gate2)) {
        best = d2;
        bj = jj;
      }
    }
    if (bj >= 0) {
      act[perm[bj]] = MERGE_SECONDARY;
      partner[i1] = perm[bj];
      paired[ji] = 1;
      paired[bj] = 1;
      ++n;
    } else {
      act[i1] = KEEP;
    }
  }
  // unpaired candidates (also those left when the budget ran out)
  for (int j = b; j < e; ++j) {
    const int i = perm[j];
    if (act[i] == MERGE_PRIMARY && !paired[j]) act[i] = KEEP;
  }
  int projected = 0;
  for (int j = b; j < e; ++j) {
    const int a = act[perm[j]];
    projected += (a == KEEP) ? 1 : (a == SPLIT) ? split_w : (a == MERGE_PRIMARY) ? 1 : 0;
  }
  while (projected < min_ppc) {
    bool undone = false;
    for (int j = b; j < e; ++j) {
      const int pp = perm[j];
      if (act[pp] == MERGE_PRIMARY) {
        const int q = partner[pp];
        if (q >= 0) act[q] = KEEP;
        partner[pp] = -1;
        act[pp] = KEEP;
        --n;
        projected += 1;
        undone = true;
        break;
      }
    }
    if (!undone) break;
  }
  return n;
}

// Counts the merge candidates (into ms_counts[2], read by the pairing) and
// the splits left after the cap (ms_counts[0]): a block reduction, then one
// global atomic per block and count.
__global__ void k_ms_count_cand(const int* act, int cap, Scalars* S) {
  if (!S->active) return;
  __shared__ unsigned long long part[2][32];
  unsigned long long c = 0, s = 0;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int a = act[i];
    c += (a == MERGE_PRIMARY);
    s += (a == SPLIT);
  }
  for (int o = 16; o > 0; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0) {
    part[0][w] = c;
    part[1][w] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tc = 0, ts = 0;
    for (int k = 0; k < nw; ++k) {
      tc += part[0][k];
      ts += part[1][k];
    }
    if (tc) atomicAdd((unsigned long long*)&S->ms_counts[2], tc);
    if (ts) atomicAdd((unsigned long long*)&S->ms_counts[0], ts);
  }
}

__global__ void k_ms_reset_counts(Scalars* S) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    S->ms_counts[0] = S->ms_counts[1] = S->ms_counts[2] = S->ms_counts[3] = 0;
  }
}

// all cells in parallel when the merge budget cannot bind
__global__ void k_ms_pair_parallel(const int* start, int ncells,
                                   const int* perm, int* act, int* partner,
                                   int* paired, Particles p, MsCfg c,
                                   Scalars* S) {
  if (!S->active) return;
  if (S->ms_counts[2] / 2 >= c.max_ops) return;  // budget may bind
  const double max_dv2 = c.max_dv * c.max_dv;
  long long local = 0;
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < ncells;
       cell += gridDim.x * blockDim.x) {
    const int b = start[cell], e = start[cell + 1];
    if (e - b < 1) continue;
    local += pair_cell(b, e, perm, act, partner, paired, p, max_dv2, c.pair_gate2,
                       c.min_ppc, c.split_w, 0x7fffffffffffffffLL);
  }
  if (local) atomicAdd((unsigned long long*)&S->ms_counts[1], (unsigned long long)local);
}

// When the merge budget may bind (candidates / 2 >= max_ops) the cells are
// paired in order by one thread, which walks only the cells holding a
// candidate: flag[j] marks sorted position j holding one, an exclusive scan
// gives rank, and list[rank[j]] = j lists them in (cell, index) order.
__device__ __forceinline__ bool budget_may_bind(const Scalars* S, const MsCfg& c) {
  return S->ms_counts[2] / 2 >= c.max_ops;
}

__global__ void k_ms_cand_flags(const int* perm, const int* act, int* flag, int cap,
                                MsCfg c, const Scalars* S) {
  if (!S->active) return;
  const bool bind = budget_may_bind(S, c);
  const int np = S->np;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cap;
       j += gridDim.x * blockDim.x)
    flag[j] = (bind && j < np && act[perm[j]] == MERGE_PRIMARY) ? 1 : 0;
}

__global__ void k_ms_cand_list(const int* rank, int* list, int cap, MsCfg c,
                               const Scalars* S) {
  if (!S->active || !budget_may_bind(S, c)) return;
  const int np = S->np;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np;
       j += gridDim.x * blockDim.x)
    if (rank[j + 1] > rank[j]) list[rank[j]] = j;
}

// One thread, the candidates' cells in order, the exact global n_merge
// budget.  A cell without a candidate pairs nothing and undoes nothing, so
// skipping it changes nothing; once the budget is spent no later cell can
// merge, and k_ms_demote turns their candidates back to KEEP (as the
// reference's per-cell loop does, :186-201).
__global__ void k_ms_pair_serial(const int* start, const int* perm, const int* list,
                                 const int* rank, int cap, int* act, int* partner,
                                 int* paired, Particles p, MsCfg c, Scalars* S) {
  if (!S->active || !budget_may_bind(S, c)) return;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double max_dv2 = c.max_dv * c.max_dv;
  const int ncand = rank[cap];
  long long n_merge = 0;
  int q = 0;
  while (q < ncand && n_merge < c.max_ops) {
    const int cell = p.key[perm[list[q]]];
    const int b = start[cell], e = start[cell + 1];
    n_merge += pair_cell(b, e, perm, act, partner, paired, p, max_dv2, c.pair_gate2,
                         c.min_ppc, c.split_w, c.max_ops - n_merge);
    while (q < ncand && list[q] < e) ++q;  // the cell's other candidates
  }
  S->ms_counts[1] = n_merge;
}

// candidates of the cells after the budget was spent: KEEP
__global__ void k_ms_demote(int* act, const int* partner, MsCfg c, const Scalars* S) {
  if (!S->active || !budget_may_bind(S, c)) return;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x)
    if (act[i] == MERGE_PRIMARY && partner[i] < 0) act[i] = KEEP;
}

// w in reference order: the weight of slot i goes to w[idx[i]] (idx is a
// permutation of [0, np)), so that the scan gives each particle its index in
// the compacted reference order; wslot in slot order, whose scan gives its
// storage slot; both are zero from np to cap.
__global__ void k_ms_weights(const int* act, const int* ridx, int* w, int* wslot, int cap,
                             int split_w, const Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap;
       i += gridDim.x * blockDim.x) {
    if (i < np) {
      const int a = act[i];
      const int wt = (a == KEEP) ? 1 : (a == SPLIT) ? split_w : (a == MERGE_PRIMARY) ? 1 : 0;
      w[ridx[i]] = wt;
      wslot[i] = wt;
    } else {
      w[i] = 0;
      wslot[i] = 0;
    }
  }
}

__global__ void k_ms_init_partner(int* partner, int cap, const Scalars* S) {
  if (!S->active) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap;
       i += gridDim.x * blockDim.x)
    partner[i] = -1;
}

struct Fields {
  double* f[kMsFields];
  int* label;
  int* level;
};

// field slots: 0 x, 1 y, 2 vpx, 3 vpy, 4 hp, 5 F11, 6 F12, 7 F22, 8 Mp,
// 9 Vp, 10 H, 11 Ap, 12 mpx, 13 mpy, 14 Fbx, 15 Fby, 16 vpx_dx, 17 vpx_dy,
// 18 vpy_dx, 19 vpy_dy, 20 xp, 21 yp
__device__ __forceinline__ bool extensive(int k) {
  return k == 8 || k == 9 || k == 11 || k == 12 || k == 13;
}

// Emitted particles are stored in the order of their parents' storage slots
// (the sorted order of the last step, so the next sort moves little): the
// fields the step moves and the momentum pair at storage slot os, the
// fields kept in reference order (Ap, Fb, xp, yp: slots 11, 14, 15, 20, 21;
// label, level) at the particle's index orf of the compacted reference
// order, and idx[os] = orf.
__device__ __forceinline__ bool ms_ref_slot(int k) {
  return k == 11 || k == 14 || k == 15 || k == 20 || k == 21;
}
__device__ __forceinline__ void store_particle(const Fields& out, int* __restrict__ out_idx,
                                               const double (&v)[kMsFields], int label,
                                               int level, int os, int orf) {
#pragma unroll
  for (int k = 0; k < kMsFields; ++k) out.f[k][ms_ref_slot(k) ? orf : os] = v[k];
  out.label[orf] = label;
  out.level[orf] = level;
  out_idx[os] = orf;
}

// every particle as it is (slot i, index idx[i]); the grid's share
__device__ __forceinline__ void emit_identity(const Fields& in, const Fields& out, int np,
                                              const int* ridx, int* out_idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    double v[kMsFields];
#pragma unroll
    for (int k = 0; k < kMsFields; ++k) v[k] = in.f[k][i];
    store_particle(out, out_idx, v, in.label[i], in.level[i], i, ridx[i]);
  }
}

// oslot: exclusive scan of the weights in storage-slot order; offs: the same
// in reference order (scattered through idx)
__global__ void k_ms_emit(Fields in, Fields out, const int* act, const int* partner,
                          const int* offs, const int* oslot, const int* ridx,
                          int* out_idx, Geom G, long long cap, Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  const int nnew = offs[cap];
  if (nnew > cap) {  // the state goes through unchanged (the caller exchanges buffers)
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&S->status, kStatusCapacity);
    emit_identity(in, out, np, ridx, out_idx);
    return;
  }
  const double eps = 1e-10;
  const double Lx = G.ncols * G.hx, Ly = G.nrows * G.hy;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int a = act[i];
    const int os = oslot[i], orf = offs[ridx[i]];
    double v[kMsFields];
    if (a == KEEP) {
#pragma unroll
      for (int k = 0; k < kMsFields; ++k) v[k] = in.f[k][i];
      store_particle(out, out_idx, v, in.label[i], in.level[i], os, orf);
    } else if (a == SPLIT) {
      const int level = in.level[i];
      // principal_stretch_dir (merge_split_ops_cmes.h:93-110)
      const double exx = in.f[16][i], eyy = in.f[19][i];
      const double exy = 0.5 * (in.f[17][i] + in.f[18][i]);
      const double tr = exx + eyy;
      const double diff = 0.5 * (exx - eyy);
      const double disc = sqrt(diff * diff + exy * exy);
      const double l1 = 0.5 * tr + disc;
      const double vx = l1 - eyy, vy = exy;
      const double nrm = sqrt(vx * vx + vy * vy);
      double ux = 1.0, uy = 0.0;
      if (!(nrm < 1e-12)) {
        ux = vx / nrm;
        uy = vy / nrm;
      }
      const double r_i = sqrt(in.f[11][i]);
      const double off = 0.25 * r_i;
      const double cx = in.f[0][i], cy = in.f[1][i];
      auto clampx = [&](double w) { return w < eps ? eps : (w > Lx - eps ? Lx - eps : w); };
      auto clampy = [&](double w) { return w < eps ? eps : (w > Ly - eps ? Ly - eps : w); };
      const double nx1 = clampx(cx + off * ux), ny1 = clampy(cy + off * uy);
      const double nx2 = clampx(cx - off * ux), ny2 = clampy(cy - off * uy);
#pragma unroll
      for (int k = 0; k < kMsFields; ++k) v[k] = in.f[k][i] / (extensive(k) ? 2.0 : 1.0);
      v[11] = v[9] / v[4];  // Ap = Vp / hp
      v[12] = v[8] * v[2];
      v[13] = v[8] * v[3];
      v[0] = nx1; v[1] = ny1; v[20] = nx1; v[21] = ny1;
      store_particle(out, out_idx, v, -1, level - 1, os, orf);
      v[0] = nx2; v[1] = ny2; v[20] = nx2; v[21] = ny2;
      store_particle(out, out_idx, v, -1, level - 1, os + 1, orf + 1);
    } else if (a == MERGE_PRIMARY) {
      const int j = partner[i];
      const int level = in.level[i];
      const double M1 = in.f[8][i], M2 = in.f[8][j];
      const double Mt = M1 + M2;
      const double nx = (M1 * in.f[0][i] + M2 * in.f[0][j]) / Mt;
      const double ny = (M1 * in.f[1][i] + M2 * in.f[1][j]) / Mt;
#pragma unroll
      for (int k = 0; k < kMsFields; ++k)
        v[k] = extensive(k) ? (in.f[k][i] + in.f[k][j])
                            : (M1 * in.f[k][i] + M2 * in.f[k][j]) / Mt;
      v[4] = v[9] / v[11];  // hp = Vp / Ap
      v[0] = nx; v[1] = ny; v[20] = nx; v[21] = ny;
      v[12] = v[8] * v[2];
      v[13] = v[8] * v[3];
      store_particle(out, out_idx, v, -1, level + 1, os, orf);
    }
  }
}

// The emit writes the moving fields straight into the free half of the
// double buffer (which then becomes the state); the fields kept in
// reference order (Ap, Fb, xp, yp, label, level) come back from scratch.
__global__ void k_ms_copy_back(Fields from, Fields to, const int* offs,
                               long long cap, Scalars* S) {
  if (!S->active) return;
  const int nnew = offs[cap];
  if (nnew > cap) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnew;
       i += gridDim.x * blockDim.x) {
    to.f[11][i] = from.f[11][i];
    to.f[14][i] = from.f[14][i];
    to.f[15][i] = from.f[15][i];
    to.f[20][i] = from.f[20][i];
    to.f[21][i] = from.f[21][i];
    to.label[i] = from.label[i];
    to.level[i] = from.level[i];
  }
}

__global__ void k_ms_finish(const int* offs, long long cap, Scalars* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (!S->active) return;
  const int nnew = offs[cap];
  S->ms_counts[2] = S->np;
  if (nnew > cap) {
    S->ms_counts[3] = S->np;
    return;
  }
  S->np = nnew;
  S->ms_counts[3] = nnew;
  S->fresh = 1;
}

// ---- ELFS variant (main/merge_split_ops.h) -------------------------------

// Root of empty cell v in the union-find forest uf (every link points to a
// smaller cell id, roots to themselves), halving the path on the way.
// Reads go through L2 (other blocks link concurrently); a stale read only
// returns an older ancestor, which the callers' compare-and-swap corrects.
__device__ __forceinline__ int uf_find(int* uf, int v) {
  volatile int* vu = uf;
  int par = vu[v];
  if (par != v) {
    int prev = v, next;
    while (par > (next = vu[par])) {
      vu[prev] = next;
      prev = par;
      par = next;
    }
  }
  return par;
}

// Joins the sets of empty cells a and b: the larger root is linked to the
// smaller by compare-and-swap; a failed swap returns the root's new
// (smaller) parent and the loop goes on with it.  Every retry lowers one of
// the two ids, so the loop ends within `limit` rounds (twice the cell
// count); past it the status word takes kStatusMsLimit.
__device__ __forceinline__ void uf_unite(int* uf, int a, int b, int limit, Scalars* S) {
  int ra = uf_find(uf, a), rb = uf_find(uf, b);
  for (int guard = 0; ra != rb; ++guard) {
    if (guard > limit) {
      atomicOr(&S->status, kStatusMsLimit);
      return;
    }
    if (ra < rb) {
      const int old = atomicCAS(&uf[rb], rb, ra);
      if (old == rb) return;
      rb = old;
    } else {
      const int old = atomicCAS(&uf[ra], ra, rb);
      if (old == ra) return;
      ra = old;
    }
  }
}

// Per cell: empty cells start as their own set, cells with particles are
// out of the forest (-1); no root reaches the edge yet; no hop count.
__global__ void k_elfs_cells(const int* __restrict__ start, int ncells, int* uf, int* eroot,
                             int* hops, int* bqn, const Scalars* S) {
  if (!S->active) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) bqn[0] = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += gridDim.x * blockDim.x) {
    uf[c] = start[c + 1] > start[c] ? -1 : c;
    eroot[c] = 0;
    hops[c] = -1;
  }
}

// Each empty cell joins its lower and right neighbours when they are empty.
__global__ void k_elfs_union(int* uf, int nrows, int ncols, Scalars* S) {
  if (!S->active) return;
  const int ncells = nrows * ncols;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += gridDim.x * blockDim.x) {
    if (uf[c] < 0) continue;
    const int r = c % nrows, col = c / nrows;
    if (r + 1 < nrows && uf[c + 1] >= 0) uf_unite(uf, c, c + 1, 2 * ncells + 2, S);
    if (col + 1 < ncols && uf[c + nrows] >= 0) uf_unite(uf, c, c + nrows, 2 * ncells + 2, S);
  }
}

// Every empty cell points to its root; the roots of empty edge cells are
// marked (mark_exterior_cells' seeds, :103-121).
__global__ void k_elfs_roots(int* uf, int* eroot, int nrows, int ncols, const Scalars* S) {
  if (!S->active) return;
  const int ncells = nrows * ncols;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += gridDim.x * blockDim.x) {
    if (uf[c] < 0) continue;
    const int root = uf_find(uf, c);
    uf[c] = root;
    const int r = c % nrows, col = c / nrows;
    if (r == 0 || r == nrows - 1 || col == 0 || col == ncols - 1) eroot[root] = 1;
  }
}

// exterior cell: empty, in a set that reaches the edge (uf flattened)
__device__ __forceinline__ bool elfs_exterior(const int* uf, const int* eroot, int q) {
  const int r = uf[q];
  return r >= 0 && eroot[r] != 0;
}

// The search's first level: cells with particles off the grid edge with an
// exterior cell left or right of them (compute_boundary_distance, :194-225).
__global__ void k_elfs_seeds(const int* uf, const int* eroot, int* hops, int* bq, int* bqn,
                             int nrows, int ncols, const Scalars* S) {
  if (!S->active) return;
  const int ncells = nrows * ncols;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += gridDim.x * blockDim.x) {
    if (uf[c] >= 0) continue;  // empty
    const int r = c % nrows, col = c / nrows;
    if (r == 0 || r == nrows - 1 || col == 0 || col == ncols - 1) continue;
    if (elfs_exterior(uf, eroot, c - nrows) || elfs_exterior(uf, eroot, c + nrows)) {
      hops[c] = 0;
      bq[atomicAdd(bqn, 1)] = c;
    }
  }
}

// Breadth-first search by levels through the cells with particles (:228-
// 259), in one block: each level's frontier claims its unreached
// neighbours by compare-and-swap (hop count level + 1) and lists them for
// the next level.  A cell is listed once, so there are at most ncells
// levels; the hop counts do not depend on the order inside a level.
__global__ void __launch_bounds__(1024)
    k_elfs_bfs(const int* uf, int* hops, int* bq, const int* bqn, int nrows, int ncols,
               const Scalars* S) {
  if (!S->active) return;
  const int ncells = nrows * ncols;
  __shared__ int nnext;
  int* src = bq;
  int* dst = bq + ncells;
  int n = *bqn;
  for (int level = 0; n > 0 && level < ncells; ++level) {
    if (threadIdx.x == 0) nnext = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int k = src[i];
      const int r = k % nrows, col = k / nrows;
      const int nb[4] = {r > 0 ? k - 1 : -1, r + 1 < nrows ? k + 1 : -1,
                         col > 0 ? k - nrows : -1, col + 1 < ncols ? k + nrows : -1};
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int q = nb[t];
        if (q < 0 || uf[q] >= 0) continue;  // outside, or empty
        if (atomicCAS(&hops[q], -1, level + 1) == -1) dst[atomicAdd(&nnext, 1)] = q;
      }
    }
    __syncthreads();
    n = nnext;
    int* t = src;
    src = dst;
    dst = t;
    __syncthreads();
  }
}

// decide_actions' marks (:385-402) with compute_elfs (:266-343): the
// cell's distance (hops * min(hx, hy), DBL_MAX where no hop reached),
// refined within max(hx, hy) of the surface by the distance to the nearest
// exterior cell box among the two cells left and right in the row.
__global__ void k_elfs_mark(Particles p, const int* __restrict__ hops, const int* uf,
                            const int* eroot, Geom G, MsCfg c, int* act, int cap,
                            Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  const int nrows = G.nrows, ncols = G.ncols;
  const double hx = G.hx, hy = G.hy;
  const double h = (hx < hy) ? hx : hy;
  const double refine = (hx < hy) ? hy : hx;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap;
       i += gridDim.x * blockDim.x) {
    int a = KEEP;
    if (i < np) {
      const int cell = p.key[i];
      const int hc = hops[cell];
      const double base = hc >= 0 ? hc * h : DBL_MAX;
      double e = base;
      if (!(base > refine)) {
        const double px = p.x[i], py = p.y[i];
        const int r = cell % nrows, c0 = cell / nrows;
        for (int dc = -2; dc <= 2; ++dc) {
          const int cc = c0 + dc;
          if (cc < 0 || cc >= ncols) continue;
          if (!elfs_exterior(uf, eroot, r + nrows * cc)) continue;
          const double cx_lo = cc * hx, cx_hi = (cc + 1) * hx;
          const double cy_lo = r * hy, cy_hi = (r + 1) * hy;
          const double qx = px < cx_lo ? cx_lo : (px > cx_hi ? cx_hi : px);
          const double qy = py < cy_lo ? cy_lo : (py > cy_hi ? cy_hi : py);
          const double dx = px - qx, dy = py - qy;
          const double d = sqrt(dx * dx + dy * dy);
          if (d < e) e = d;
        }
      }
      const double r_i = sqrt(p.Ap[i]);
      const double div = p.vpx_dx[i] + p.vpy_dy[i];
      const int lvl = p.level[i];
      if ((e < c.alpha * r_i) || (div > c.stretch)) {
        if (lvl > c.min_level) a = SPLIT;
      } else if (e > c.beta * r_i && p.hp[i] > c.hp_min) {
        if (lvl < c.max_level) a = MERGE_PRIMARY;
      }
    }
    act[i] = a;
  }
}

// execute_merge_split (:513-717) for the field slots of k_ms_emit: a split
// leaves four children at (+-r/2, +-r/2) around the parent (r = sqrt(Ap),
// clamped into the domain) with the extensive fields divided by 4 and the
// momentum rebuilt; a merge leaves the centre of mass with the extensive
// fields summed, the rest mass-averaged and the primary's label.
__global__ void k_ms_emit_elfs(Fields in, Fields out, const int* act, const int* partner,
                               const int* offs, const int* oslot, const int* ridx,
                               int* out_idx, Geom G, long long cap, Scalars* S) {
  if (!S->active) return;
  const int np = S->np;
  const int nnew = offs[cap];
  if (nnew > cap) {  // the state goes through unchanged (the caller exchanges buffers)
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&S->status, kStatusCapacity);
    emit_identity(in, out, np, ridx, out_idx);
    return;
  }
  const double eps = 1e-10;
  const double Lx = G.ncols * G.hx, Ly = G.nrows * G.hy;
  auto clampx = [&](double w) { return w < eps ? eps : (w > Lx - eps ? Lx - eps : w); };
  auto clampy = [&](double w) { return w < eps ? eps : (w > Ly - eps ? Ly - eps : w); };
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const int a = act[i];
    const int os = oslot[i], orf = offs[ridx[i]];
    double v[kMsFields];
    if (a == KEEP) {
#pragma unroll
      for (int k = 0; k < kMsFields; ++k) v[k] = in.f[k][i];
      store_particle(out, out_idx, v, in.label[i], in.level[i], os, orf);
    } else if (a == SPLIT) {
      const double off = sqrt(in.f[11][i]) / 2.0;
      const double px = in.f[0][i], py = in.f[1][i];
      const double xs[4] = {clampx(px + off), clampx(px + off), clampx(px - off),
                            clampx(px - off)};
      const double ys[4] = {clampy(py + off), clampy(py - off), clampy(py + off),
                            clampy(py - off)};
      const int level = in.level[i];
#pragma unroll
      for (int k = 0; k < kMsFields; ++k) v[k] = in.f[k][i] / (extensive(k) ? 4.0 : 1.0);
      v[12] = v[8] * v[2];
      v[13] = v[8] * v[3];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        v[0] = xs[q]; v[1] = ys[q]; v[20] = xs[q]; v[21] = ys[q];
        store_particle(out, out_idx, v, -1, level - 1, os + q, orf + q);
      }
    } else if (a == MERGE_PRIMARY) {
      const int j = partner[i];
      const double M1 = in.f[8][i], M2 = in.f[8][j];
      const double Mt = M1 + M2;
#pragma unroll
      for (int k = 0; k < kMsFields; ++k)
        v[k] = extensive(k) ? (in.f[k][i] + in.f[k][j])
                            : (M1 * in.f[k][i] + M2 * in.f[k][j]) / Mt;
      v[20] = v[0];
      v[21] = v[1];
      v[12] = v[8] * v[2];
      v[13] = v[8] * v[3];
      store_particle(out, out_idx, v, in.label[i], in.level[i] + 1, os, orf);
    }
  }
}

bool ms_moving_slot_host(int k) { return k <= 10 || (k >= 16 && k <= 19); }

int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return int(b);
}

// exclusive scan of a[0..n) -> out[0..n] (a is zeroed), n = cap
int scan_enqueue(int* a, int* out, int n, int* tile_sum, int ntiles,
                 const Scalars* S, cudaStream_t st) {
  k_scan_sums<<<ntiles, kScanThreads, 0, st>>>(a, n, tile_sum, nullptr, S, 0, nullptr);
  k_scan_apply<<<ntiles, kScanThreads, 0, st>>>(a, n, tile_sum, out, nullptr, nullptr, S, 0,
                                                nullptr);
  return 2;
}

}  // namespace

int ms_enqueue(MsBuffers& m, Particles p, Particles q, const int* start, const int* perm,
               int ncells, Geom G, Phys P, const double* Z,
               const dampm_ms_params& cfg, Scalars* S, long long cap,
               cudaStream_t st, int use_step_dt, double dt, int variant,
               double stretch_thresh) {
  const bool elfs = variant == kMsElfs;
  MsCfg c{};
  c.alpha = cfg.alpha;
  c.beta = cfg.beta;
  c.split_hp_min = cfg.split_hp_min;
  c.shear_split = cfg.shear_split;
  c.hp_min = cfg.hp_min;
  c.max_dv = cfg.max_dv;
  c.min_level = cfg.min_level;
  c.max_level = cfg.max_level;
  c.min_ppc = cfg.min_particles_per_cell;
  c.max_ops = (long long)(int)cfg.max_ops;
  {
    const double min_h = (G.hy < G.hx) ? G.hy : G.hx;
    const double r = cfg.pair_dist * min_h;
    c.pair_gate2 = cfg.pair_dist > 0.0 ? r * r : 0.0;
  }
  c.dt_host = dt;
  c.use_step_dt = use_step_dt;
  c.split_w = 2;
  c.stretch = stretch_thresh;
  if (elfs) {  // main/merge_split_ops.h:406-497: a split counts 4, at least 2 per cell
    c.split_w = 4;
    c.min_ppc = 2;
    c.pair_gate2 = 0.0;
  }
  int n = 0;
  const int gp = grid_for(cap, 256);
  const int ic = int(cap);
  k_ms_reset_counts<<<1, 1, 0, st>>>(S);
  k_ms_materialize<<<gp, 256, 0, st>>>(p, P, S, m);
  // the state as the decision and the emit read it: moving fields at their
  // storage slots, the reference-order ones from the per-slot scratch
  Particles pv = p;
  pv.Ap = m.aps;
  pv.Fbx = m.fbxs;
  pv.Fby = m.fbys;
  pv.xp = m.xps;
  pv.yp = m.yps;
  pv.label = m.labs;
  pv.level = m.levs;
  n += 2;
  if (elfs) {
    const int gc = grid_for(ncells, 256);
    k_elfs_cells<<<gc, 256, 0, st>>>(start, ncells, m.uf, m.eroot, m.hops, m.bqn, S);
    k_elfs_union<<<gc, 256, 0, st>>>(m.uf, G.nrows, G.ncols, S);
    k_elfs_roots<<<gc, 256, 0, st>>>(m.uf, m.eroot, G.nrows, G.ncols, S);
    k_elfs_seeds<<<gc, 256, 0, st>>>(m.uf, m.eroot, m.hops, m.bq, m.bqn, G.nrows, G.ncols, S);
    k_elfs_bfs<<<1, 1024, 0, st>>>(m.uf, m.hops, m.bq, m.bqn, G.nrows, G.ncols, S);
    k_elfs_mark<<<gp, 256, 0, st>>>(pv, m.hops, m.uf, m.eroot, G, c, m.act, ic, S);
    n += 5;
  } else {
    k_ms_mark<<<gp, 256, 0, st>>>(pv, G, c, m.act, ic, S);
  }
  k_ms_init_partner<<<gp, 256, 0, st>>>(m.partner, ic, S);
  k_ms_split_flags<<<gp, 256, 0, st>>>(perm, m.act, m.flag, ic, S);
  n += 3;
  n += scan_enqueue(m.flag, m.rank, ic, m.tile_sum, m.ntiles, S, st);
  k_ms_split_cap<<<gp, 256, 0, st>>>(perm, m.rank, m.act, c, S);
  k_ms_count_cand<<<gp, 256, 0, st>>>(m.act, ic, S);
  k_ms_pair_parallel<<<grid_for(ncells, 128), 128, 0, st>>>(
      start, ncells, perm, m.act, m.partner, m.paired, p, c, S);
  k_ms_cand_flags<<<gp, 256, 0, st>>>(perm, m.act, m.flag, ic, c, S);
  n += 1 + scan_enqueue(m.flag, m.rank, ic, m.tile_sum, m.ntiles, S, st);
  k_ms_cand_list<<<gp, 256, 0, st>>>(m.rank, m.w, ic, c, S);
  k_ms_pair_serial<<<1, 1, 0, st>>>(start, perm, m.w, m.rank, ic, m.act, m.partner,
                                    m.paired, p, c, S);
  k_ms_demote<<<gp, 256, 0, st>>>(m.act, m.partner, c, S);
  n += 2;
  k_ms_weights<<<gp, 256, 0, st>>>(m.act, p.idx, m.w, m.flag, ic, c.split_w, S);
  n += 5;
  n += scan_enqueue(m.w, m.offs, ic, m.tile_sum, m.ntiles, S, st);
  n += scan_enqueue(m.flag, m.rank, ic, m.tile_sum, m.ntiles, S, st);
  Fields in{}, out{};
  double* pf[kMsFields] = {pv.x,   pv.y,   pv.vpx, pv.vpy, pv.hp,     pv.F11,
                           pv.F12, pv.F22, pv.Mp,  pv.Vp,  pv.H,      pv.Ap,
                           m.mx,   m.my,   pv.Fbx, pv.Fby, pv.vpx_dx, pv.vpx_dy,
                           pv.vpy_dx, pv.vpy_dy, pv.xp, pv.yp};
  double* qf[kMsFields] = {q.x,   q.y,   q.vpx, q.vpy, q.hp,     q.F11,
                           q.F12, q.F22, q.Mp,  q.Vp,  q.H,      nullptr,
                           nullptr, nullptr, nullptr, nullptr, q.vpx_dx, q.vpx_dy,
                           q.vpy_dx, q.vpy_dy, nullptr, nullptr};
  for (int k = 0; k < kMsFields; ++k) {
    in.f[k] = pf[k];
    out.f[k] = ms_moving_slot_host(k) ? qf[k] : m.sd[k];
  }
  in.label = pv.label;
  in.level = pv.level;
  out.label = m.slabel;
  out.level = m.slevel;
  if (elfs)
    k_ms_emit_elfs<<<gp, 256, 0, st>>>(in, out, m.act, m.partner, m.offs, m.rank, p.idx,
                                       q.idx, G, cap, S);
  else
    k_ms_emit<<<gp, 256, 0, st>>>(in, out, m.act, m.partner, m.offs, m.rank, p.idx, q.idx, G,
                                  cap, S);
  // the reference-order fields back into their arrays
  Fields fixed{};
  fixed.f[11] = p.Ap;
  fixed.f[14] = p.Fbx;
  fixed.f[15] = p.Fby;
  fixed.f[20] = p.xp;
  fixed.f[21] = p.yp;
  fixed.label = p.label;
  fixed.level = p.level;
  k_ms_copy_back<<<gp, 256, 0, st>>>(out, fixed, m.offs, cap, S);
  k_ms_finish<<<1, 1, 0, st>>>(m.offs, cap, S);
  // q (its moving fields written by the emit, the others shared) is the
  // state from here on
  k_ms_pair_mom<<<gp, 256, 0, st>>>(m.sd[12], m.sd[13], q, S);
  launch_prep<double>(gp, 256, st, q, Z, G, P, S, 0);
  n += 5;
  return n;
}

}  // namespace dampm
