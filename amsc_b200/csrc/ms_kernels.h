// ms_kernels.h -- adaptive merge/split on the device
// (main/merge_split_ops_cmes.h:116-447).
#pragma once
#include <cuda_runtime.h>

#include "../../include/dampm_cuda.h"
#include "dampm_kernels.h"

namespace dampm {

// particle fields carried through a merge/split emit (doubles)
constexpr int kMsFields = 22;

struct MsBuffers {
  int *act = nullptr, *partner = nullptr, *w = nullptr, *offs = nullptr;
  int *flag = nullptr, *rank = nullptr, *paired = nullptr, *tile_sum = nullptr;
  int ntiles = 0;
  long long cap = 0;
  double* stage = nullptr;  // one field of scratch (also a download staging area)
  double* sd[kMsFields] = {};
  double *mx = nullptr, *my = nullptr;  // the momentum pair as two fields
  int *slabel = nullptr, *slevel = nullptr;
  // the reference-order fields of each storage slot for the decision and
  // the emit (Ap and Fb derived or gathered, xp, yp, label, level gathered
  // through idx), so that a call works on the sorted storage as it lies
  double *aps = nullptr, *fbxs = nullptr, *fbys = nullptr, *xps = nullptr, *yps = nullptr;
  int *labs = nullptr, *levs = nullptr;
  // the ELFS variant's cell arrays (allocated when it is selected): the
  // empty cells' union-find forest (-1: a cell with particles), the roots
  // that reach the grid edge, the hop counts from the free surface, the
  // two frontier queues of the search and its counter
  int *uf = nullptr, *eroot = nullptr, *hops = nullptr, *bq = nullptr, *bqn = nullptr;
  int elfs_cells = 0;
};

template <class Alloc>
int ms_alloc(MsBuffers& m, long long cap, int /*ncells*/, Alloc alloc) {
  m.cap = cap;
  m.ntiles = int((cap + kScanTile - 1) / kScanTile);
  int** ints[] = {&m.act, &m.partner, &m.w, &m.offs, &m.flag, &m.rank,
                        &m.paired, &m.slabel, &m.slevel, &m.labs, &m.levs};
  for (int** q : ints) {
    int rc = alloc((void**)q, sizeof(int) * size_t(cap + 1));
    if (rc) return rc;
  }
  int rc = alloc((void**)&m.tile_sum, sizeof(int) * size_t(m.ntiles + 1));
  if (rc) return rc;
  rc = alloc((void**)&m.stage, sizeof(double) * size_t(cap));
  if (rc) return rc;
  for (int k = 0; k < kMsFields; ++k) {
    rc = alloc((void**)&m.sd[k], sizeof(double) * size_t(cap));
    if (rc) return rc;
  }
  rc = alloc((void**)&m.mx, sizeof(double) * size_t(cap));
  if (rc) return rc;
  rc = alloc((void**)&m.my, sizeof(double) * size_t(cap));
  if (rc) return rc;
  double** dd[] = {&m.aps, &m.fbxs, &m.fbys, &m.xps, &m.yps};
  for (double** q : dd) {
    rc = alloc((void**)q, sizeof(double) * size_t(cap));
    if (rc) return rc;
  }
  return 0;
}

template <class Alloc>
int ms_alloc_elfs(MsBuffers& m, int ncells, Alloc alloc) {
  if (m.elfs_cells >= ncells) return 0;
  int** arr[] = {&m.uf, &m.eroot, &m.hops};
  for (int** q : arr) {
    int rc = alloc((void**)q, sizeof(int) * size_t(ncells + 1));
    if (rc) return rc;
  }
  int rc = alloc((void**)&m.bq, sizeof(int) * 2 * size_t(ncells + 1));
  if (rc) return rc;
  rc = alloc((void**)&m.bqn, sizeof(int) * 4);
  if (rc) return rc;
  m.elfs_cells = ncells;
  return 0;
}

// The merge/split a context runs: the one gpu_offload calls
// (main/merge_split_ops_cmes.h) or the ELFS variant (main/merge_split_ops.h).
enum MsVariant { kMsCmes = DAMPM_MS_CMES, kMsElfs = DAMPM_MS_ELFS };

// Enqueues one adaptive_merge_split on the current binning (start/perm must
// describe the current positions).  dt comes from the step's device scalar
// when use_step_dt, else `dt`.  Returns the number of kernel launches.
// p: the state (its storage in the sorted order of the last step, idx the
// reference index of each slot), q: the free half of its double buffer,
// which receives the emitted particles in the compacted reference order and
// holds the state afterwards (the caller exchanges the two).
int ms_enqueue(MsBuffers& m, Particles p, Particles q, const int* start, const int* perm,
               int ncells, Geom G, Phys P, const double* Z,
               const dampm_ms_params& cfg, Scalars* S, long long cap,
               cudaStream_t stream, int use_step_dt, double dt, int variant = kMsCmes,
               double stretch_thresh = 1e7);

}  // namespace dampm
