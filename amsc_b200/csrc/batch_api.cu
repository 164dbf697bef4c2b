// batch_api.cu -- the extern "C" boundary of batches of independent scenarios
// (include/dampm_cuda.h, dampm_batch_*).
//
// A batch packs many scenarios (each its own grid, terrain, particles,
// rheology and loop: fixed dt for NSTEPS or CFL until T) back to back in one
// set of device arrays and advances all of them with one launch per kernel
// and pass.  Scenarios join at the end of the packed arrays (dampm_batch_add)
// and leave by being marked dead (dampm_batch_remove); dampm_batch_compact
// moves the live ones into the other half of a double buffer so that the
// freed room can be reused.  Merge/split and recorded outputs are not part of
// a batch.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dampm_cuda.h"
#include "dampm_kernels.h"
#include "host_util.h"

using namespace dampm;

namespace {

struct HostScn {
  int handle = -1;
  Scn d{};  // the device table entry
  dampm_grid grid{};
  dampm_params params{};
  long long nn = 0, nc = 0;
};

}  // namespace

struct dampm_batch {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long P_cap = 0, N_cap = 0;
  int S_cap = 0, STRIP_cap = 0, B_cap = 0;
  long long USEG_cap = 0;
  // packed totals (live and dead scenarios)
  long long P_tot = 0, N_tot = 0, C_tot = 0, useg_tot = 0;
  int strips_tot = 0, nblk = 0;
  std::vector<HostScn> scns;  // packed order = device table order
  int next_handle = 0;
  // device
  int precision = DAMPM_FP64;
  // the two halves of the double buffer of the moving particle fields: each
  // pass's G2P reads half `cur` and writes the other, and so does a
  // compaction; the fields that only an upload uses are shared
  ParticlesT<double> p64[2]{};  // FP64
  ParticlesT<float> p32[2]{};   // FP32 form
  double* Z[2] = {nullptr, nullptr};
  int cur = 0;  // half holding the particles; also the terrain's half
  int zcur = 0;
  void* vvL = nullptr;  // pairs (vvxL, vvyL) of the precision's real type
  double* stage = nullptr;  // one field in reference order, for downloads
  unsigned long long* sortbuf = nullptr;  // 2 x capacity: crowded cells' order
  int *count = nullptr, *start = nullptr, *perm = nullptr;
  int* skey = nullptr;  // the cell key of each sorted position
  int *tile_sum = nullptr, *clist = nullptr, *clist_n = nullptr, *cbig = nullptr;
  unsigned char* tflag = nullptr;  // the scan tiles of a pass (k_b_tile_flags)
  int* cmid = nullptr;  // cells with more than 16 particles
  int* ustart = nullptr;
  long long* upex = nullptr;
  int4* uplan = nullptr;  // {cA, cB, heavy, 0}
  int4* ulist = nullptr;
  int* uorder = nullptr;  // the order P2G takes the units in
  int *strip_n = nullptr, *ucount = nullptr, *strip_scn = nullptr;
  double* led_part = nullptr;
  int2 *scn_units = nullptr, *gblk = nullptr;
  int4 *mblk = nullptr, *nmove = nullptr;
  Scn* scn = nullptr;
  Scalars *S = nullptr, *Sg = nullptr;
  Scalars* Sh = nullptr;  // pinned mirror of S
  int p2g_grid = 1;
  long long launches = 0;
  // tuning: P2G units per CTA and the weight of a column in the unit plan
  int units_per_cta = kUnitsPerCta, col_weight = kColWeight;
  // kBatchGraphPasses passes captured in a CUDA graph, replayed while the
  // layout holds; one graph per half the passes start from
  int use_graphs = 1;
  bool graph_dirty[2] = {true, true};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  std::vector<void*> allocs;
  std::string err;
};

namespace {

#define BCK(call)                                                         \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      b->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      return DAMPM_ERR_CUDA;                                              \
    }                                                                     \
  } while (0)

int bfail(dampm_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

template <class T>
int balloc(dampm_batch* b, T** ptr, size_t n) {
  void* q = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess) {
    b->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return DAMPM_ERR_CUDA;
  }
  b->allocs.push_back(q);
  *ptr = static_cast<T*>(q);
  return DAMPM_OK;
}

template <class R>
ParticlesT<R>* halves(dampm_batch* b);
template <>
ParticlesT<double>* halves<double>(dampm_batch* b) { return b->p64; }
template <>
ParticlesT<float>* halves<float>(dampm_batch* b) { return b->p32; }

// the particle arrays of both halves: the moving fields of each half, and
// the fields only an upload uses (Ap, Fb, label, level) shared
template <class R>
int alloc_particles(dampm_batch* b, ParticlesT<R>* h) {
  for (int k = 0; k < 2; ++k) {
    MovingRefs<R> m = moving_refs(h[k]);
    for (int f = 0; f < kMovingR; ++f) {
      if (m.r[f] == &h[k].vpx_dx || m.r[f] == &h[k].vpx_dy || m.r[f] == &h[k].vpy_dx ||
          m.r[f] == &h[k].vpy_dy)
        continue;  // no gradients in a batch (no merge/split)
      int rc = balloc(b, m.r[f], size_t(b->P_cap));
      if (rc) return rc;
    }
    for (int f = 0; f < kMovingI; ++f) {
      int rc = balloc(b, m.i[f], size_t(b->P_cap));
      if (rc) return rc;
    }
    for (int f = 0; f < kMovingV; ++f) {
      int rc = balloc(b, m.v[f], size_t(b->P_cap));
      if (rc) return rc;
    }
  }
  R** f[] = {&h[0].Ap, &h[0].Fbx, &h[0].Fby};
  for (R** q : f) {
    int rc = balloc(b, q, size_t(b->P_cap));
    if (rc) return rc;
  }
  int** fi[] = {&h[0].label, &h[0].level};
  for (int** q : fi) {
    int rc = balloc(b, q, size_t(b->P_cap));
    if (rc) return rc;
  }
  h[1].Ap = h[0].Ap;
  h[1].Fbx = h[0].Fbx;
  h[1].Fby = h[0].Fby;
  h[1].label = h[0].label;
  h[1].level = h[0].level;
  return DAMPM_OK;
}

template <class R>
ParticlesT<R> shifted(const ParticlesT<R>& p, long long off) {
  ParticlesT<R> q = p;
  MovingRefs<R> m = moving_refs(q);
  for (R** d : m.r)
    if (*d) *d += off;
  for (int** d : m.i)
    if (*d) *d += off;
  for (V2<R>** d : m.v)
    if (*d) *d += off;
  R** f[] = {&q.Ap, &q.Fbx, &q.Fby};
  for (R** d : f)
    if (*d) *d += off;
  int** fi[] = {&q.label, &q.level};
  for (int** d : fi)
    if (*d) *d += off;
  return q;
}

int strips_of(const dampm_grid& g) { return (g.Ney + 1 + kTR - 1) / kTR; }

// Rebuilds the strip and G2P block tables from the host scenario list and
// uploads them with the scenario table and the batch totals.
int upload_tables(dampm_batch* b) {
  std::vector<int> strip_scn(std::max(b->strips_tot, 1));
  std::vector<int2> gblk;
  gblk.reserve(b->nblk);
  std::vector<Scn> tab(b->scns.size());
  for (size_t s = 0; s < b->scns.size(); ++s) {
    const Scn& d = b->scns[s].d;
    tab[s] = d;
    for (int k = 0; k < d.nstrips; ++k) strip_scn[d.strip_off + k] = int(s);
    for (int f = 0; f < d.np; f += kG2PThreads) gblk.push_back(make_int2(int(s), f));
  }
  b->nblk = int(gblk.size());
  if (!tab.empty())
    BCK(cudaMemcpyAsync(b->scn, tab.data(), sizeof(Scn) * tab.size(),
                        cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->strip_scn, strip_scn.data(), sizeof(int) * strip_scn.size(),
                      cudaMemcpyHostToDevice, b->stream));
  if (!gblk.empty())
    BCK(cudaMemcpyAsync(b->gblk, gblk.data(), sizeof(int2) * gblk.size(),
                        cudaMemcpyHostToDevice, b->stream));
  Scalars g{};
  g.np = int(b->P_tot);
  g.active = 1;
  // the next sort scans every cell of the new layout
  g.krange[0] = 0x7fffffff;
  g.krange[1] = -1;
  g.knext[0] = 0;
  g.knext[1] = int(std::max<long long>(b->C_tot, 1)) - 1;
  BCK(cudaMemcpyAsync(b->Sg, &g, sizeof(Scalars), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));  // host vectors die here
  b->graph_dirty[0] = b->graph_dirty[1] = true;  // launch sizes or buffers changed
  return DAMPM_OK;
}

int find(dampm_batch* b, int handle) {
  for (size_t s = 0; s < b->scns.size(); ++s)
    if (b->scns[s].handle == handle) return int(s);
  return -1;
}

int read_scalars(dampm_batch* b) {
  if (b->scns.empty()) return DAMPM_OK;
  BCK(cudaMemcpyAsync(b->Sh, b->S, sizeof(Scalars) * b->scns.size(),
                      cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return DAMPM_OK;
}

// One pass of every live scenario: kPassLaunches kernel launches.
constexpr int kPassLaunches = 14;
int enqueue_pass(dampm_batch* b) {
  cudaStream_t st = b->stream;
  const int nscn = int(b->scns.size());
  const int ncell = int(std::max<long long>(b->C_tot, 1));
  const int ntiles = (ncell + kScanTile - 1) / kScanTile;
  const int nxt = 1 - b->cur;
  const int* key = b->precision == DAMPM_FP32 ? b->p32[b->cur].key : b->p64[b->cur].key;
  const int* slot = b->precision == DAMPM_FP32 ? b->p32[b->cur].slot : b->p64[b->cur].slot;
  const int* idx = b->precision == DAMPM_FP32 ? b->p32[b->cur].idx : b->p64[b->cur].idx;
  k_b_step_begin<<<1, 1024, 0, st>>>(b->scn, b->S, nscn, b->Sg);
  const int gp = grid_blocks(b->P_tot, 256);
  // the counting sort of every scenario at once (G2P counted the keys), over
  // the tiles the scenarios' key ranges meet
  k_b_tile_flags<<<grid_blocks(ntiles, 256), 256, 0, st>>>(b->scn, b->S, nscn, b->Sg,
                                                            b->tflag, ntiles);
  k_scan_sums<<<ntiles, kScanThreads, 0, st>>>(b->count, ncell, b->tile_sum, b->clist_n,
                                               b->Sg, 0, b->tflag);
  k_scan_apply<<<ntiles, kScanThreads, 0, st>>>(b->count, ncell, b->tile_sum, b->start,
                                                b->clist, b->clist_n, b->Sg, 0, b->tflag);
  k_scatter<<<gp, 256, 0, st>>>(key, slot, idx, b->start, b->perm, b->skey, b->sortbuf,
                                b->Sg);
  k_segment_order<<<148 * 4, 256, 0, st>>>(b->start, b->clist, b->clist_n, b->perm,
                                            b->sortbuf, b->cmid, b->Sg);
  k_segment_order_mid<<<148 * 8, 256, 0, st>>>(b->start, b->cmid, b->clist_n, b->perm,
                                                b->sortbuf, b->cbig, b->Sg);
  k_segment_order_big<<<148, 1024, sort_big_smem_bytes(), st>>>(b->start, b->cbig, b->clist_n, b->perm,
                                            b->sortbuf, b->P_cap, b->Sg);
  k_b_units_plan<<<b->strips_tot, kPlanThreads, 0, st>>>(
      b->start, b->scn, b->S, b->strip_scn, b->Sg, b->units_per_cta * b->p2g_grid,
      b->col_weight, b->ustart, b->upex, b->uplan, b->strip_n, b->ucount + 3);
  k_b_units_flat<<<1, kPlanThreads, sizeof(int) * (b->strips_tot + 1), st>>>(
      b->strip_n, b->strips_tot, b->strip_scn, b->scn, nscn, b->uplan, b->ulist, b->uorder,
      b->ucount, b->scn_units, b->S, b->Sg);
  if (b->precision == DAMPM_FP32)
    launch_b_p2g<float>(b->p2g_grid, st, b->p32[b->cur], b->perm, b->start,
                        static_cast<float2*>(b->vvL),
                        b->led_part, b->scn, b->S, b->ulist, b->uorder, b->ucount, b->Sg);
  else
    launch_b_p2g<double>(b->p2g_grid, st, b->p64[b->cur], b->perm, b->start,
                         static_cast<double2*>(b->vvL),
                         b->led_part, b->scn, b->S, b->ulist, b->uorder, b->ucount, b->Sg);
  k_b_ledger<<<nscn, 256, 0, st>>>(b->led_part, b->scn_units, b->scn, b->S, nscn,
                                   b->Sg);
  if (b->precision == DAMPM_FP32)
    launch_b_g2p<float>(b->nblk, st, b->p32[b->cur], b->p32[nxt], b->perm, b->skey,
                        static_cast<const float2*>(b->vvL), b->Z[b->zcur], b->scn, b->S,
                        b->gblk, b->Sg, b->count);
  else
    launch_b_g2p<double>(b->nblk, st, b->p64[b->cur], b->p64[nxt], b->perm, b->skey,
                         static_cast<const double2*>(b->vvL), b->Z[b->zcur], b->scn, b->S,
                         b->gblk, b->Sg, b->count);
  k_b_step_end<<<1, 1024, 0, st>>>(b->scn, b->S, nscn);
  b->cur = nxt;
  b->launches += kPassLaunches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(b, DAMPM_ERR_CUDA, cudaGetErrorString(e));
  return DAMPM_OK;
}

// Particles of one scenario into the current half (converted to R on the
// host), then the initial state of main/optim_par.cpp:239-264 on the device.
template <class R>
int upload_scenario(dampm_batch* b, const Scn& d, int pos, long long np,
                    const double* const* in, double* Zs) {
  ParticlesT<R> p = shifted(halves<R>(b)[b->cur], d.p_off);
  // in: x, y, Mp, Ap, vpx, vpy, hp, mom_px, mom_py, Vp
  R* dst[10] = {p.x, p.y, p.Mp, p.Ap, p.vpx, p.vpy, p.hp, nullptr, nullptr, p.Vp};
  cudaStream_t st = b->stream;
  std::vector<R> tmp, tmp2;
  auto host_r = [&](int k, std::vector<R>& t) -> const R* {
    if (sizeof(R) == sizeof(double)) return reinterpret_cast<const R*>(in[k]);
    t.assign(in[k], in[k] + np);
    return t.data();
  };
  for (int k = 0; k < 10; ++k) {
    if (!dst[k]) continue;
    BCK(cudaMemcpyAsync(dst[k], host_r(k, tmp), sizeof(R) * size_t(np),
                        cudaMemcpyHostToDevice, st));
    if (sizeof(R) != sizeof(double)) BCK(cudaStreamSynchronize(st));  // tmp is reused
  }
  BCK(upload_pair(p.mp, host_r(7, tmp), host_r(8, tmp2), np, st));
  BCK(cudaStreamSynchronize(st));
  // (the terrain gradients only feed recorded outputs, which a batch does
  // not keep, so Z stands in for them)
  launch_init_particles<R>(grid_blocks(np, 256), 256, st, p, Zs, Zs, Zs, d.G, d.P,
                           b->S + pos, int(np), d.c_off);
  // the new keys join the counts the last pass left for the next sort
  k_count_n<<<grid_blocks(np, 256), 256, 0, st>>>(p.key, b->count, p.slot, int(np));
  launch_prep<R>(grid_blocks(np, 256), 256, st, p, Zs, d.G, d.P, b->S + pos, 0);
  b->launches += 3;
  BCK(cudaGetLastError());
  return DAMPM_OK;
}

// out[idx[j]] = a[j] over one scenario's n particles (idx: its reference
// index), converted to double
template <class R>
__global__ void k_b_to_ref(const R* __restrict__ a, const int* __restrict__ idx,
                           double* __restrict__ out, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    out[idx[j]] = double(a[j]);
}

template <class R>
__global__ void k_b_pair_to_ref(const V2<R>* __restrict__ a, int half,
                                const int* __restrict__ idx, double* __restrict__ out,
                                int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const V2<R> v = a[j];
    out[idx[j]] = double(half ? v.y : v.x);
  }
}

template <class R>
int download_field(dampm_batch* b, const Scn& d, const std::string& f, double* out) {
  const ParticlesT<R> p = shifted(halves<R>(b)[b->cur], d.p_off);
  const R* src = nullptr;
  int pair_half = -1;  // mom_px / mom_py: one half of the momentum pair
  if (f == "x") src = p.x;
  else if (f == "y") src = p.y;
  else if (f == "vpx") src = p.vpx;
  else if (f == "vpy") src = p.vpy;
  else if (f == "hp") src = p.hp;
  else if (f == "F_11") src = p.F11;
  else if (f == "F_12" || f == "F_21") src = p.F12;
  else if (f == "F_22") src = p.F22;
  else if (f == "Mp") src = p.Mp;
  else if (f == "Vp") src = p.Vp;
  else if (f == "H") src = p.H;
  else if (f == "mom_px" || f == "mom_py") pair_half = f == "mom_px" ? 0 : 1;
  if (!src && pair_half < 0)
    return bfail(b, DAMPM_ERR_UNKNOWN_FIELD, "unknown batch field " + f);
  if (d.np == 0) return DAMPM_OK;
  const int gp = grid_blocks(d.np, 256);
  if (pair_half >= 0)
    k_b_pair_to_ref<R><<<gp, 256, 0, b->stream>>>(p.mp, pair_half, p.idx, b->stage, d.np);
  else
    k_b_to_ref<R><<<gp, 256, 0, b->stream>>>(src, p.idx, b->stage, d.np);
  BCK(cudaGetLastError());
  BCK(cudaMemcpyAsync(out, b->stage, sizeof(double) * size_t(d.np), cudaMemcpyDeviceToHost,
                      b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return DAMPM_OK;
}

}  // namespace

extern "C" {

int dampm_batch_create(long long particle_cap, long long node_cap, int scenario_cap,
                       int precision, void* cuda_stream, dampm_batch** out) {
  if (!out || particle_cap < 1 || node_cap < 4 || scenario_cap < 1 ||
      particle_cap > 0x7fffffffLL || node_cap > 0x7fffffffLL)
    return DAMPM_ERR_ARG;
  if (precision != DAMPM_FP64 && precision != DAMPM_FP32) return DAMPM_ERR_ARG;
  dampm_batch* b = new dampm_batch();
  b->precision = precision;
  const bool f32 = precision == DAMPM_FP32;
  const size_t rsz = f32 ? sizeof(float) : sizeof(double);
  b->P_cap = particle_cap;
  b->N_cap = node_cap;
  b->S_cap = scenario_cap;
  b->STRIP_cap = kMaxStrips;
  // unit-plan slots: a scenario takes ceil((Ney+1)/30) * (Nex+1) of them,
  // at most nn/30 + (Nex+1)
  b->USEG_cap = node_cap / 24 + 2048LL * scenario_cap + 1024;
  b->B_cap = int(particle_cap / kG2PThreads) + scenario_cap + 1;
  if (cuda_stream) {
    b->stream = static_cast<cudaStream_t>(cuda_stream);
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete b;
      return DAMPM_ERR_CUDA;
    }
    b->own_stream = true;
  }
  int rc = f32 ? alloc_particles(b, b->p32) : alloc_particles(b, b->p64);
  const size_t nn = size_t(node_cap), pc = size_t(particle_cap);
  rc = rc ? rc : balloc(b, &b->stage, pc);
  rc = rc ? rc : balloc(b, &b->sortbuf, 2 * pc);
  rc = rc ? rc : balloc(b, &b->Z[0], nn);
  rc = rc ? rc : balloc(b, &b->Z[1], nn);
  rc = rc ? rc : balloc(b, reinterpret_cast<unsigned char**>(&b->vvL), 2 * nn * rsz);
  // cells of all scenarios: fewer than their nodes
  rc = rc ? rc : balloc(b, &b->count, nn + 4);
  rc = rc ? rc : balloc(b, &b->start, nn + 1);
  rc = rc ? rc : balloc(b, &b->clist, nn + 4);
  rc = rc ? rc : balloc(b, &b->clist_n, 4);
  rc = rc ? rc : balloc(b, &b->tile_sum, nn / kScanTile + 2);
  rc = rc ? rc : balloc(b, &b->tflag, nn / kScanTile + 2);
  rc = rc ? rc : balloc(b, &b->perm, pc);
  rc = rc ? rc : balloc(b, &b->skey, pc);
  rc = rc ? rc : balloc(b, &b->cbig, pc / 256 + 4);
  rc = rc ? rc : balloc(b, &b->cmid, pc / 17 + 4);
  const size_t us = size_t(b->USEG_cap);
  rc = rc ? rc : balloc(b, &b->ustart, us);
  rc = rc ? rc : balloc(b, &b->upex, us);
  rc = rc ? rc : balloc(b, &b->uplan, us);
  rc = rc ? rc : balloc(b, &b->ulist, us);
  rc = rc ? rc : balloc(b, &b->uorder, us);
  rc = rc ? rc : balloc(b, &b->led_part, us * 6);
  rc = rc ? rc : balloc(b, &b->strip_n, size_t(b->STRIP_cap));
  rc = rc ? rc : balloc(b, &b->strip_scn, size_t(b->STRIP_cap));
  rc = rc ? rc : balloc(b, &b->ucount, 4);
  if (rc == DAMPM_OK && cudaMemsetAsync(b->ucount, 0, sizeof(int) * 4, b->stream) != cudaSuccess)
    rc = bfail(b, DAMPM_ERR_CUDA, "cudaMemsetAsync failed");
  rc = rc ? rc : balloc(b, &b->scn_units, size_t(scenario_cap));
  rc = rc ? rc : balloc(b, &b->gblk, size_t(b->B_cap));
  rc = rc ? rc : balloc(b, &b->mblk, size_t(b->B_cap));
  rc = rc ? rc : balloc(b, &b->nmove, nn / kG2PThreads + size_t(scenario_cap) + 1);
  rc = rc ? rc : balloc(b, &b->scn, size_t(scenario_cap));
  rc = rc ? rc : balloc(b, &b->S, size_t(scenario_cap));
  rc = rc ? rc : balloc(b, &b->Sg, 1);
  if (rc == DAMPM_OK &&
      cudaMallocHost(&b->Sh, sizeof(Scalars) * size_t(scenario_cap)) != cudaSuccess)
    rc = bfail(b, DAMPM_ERR_CUDA, "cudaMallocHost failed");
  if (rc == DAMPM_OK) {
    cudaMemsetAsync(b->count, 0, sizeof(int) * (nn + 4), b->stream);
    cudaMemsetAsync(b->vvL, 0, 2 * rsz * nn, b->stream);
    cudaMemsetAsync(b->S, 0, sizeof(Scalars) * size_t(scenario_cap), b->stream);
    cudaMemsetAsync(b->Sg, 0, sizeof(Scalars), b->stream);
    const int per_sm = f32 ? setup_b_p2g<float>() : setup_b_p2g<double>();
    if (per_sm == 0) rc = bfail(b, DAMPM_ERR_CUDA, "cannot configure P2G shared memory");
    if (!setup_sort()) rc = bfail(b, DAMPM_ERR_CUDA, "cannot configure the sort's shared memory");
    int nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    b->p2g_grid = std::max(1, nsm * std::max(per_sm, 1));
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) rc = DAMPM_ERR_CUDA;
  }
  if (rc != DAMPM_OK) {
    dampm_batch_destroy(b);
    return rc;
  }
  *out = b;
  return DAMPM_OK;
}

int dampm_batch_destroy(dampm_batch* b) {
  if (!b) return DAMPM_ERR_ARG;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (cudaGraphExec_t g : b->graph)
    if (g) cudaGraphExecDestroy(g);
  for (void* q : b->allocs) cudaFree(q);
  if (b->Sh) cudaFreeHost(b->Sh);
  if (b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return DAMPM_OK;
}

const char* dampm_batch_last_error(dampm_batch* b) {
  return b ? b->err.c_str() : "null batch";
}

int dampm_batch_add(dampm_batch* b, const dampm_grid* grid, const dampm_params* params,
                    const double* Z, long long np, const double* x, const double* y,
                    const double* Mp, const double* Ap, const double* vpx,
                    const double* vpy, const double* hp, const double* mom_px,
                    const double* mom_py, const double* Vp, int* handle) {
  if (!b || !grid || !params || !Z || !handle || np < 1) return DAMPM_ERR_ARG;
  if (!x || !y || !Mp || !Ap || !vpx || !vpy || !hp || !mom_px || !mom_py || !Vp)
    return DAMPM_ERR_ARG;
  if (grid->Nex < 1 || grid->Ney < 1 || !(grid->hx > 0) || !(grid->hy > 0))
    return bfail(b, DAMPM_ERR_ARG, "bad grid");
  HostScn h;
  h.grid = *grid;
  h.params = *params;
  h.nn = (long long)(grid->Nex + 1) * (grid->Ney + 1);
  h.nc = (long long)grid->Nex * grid->Ney;
  const int nstrips = strips_of(*grid);
  const long long useg = (long long)nstrips * (grid->Nex + 1);
  const int blocks = int((np + kG2PThreads - 1) / kG2PThreads);
  if (int(b->scns.size()) >= b->S_cap || b->P_tot + np > b->P_cap ||
      b->N_tot + h.nn > b->N_cap || b->strips_tot + nstrips > b->STRIP_cap ||
      b->useg_tot + useg > b->USEG_cap || b->nblk + blocks > b->B_cap)
    return bfail(b, DAMPM_ERR_CAPACITY,
                 "batch full: remove finished scenarios and compact, or create a larger batch");
  Scn& d = h.d;
  d.G = make_geom(*grid);
  d.P = make_phys(*params);
  d.p_off = int(b->P_tot);
  d.np = int(np);
  d.n_off = int(b->N_tot);
  d.c_off = int(b->C_tot);
  d.strip_off = b->strips_tot;
  d.nstrips = nstrips;
  d.useg_off = int(b->useg_tot);
  d.live = 1;
  h.handle = b->next_handle++;
  const int pos = int(b->scns.size());
  // particles and terrain into the current half
  cudaStream_t st = b->stream;
  double* Zs = b->Z[b->zcur] + d.n_off;
  BCK(cudaMemcpyAsync(Zs, Z, sizeof(double) * size_t(h.nn), cudaMemcpyHostToDevice, st));
  Scalars s0{};
  s0.fresh = 1;
  s0.np = int(np);
  // the first plan covers all of the scenario's cells
  s0.krange[0] = 0x7fffffff;
  s0.krange[1] = -1;
  s0.knext[0] = d.c_off;
  s0.knext[1] = d.c_off + int(h.nc) - 1;
  b->Sh[pos] = s0;
  BCK(cudaMemcpyAsync(b->S + pos, b->Sh + pos, sizeof(Scalars), cudaMemcpyHostToDevice,
                      st));
  const double* in[10] = {x, y, Mp, Ap, vpx, vpy, hp, mom_px, mom_py, Vp};
  int urc = b->precision == DAMPM_FP32 ? upload_scenario<float>(b, d, pos, np, in, Zs)
                                       : upload_scenario<double>(b, d, pos, np, in, Zs);
  if (urc) return urc;
  BCK(cudaGetLastError());
  b->scns.push_back(h);
  b->P_tot += np;
  b->N_tot += h.nn;
  b->C_tot += h.nc;
  b->strips_tot += nstrips;
  b->useg_tot += useg;
  int rc = upload_tables(b);
  if (rc) return rc;
  *handle = h.handle;
  return DAMPM_OK;
}

int dampm_batch_remove(dampm_batch* b, int handle) {
  if (!b) return DAMPM_ERR_ARG;
  const int s = find(b, handle);
  if (s < 0) return bfail(b, DAMPM_ERR_ARG, "unknown scenario handle");
  b->scns[s].d.live = 0;
  b->scns[s].handle = -1;
  const int live = 0;
  BCK(cudaMemcpyAsync(reinterpret_cast<char*>(b->scn + s) + offsetof(Scn, live), &live,
                      sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return DAMPM_OK;
}

int dampm_batch_compact(dampm_batch* b) {
  if (!b) return DAMPM_ERR_ARG;
  bool any_dead = false;
  for (const HostScn& h : b->scns) any_dead |= !h.d.live;
  if (!any_dead) return DAMPM_OK;
  int rc = read_scalars(b);
  if (rc) return rc;
  std::vector<HostScn> keep;
  std::vector<Scalars> S;
  std::vector<int4> mv, nm;
  long long P = 0, N = 0, C = 0, U = 0;
  int strips = 0;
  for (size_t s = 0; s < b->scns.size(); ++s) {
    HostScn h = b->scns[s];
    if (!h.d.live) continue;
    const Scn old = h.d;
    h.d.p_off = int(P);
    h.d.n_off = int(N);
    h.d.c_off = int(C);
    h.d.strip_off = strips;
    h.d.useg_off = int(U);
    for (int f = 0; f < old.np; f += kG2PThreads)
      mv.push_back(make_int4(h.d.p_off + f, old.p_off + f,
                             std::min(kG2PThreads, old.np - f), h.d.c_off - old.c_off));
    for (long long f = 0; f < h.nn; f += kG2PThreads)
      nm.push_back(make_int4(int(h.d.n_off + f), int(old.n_off + f),
                             int(std::min<long long>(kG2PThreads, h.nn - f)), 0));
    P += old.np;
    N += h.nn;
    C += h.nc;
    strips += old.nstrips;
    U += (long long)old.nstrips * (h.grid.Nex + 1);
    S.push_back(b->Sh[s]);
    // its cells move: the first plan after the move covers all of them
    S.back().krange[0] = 0x7fffffff;
    S.back().krange[1] = -1;
    S.back().knext[0] = h.d.c_off;
    S.back().knext[1] = h.d.c_off + int(h.nc) - 1;
    keep.push_back(h);
  }
  const int nxt = 1 - b->cur, znxt = 1 - b->zcur;
  // the counts of the moved keys, for the next sort (the whole array: cells
  // beyond the new total may hold counts of removed scenarios, which a later
  // scenario's cells would otherwise inherit)
  BCK(cudaMemsetAsync(b->count, 0, sizeof(int) * size_t(b->N_cap + 4), b->stream));
  if (!mv.empty()) {
    BCK(cudaMemcpyAsync(b->mblk, mv.data(), sizeof(int4) * mv.size(),
                        cudaMemcpyHostToDevice, b->stream));
    if (b->precision == DAMPM_FP32)
      launch_b_move<float>(int(mv.size()), b->stream, b->p32[nxt], b->p32[b->cur], b->mblk);
    else
      launch_b_move<double>(int(mv.size()), b->stream, b->p64[nxt], b->p64[b->cur],
                            b->mblk);
    const int* key = b->precision == DAMPM_FP32 ? b->p32[nxt].key : b->p64[nxt].key;
    int* slot = b->precision == DAMPM_FP32 ? b->p32[nxt].slot : b->p64[nxt].slot;
    k_count_n<<<grid_blocks(P, 256), 256, 0, b->stream>>>(key, b->count, slot, int(P));
  }
  if (!nm.empty()) {
    BCK(cudaMemcpyAsync(b->nmove, nm.data(), sizeof(int4) * nm.size(),
                        cudaMemcpyHostToDevice, b->stream));
    k_b_move_nodes<<<int(nm.size()), kG2PThreads, 0, b->stream>>>(b->Z[znxt], b->Z[b->zcur],
                                                                  b->nmove);
  }
  for (size_t s = 0; s < S.size(); ++s) b->Sh[s] = S[s];
  if (!S.empty())
    BCK(cudaMemcpyAsync(b->S, b->Sh, sizeof(Scalars) * S.size(), cudaMemcpyHostToDevice,
                        b->stream));
  BCK(cudaGetLastError());
  b->cur = nxt;
  b->zcur = znxt;
  b->scns = keep;
  b->P_tot = P;
  b->N_tot = N;
  b->C_tot = C;
  b->strips_tot = strips;
  b->useg_tot = U;
  return upload_tables(b);
}

// Passes per graph: even, so that a replay ends on the half it began.
constexpr int kBatchGraphPasses = 16;

// The graph of kBatchGraphPasses passes from half h, captured after any
// change of layout (the launches' sizes and pointers depend only on the
// layout and on the half the passes start from; every other change lives in
// device memory).  Nothing runs.
int ensure_batch_graph(dampm_batch* b, int h) {
  if (!b->graph_dirty[h] && b->graph[h]) return DAMPM_OK;
  if (b->graph[h]) {
    cudaGraphExecDestroy(b->graph[h]);
    b->graph[h] = nullptr;
  }
  const int cur0 = b->cur;
  const long long l0 = b->launches;
  b->cur = h;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = DAMPM_OK;
  for (int k = 0; k < kBatchGraphPasses && rc == DAMPM_OK; ++k) rc = enqueue_pass(b);
  b->launches = l0;
  b->cur = cur0;  // nothing ran
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return bfail(b, DAMPM_ERR_CUDA, cudaGetErrorString(e));
  const cudaError_t ei = cudaGraphInstantiate(&b->graph[h], g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    b->graph[h] = nullptr;
    return bfail(b, DAMPM_ERR_CUDA, cudaGetErrorString(ei));
  }
  b->graph_dirty[h] = false;
  return DAMPM_OK;
}

int dampm_batch_step(dampm_batch* b, int nsteps) {
  if (!b || nsteps < 0) return DAMPM_ERR_ARG;
  if (b->scns.empty() || nsteps == 0) return DAMPM_OK;
  // no graph of our own inside the caller's capture
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool graphs = b->use_graphs &&
                      cudaStreamIsCapturing(b->stream, &cs) == cudaSuccess &&
                      cs == cudaStreamCaptureStatusNone;
  int left = nsteps;
  if (graphs && left >= kBatchGraphPasses) {
    const int h = b->cur;
    int rc = ensure_batch_graph(b, h);
    if (rc) return rc;
    for (; left >= kBatchGraphPasses; left -= kBatchGraphPasses) {
      BCK(cudaGraphLaunch(b->graph[h], b->stream));
      b->launches += (long long)kPassLaunches * kBatchGraphPasses;
    }
  }
  for (; left > 0; --left) {
    int rc = enqueue_pass(b);
    if (rc) return rc;
  }
  // the graph the next call starts from, captured now rather than inside it
  if (graphs) return ensure_batch_graph(b, b->cur);
  return DAMPM_OK;
}

int dampm_batch_tune(dampm_batch* b, int units_per_cta, int col_weight, int use_graphs) {
  if (!b || units_per_cta < 0 || col_weight < 0 || use_graphs < -1) return DAMPM_ERR_ARG;
  if (units_per_cta > 0) b->units_per_cta = units_per_cta;
  if (col_weight > 0) b->col_weight = col_weight;
  if (use_graphs >= 0) b->use_graphs = use_graphs;
  b->graph_dirty[0] = b->graph_dirty[1] = true;
  return DAMPM_OK;
}

int dampm_batch_sync(dampm_batch* b) {
  if (!b) return DAMPM_ERR_ARG;
  int rc = read_scalars(b);
  if (rc) return rc;
  for (size_t s = 0; s < b->scns.size(); ++s)
    if (b->scns[s].d.live && b->Sh[s].status)
      return bfail(b, DAMPM_ERR_DEVICE,
                   "a scenario's state diverged (non-finite or negative) and was stopped");
  return DAMPM_OK;
}

int dampm_batch_query(dampm_batch* b, int handle, int* it, double* t, double* dt_last,
                      int* running, long long* np) {
  if (!b) return DAMPM_ERR_ARG;
  const int s = find(b, handle);
  if (s < 0) return bfail(b, DAMPM_ERR_ARG, "unknown scenario handle");
  int rc = read_scalars(b);
  if (rc) return rc;
  const Scalars& S = b->Sh[s];
  const Phys& P = b->scns[s].d.P;
  if (it) *it = S.it;
  if (t) *t = S.t;
  if (dt_last) *dt_last = S.dt;
  // the loop condition of the next pass (main/optim_par.cpp:281)
  if (running) *running = (S.status == 0) && (P.fixed ? (S.it < P.NSTEPS) : (S.t < P.T));
  if (np) *np = b->scns[s].d.np;
  return S.status ? bfail(b, DAMPM_ERR_DEVICE, "device status word set") : DAMPM_OK;
}

int dampm_batch_download(dampm_batch* b, int handle, const char* field, double* out) {
  if (!b || !field || !out) return DAMPM_ERR_ARG;
  const int s = find(b, handle);
  if (s < 0) return bfail(b, DAMPM_ERR_ARG, "unknown scenario handle");
  const std::string f(field);
  return b->precision == DAMPM_FP32 ? download_field<float>(b, b->scns[s].d, f, out)
                                    : download_field<double>(b, b->scns[s].d, f, out);
}

int dampm_batch_ledgers(dampm_batch* b, int handle, double out[9]) {
  if (!b || !out) return DAMPM_ERR_ARG;
  const int s = find(b, handle);
  if (s < 0) return bfail(b, DAMPM_ERR_ARG, "unknown scenario handle");
  int rc = read_scalars(b);
  if (rc) return rc;
  for (int k = 0; k < 9; ++k) out[k] = b->Sh[s].ledger[k];
  return DAMPM_OK;
}

int dampm_batch_states(dampm_batch* b, int cap, int* handles, int* running, int* its,
                       double* ts, int* count) {
  if (!b || !count || cap < 0 || (cap > 0 && (!handles || !running || !its || !ts)))
    return DAMPM_ERR_ARG;
  int rc = read_scalars(b);
  if (rc) return rc;
  int n = 0;
  for (size_t s = 0; s < b->scns.size(); ++s) {
    const HostScn& h = b->scns[s];
    if (!h.d.live) continue;
    if (n >= cap) return bfail(b, DAMPM_ERR_ARG, "state arrays shorter than the live count");
    const Scalars& S = b->Sh[s];
    const Phys& P = h.d.P;
    handles[n] = h.handle;
    // a scenario stopped by its status word reports -1; the others go on
    running[n] = S.status ? -1 : (P.fixed ? (S.it < P.NSTEPS) : (S.t < P.T)) ? 1 : 0;
    its[n] = S.it;
    ts[n] = S.t;
    ++n;
  }
  *count = n;
  return DAMPM_OK;
}

int dampm_batch_usage(dampm_batch* b, long long out[8]) {
  if (!b || !out) return DAMPM_ERR_ARG;
  long long live = 0, dead = 0;
  for (const HostScn& h : b->scns) (h.d.live ? live : dead) += 1;
  out[0] = live;
  out[1] = dead;
  out[2] = b->P_tot;
  out[3] = b->P_cap;
  out[4] = b->N_tot;
  out[5] = b->N_cap;
  out[6] = b->S_cap;
  out[7] = b->launches;
  return DAMPM_OK;
}

}  // extern "C"
