// dampm_api.cu -- the extern "C" boundary (include/dampm_cuda.h).
//
// Host orchestration of the sm_100a step: device buffers owned by the
// context, all kernels enqueued on one stream, loop state kept on the device
// (Scalars) so that dampm_step() never synchronises.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dampm_cuda.h"
#include "dampm_kernels.h"
#include "ms_kernels.h"
#include "host_util.h"

using namespace dampm;

struct dampm_ctx {
  dampm_grid grid{};
  dampm_params params{};
  dampm_ms_params ms{};
  int precision = DAMPM_FP64;
  Geom G{};
  Phys P{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long cap = 0;
  int nn = 0, nc = 0;
  // p: the particles as the last pass left them (sorted by the cell of the
  // last binning); q: the other buffer of the moving fields, which the next
  // G2P (or a reordering) writes; the two are exchanged after each.
  Particles p{}, q{};
  Nodes nodes{};
  double *Z = nullptr, *dZdx = nullptr, *dZdy = nullptr;
  int *count = nullptr, *start = nullptr, *perm = nullptr, *tile_sum = nullptr;
  int* skey = nullptr;  // the cell of each sorted position
  unsigned long long* sortbuf = nullptr;  // 2 x capacity: crowded cells' order
  int ntiles = 0;
  double* led_part = nullptr;
  int n_led = 0;
  int strips = 0, useg = 0;  // strips; unit slots per strip (ncols + 1)
  int *ustart = nullptr, *strip_n = nullptr, *ucount = nullptr;
  long long* upex = nullptr;
  int4* uplan = nullptr;  // {cA, cB, heavy, 0}
  int4* ulist = nullptr;
  int* uorder = nullptr;  // the order P2G takes the units in
  int *clist = nullptr, *clist_n = nullptr;  // cells with >= 2 particles
  int* cbig = nullptr;  // cells with more than 256 particles (capacity / 256)
  int* cmid = nullptr;  // cells with more than 16 particles (capacity / 17)
  double* ledger_log = nullptr;  // kLedgerLog rows {t, err_mass, err_mom}
  int p2g_grid = 0;
  Scalars* S = nullptr;
  Scalars* Sh = nullptr;  // pinned host mirror
  MsBuffers msb{};
  bool terrain_ok = false, particles_ok = false;
  bool ms_enabled = false;
  int ms_variant = kMsCmes;       // which merge/split runs (ms_kernels.h)
  double ms_stretch = 1e7;        // the ELFS variant's divergence trigger
  bool record = false;
  bool record_alloc = false;
  long long it_host = 0;  // passes enqueued since upload (= device it while active)
  long long launches = 0;
  std::string err;
  std::vector<void*> allocs;
  // CUDA graphs of `passes` passes (kGraphPasses identical ones, or one
  // merge/split cycle from a given phase), each valid while its key (the
  // values the captured launches took by value -- buffers included, so the
  // parity of the particle buffers -- the cycle and its phase) is unchanged.
  // Two are kept: a merge/split cycle of odd length leaves the buffers
  // exchanged, so consecutive cycles alternate between two graphs.
  bool use_graphs = true;
  static constexpr int kKeyBytes = 2 * sizeof(Particles) + sizeof(Nodes) + sizeof(Geom) +
                                   sizeof(Phys) + sizeof(long long) + sizeof(int) +
                                   sizeof(dampm_ms_params) + sizeof(int) + sizeof(double) +
                                   3 * sizeof(int);
  struct GraphSlot {
    cudaGraphExec_t exec = nullptr;
    int passes = 0, phase = 0;
    long long launches = 0, used = 0;
    unsigned char key[kKeyBytes] = {};
  } graphs[2];
  long long graph_clock = 0;
  // slab mode (one scenario split over contexts by cell columns): the
  // leaver list G2P fills, scratch for the route, the particle count
  bool slab = false;
  int* leave = nullptr;
  int* sel = nullptr;        // slot lists (capacity)
  int* selcount = nullptr;   // one counter
  int2* moves = nullptr;     // hole fills (capacity)
  // staged downloads (dampm_stage_download): fields gathered into reference
  // order in `outbuf` on the step stream, copied to the host on `side`
  cudaStream_t side = nullptr;
  cudaEvent_t staged = nullptr;
  double* outbuf = nullptr;
  int outbuf_fields = 0;
  long long outbuf_cap = 0;
  bool side_pending = false;
  // timing
  bool timing = false;
  std::vector<cudaEvent_t> evpool;
  int evused = 0;
  std::vector<int> evclass;  // class of the interval ending at event k
};

namespace {

#define CK(call)                                                          \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
      return DAMPM_ERR_CUDA;                                              \
    }                                                                     \
  } while (0)

int fail(dampm_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

template <class T>
int dalloc(dampm_ctx* ctx, T** ptr, size_t n) {
  void* q = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess) {
    ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return DAMPM_ERR_CUDA;
  }
  ctx->allocs.push_back(q);
  *ptr = static_cast<T*>(q);
  return DAMPM_OK;
}

int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return int(b);
}

void ev_mark(dampm_ctx* ctx, int cls) {
  if (!ctx->timing) return;
  if (ctx->evused == (int)ctx->evpool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ctx->evpool.push_back(e);
    ctx->evclass.push_back(0);
  }
  ctx->evclass[ctx->evused] = cls;
  cudaEventRecord(ctx->evpool[ctx->evused], ctx->stream);
  ctx->evused++;
}

// q shares p's fields that the step does not move
void share_fixed(dampm_ctx* ctx) {
  Particles& p = ctx->p;
  Particles& q = ctx->q;
  q.label = p.label;
  q.level = p.level;
  q.xp = p.xp;
  q.yp = p.yp;
  q.Ap = p.Ap;
  q.Fbx = p.Fbx;
  q.Fby = p.Fby;
  q.apx = p.apx;
  q.apy = p.apy;
  q.Zp = p.Zp;
  q.hpZ = p.hpZ;
  q.dZxp = p.dZxp;
  q.dZyp = p.dZyp;
  q.Fpx = p.Fpx;
  q.Fpy = p.Fpy;
  q.Frx = p.Frx;
  q.Fry = p.Fry;
}

int alloc_record(dampm_ctx* ctx) {
  if (ctx->record_alloc) return DAMPM_OK;
  const long long cap = ctx->cap;
  Particles& p = ctx->p;
  double** pf[] = {&p.apx, &p.apy, &p.Zp, &p.hpZ, &p.dZxp, &p.dZyp,
                   &p.Fpx, &p.Fpy, &p.Frx, &p.Fry};
  for (double** q : pf) {
    int rc = dalloc(ctx, q, cap);
    if (rc) return rc;
    CK(cudaMemsetAsync(*q, 0, cap * sizeof(double), ctx->stream));
  }
  Nodes& n = ctx->nodes;
  double** nf[] = {&n.Mv,   &n.mvx,  &n.mvy,   &n.avx,   &n.avy,
                   &n.vvx,  &n.vvy,  &n.FPxv,  &n.FPyv,  &n.Fricx,
                   &n.Fricy, &n.Fintx, &n.Finty, &n.HV};
  for (double** q : nf) {
    int rc = dalloc(ctx, q, ctx->nn);
    if (rc) return rc;
    CK(cudaMemsetAsync(*q, 0, ctx->nn * sizeof(double), ctx->stream));
  }
  share_fixed(ctx);
  ctx->record_alloc = true;
  return DAMPM_OK;
}

int alloc_particles(dampm_ctx* ctx, long long cap) {
  ctx->cap = cap;
  for (Particles* pp : {&ctx->p, &ctx->q}) {
    MovingRefs<double> m = moving_refs(*pp);
    for (double** f : m.r) {
      int rc = dalloc(ctx, f, cap);
      if (rc) return rc;
      CK(cudaMemsetAsync(*f, 0, cap * sizeof(double), ctx->stream));
    }
    for (int** f : m.i) {
      int rc = dalloc(ctx, f, cap);
      if (rc) return rc;
      CK(cudaMemsetAsync(*f, 0, cap * sizeof(int), ctx->stream));
    }
    for (double2** f : m.v) {
      int rc = dalloc(ctx, f, cap);
      if (rc) return rc;
      CK(cudaMemsetAsync(*f, 0, cap * sizeof(double2), ctx->stream));
    }
  }
  Particles& p = ctx->p;
  double** f[] = {&p.Ap, &p.Fbx, &p.Fby, &p.xp, &p.yp};
  for (double** q : f) {
    int rc = dalloc(ctx, q, cap);
    if (rc) return rc;
    CK(cudaMemsetAsync(*q, 0, cap * sizeof(double), ctx->stream));
  }
  int** fi[] = {&p.label, &p.level, &ctx->perm, &ctx->skey};
  for (int** q : fi) {
    int rc = dalloc(ctx, q, cap);
    if (rc) return rc;
  }
  {
    int rc = dalloc(ctx, &ctx->sortbuf, size_t(2 * cap));
    if (rc) return rc;
    rc = dalloc(ctx, &ctx->cbig, size_t(cap / 256 + 4));
    if (rc) return rc;
    rc = dalloc(ctx, &ctx->cmid, size_t(cap / 17 + 4));
    if (rc) return rc;
  }
  share_fixed(ctx);
  int rc = ms_alloc(ctx->msb, cap, ctx->nc, [&](void** q, size_t bytes) {
    return dalloc(ctx, reinterpret_cast<unsigned char**>(q), bytes);
  });
  if (rc) return rc;
  if (ctx->record) return alloc_record(ctx);
  return DAMPM_OK;
}

// Enqueues the binning of the current particles (SORT), whose slots and
// counts are in hand (from G2P, or from k_count after an upload, a state
// upload or a merge/split).
void enqueue_sort(dampm_ctx* ctx) {
  const int gp = grid_for(ctx->cap, 256);
  k_scan_sums<<<ctx->ntiles, kScanThreads, 0, ctx->stream>>>(ctx->count, ctx->nc,
                                                             ctx->tile_sum, ctx->clist_n,
                                                             ctx->S, 1, nullptr);
  k_scan_apply<<<ctx->ntiles, kScanThreads, 0, ctx->stream>>>(
      ctx->count, ctx->nc, ctx->tile_sum, ctx->start, ctx->clist, ctx->clist_n, ctx->S, 1,
      nullptr);
  k_scatter<<<gp, 256, 0, ctx->stream>>>(ctx->p.key, ctx->p.slot, ctx->p.idx, ctx->start,
                                         ctx->perm, ctx->skey, ctx->sortbuf, ctx->S);
  k_segment_order<<<148 * 4, 256, 0, ctx->stream>>>(ctx->start, ctx->clist,
                                                   ctx->clist_n, ctx->perm, ctx->sortbuf,
                                                   ctx->cmid, ctx->S);
  k_segment_order_mid<<<148 * 8, 256, 0, ctx->stream>>>(ctx->start, ctx->cmid,
                                                       ctx->clist_n, ctx->perm, ctx->sortbuf,
                                                       ctx->cbig, ctx->S);
  k_segment_order_big<<<148, 1024, sort_big_smem_bytes(), ctx->stream>>>(ctx->start, ctx->cbig, ctx->clist_n,
                                                     ctx->perm, ctx->sortbuf, ctx->cap,
                                                     ctx->S);
  ctx->launches += 6;
}

// One pass of the loop body in two halves: step start, sort and P2G; then
// G2P and step end (slab mode exchanges node columns between them).
int enqueue_front(dampm_ctx* ctx) {
  const long long it_next = ctx->it_host + 1;
  const bool ms_due = ctx->ms_enabled && ctx->params.MERGE_SPLIT_ON != 0 &&
                      ctx->ms.call_interval > 0 &&
                      (it_next % ctx->ms.call_interval) == 0;
  ev_mark(ctx, 3);
  k_step_begin<<<1, 1, 0, ctx->stream>>>(ctx->S, ctx->G, ctx->P);
  ctx->launches += 1;
  if (ms_due) {  // on the binning of the particles as they lie in storage
    enqueue_sort(ctx);
    ctx->launches += ms_enqueue(ctx->msb, ctx->p, ctx->q, ctx->start, ctx->perm, ctx->nc,
                                ctx->G, ctx->P, ctx->Z, ctx->ms, ctx->S, ctx->cap,
                                ctx->stream, /*use_step_dt=*/1, 0.0, ctx->ms_variant,
                                ctx->ms_stretch);
    swap_moving(ctx->p, ctx->q);
    k_keys<<<grid_for(ctx->cap, 256), 256, 0, ctx->stream>>>(ctx->p, ctx->G, ctx->S, 0);
    k_count<<<grid_for(ctx->cap, 256), 256, 0, ctx->stream>>>(ctx->p.key, ctx->count,
                                                             ctx->p.slot, ctx->S);
    ctx->launches += 2;
  }
  ev_mark(ctx, 0);
  enqueue_sort(ctx);
  ev_mark(ctx, 1);
  k_units_plan<<<ctx->strips, kPlanThreads, 0, ctx->stream>>>(
      ctx->start, ctx->G, ctx->S, kUnitsPerCta * ctx->p2g_grid, ctx->useg, ctx->ustart,
      ctx->upex, ctx->uplan, ctx->strip_n, ctx->ucount + 3);
  k_units_flat<<<1, kPlanThreads, sizeof(int) * (ctx->strips + 1), ctx->stream>>>(
      ctx->strip_n, ctx->strips, ctx->useg, ctx->uplan, ctx->ulist, ctx->uorder, ctx->ucount,
      ctx->S);
  if (ctx->record) {
    Nodes& n = ctx->nodes;
    double* nf[] = {n.Mv,  n.mvx,  n.mvy,   n.avx,   n.avy,  n.vvx, n.vvy,
                    n.FPxv, n.FPyv, n.Fricx, n.Fricy, n.Fintx, n.Finty};
    for (double* q : nf)
      cudaMemsetAsync(q, 0, sizeof(double) * ctx->nn, ctx->stream);
    cudaMemsetAsync(n.vvL, 0, sizeof(double2) * ctx->nn, ctx->stream);
  }
  launch_p2g(ctx->p2g_grid, ctx->stream, ctx->p, ctx->perm, ctx->start, ctx->nodes,
             ctx->led_part, ctx->G, ctx->P, ctx->S, ctx->record ? 1 : 0, ctx->ulist, ctx->uorder,
             ctx->ucount);
  ctx->launches += 2;
  ev_mark(ctx, 3);
  k_ledger_final<<<1, 1024, 0, ctx->stream>>>(ctx->led_part, ctx->ucount, ctx->S,
                                               ctx->ledger_log);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, DAMPM_ERR_CUDA, cudaGetErrorString(e));
  return DAMPM_OK;
}

int enqueue_back(dampm_ctx* ctx) {
  const long long it_next = ctx->it_host + 1;
  // the pass after the merge/split call needs the gradients of this one
  const bool grad_next = ctx->ms_enabled && ctx->params.MERGE_SPLIT_ON != 0 &&
                         ctx->ms.call_interval > 0 &&
                         ((it_next + 1) % ctx->ms.call_interval) == 0;
  ev_mark(ctx, 2);
  launch_g2p(grid_for(ctx->cap, kG2PThreads), ctx->stream, ctx->p, ctx->q, ctx->perm,
             ctx->skey, ctx->nodes, ctx->Z, ctx->G, ctx->P, ctx->S, ctx->count, ctx->leave,
             ctx->record ? 1 : 0,
             (grad_next || ctx->record) ? 1 : 0);
  if (ctx->record) {
    k_hv<<<grid_for(ctx->nn, 256), 256, 0, ctx->stream>>>(ctx->q, ctx->start,
                                                           ctx->nodes.HV, ctx->G, ctx->S);
    ctx->launches += 1;
  }
  ev_mark(ctx, 3);
  k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->S);
  ctx->launches += 4;
  swap_moving(ctx->p, ctx->q);
  ctx->it_host = it_next;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, DAMPM_ERR_CUDA, cudaGetErrorString(e));
  return DAMPM_OK;
}

int enqueue_pass(dampm_ctx* ctx) {
  int rc = enqueue_front(ctx);
  return rc ? rc : enqueue_back(ctx);
}

// Passes can be replayed from a graph when they repeat: kGraphPasses alike
// without merge/split, or the call_interval passes of one merge/split cycle
// (which begin at the same phase of the cycle); not with recorded outputs or
// event timing, nor while the caller is capturing the stream.
constexpr int kGraphPasses = 16;
constexpr int kMaxGraphCycle = 64;

bool ms_cadence(const dampm_ctx* ctx) {
  return ctx->ms_enabled && ctx->params.MERGE_SPLIT_ON != 0 && ctx->ms.call_interval > 0;
}

// passes per graph (0: no graph) and the cycle phase the graph starts at
int graph_shape(const dampm_ctx* ctx, int* phase) {
  *phase = 0;
  if (!ms_cadence(ctx)) return kGraphPasses;
  const int L = ctx->ms.call_interval;
  if (L < 2 || L > kMaxGraphCycle) return 0;
  *phase = int(ctx->it_host % L);
  return L;
}

bool graph_eligible(dampm_ctx* ctx) {
  if (!ctx->use_graphs || ctx->timing || ctx->record) return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess ||
      cs != cudaStreamCaptureStatusNone)
    return false;
  return true;
}

void graph_key_of(const dampm_ctx* ctx, int passes, int phase, unsigned char* k) {
  size_t o = 0;
  auto put = [&](const void* v, size_t n) {
    std::memcpy(k + o, v, n);
    o += n;
  };
  put(&ctx->p, sizeof(Particles));
  put(&ctx->q, sizeof(Particles));
  put(&ctx->nodes, sizeof(Nodes));
  put(&ctx->G, sizeof(Geom));
  put(&ctx->P, sizeof(Phys));
  put(&ctx->cap, sizeof(long long));
  put(&ctx->p2g_grid, sizeof(int));
  put(&ctx->ms, sizeof(dampm_ms_params));
  put(&ctx->ms_variant, sizeof(int));
  put(&ctx->ms_stretch, sizeof(double));
  const int cyc[3] = {ms_cadence(ctx) ? 1 : 0, passes, phase};
  put(cyc, sizeof(cyc));
}

void drop_graphs(dampm_ctx* ctx) {
  for (auto& g : ctx->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = dampm_ctx::GraphSlot{};
  }
}

// A stream that cannot be captured (or a graph that cannot be built): the
// context launches plainly from then on.
int graphs_off(dampm_ctx* ctx) {
  cudaGetLastError();  // the capture's error is not the step's
  ctx->use_graphs = false;
  drop_graphs(ctx);
  return DAMPM_OK;
}

// The graph of `passes` passes from the current pass, captured unless one in
// hand was captured with the same buffers, parameters, cycle and phase
// (*out = null when graphs were turned off).
int ensure_graph(dampm_ctx* ctx, int passes, int phase, dampm_ctx::GraphSlot** out) {
  *out = nullptr;
  unsigned char key[dampm_ctx::kKeyBytes];
  graph_key_of(ctx, passes, phase, key);
  for (auto& g : ctx->graphs)
    if (g.exec && std::memcmp(key, g.key, sizeof(key)) == 0) {
      g.used = ++ctx->graph_clock;
      *out = &g;
      return DAMPM_OK;
    }
  dampm_ctx::GraphSlot* slot = &ctx->graphs[0];
  for (auto& g : ctx->graphs)
    if (!g.exec || g.used < slot->used) slot = &g;  // an empty slot, else the oldest
  if (slot->exec) cudaGraphExecDestroy(slot->exec);
  *slot = dampm_ctx::GraphSlot{};
  const long long it0 = ctx->it_host, l0 = ctx->launches;
  const Particles p0 = ctx->p, q0 = ctx->q;
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return graphs_off(ctx);
  int rc = DAMPM_OK;
  for (int k = 0; k < passes && rc == DAMPM_OK; ++k) rc = enqueue_pass(ctx);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  const long long captured = ctx->launches - l0;
  // nothing ran: the host's view of the passes and buffers goes back
  ctx->it_host = it0;
  ctx->launches = l0;
  ctx->p = p0;
  ctx->q = q0;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return graphs_off(ctx);
  }
  const cudaError_t ei = cudaGraphInstantiate(&slot->exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    slot->exec = nullptr;
    return graphs_off(ctx);
  }
  std::memcpy(slot->key, key, sizeof(key));
  slot->passes = passes;
  slot->phase = phase;
  slot->launches = captured;
  slot->used = ++ctx->graph_clock;
  *out = slot;
  return DAMPM_OK;
}

// The buffers after `passes` passes replayed from a graph: each pass
// exchanges them once, a merge/split pass once more (its emit writes the
// free half).
void advance_buffers(dampm_ctx* ctx, int passes) {
  int swaps = passes;
  if (ms_cadence(ctx)) {
    const int L = ctx->ms.call_interval;
    for (long long it = ctx->it_host + 1; it <= ctx->it_host + passes; ++it)
      if (it % L == 0) ++swaps;
  }
  if (swaps & 1) swap_moving(ctx->p, ctx->q);
}

// Reads the device scalars.  strict: a set status bit is returned as an
// error (the calls that report the status word); the data-out calls pass
// false so that a diverged state can still be inspected.
// The next sort scans every cell (after new particles or a new count).
void full_scan_next(const dampm_ctx* ctx, Scalars& s) {
  s.krange[0] = 0x7fffffff;
  s.krange[1] = -1;
  s.knext[0] = 0;
  s.knext[1] = ctx->nc - 1;
}

int sync_status(dampm_ctx* ctx, bool strict = true) {
  CK(cudaMemcpyAsync(ctx->Sh, ctx->S, sizeof(Scalars), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (!strict) return DAMPM_OK;
  if (ctx->Sh->status & kStatusCapacity)
    return fail(ctx, DAMPM_ERR_CAPACITY, "particle capacity exceeded by merge/split");
  if (ctx->Sh->status & kStatusNonFinite)
    return fail(ctx, DAMPM_ERR_DEVICE,
                "non-finite or negative particle state: the run diverged and was stopped");
  if (ctx->Sh->status)
    return fail(ctx, DAMPM_ERR_DEVICE, "device status word set");
  return DAMPM_OK;
}


// out[idx[j]] = a[j]: a field of the sorted slots into reference order
__global__ void k_to_ref(const double* __restrict__ a, const int* __restrict__ idx,
                         double* __restrict__ out, const Scalars* S) {
  const int np = S->np;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += gridDim.x * blockDim.x)
    out[idx[j]] = a[j];
}

// one half of a pair field into reference order
__global__ void k_pair_to_ref(const double2* __restrict__ a, int half,
                              const int* __restrict__ idx, double* __restrict__ out,
                              const Scalars* S) {
  const int np = S->np;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += gridDim.x * blockDim.x) {
    const double2 v = a[j];
    out[idx[j]] = half ? v.y : v.x;
  }
}

__global__ void k_int_to_double(const int* a, double* b, const Scalars* S) {
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x)
    b[i] = double(a[i]);
}

// Ap (which 0) and Fb as the reference stores them at the end of a step
// (main/optim_par.cpp:600-626), from the persistent state, into reference
// order.
__global__ void k_derived(Particles p, Phys P, const Scalars* S, int which,
                          double* out) {
  const int np = S->np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const double hp = p.hp[i];
    double v = 0.0;
    if (which == 0) {
      v = hp > 1.e-2 ? p.Vp[i] / hp : 0.0;
    }
    else {
      double fx, fy;
      voellmy(P, p.vpx[i], p.vpy[i], hp, fx, fy);
      v = (which == 3) ? fx : fy;  // which 3, 4: Fb_x, Fb_y
    }
    out[p.idx[i]] = v;
  }
}

constexpr int kMaxStaged = 64;  // fields per dampm_stage_download call

// Where a particle field comes from, as dampm_download names it.
struct FieldSrc {
  const double* sorted = nullptr;  // a field of the sorted slots
  const double* ref = nullptr;     // a field already in reference order
  const int* iref = nullptr;       // an integer field in reference order
  int derived = -1;                // Ap / Fb formed from the state
  int pair_half = -1;              // one half of the stored momentum pair
};

int resolve_field(dampm_ctx* ctx, const std::string& f, bool fresh, FieldSrc& r) {
  Particles& p = ctx->p;
  if (f == "x") r.sorted = p.x;
  else if (f == "y") r.sorted = p.y;
  else if (f == "Mp") r.sorted = p.Mp;
  else if (f == "Vp") r.sorted = p.Vp;
  else if (f == "H") r.sorted = p.H;
  else if (f == "hp") r.sorted = p.hp;
  else if (f == "vpx" || f == "vpxL") r.sorted = p.vpx;
  else if (f == "vpy" || f == "vpyL") r.sorted = p.vpy;
  else if (f == "F_11") r.sorted = p.F11;
  else if (f == "F_12" || f == "F_21") r.sorted = p.F12;
  else if (f == "F_22") r.sorted = p.F22;
  else if (f == "xp") r.ref = p.xp;
  else if (f == "yp") r.ref = p.yp;
  else if (f == "vpx_dx") r.sorted = p.vpx_dx;
  else if (f == "vpx_dy") r.sorted = p.vpx_dy;
  else if (f == "vpy_dx") r.sorted = p.vpy_dx;
  else if (f == "vpy_dy") r.sorted = p.vpy_dy;
  else if (f == "label") r.iref = p.label;
  else if (f == "level") r.iref = p.level;
  // fresh values (uploaded or emitted by merge/split) are kept in reference order
  else if (f == "Ap") { if (fresh) r.ref = p.Ap; else r.derived = 0; }
  else if (f == "mom_px" || f == "mom_py") r.pair_half = f == "mom_px" ? 0 : 1;
  else if (f == "Fb_x") { if (fresh) r.ref = p.Fbx; else r.derived = 3; }
  else if (f == "Fb_y") { if (fresh) r.ref = p.Fby; else r.derived = 4; }
  else if (ctx->record_alloc) {
    if (f == "apx") r.sorted = p.apx;
    else if (f == "apy") r.sorted = p.apy;
    else if (f == "Zp") r.sorted = p.Zp;
    else if (f == "hpZ") r.sorted = p.hpZ;
    else if (f == "dZxp") r.sorted = p.dZxp;
    else if (f == "dZyp") r.sorted = p.dZyp;
    else if (f == "Fpx") r.sorted = p.Fpx;
    else if (f == "Fpy") r.sorted = p.Fpy;
    else if (f == "Fric_px") r.sorted = p.Frx;
    else if (f == "Fric_py") r.sorted = p.Fry;
  }
  if (!r.sorted && !r.ref && !r.iref && r.derived < 0 && r.pair_half < 0)
    return fail(ctx, DAMPM_ERR_UNKNOWN_FIELD, "unknown particle field " + f);
  return DAMPM_OK;
}

// The field into reference order at dst (np doubles), on the context stream.
void enqueue_to_ref(dampm_ctx* ctx, const FieldSrc& r, double* dst, int np) {
  Particles& p = ctx->p;
  const int gp = grid_for(np, 256);
  if (r.sorted)
    k_to_ref<<<gp, 256, 0, ctx->stream>>>(r.sorted, p.idx, dst, ctx->S);
  else if (r.pair_half >= 0)
    k_pair_to_ref<<<gp, 256, 0, ctx->stream>>>(p.mp, r.pair_half, p.idx, dst, ctx->S);
  else if (r.iref)
    k_int_to_double<<<gp, 256, 0, ctx->stream>>>(r.iref, dst, ctx->S);
  else if (r.derived >= 0)
    k_derived<<<gp, 256, 0, ctx->stream>>>(p, ctx->P, ctx->S, r.derived, dst);
  else
    cudaMemcpyAsync(dst, r.ref, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream);
}

}  // namespace

extern "C" {

const char* dampm_version(void) { return "dampm-b200 0.1 (sm_100a)"; }

const char* dampm_last_error(dampm_ctx* ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

int dampm_ctx_create(const dampm_grid* grid, const dampm_params* params,
                     const dampm_ms_params* ms, int precision,
                     long long capacity, void* cuda_stream, dampm_ctx** out) {
  if (!grid || !params || !out) return DAMPM_ERR_ARG;
  if (grid->Nex < 1 || grid->Ney < 1 || !(grid->hx > 0) || !(grid->hy > 0))
    return DAMPM_ERR_ARG;
  if (precision != DAMPM_FP64) return DAMPM_ERR_ARG;
  const long long nn = (long long)(grid->Nex + 1) * (grid->Ney + 1);
  if (nn > 0x7fffffffLL) return DAMPM_ERR_ARG;
  dampm_ctx* ctx = new dampm_ctx();
  ctx->grid = *grid;
  ctx->params = *params;
  if (ms) {
    ctx->ms = *ms;
  } else {  // main/mpm_data.h:102-112
    ctx->ms = dampm_ms_params{0.9, 0.30, 0.0, 1e30, 0.05, 0.01, -2, 2, 2, 10, 1e9, 0.0};
  }
  ctx->precision = precision;
  ctx->G = make_geom(*grid);
  ctx->P = make_phys(*params);
  ctx->nn = int(nn);
  ctx->nc = grid->Nex * grid->Ney;
  ctx->cap = capacity;
  if (cuda_stream) {
    ctx->stream = static_cast<cudaStream_t>(cuda_stream);
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return DAMPM_ERR_CUDA;
    }
    ctx->own_stream = true;
  }
  int rc = DAMPM_OK;
  rc = rc ? rc : dalloc(ctx, &ctx->Z, nn);
  rc = rc ? rc : dalloc(ctx, &ctx->dZdx, nn);
  rc = rc ? rc : dalloc(ctx, &ctx->dZdy, nn);
  rc = rc ? rc : dalloc(ctx, &ctx->nodes.vvL, nn);
  ctx->ntiles = (ctx->nc + kScanTile - 1) / kScanTile;
  rc = rc ? rc : dalloc(ctx, &ctx->count, size_t(ctx->nc) + 4);
  rc = rc ? rc : dalloc(ctx, &ctx->clist, size_t(ctx->nc) + 4);
  rc = rc ? rc : dalloc(ctx, &ctx->clist_n, 4);
  rc = rc ? rc : dalloc(ctx, &ctx->start, size_t(ctx->nc) + 1);
  rc = rc ? rc : dalloc(ctx, &ctx->tile_sum, size_t(ctx->ntiles) + 1);
  ctx->strips = (grid->Ney + 1 + kTR - 1) / kTR;
  ctx->useg = grid->Nex + 1;
  ctx->n_led = ctx->strips * ctx->useg;  // most units a step can list
  if (ctx->strips > kMaxStrips)
    rc = fail(ctx, DAMPM_ERR_ARG, "grid has too many rows for the P2G unit planner");
  rc = rc ? rc : dalloc(ctx, &ctx->led_part, size_t(ctx->n_led) * 6);
  rc = rc ? rc : dalloc(ctx, &ctx->ustart, size_t(ctx->n_led));
  rc = rc ? rc : dalloc(ctx, &ctx->upex, size_t(ctx->n_led));
  rc = rc ? rc : dalloc(ctx, &ctx->uplan, size_t(ctx->n_led));
  rc = rc ? rc : dalloc(ctx, &ctx->ulist, size_t(ctx->n_led));
  rc = rc ? rc : dalloc(ctx, &ctx->uorder, size_t(ctx->n_led));
  rc = rc ? rc : dalloc(ctx, &ctx->strip_n, size_t(ctx->strips));
  rc = rc ? rc : dalloc(ctx, &ctx->ucount, 4);
  rc = rc ? rc : dalloc(ctx, &ctx->ledger_log, size_t(kLedgerLog) * 3);
  rc = rc ? rc : dalloc(ctx, &ctx->S, 1);
  if (rc == DAMPM_OK) {
    if (cudaMallocHost(&ctx->Sh, sizeof(Scalars)) != cudaSuccess) rc = DAMPM_ERR_CUDA;
  }
  if (rc == DAMPM_OK) {
    cudaMemsetAsync(ctx->count, 0, sizeof(int) * ctx->nc, ctx->stream);
    cudaMemsetAsync(ctx->ucount, 0, sizeof(int) * 4, ctx->stream);
    cudaMemsetAsync(ctx->nodes.vvL, 0, sizeof(double2) * nn, ctx->stream);
    cudaMemsetAsync(ctx->S, 0, sizeof(Scalars), ctx->stream);
    int per_sm = setup_p2g(), nsm = 0, dev = 0;
    if (per_sm == 0) rc = fail(ctx, DAMPM_ERR_CUDA, "cannot configure P2G shared memory");
    if (!setup_sort()) rc = fail(ctx, DAMPM_ERR_CUDA, "cannot configure the sort's shared memory");
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (per_sm < 1) per_sm = 1;
    ctx->p2g_grid = std::max(1, std::min(nsm * per_sm, ctx->n_led));
  }
  if (rc != DAMPM_OK) {
    dampm_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return DAMPM_OK;
}

int dampm_ctx_destroy(dampm_ctx* ctx) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->staged) cudaEventDestroy(ctx->staged);
  for (void* q : ctx->allocs) cudaFree(q);
  for (cudaEvent_t e : ctx->evpool) cudaEventDestroy(e);
  drop_graphs(ctx);
  if (ctx->Sh) cudaFreeHost(ctx->Sh);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return DAMPM_OK;
}

int dampm_upload_terrain(dampm_ctx* ctx, const double* Z, const double* dZdx,
                         const double* dZdy) {
  if (!ctx || !Z || !dZdx || !dZdy) return DAMPM_ERR_ARG;
  const size_t b = sizeof(double) * ctx->nn;
  CK(cudaMemcpyAsync(ctx->Z, Z, b, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->dZdx, dZdx, b, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->dZdy, dZdy, b, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->terrain_ok = true;
  return DAMPM_OK;
}

int dampm_upload_particles(dampm_ctx* ctx, long long np, const double* x,
                           const double* y, const double* Mp, const double* Ap,
                           const double* vpx, const double* vpy,
                           const double* hp, const double* mom_px,
                           const double* mom_py, const double* Vp) {
  if (!ctx || np < 0 || np > 0x7fffffffLL) return DAMPM_ERR_ARG;
  if (np > 0 && (!x || !y || !Mp || !Ap || !vpx || !vpy || !hp || !mom_px ||
                 !mom_py || !Vp))
    return DAMPM_ERR_ARG;
  if (!ctx->terrain_ok) return fail(ctx, DAMPM_ERR_STATE, "upload terrain first");
  if (ctx->p.x == nullptr) {
    long long cap = ctx->cap > 0 ? ctx->cap : 2 * np + 1024;
    if (cap < np) return fail(ctx, DAMPM_ERR_CAPACITY, "capacity below particle count");
    int rc = alloc_particles(ctx, cap);
    if (rc) return rc;
  } else if (np > ctx->cap) {
    return fail(ctx, DAMPM_ERR_CAPACITY, "capacity below particle count");
  }
  const size_t b = sizeof(double) * np;
  Particles& p = ctx->p;
  if (np > 0) {
    CK(cudaMemcpyAsync(p.x, x, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.y, y, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.xp, x, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.yp, y, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.Mp, Mp, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.Ap, Ap, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.vpx, vpx, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.vpy, vpy, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.hp, hp, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(upload_pair(p.mp, mom_px, mom_py, np, ctx->stream));
    CK(cudaMemcpyAsync(p.Vp, Vp, b, cudaMemcpyHostToDevice, ctx->stream));
  }
  Scalars s0{};
  s0.fresh = 1;
  s0.np = int(np);
  full_scan_next(ctx, s0);
  *ctx->Sh = s0;
  CK(cudaMemcpyAsync(ctx->S, ctx->Sh, sizeof(Scalars), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaMemsetAsync(ctx->count, 0, sizeof(int) * ctx->nc, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // Sh is reused below
  if (np > 0) {
    // the slots hold the particles in DATA order (idx = slot)
    launch_init_particles<double>(grid_for(np, 256), 256, ctx->stream, p, ctx->Z,
                                  ctx->dZdx, ctx->dZdy, ctx->G, ctx->P, ctx->S, int(np), 0);
    k_count_n<<<grid_for(np, 256), 256, 0, ctx->stream>>>(p.key, ctx->count, p.slot,
                                                           int(np));
    launch_prep<double>(grid_for(np, 256), 256, ctx->stream, p, ctx->Z, ctx->G, ctx->P,
                        ctx->S, 0);
    CK(cudaGetLastError());
  }
  ctx->it_host = 0;
  ctx->particles_ok = true;
  return sync_status(ctx);
}

int dampm_enable_merge_split(dampm_ctx* ctx, int enable) {
  if (!ctx) return DAMPM_ERR_ARG;
  ctx->ms_enabled = enable != 0;
  return DAMPM_OK;
}

int dampm_set_ms_variant(dampm_ctx* ctx, int variant, double stretch_thresh) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (variant != DAMPM_MS_CMES && variant != DAMPM_MS_ELFS)
    return fail(ctx, DAMPM_ERR_ARG, "unknown merge/split variant");
  if (variant == DAMPM_MS_ELFS) {
    const int rc = ms_alloc_elfs(ctx->msb, ctx->nc, [&](void** q, size_t bytes) {
      return dalloc(ctx, reinterpret_cast<unsigned char**>(q), bytes);
    });
    if (rc) return rc;
  }
  ctx->ms_variant = variant;
  ctx->ms_stretch = stretch_thresh;
  return DAMPM_OK;
}

int dampm_record_outputs(dampm_ctx* ctx, int enable) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (ctx->slab && enable) return fail(ctx, DAMPM_ERR_STATE, "slab mode records no outputs");
  ctx->record = enable != 0;
  if (ctx->record && ctx->p.x) return alloc_record(ctx);
  return DAMPM_OK;
}

int dampm_step(dampm_ctx* ctx, int nsteps) {
  if (!ctx || nsteps < 0) return DAMPM_ERR_ARG;
  if (ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "slab mode: use the dampm_slab_* calls");
  if (!ctx->particles_ok) return fail(ctx, DAMPM_ERR_STATE, "upload particles first");
  ctx->launches = 0;
  ctx->evused = 0;
  int s = 0;
  int phase = 0;
  const int len = graph_eligible(ctx) ? graph_shape(ctx, &phase) : 0;
  if (len > 0) {
    bool aligned = true;
    if (ms_cadence(ctx)) {
      // graphs of this cycle in hand: plain passes up to their phase
      for (const auto& g : ctx->graphs)
        if (g.exec && g.passes == len) phase = g.phase;
      for (; s < nsteps && int(ctx->it_host % len) != phase; ++s) {
        int rc = enqueue_pass(ctx);
        if (rc) return rc;
      }
      aligned = int(ctx->it_host % len) == phase;
    }
    // captured on the first eligible call, whatever its length (a short call
    // captures the graph for the calls to come and runs plainly)
    bool first = true;
    while (aligned && (first || s + len <= nsteps)) {
      first = false;
      dampm_ctx::GraphSlot* g = nullptr;
      int rc = ensure_graph(ctx, len, phase, &g);
      if (rc) return rc;
      if (!g || s + len > nsteps) break;
      CK(cudaGraphLaunch(g->exec, ctx->stream));
      advance_buffers(ctx, len);
      ctx->it_host += len;
      ctx->launches += g->launches;
      s += len;
    }
  }
  for (; s < nsteps; ++s) {
    int rc = enqueue_pass(ctx);
    if (rc) return rc;
  }
  // without merge/split, the graph the next call starts from (the buffers of
  // an odd count of passes are exchanged), captured now rather than inside it
  if (len > 0 && !ms_cadence(ctx)) {
    dampm_ctx::GraphSlot* g = nullptr;
    int rc = ensure_graph(ctx, len, phase, &g);
    if (rc) return rc;
  }
  ev_mark(ctx, 3);
  return DAMPM_OK;
}

int dampm_set_graphs(dampm_ctx* ctx, int enable) {
  if (!ctx) return DAMPM_ERR_ARG;
  ctx->use_graphs = enable != 0;
  return DAMPM_OK;
}

int dampm_sync(dampm_ctx* ctx) {
  if (!ctx) return DAMPM_ERR_ARG;
  return sync_status(ctx);
}

int dampm_run(dampm_ctx* ctx, long long max_steps, int chunk,
              long long* steps_done) {
  if (!ctx || chunk < 1) return DAMPM_ERR_ARG;
  long long done = 0;
  int it0 = 0;
  int rc = sync_status(ctx);
  if (rc) return rc;
  it0 = ctx->Sh->it;
  while (done < max_steps) {
    const int n = int(std::min<long long>(chunk, max_steps - done));
    rc = dampm_step(ctx, n);
    if (rc) return rc;
    rc = sync_status(ctx);
    if (rc) return rc;
    done += n;
    if (!ctx->Sh->active) break;
  }
  // passes whose loop condition failed did nothing: realign the host count
  ctx->it_host = ctx->Sh->it;
  if (steps_done) *steps_done = ctx->Sh->it - it0;
  return DAMPM_OK;
}

int dampm_status(dampm_ctx* ctx, int* it, double* t, double* dt_last,
                 long long* np) {
  if (!ctx) return DAMPM_ERR_ARG;
  int rc = sync_status(ctx, false);
  if (rc) return rc;
  if (it) *it = ctx->Sh->it;
  if (t) *t = ctx->Sh->t;
  if (dt_last) *dt_last = ctx->Sh->dt;
  if (np) *np = ctx->Sh->np;
  // the loop state is filled in either way; a set status bit is reported
  return ctx->Sh->status ? sync_status(ctx) : DAMPM_OK;
}

int dampm_merge_split(dampm_ctx* ctx, double dt, long long counts[4]) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "slab mode: use the dampm_slab_* calls");
  if (!ctx->particles_ok) return fail(ctx, DAMPM_ERR_STATE, "upload particles first");
  // bin with the current positions, then decide + emit (an always-active
  // pass: the loop condition does not apply to a standalone call)
  Scalars* S = ctx->S;
  int rc = sync_status(ctx);
  if (rc) return rc;
  const int active_save = ctx->Sh->active;
  ctx->Sh->active = 1;
  CK(cudaMemcpyAsync(&S->active, &ctx->Sh->active, sizeof(int),
                     cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  enqueue_sort(ctx);
  ms_enqueue(ctx->msb, ctx->p, ctx->q, ctx->start, ctx->perm, ctx->nc, ctx->G, ctx->P,
             ctx->Z, ctx->ms, ctx->S, ctx->cap, ctx->stream, /*use_step_dt=*/0, dt,
             ctx->ms_variant, ctx->ms_stretch);
  swap_moving(ctx->p, ctx->q);
  k_keys<<<grid_for(ctx->cap, 256), 256, 0, ctx->stream>>>(ctx->p, ctx->G, ctx->S, 0);
  k_count<<<grid_for(ctx->cap, 256), 256, 0, ctx->stream>>>(ctx->p.key, ctx->count,
                                                           ctx->p.slot, ctx->S);
  CK(cudaGetLastError());
  rc = sync_status(ctx);
  if (rc) return rc;
  ctx->Sh->active = active_save;
  CK(cudaMemcpyAsync(&S->active, &ctx->Sh->active, sizeof(int),
                     cudaMemcpyHostToDevice, ctx->stream));
  if (counts)
    for (int k = 0; k < 4; ++k) counts[k] = ctx->Sh->ms_counts[k];
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

int dampm_download(dampm_ctx* ctx, const char* field, double* out) {
  if (!ctx || !field || !out) return DAMPM_ERR_ARG;
  if (ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "slab mode: use the dampm_slab_* calls");
  if (!ctx->particles_ok) return fail(ctx, DAMPM_ERR_STATE, "no particles");
  int rc = sync_status(ctx, false);
  if (rc) return rc;
  const int np = ctx->Sh->np;
  FieldSrc r;
  rc = resolve_field(ctx, field, ctx->Sh->fresh != 0, r);
  if (rc) return rc;
  if (np == 0) return DAMPM_OK;
  double* tmp = ctx->msb.stage;  // the merge/split scratch as a staging buffer
  enqueue_to_ref(ctx, r, tmp, np);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, tmp, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

int dampm_download_nodal(dampm_ctx* ctx, const char* field, double* out) {
  if (!ctx || !field || !out) return DAMPM_ERR_ARG;
  const std::string f(field);
  const double* src = nullptr;
  Nodes& n = ctx->nodes;
  if (f == "vvxL" || f == "vvyL") {
    CK(download_pair_half(out, n.vvL, f == "vvxL" ? 0 : 1, ctx->nn, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DAMPM_OK;
  }
  if (f == "Z") src = ctx->Z;
  else if (f == "dZdx") src = ctx->dZdx;
  else if (f == "dZdy") src = ctx->dZdy;
  else if (ctx->record_alloc) {
    if (f == "Mv") src = n.Mv;
    else if (f == "mom_vx") src = n.mvx;
    else if (f == "mom_vy") src = n.mvy;
    else if (f == "avx") src = n.avx;
    else if (f == "avy") src = n.avy;
    else if (f == "vvx") src = n.vvx;
    else if (f == "vvy") src = n.vvy;
    else if (f == "FPxv") src = n.FPxv;
    else if (f == "FPyv") src = n.FPyv;
    else if (f == "Fric_x") src = n.Fricx;
    else if (f == "Fric_y") src = n.Fricy;
    else if (f == "F_int_vx") src = n.Fintx;
    else if (f == "F_int_vy") src = n.Finty;
    else if (f == "HV") src = n.HV;
  }
  if (!src) return fail(ctx, DAMPM_ERR_UNKNOWN_FIELD, "unknown nodal field " + f);
  CK(cudaMemcpyAsync(out, src, sizeof(double) * ctx->nn, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

int dampm_ledger_history(dampm_ctx* ctx, long long first_it, int n, double* out) {
  if (!ctx || !out || n < 0 || first_it < 1 || n > kLedgerLog) return DAMPM_ERR_ARG;
  int rc = sync_status(ctx);
  if (rc) return rc;
  const long long last = ctx->Sh->it;
  if (first_it + n - 1 > last || last - first_it >= kLedgerLog)
    return fail(ctx, DAMPM_ERR_ARG, "ledger rows outside the last 1024 steps");
  std::vector<double> all(size_t(kLedgerLog) * 3);
  CK(cudaMemcpyAsync(all.data(), ctx->ledger_log, sizeof(double) * all.size(),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < n; ++k) {
    const double* row = all.data() + 3 * ((first_it + k - 1) % kLedgerLog);
    for (int q = 0; q < 3; ++q) out[3 * k + q] = row[q];
  }
  return DAMPM_OK;
}

int dampm_ledgers(dampm_ctx* ctx, double out[9]) {
  if (!ctx || !out) return DAMPM_ERR_ARG;
  int rc = sync_status(ctx, false);
  if (rc) return rc;
  std::memcpy(out, ctx->Sh->ledger, sizeof(double) * 9);
  return DAMPM_OK;
}

int dampm_set_state(dampm_ctx* ctx, long long np, const double* const* fields,
                    const double* Ap, const double* mom_px,
                    const double* mom_py, const double* Fb_x,
                    const double* Fb_y) {
  if (ctx && ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "slab mode: use the dampm_slab_* calls");
  if (!ctx || !fields || np < 0 || np > ctx->cap) return DAMPM_ERR_ARG;
  if (!ctx->particles_ok) return fail(ctx, DAMPM_ERR_STATE, "upload particles first");
  Particles& p = ctx->p;
  double* dst[11] = {p.x, p.y, p.vpx, p.vpy, p.hp, p.F11, p.F12, p.F22,
                     p.Mp, p.Vp, p.H};
  const size_t b = sizeof(double) * np;
  for (int k = 0; k < 11; ++k) {
    if (!fields[k]) return DAMPM_ERR_ARG;
    CK(cudaMemcpyAsync(dst[k], fields[k], b, cudaMemcpyHostToDevice, ctx->stream));
  }
  const bool fresh = Ap && mom_px && mom_py && Fb_x && Fb_y;
  if (fresh) {
    CK(cudaMemcpyAsync(p.Ap, Ap, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(upload_pair(p.mp, mom_px, mom_py, np, ctx->stream));
    CK(cudaMemcpyAsync(p.Fbx, Fb_x, b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(p.Fby, Fb_y, b, cudaMemcpyHostToDevice, ctx->stream));
  }
  int rc = sync_status(ctx, false);
  if (rc) return rc;
  ctx->Sh->np = int(np);
  ctx->Sh->fresh = fresh ? 1 : 0;
  ctx->Sh->status = 0;  // a new state: an earlier divergence no longer applies
  ctx->Sh->red_cur[0] = ctx->Sh->red_cur[1] = ctx->Sh->red_cur[2] = 0ull;
  full_scan_next(ctx, *ctx->Sh);
  CK(cudaMemcpyAsync(ctx->S, ctx->Sh, sizeof(Scalars), cudaMemcpyHostToDevice,
                     ctx->stream));
  // the slots now hold the particles in reference order
  CK(cudaMemsetAsync(ctx->count, 0, sizeof(int) * ctx->nc, ctx->stream));
  k_keys<<<grid_for(np, 256), 256, 0, ctx->stream>>>(p, ctx->G, ctx->S, 1);
  k_count_n<<<grid_for(np, 256), 256, 0, ctx->stream>>>(p.key, ctx->count, p.slot, int(np));
  k_reduce_state<<<grid_for(np, 256), 256, 0, ctx->stream>>>(p, ctx->S);
  launch_prep<double>(grid_for(np, 256), 256, ctx->stream, p, ctx->Z, ctx->G, ctx->P,
                      ctx->S, fresh ? 0 : 1);
  CK(cudaGetLastError());
  return DAMPM_OK;
}

int dampm_get_state(dampm_ctx* ctx, double* const* fields) {
  if (!ctx || !fields) return DAMPM_ERR_ARG;
  if (ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "slab mode: use the dampm_slab_* calls");
  int rc = sync_status(ctx, false);
  if (rc) return rc;
  Particles& p = ctx->p;
  const double* src[11] = {p.x, p.y, p.vpx, p.vpy, p.hp, p.F11, p.F12, p.F22,
                           p.Mp, p.Vp, p.H};
  const int np = ctx->Sh->np;
  const size_t b = sizeof(double) * np;
  for (int k = 0; k < 11; ++k)
    if (!fields[k]) return DAMPM_ERR_ARG;
  if (np == 0) return DAMPM_OK;
  // into reference order in the merge/split scratch, then one copy each
  for (int k = 0; k < 11; ++k)
    k_to_ref<<<grid_for(np, 256), 256, 0, ctx->stream>>>(src[k], p.idx, ctx->msb.sd[k],
                                                         ctx->S);
  CK(cudaGetLastError());
  for (int k = 0; k < 11; ++k)
    CK(cudaMemcpyAsync(fields[k], ctx->msb.sd[k], b, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

long long dampm_last_launch_count(dampm_ctx* ctx) { return ctx ? ctx->launches : -1; }

int dampm_last_timings(dampm_ctx* ctx, int enable_events, double out[5]) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (out) {
    for (int k = 0; k < 5; ++k) out[k] = 0.0;
    if (ctx->evused > 1) {
      CK(cudaStreamSynchronize(ctx->stream));
      for (int k = 1; k < ctx->evused; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->evpool[k - 1], ctx->evpool[k]));
        // interval (k-1, k] belongs to the class recorded at event k-1
        const int cls = ctx->evclass[k - 1];
        out[cls] += ms;
        out[4] += ms;
      }
    }
  }
  ctx->timing = enable_events != 0;
  return DAMPM_OK;
}

// ---- one scenario over slabs of cell columns ------------------------------
namespace {

unsigned long long host_ordered_key(double v) {
  unsigned long long b;
  std::memcpy(&b, &v, sizeof b);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double host_ordered_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  std::memcpy(&v, &b, sizeof v);
  return v;
}

int slab_alloc(dampm_ctx* ctx) {
  if (ctx->leave || !ctx->p.x) return DAMPM_OK;
  int rc = dalloc(ctx, &ctx->leave, size_t(ctx->cap));
  rc = rc ? rc : dalloc(ctx, &ctx->sel, size_t(ctx->cap));
  rc = rc ? rc : dalloc(ctx, &ctx->selcount, 1);
  rc = rc ? rc : dalloc(ctx, &ctx->moves, size_t(ctx->cap));
  return rc;
}

int slab_ready(dampm_ctx* ctx) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (!ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "not in slab mode (dampm_slab_set)");
  if (!ctx->particles_ok) return fail(ctx, DAMPM_ERR_STATE, "upload particles first");
  return slab_alloc(ctx);
}

}  // namespace

int dampm_slab_record_doubles(void) { return kSlabRecord; }

int dampm_slab_set(dampm_ctx* ctx, int col_lo, int col_hi) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (!(0 <= col_lo && col_lo < col_hi && col_hi <= ctx->grid.Nex))
    return fail(ctx, DAMPM_ERR_ARG, "slab columns outside the grid");
  if (ctx->record || (ctx->ms_enabled && ctx->params.MERGE_SPLIT_ON))
    return fail(ctx, DAMPM_ERR_STATE, "slab mode runs without recorded outputs or merge/split");
  ctx->slab = true;
  ctx->use_graphs = false;
  ctx->G.pc_lo = col_lo;
  ctx->G.pc_hi = col_hi;
  ctx->G.nc_lo = col_lo;
  ctx->G.nc_hi = col_hi == ctx->grid.Nex ? col_hi : col_hi - 1;
  return slab_alloc(ctx);
}

int dampm_slab_set_index(dampm_ctx* ctx, const int* idx) {
  int rc = slab_ready(ctx);
  if (rc) return rc;
  if (!idx) return DAMPM_ERR_ARG;
  rc = sync_status(ctx, false);
  if (rc) return rc;
  const int np = ctx->Sh->np - ctx->Sh->nghost;
  CK(cudaMemcpyAsync(ctx->p.idx, idx, sizeof(int) * np, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

int dampm_slab_pass(dampm_ctx* ctx, int phase) {
  int rc = slab_ready(ctx);
  if (rc) return rc;
  ctx->launches = 0;
  if (phase == 0) return enqueue_front(ctx);
  if (phase == 1) return enqueue_back(ctx);
  return DAMPM_ERR_ARG;
}

int dampm_slab_node_column(dampm_ctx* ctx, int col, double* buf, int set) {
  if (!ctx || !buf || col < 0 || col > ctx->grid.Nex) return DAMPM_ERR_ARG;
  const size_t n = size_t(ctx->grid.Ney + 1);
  double2* c = ctx->nodes.vvL + (size_t)col * n;
  if (set)
    CK(cudaMemcpyAsync(c, buf, n * sizeof(double2), cudaMemcpyDeviceToDevice, ctx->stream));
  else
    CK(cudaMemcpyAsync(buf, c, n * sizeof(double2), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

int dampm_slab_cfl(dampm_ctx* ctx, double maxima[3], int set) {
  if (!ctx || !maxima) return DAMPM_ERR_ARG;
  if (set) {
    k_slab_set_red<<<1, 1, 0, ctx->stream>>>(ctx->S, host_ordered_key(maxima[0]),
                                             host_ordered_key(maxima[1]),
                                             host_ordered_key(maxima[2]));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return DAMPM_OK;
  }
  int rc = sync_status(ctx, false);
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) maxima[k] = host_ordered_value(ctx->Sh->red_cur[k]);
  return DAMPM_OK;
}

int dampm_slab_route(dampm_ctx* ctx, double* left, double* right, long long cap,
                     long long* n_left, long long* n_right) {
  int rc = slab_ready(ctx);
  if (rc) return rc;
  if (!n_left || !n_right || cap < 0) return DAMPM_ERR_ARG;
  rc = sync_status(ctx, false);
  if (rc) return rc;
  const int np = ctx->Sh->np, L = ctx->Sh->nleave;
  *n_left = *n_right = 0;
  if (L == 0) return DAMPM_OK;
  std::vector<int> slots(L), keys(L);
  CK(cudaMemcpyAsync(slots.data(), ctx->leave, sizeof(int) * L, cudaMemcpyDeviceToHost,
                     ctx->stream));
  k_slab_keys<<<grid_for(L, 256), 256, 0, ctx->stream>>>(ctx->p.key, ctx->leave, L, ctx->sel);
  CK(cudaMemcpyAsync(keys.data(), ctx->sel, sizeof(int) * L, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // leavers by side, in slot order
  std::vector<int> order(L);
  for (int k = 0; k < L; ++k) order[k] = k;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return slots[a] < slots[b]; });
  std::vector<int> lefts, rights, sorted_slots;
  for (int k : order) {
    sorted_slots.push_back(slots[k]);
    (keys[k] / ctx->grid.Ney < ctx->G.pc_lo ? lefts : rights).push_back(slots[k]);
  }
  if ((long long)lefts.size() > cap || (long long)rights.size() > cap)
    return fail(ctx, DAMPM_ERR_CAPACITY, "route buffers smaller than the migrants");
  if ((!left && !lefts.empty()) || (!right && !rights.empty()))
    return fail(ctx, DAMPM_ERR_STATE, "particles left the slab on a side without a neighbour");
  // pack the migrants, then fill the holes below the new count with the
  // particles that stay above it
  const int keep = np - L;
  std::vector<int2> mv;
  {
    size_t h = 0;  // leavers below `keep`, in slot order, are the holes
    size_t li = 0;
    for (int src = keep; src < np; ++src) {
      while (li < sorted_slots.size() && sorted_slots[li] < src) ++li;
      if (li < sorted_slots.size() && sorted_slots[li] == src) continue;  // a leaver
      while (h < sorted_slots.size() && sorted_slots[h] >= keep) ++h;
      mv.push_back(make_int2(src, sorted_slots[h++]));
    }
  }
  for (int side = 0; side < 2; ++side) {
    const std::vector<int>& v = side ? rights : lefts;
    if (v.empty()) continue;
    CK(cudaMemcpyAsync(ctx->sel, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    k_slab_pack<<<grid_for(long(v.size()), 256), 256, 0, ctx->stream>>>(
        ctx->p, ctx->sel, int(v.size()), side ? right : left);
    CK(cudaStreamSynchronize(ctx->stream));  // sel is reused
  }
  if (!mv.empty()) {
    CK(cudaMemcpyAsync(ctx->moves, mv.data(), sizeof(int2) * mv.size(),
                       cudaMemcpyHostToDevice, ctx->stream));
    k_slab_move<<<grid_for(long(mv.size()), 256), 256, 0, ctx->stream>>>(ctx->p, ctx->moves,
                                                                         int(mv.size()));
  }
  k_slab_scalars<<<1, 1, 0, ctx->stream>>>(ctx->S, keep, 0, ctx->nc);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  *n_left = (long long)lefts.size();
  *n_right = (long long)rights.size();
  return DAMPM_OK;
}

int dampm_slab_ghosts(dampm_ctx* ctx, double* buf, long long cap, long long* n) {
  int rc = slab_ready(ctx);
  if (rc) return rc;
  if (!buf || !n) return DAMPM_ERR_ARG;
  rc = sync_status(ctx, false);
  if (rc) return rc;
  const int np = ctx->Sh->np - ctx->Sh->nghost;
  CK(cudaMemsetAsync(ctx->selcount, 0, sizeof(int), ctx->stream));
  k_slab_select<<<grid_for(np, 256), 256, 0, ctx->stream>>>(
      ctx->p.key, np, ctx->G.pc_hi - 1, ctx->grid.Ney, ctx->sel, ctx->selcount);
  int cnt = 0;
  CK(cudaMemcpyAsync(&ctx->Sh->np_next, ctx->selcount, sizeof(int), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  cnt = ctx->Sh->np_next;
  if (cnt > cap) return fail(ctx, DAMPM_ERR_CAPACITY, "ghost buffer smaller than the column");
  if (cnt > 0)
    k_slab_pack<<<grid_for(cnt, 256), 256, 0, ctx->stream>>>(ctx->p, ctx->sel, cnt, buf);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  *n = cnt;
  return DAMPM_OK;
}

int dampm_slab_import(dampm_ctx* ctx, const double* buf, long long n, int ghosts) {
  int rc = slab_ready(ctx);
  if (rc) return rc;
  if (n < 0 || (n > 0 && !buf)) return DAMPM_ERR_ARG;
  rc = sync_status(ctx, false);
  if (rc) return rc;
  const long long base = ctx->Sh->np;
  if (base + n > ctx->cap)
    return fail(ctx, DAMPM_ERR_CAPACITY, "slab capacity below its particles and imports");
  if (n > 0) {
    k_slab_unpack<<<grid_for(n, 256), 256, 0, ctx->stream>>>(ctx->p, buf, int(n), int(base));
    // ghosts: the left neighbour's last column; migrants: this slab's columns
    const int lo = ghosts ? ctx->G.pc_lo - 1 : ctx->G.pc_lo;
    const int hi = ghosts ? ctx->G.pc_lo : ctx->G.pc_hi;
    k_slab_check<<<grid_for(n, 256), 256, 0, ctx->stream>>>(ctx->p.key + base, int(n), lo, hi,
                                                            ctx->grid.Ney, ctx->S);
    k_count_n<<<grid_for(n, 256), 256, 0, ctx->stream>>>(ctx->p.key + base, ctx->count,
                                                         ctx->p.slot + base, int(n));
  }
  k_slab_scalars<<<1, 1, 0, ctx->stream>>>(ctx->S, int(base + n), ghosts ? int(n) : 0,
                                           ctx->nc);
  CK(cudaGetLastError());
  rc = sync_status(ctx, false);
  if (rc) return rc;
  if (ctx->Sh->status & kStatusSlab)
    return fail(ctx, DAMPM_ERR_STATE, "a particle moved more than one slab in a step");
  return DAMPM_OK;
}

int dampm_slab_download(dampm_ctx* ctx, const char* field, double* out, long long* idx) {
  int rc = slab_ready(ctx);
  if (rc) return rc;
  if (!field || !out) return DAMPM_ERR_ARG;
  rc = sync_status(ctx, false);
  if (rc) return rc;
  const int np = ctx->Sh->np - ctx->Sh->nghost;
  const std::string f(field);
  Particles& p = ctx->p;
  const double* src = f == "x" ? p.x : f == "y" ? p.y : f == "vpx" ? p.vpx
                    : f == "vpy" ? p.vpy : f == "hp" ? p.hp : f == "F_11" ? p.F11
                    : (f == "F_12" || f == "F_21") ? p.F12 : f == "F_22" ? p.F22
                    : f == "Mp" ? p.Mp : f == "Vp" ? p.Vp : f == "H" ? p.H : nullptr;
  if (!src) return fail(ctx, DAMPM_ERR_UNKNOWN_FIELD, "unknown slab field " + f);
  if (np == 0) return DAMPM_OK;
  CK(cudaMemcpyAsync(out, src, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
  if (idx) {
    std::vector<int> ix(np);
    CK(cudaMemcpyAsync(ix.data(), p.idx, sizeof(int) * np, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < np; ++k) idx[k] = ix[k];
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return DAMPM_OK;
}

// ---- output without stalling the step loop ---------------------------------
int dampm_staged_wait(dampm_ctx* ctx) {
  if (!ctx) return DAMPM_ERR_ARG;
  if (ctx->side_pending) {
    CK(cudaStreamSynchronize(ctx->side));
    ctx->side_pending = false;
  }
  return DAMPM_OK;
}

int dampm_stage_download(dampm_ctx* ctx, int n, const char* const* fields,
                         double* const* host_out, long long* np_out) {
  if (!ctx || n < 0 || n > kMaxStaged || (n > 0 && (!fields || !host_out)))
    return DAMPM_ERR_ARG;
  if (ctx->slab) return fail(ctx, DAMPM_ERR_STATE, "slab mode: use the dampm_slab_* calls");
  if (!ctx->particles_ok) return fail(ctx, DAMPM_ERR_STATE, "no particles");
  int rc = dampm_staged_wait(ctx);  // the buffer of the last call is free again
  if (rc) return rc;
  rc = sync_status(ctx, false);
  if (rc) return rc;
  const int np = ctx->Sh->np;
  const bool fresh = ctx->Sh->fresh != 0;
  std::vector<FieldSrc> src(n);
  for (int k = 0; k < n; ++k) {
    if (!fields[k] || !host_out[k]) return DAMPM_ERR_ARG;
    rc = resolve_field(ctx, fields[k], fresh, src[k]);
    if (rc) return rc;
  }
  if (np_out) *np_out = np;
  if (n == 0 || np == 0) return DAMPM_OK;
  if (!ctx->side) {
    CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->staged, cudaEventDisableTiming));
  }
  if (ctx->outbuf_fields < n || ctx->outbuf_cap != ctx->cap) {  // grows, then stays
    if (ctx->outbuf) {
      CK(cudaStreamSynchronize(ctx->stream));
      cudaFree(ctx->outbuf);
      ctx->allocs.erase(std::remove(ctx->allocs.begin(), ctx->allocs.end(),
                                    static_cast<void*>(ctx->outbuf)),
                        ctx->allocs.end());
      ctx->outbuf = nullptr;
    }
    rc = dalloc(ctx, &ctx->outbuf, size_t(n) * size_t(ctx->cap));
    if (rc) return rc;
    ctx->outbuf_fields = n;
    ctx->outbuf_cap = ctx->cap;
  }
  for (int k = 0; k < n; ++k)
    enqueue_to_ref(ctx, src[k], ctx->outbuf + size_t(k) * size_t(ctx->cap), np);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->staged, ctx->stream));
  CK(cudaStreamWaitEvent(ctx->side, ctx->staged, 0));
  for (int k = 0; k < n; ++k)
    CK(cudaMemcpyAsync(host_out[k], ctx->outbuf + size_t(k) * size_t(ctx->cap),
                       sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->side));
  ctx->side_pending = true;
  return DAMPM_OK;
}

}  // extern "C"
