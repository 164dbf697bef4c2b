// dampm_kernels.h -- device buffers and kernel entry points of the step.
#pragma once
#include <cstddef>
#include <utility>

#include "dampm_device.cuh"

namespace dampm {

// P2G tiling: kTR node rows per strip (one lane per row in each of the four
// warps, one per quantity group, finishing and starting chains); units of
// variable column width cut to about np / (kUnitsPerCta * CTAs) particles
// (at least kUnitMinWeight), a column weighing its particles + kColWeight;
// particle records staged in shared memory kCap at a time.
constexpr int kTR = 30;
#ifndef DAMPM_UNITS_PER_CTA
#define DAMPM_UNITS_PER_CTA 2
#endif
#ifndef DAMPM_COL_WEIGHT
#define DAMPM_COL_WEIGHT 192
#endif
constexpr int kUnitsPerCta = DAMPM_UNITS_PER_CTA;
constexpr int kUnitMinWeight = 1024;
constexpr int kColWeight = DAMPM_COL_WEIGHT;
constexpr int kPlanThreads = 1024;
constexpr int kMaxStrips = 8192;  // strip offsets of the unit list in shared memory
constexpr int kP2GThreads = 128;
#ifndef DAMPM_P2G_CAP
#define DAMPM_P2G_CAP 512
#endif
#ifndef DAMPM_P2G_MIN_BLOCKS
#define DAMPM_P2G_MIN_BLOCKS 4
#endif
#ifndef DAMPM_CHAIN_UNROLL
#define DAMPM_CHAIN_UNROLL 2  // P2G chain steps unrolled per loop trip
#endif
constexpr int kChainUnroll = DAMPM_CHAIN_UNROLL;
constexpr int kCap = DAMPM_P2G_CAP;
constexpr int kP2GMinBlocks = DAMPM_P2G_MIN_BLOCKS;
constexpr int kG2PThreads = 256;
#ifndef DAMPM_G2P_MIN_BLOCKS
#define DAMPM_G2P_MIN_BLOCKS 4
#endif
constexpr int kG2PMinBlocks = DAMPM_G2P_MIN_BLOCKS;
constexpr int kScanTile = 4096;
constexpr int kScanThreads = 1024;

// Two values of R side by side (one 16-byte load in FP64, 8 in FP32).
template <class R>
struct Vec2T;
template <>
struct Vec2T<double> {
  using type = double2;
};
template <>
struct Vec2T<float> {
  using type = float2;
};
template <class R>
using V2 = typename Vec2T<R>::type;

// Particle SoA.  The moving fields are kept in cell-sorted order -- by
// (cell of the last binning, reference index) -- in two buffers: each step's
// G2P reads one through the sort permutation and writes the other in the new
// sorted order, so P2G and G2P stream contiguous runs of a cell column
// instead of gathering across the whole set.  `idx` is each slot's index in
// the reference's particle order (DATA order, then the compacted order
// merge/split produces); data going in and out of the library is in that
// order.  R = double is the FP64 path, R = float the FP32 form (batches).
template <class R>
struct ParticlesT {
  // ---- moving (double-buffered, sorted order) ----
  R *x, *y, *vpx, *vpy, *hp, *F11, *F12, *F22, *Mp, *Vp, *H;
  // key: cell of the next binning; idx: reference index; slot: rank among
  // the particles of its cell from the counting sort's atomics
  int *key, *idx, *slot;
  // the record the next P2G transfers, written by G2P (or by k_prep after an
  // upload, a state upload or a merge/split), as pairs that P2G gathers
  // with one copy each:
  //   mp = (mom_px, mom_py)  momentum v*Mp, and qf = (Ap*Fb_x, Ap*Fb_y) the
  //        friction force, as the reference stores them at the end of a
  //        step (main/optim_par.cpp:456-459,600-626);
  //   xe = (xi, eta)  local coordinates in the cell of the next binning;
  //   qg = gravity force -g*Vp*rho*grad(Z)*(1 - H/hp) there
  //        (main/optim_par.cpp:387,447-454).
  V2<R> *mp, *qf, *xe, *qg;
  // velocity gradients (merge/split input, outputs); null in batches
  R *vpx_dx, *vpx_dy, *vpy_dx, *vpy_dy;
  // ---- reference order (not moved by the step) ----
  int *label, *level;
  R *xp, *yp;
  // Ap and Fb as stored at upload / merge/split: valid while Scalars::fresh
  // is set, when the slots are in reference order (otherwise they are
  // derived from the state)
  R *Ap, *Fbx, *Fby;
  // ---- output-only fields of a recorded step (G2P's sorted order) ----
  R *apx, *apy, *Zp, *hpZ, *dZxp, *dZyp, *Fpx, *Fpy, *Frx, *Fry;
};

// Pointers to the moving fields of p, in a fixed order.
constexpr int kMovingR = 15, kMovingI = 3, kMovingV = 4;
template <class R>
struct MovingRefs {
  R** r[kMovingR];
  int** i[kMovingI];
  V2<R>** v[kMovingV];
};
template <class R>
inline MovingRefs<R> moving_refs(ParticlesT<R>& p) {
  return MovingRefs<R>{{&p.x, &p.y, &p.vpx, &p.vpy, &p.hp, &p.F11, &p.F12, &p.F22, &p.Mp,
                        &p.Vp, &p.H, &p.vpx_dx, &p.vpx_dy, &p.vpy_dx, &p.vpy_dy},
                       {&p.key, &p.idx, &p.slot},
                       {&p.mp, &p.qf, &p.xe, &p.qg}};
}
// exchanges the moving buffers of a and b (the other pointers are shared)
template <class R>
inline void swap_moving(ParticlesT<R>& a, ParticlesT<R>& b) {
  MovingRefs<R> ra = moving_refs(a), rb = moving_refs(b);
  for (int k = 0; k < kMovingR; ++k) std::swap(*ra.r[k], *rb.r[k]);
  for (int k = 0; k < kMovingI; ++k) std::swap(*ra.i[k], *rb.i[k]);
  for (int k = 0; k < kMovingV; ++k) std::swap(*ra.v[k], *rb.v[k]);
}
using Particles = ParticlesT<double>;

// Nodal fields, quadgrid node order.
template <class R>
struct NodesT {
  V2<R>* vvL;  // (vvxL, vvyL): the velocities G2P interpolates, one load per node
  // recorded only on output steps
  R *Mv, *mvx, *mvy, *avx, *avy, *vvx, *vvy, *FPxv, *FPyv, *Fricx,
      *Fricy, *Fintx, *Finty, *HV;
};
using Nodes = NodesT<double>;

__global__ void k_step_begin(Scalars* S, Geom G, Phys P);
__global__ void k_step_end(Scalars* S);
// Host launchers of the kernels that exist in both precisions (the kernel
// templates are instantiated in step_kernels.cu, next to their definitions).
template <class R>
void launch_init_particles(int grid, int block, cudaStream_t st, ParticlesT<R> p,
                           const double* Z, const double* dZdx, const double* dZdy,
                           Geom G, Phys P, Scalars* S, int np, int key_off);
// cell keys of the current positions (and idx = slot when set_idx: slots
// in reference order); the next sort scans every cell
__global__ void k_keys(Particles p, Geom G, Scalars* S, int set_idx);
__global__ void k_reduce_state(Particles p, Scalars* S);
template <class R>
void launch_prep(int grid, int block, cudaStream_t st, ParticlesT<R> p, const double* Z,
                 Geom G, Phys P, const Scalars* S, int derive);
// counting sort: slots and counts (after an upload, a state upload or a
// merge/split; a step's G2P counts the keys it makes), the scan of the
// counts over the key range (ranged != 0; else over all n), the scatter into
// perm, and the order by reference index inside each cell
__global__ void k_count(const int* key, int* count, int* slot,
                        const Scalars* S);
__global__ void k_count_n(const int* key, int* count, int* slot, int n);
// tflag (may be null): scan only the flagged tiles (k_b_tile_flags)
__global__ void k_scan_sums(const int* count, int n, int* tile_sum, int* list_n,
                            const Scalars* S, int ranged, const unsigned char* tflag);
__global__ void k_scan_apply(int* count, int n, const int* tile_sum,
                             int* start, int* list, int* list_n,
                             const Scalars* S, int ranged, const unsigned char* tflag);
// pk: 2 x capacity entries; the scatter writes the first half, which the
// per-cell ordering sorts (the crowded cells use both halves)
__global__ void k_scatter(const int* key, const int* slot, const int* idx, const int* start,
                          int* perm, int* skey, unsigned long long* pk, Scalars* S);
__global__ void k_segment_order(const int* start, const int* list, int* list_n,
                                int* perm, const unsigned long long* pk, int* mid,
                                const Scalars* S);
__global__ void k_segment_order_mid(const int* start, const int* mid, int* list_n,
                                    int* perm, const unsigned long long* pk, int* big,
                                    const Scalars* S);
__global__ void k_segment_order_big(const int* start, const int* big,
                                    const int* list_n, int* perm, unsigned long long* pk,
                                    long long cap, const Scalars* S);
// dynamic shared memory of k_segment_order_big; setup_sort sets its limit
// (0 on failure)
size_t sort_big_smem_bytes();
int setup_sort();
__global__ void k_units_plan(const int* cstart, Geom G, const Scalars* S,
                             int target_units, int seg, int* ustart,
                             long long* upex, int4* plan, int* strip_n, int* heavy_n);
// the flat unit list and uorder, the order P2G hands the units out in
// (heavy units first)
__global__ void k_units_flat(const int* strip_n, int strips, int seg,
                             const int4* plan, int4* ulist, int* uorder, int* ucount,
                             const Scalars* S);
// P2G of the single-scenario step (k_p2g specialised for recorded outputs);
// setup_p2g sets its shared-memory attributes and returns the resident CTAs
// per SM (0 on failure)
void launch_p2g(int grid, cudaStream_t st, Particles p, const int* perm, const int* cstart,
                Nodes nodes, double* led_part, Geom G, Phys P, const Scalars* S, int record,
                const int4* ulist, const int* uorder, const int* ucount);
int setup_p2g();
constexpr int kLedgerLog = 1024;  // rows of the per-step ledger log
__global__ void k_ledger_final(const double* led_part, const int* ucount,
                               Scalars* S, double* log);
// G2P of the single-scenario step (k_g2p_t specialised for the two flags):
// reads `cur` through perm, writes `nxt` in this step's sorted order and
// counts the next binning's keys
void launch_g2p(int grid, cudaStream_t st, Particles cur, Particles nxt, const int* perm,
                const int* skey, Nodes nodes, const double* Z, Geom G, Phys P, Scalars* S,
                int* count, int* leave, int record, int want_grad);

// ---- batches of independent scenarios --------------------------------------
// One scenario of a batch: its geometry, physics and place in the packed
// arrays (particles, nodes and cells of all scenarios, back to back).
struct Scn {
  Geom G;
  Phys P;
  int p_off, np;           // particles [p_off, p_off + np)
  int n_off;               // first node
  int c_off;               // first cell (cell keys are c_off + r + c*nrows)
  int strip_off, nstrips;  // its strips in the batch's strip order
  int useg_off;            // first unit-plan slot of its first strip
  int live;                // 0 once removed
};

__global__ void k_b_step_begin(const Scn* scn, Scalars* S, int nscn, Scalars* Sg);
__global__ void k_b_step_end(const Scn* scn, Scalars* S, int nscn);
__global__ void k_b_units_plan(const int* cstart, const Scn* scn, const Scalars* S,
                               const int* strip_scn, const Scalars* Sg,
                               int target_units, int col_weight, int* ustart,
                               long long* upex, int4* plan, int* strip_n, int* heavy_n);
__global__ void k_b_units_flat(const int* strip_n, int strips, const int* strip_scn,
                               const Scn* scn, int nscn, const int4* plan,
                               int4* ulist, int* uorder, int* ucount, int2* scn_units,
                               Scalars* S, const Scalars* Sg);
__global__ void k_b_tile_flags(const Scn* scn, const Scalars* S, int nscn, const Scalars* Sg,
                               unsigned char* tflag, int ntiles);
template <class R>
void launch_b_p2g(int grid, cudaStream_t st, ParticlesT<R> p, const int* perm,
                  const int* cstart, V2<R>* vvL, double* led_part, const Scn* scn,
                  Scalars* S, const int4* ulist, const int* uorder, const int* ucount,
                  const Scalars* Sg);
// sets the batched P2G kernel's shared-memory attributes; returns the
// resident CTAs per SM (0 on failure)
template <class R>
int setup_b_p2g();
__global__ void k_b_ledger(const double* led_part, const int2* scn_units,
                           const Scn* scn, Scalars* S, int nscn,
                           const Scalars* Sg);
template <class R>
void launch_b_g2p(int grid, cudaStream_t st, ParticlesT<R> cur, ParticlesT<R> nxt,
                  const int* perm, const int* skey, const V2<R>* vvL, const double* Z,
                  const Scn* scn, Scalars* S, const int2* gblk, Scalars* Sg, int* count);
template <class R>
void launch_b_move(int grid, cudaStream_t st, ParticlesT<R> dst, ParticlesT<R> src,
                   const int4* mblk);
// float <-> double copies of one particle field (FP32 batch upload/download)
__global__ void k_to_f32(const double* a, float* b, long long n);
__global__ void k_to_f64(const float* a, double* b, long long n);
__global__ void k_b_move_nodes(double* dst, const double* src, const int4* nblk);

__global__ void k_hv(const Particles p, const int* cstart, double* HV, Geom G,
                     const Scalars* S);

size_t p2g_smem_bytes();  // FP64 P2G staging (the single-scenario path)

// ---- one scenario over slabs of cell columns (slab_kernels.cu) ---------------
constexpr int kSlabRecord = 20;  // doubles per particle record that travels
__global__ void k_slab_pack(Particles p, const int* slots, int n, double* buf);
__global__ void k_slab_unpack(Particles p, const double* buf, int n, int base);
__global__ void k_slab_select(const int* key, int n, int col, int nrows, int* slots,
                              int* count);
__global__ void k_slab_keys(const int* key, const int* slots, int n, int* out);
__global__ void k_slab_check(const int* key, int n, int col_lo, int col_hi, int nrows,
                             Scalars* S);
__global__ void k_slab_move(Particles p, const int2* moves, int n);
__global__ void k_slab_scalars(Scalars* S, int np, int ghosts_added, int ncells);
__global__ void k_slab_set_red(Scalars* S, unsigned long long a, unsigned long long b,
                               unsigned long long c);

}  // namespace dampm
