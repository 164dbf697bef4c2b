/*
 * dampm_cuda.h -- C ABI of the B200 (sm_100a) depth-averaged MPM time step.
 *
 * Drop-in boundary for the step loop of dampm (lucadiprofio/AMSC).  It
 * replaces, in the reference project:
 *   - the 17 `gpu_kernels::` free functions (main/gpu_kernels.h:7-196) that
 *     main/gpu_offload.cpp:410-540 launches once per step;
 *   - the per-step host binning `particles_t::init_particle_mesh` and its
 *     PCIe round trip (main/gpu_offload.cpp:546-558);
 *   - the host CFL reduction (main/gpu_offload.cpp:285-300,
 *     main/optim_par.cpp:285-308);
 *   - the host merge/split `adaptive_merge_split` (main/merge_split_ops_cmes.h
 *     :432-447, called from main/gpu_offload.cpp:321-401);
 *   - the loop body of main/optim_par.cpp:281-668 (whose numbers the FP64
 *     path reproduces).
 *
 * Conventions
 *   - Plain C types only; host pointers are host memory, never retained.
 *   - Every function returns 0 (DAMPM_OK) or a negative dampm_status code;
 *     dampm_last_error() gives a one-line message.  Device-side problems are
 *     reported through a device status word, never by a trap: G2P sets it
 *     when any particle's x, y, vpx, vpy or hp is NaN or infinite, or hp is
 *     negative (DAMPM_ERR_DEVICE); merge/split sets it when the particle
 *     capacity would be exceeded (DAMPM_ERR_CAPACITY).  A flagged run does
 *     no further passes.  dampm_sync(), dampm_run() and dampm_status()
 *     return the code; the data-out calls still copy the (diverged) state.
 *   - A context owns all of its device memory and is used from one host
 *     thread at a time.  Work is enqueued on the stream given at creation
 *     (NULL = a stream the context creates).
 *   - Node arrays are in quadgrid order: node (r, c) at r + c*(Ney+1)
 *     (main/gpu_kernels.cpp:7-16); the cell of (r, c) is r + c*Ney.
 *   - Particle arrays passed in and out are in the reference's particle
 *     index order (DATA order, then the compacted order that merge/split
 *     produces, main/merge_split_ops_cmes.h:268-274).
 */
#ifndef DAMPM_CUDA_H
#define DAMPM_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

enum dampm_status {
  DAMPM_OK = 0,
  DAMPM_ERR_ARG = -1,      /* bad argument (null pointer, bad size, ...)   */
  DAMPM_ERR_CUDA = -2,     /* CUDA runtime error                           */
  DAMPM_ERR_STATE = -3,    /* call out of order (e.g. step before upload)  */
  DAMPM_ERR_CAPACITY = -4, /* particle capacity exceeded (merge/split)     */
  DAMPM_ERR_DEVICE = -5,   /* device status word flagged a problem         */
  DAMPM_ERR_UNKNOWN_FIELD = -6
};

/* Grid of main/mpm_data.h:14-17 (grid.set_sizes(Ney, Nex, hx, hy),
 * main/optim_par.cpp:136). */
typedef struct {
  int Nex;
  int Ney;
  double hx;
  double hy;
} dampm_grid;

/* Scalar physics/run parameters of struct DATA (main/mpm_data.h:21-44). */
typedef struct {
  double g, T, rho, xi, mu, phi, tauy;
  double BINGHAM_ON, FRICTION_ON, CFL;
  int BC_FLAG;
  int MERGE_SPLIT_ON;
  double eq_level;
  double DT_FIXED; /* > 0: fixed dt for NSTEPS steps; else CFL until T     */
  int NSTEPS;
} dampm_params;

/* ms_* parameters (main/mpm_data.h:46-56 defaults at :102-112; used as
 * ms_config, main/merge_split_ops_cmes.h:14-37, main/gpu_offload.cpp:308-319).
 */
typedef struct {
  double alpha, beta, split_hp_min, shear_split, hp_min, max_dv;
  int min_level, max_level, min_particles_per_cell, call_interval;
  double max_ops;
  /* Merge only pairs closer than pair_dist * min(hx, hy); 0 (what a
   * positional initialiser of the fields above leaves) = no distance limit,
   * the reference's pairing of the nearest co-moving candidate in the cell
   * (main/merge_split_ops_cmes.h:192-210).  No counterpart in the reference:
   * the benchmark's merge/split configuration asks for 0.25. */
  double pair_dist;
} dampm_ms_params;

typedef struct dampm_ctx dampm_ctx;

/* Precision of particle storage and arithmetic. */
enum dampm_precision { DAMPM_FP64 = 0, DAMPM_FP32 = 1 };

/* Creates a context for one scenario.  `capacity` is the largest particle
 * count the context may hold (merge/split may grow it); 0 = chosen at upload
 * (2x the uploaded count).  Replaces the `target data` region set-up of
 * main/gpu_offload.cpp:258-271. */
int dampm_ctx_create(const dampm_grid* grid, const dampm_params* params,
                     const dampm_ms_params* ms, int precision,
                     long long capacity, void* cuda_stream, dampm_ctx** out);

int dampm_ctx_destroy(dampm_ctx* ctx);

/* Terrain on the nodes, quadgrid node order, (Nex+1)*(Ney+1) values each.
 * Replaces vars["Z"/"dZdx"/"dZdy"] = data.* (main/optim_par.cpp:235-237). */
int dampm_upload_terrain(dampm_ctx* ctx, const double* Z, const double* dZdx,
                         const double* dZdy);

/* Particles in DATA order, then the initialisation of
 * main/optim_par.cpp:147-264 on the device (Zp, H, hpZ, initial stress,
 * label = index, level = 0).  Resets it = 0, t = 0. */
int dampm_upload_particles(dampm_ctx* ctx, long long np, const double* x,
                           const double* y, const double* Mp, const double* Ap,
                           const double* vpx, const double* vpy,
                           const double* hp, const double* mom_px,
                           const double* mom_py, const double* Vp);

/* Enqueues `nsteps` passes of the loop body (dt, it++, merge/split at the
 * gpu_offload cadence when MERGE_SPLIT_ON and enabled, sort, P2G + nodal
 * update, G2P + rheology, t += dt).  A pass whose loop condition
 * (fixed ? it < NSTEPS : t < T) fails on the device does nothing, so this
 * never overshoots.  Asynchronous: returns once the work is enqueued.
 * Without recorded outputs or event timing, passes are replayed from a CUDA
 * graph: 16 at a time, or with merge/split one cycle of call_interval passes
 * at a time from the cycle phase the graph was captured at (passes before
 * that phase run plainly).  The graph is captured by the first call in that
 * mode, whatever its nsteps (a few milliseconds of host time, nothing runs),
 * and again whenever the buffers or parameters change.  The results are the
 * same as with plain launches.  Called while the context's stream is itself
 * being captured, it launches plainly; a stream that cannot be captured, or
 * a graph that cannot be built, turns graphs off for the context. */
int dampm_step(dampm_ctx* ctx, int nsteps);

/* enable = 0: every pass is launched plainly (no CUDA graph); 1 (default):
 * graphs as described at dampm_step.  No counterpart in the reference. */
int dampm_set_graphs(dampm_ctx* ctx, int enable);

/* Runs until the loop condition fails (or max_steps passes), synchronising
 * every `chunk` steps.  *steps_done (may be NULL) receives the count. */
int dampm_run(dampm_ctx* ctx, long long max_steps, int chunk,
              long long* steps_done);

/* Waits for the stream and checks the device status word. */
int dampm_sync(dampm_ctx* ctx);

/* Loop state: iteration, time, last dt, particle count (synchronises).  The
 * outputs are filled in even when the status word is set, which is then
 * returned as the error code. */
int dampm_status(dampm_ctx* ctx, int* it, double* t, double* dt_last,
                 long long* np);

/* Enables merge/split at the gpu_offload cadence (main/gpu_offload.cpp:321)
 * when MERGE_SPLIT_ON != 0.  Off by default: main/optim_par.cpp reads the
 * flag but never splits or merges. */
int dampm_enable_merge_split(dampm_ctx* ctx, int enable);

/* One standalone adaptive_merge_split(dt) on the current state
 * (main/merge_split_ops_cmes.h:432-447; with DAMPM_MS_ELFS selected,
 * main/merge_split_ops.h:720-755, which takes no dt).  counts (may be NULL)
 * receives {splits, merges, np_before, np_after}. */
int dampm_merge_split(dampm_ctx* ctx, double dt, long long counts[4]);

/* Which merge/split the context runs, at the cadence and standalone:
 *   DAMPM_MS_CMES  the one gpu_offload calls, adaptive_merge_split of
 *                  main/merge_split_ops_cmes.h (the default);
 *   DAMPM_MS_ELFS  the ELFS variant, adaptive_merge_split of
 *                  main/merge_split_ops.h:720-755 (the reference builds it
 *                  but calls it nowhere): split where the particle is
 *                  within alpha*sqrt(Ap) of the free surface or its velocity
 *                  divergence exceeds stretch_thresh, merge pairs beyond
 *                  beta*sqrt(Ap); splits are 1 -> 4.
 * The ELFS variant reads alpha, beta, hp_min, max_dv, min_level, max_level,
 * max_ops and call_interval of dampm_ms_params as the fields of the same
 * names of its ms_config (main/merge_split_ops.h:17-30) and ignores the
 * others; stretch_thresh is its ms_config::stretch_thresh (default 1e7).
 * Selecting it allocates four ints per cell of device memory. */
enum dampm_ms_variant { DAMPM_MS_CMES = 0, DAMPM_MS_ELFS = 1 };
int dampm_set_ms_variant(dampm_ctx* ctx, int variant, double stretch_thresh);

/* Copies one particle field to host memory in reference index order.
 * Names: x, y, Mp, Vp, H, hp, vpx, vpy, F_11, F_12, F_21, F_22, Ap, mom_px,
 * mom_py, Fb_x, Fb_y, label, level (as double), and, after a step run with
 * dampm_record_outputs(ctx, 1): vpx_dx, vpx_dy, vpy_dx, vpy_dy, apx, apy, Zp,
 * hpZ, dZxp, dZyp, Fpx, Fpy, Fric_px, Fric_py, vpxL, vpyL, xp, yp.
 * `out` must hold the current particle count. */
int dampm_download(dampm_ctx* ctx, const char* field, double* out);

/* Output without stalling the step loop (the reference writes its output
 * files from inside the step loop, main/optim_par.cpp:311-337): gathers up
 * to 64 particle fields (the names of dampm_download) into reference order
 * on the context's stream, copies them to host_out[k] on a second stream
 * and returns once that is enqueued.  Steps enqueued afterwards run while
 * the copies proceed (host_out must be page-locked for the copies to be
 * asynchronous).  dampm_staged_wait() waits for the copies; the next
 * dampm_stage_download waits for the previous one's first.  *np (may be
 * NULL) receives the count of values each host_out array receives. */
int dampm_stage_download(dampm_ctx* ctx, int n, const char* const* fields,
                         double* const* host_out, long long* np);
int dampm_staged_wait(dampm_ctx* ctx);

/* Copies one nodal field ((Nex+1)*(Ney+1) values) of the last step:
 * vvxL, vvyL always; Mv, mom_vx, mom_vy, avx, avy, vvx, vvy, Ftot_vx,
 * Ftot_vy, F_ext_vx, F_ext_vy, F_int_vx, F_int_vy, FPxv, FPyv, Fric_x,
 * Fric_y, HV after a step run with dampm_record_outputs(ctx, 1); Z, dZdx,
 * dZdy always. */
int dampm_download_nodal(dampm_ctx* ctx, const char* field, double* out);

/* When on, the following steps also materialise the output-only and
 * intermediate fields listed above (the nc_particles / nc_grid columns). */
int dampm_record_outputs(dampm_ctx* ctx, int enable);

/* Conservation ledger of the last step (main/optim_par.cpp:395-425):
 * {sum Mp, sum mom_px, sum mom_py, sum Mv, sum mom_vx, sum mom_vy,
 *  err_mass, err_mom, t}. */
int dampm_ledgers(dampm_ctx* ctx, double out[9]);

/* The conservation_errors.csv rows of steps first_it .. first_it+n-1 (step
 * numbers from 1; any of the last 1024 steps; synchronises): n rows of
 * {t at the step's start, err_mass, err_mom} (main/optim_par.cpp:395-428). */
int dampm_ledger_history(dampm_ctx* ctx, long long first_it, int n, double* out);

/* Overwrites / reads the whole persistent particle state (checkpoint and
 * host round trip).  Arrays in reference index order, np values each:
 * x, y, vpx, vpy, hp, F_11, F_12, F_22, Mp, Vp, H.  set_state marks the
 * next step as reading Ap/mom/Fb from the supplied fresh arrays when they
 * are non-NULL, else recomputing them as the step does. */
int dampm_set_state(dampm_ctx* ctx, long long np, const double* const* fields,
                    const double* Ap, const double* mom_px,
                    const double* mom_py, const double* Fb_x,
                    const double* Fb_y);
int dampm_get_state(dampm_ctx* ctx, double* const* fields);

/* Number of this library's kernel launches enqueued by the last dampm_step
 * call (for launch accounting). */
long long dampm_last_launch_count(dampm_ctx* ctx);

/* Wall time of the kernels of the last dampm_step call, measured with CUDA
 * events on the context stream (ms, synchronises); per kernel class:
 * out[0] sort, out[1] p2g, out[2] g2p, out[3] other, out[4] total. */
int dampm_last_timings(dampm_ctx* ctx, int enable_events, double out[5]);

const char* dampm_last_error(dampm_ctx* ctx);
const char* dampm_version(void);

/* ---- DATA.json at scale ----------------------------------------------------
 * Replaces DATA::DATA(const char*) (main/mpm_data.h:61-122, nlohmann::json)
 * for large files: the file is streamed and each number parsed straight into
 * a double array (std::from_chars: the same rounding as strtod), so a
 * 1 GB DATA.json needs no per-number objects.  Values are numbers or
 * (nested, flattened) arrays of numbers; anything else is an error whose
 * message dampm_json_error gives (free the handle afterwards). */
typedef struct dampm_json dampm_json;
int dampm_json_read(const char* path, dampm_json** out);
/* *n = number of values (a scalar counts 1), or -1 when the key is absent */
int dampm_json_size(const dampm_json* j, const char* key, long long* n);
/* *is_array = 1 for an array value, 0 for a scalar */
int dampm_json_kind(const dampm_json* j, const char* key, int* is_array);
int dampm_json_get(const dampm_json* j, const char* key, double* out);
const char* dampm_json_error(const dampm_json* j);
int dampm_json_free(dampm_json* j);

/* CFL time step from particle arrays held by the caller on the current
 * device, computed on the device without allocating any device memory.
 * No counterpart in the reference: its GPU driver copies vpx, vpy and hp to
 * the host every step and takes the maxima there
 * (main/gpu_offload.cpp:284-300).
 *
 * vpx, vpy, hp: np device values each (1 <= np <= 2^31-1; np beyond that
 * returns DAMPM_ERR_CAPACITY, np < 1 DAMPM_ERR_ARG).  out: 5 doubles in
 * device-writable memory, written asynchronously on cuda_stream (NULL = the
 * legacy default stream of the current device; a non-NULL stream must
 * belong to the current device, else DAMPM_ERR_DEVICE):
 * {CFL*min(hx,hy)/(1e-2+cel), cel, max|vpx|, max|vpy|, max hp} with
 * cel = |max(sqrt(g*hmax)+max|vpx|, sqrt(g*hmax)+max|vpy|)|, the step's own
 * dt formula (main/optim_par.cpp:289-304).
 *
 * Non-finite input: any NaN in vpx or vpy, or a NaN with a clear sign bit in
 * hp, makes the maxima and dt NaN (a sign-set NaN in hp is ignored).  The
 * reference's std::max_element keeps a NaN only where it is the first
 * element, so on a diverged state the two differ; dt is then meaningless
 * either way.
 *
 * The reduction scratch is a fixed 28,416-byte array inside this library,
 * one copy per device; nothing in it has to start at zero.  Its address is
 * looked up in the current context on every call (cudaGetSymbolAddress, a
 * host-side query); the first lookup in a context may load the library's
 * kernels, so make the first call before any stream capture.  Calls whose
 * work can overlap on one device (other streams, other host threads) share
 * the scratch and race: order them on one stream.  Returns DAMPM_ERR_CUDA
 * if the lookup or a launch fails. */
int dampm_cfl_dt_noalloc(const double* vpx, const double* vpy,
                         const double* hp, long long np, double g, double CFL,
                         double hx, double hy, double* out, void* cuda_stream);

/* ---- One scenario over slabs of cell columns --------------------------------
 * A scenario too large for one GPU (or one that should run on several)
 * splits along x: each context in slab mode holds the whole grid's nodes
 * and terrain and the particles of its cell columns [col_lo, col_hi).  The
 * reference has no counterpart (one domain per process, main/optim_par.cpp
 * :128-682, main/gpu_offload.cpp:258-271); with the exchanges below every
 * particle's numbers equal the single-context run bit for bit.  A step is,
 * for all slabs, in this order:
 *   1. dampm_slab_ghosts on slab r, dampm_slab_import(.., ghosts=1) of the
 *      result on slab r+1 (copies of slab r's last column, which P2G of
 *      slab r+1 reads first);
 *   2. dampm_slab_pass(ctx, 0): step start, sort, P2G;
 *   3. dampm_slab_node_column(get) of column col_lo on slab r, (set) on slab
 *      r-1 -- the (vvxL, vvyL) pairs G2P of slab r-1 interpolates;
 *   4. dampm_slab_pass(ctx, 1): G2P, step end;
 *   5. dampm_slab_route on every slab, dampm_slab_import(.., ghosts=0) of
 *      its left / right output on slab r-1 / r+1 (particles that moved);
 *   6. dampm_slab_cfl(get) on every slab, the element-wise maximum set on
 *      every slab (the next CFL step).
 * Buffers are device memory on the context's device holding particle
 * records of dampm_slab_record_doubles() doubles.  A particle may move at
 * most one slab per step (DAMPM_ERR_STATE otherwise).  Slab mode excludes
 * merge/split, recorded outputs and CUDA graphs; dampm_step, dampm_download
 * and the state calls return DAMPM_ERR_STATE in it. */
int dampm_slab_record_doubles(void);
/* After dampm_upload_particles of the slab's own particles (any order). */
int dampm_slab_set(dampm_ctx* ctx, int col_lo, int col_hi);
/* The reference index of each uploaded particle (np host ints). */
int dampm_slab_set_index(dampm_ctx* ctx, const int* idx);
int dampm_slab_ghosts(dampm_ctx* ctx, double* buf, long long cap, long long* n);
int dampm_slab_import(dampm_ctx* ctx, const double* buf, long long n, int ghosts);
int dampm_slab_pass(dampm_ctx* ctx, int phase);
/* (Ney+1) pairs (vvxL, vvyL) of node column col: set != 0 writes them. */
int dampm_slab_node_column(dampm_ctx* ctx, int col, double* buf, int set);
/* Particles whose new cell is left of col_lo go to `left`, right of
 * col_hi - 1 to `right` (NULL at the domain's edges); cap records each. */
int dampm_slab_route(dampm_ctx* ctx, double* left, double* right, long long cap,
                     long long* n_left, long long* n_right);
/* {max |vpx|, max |vpy|, max hp} of the slab's last G2P (get), or the
 * maxima over all slabs for the next step's CFL dt (set != 0). */
int dampm_slab_cfl(dampm_ctx* ctx, double maxima[3], int set);
/* One field of the slab's own particles in storage order, with their
 * reference indices in idx (may be NULL).  Fields as dampm_get_state. */
int dampm_slab_download(dampm_ctx* ctx, const char* field, double* out, long long* idx);

/* ---- Batches of independent scenarios -------------------------------------
 * One set of device arrays holds many scenarios back to back, each with its
 * own grid, terrain, particles, physics and loop (fixed dt for NSTEPS passes,
 * or CFL until T); one launch per kernel advances all of them.  A scenario's
 * numbers are the same alone (dampm_ctx) and in a batch.  There is no
 * counterpart in the reference, which runs one DATA per process
 * (main/optim_par.cpp:128-682); the batch applies that loop body to each
 * scenario.  Merge/split and recorded outputs are not part of a batch. */
typedef struct dampm_batch dampm_batch;

/* Capacities: total particles and total nodes over the scenarios the batch
 * holds at once (live and removed-but-not-compacted), and scenario slots.
 * Device memory is allocated here once: ~390 B per particle and ~56 B per
 * node of capacity. */
int dampm_batch_create(long long particle_cap, long long node_cap,
                       int scenario_cap, int precision, void* cuda_stream,
                       dampm_batch** out);
int dampm_batch_destroy(dampm_batch* b);

/* Appends one scenario (DATA arrays in DATA order, terrain Z in quadgrid node
 * order; the gradients dZdx/dZdy only feed recorded outputs and are not
 * taken).  Returns DAMPM_ERR_CAPACITY when the batch is full.  *handle
 * identifies the scenario in later calls. */
int dampm_batch_add(dampm_batch* b, const dampm_grid* grid,
                    const dampm_params* params, const double* Z, long long np,
                    const double* x, const double* y, const double* Mp,
                    const double* Ap, const double* vpx, const double* vpy,
                    const double* hp, const double* mom_px, const double* mom_py,
                    const double* Vp, int* handle);

/* Stops a scenario; its room is reclaimed by dampm_batch_compact, which moves
 * the live scenarios together (a synchronising call). */
int dampm_batch_remove(dampm_batch* b, int handle);
int dampm_batch_compact(dampm_batch* b);

/* Enqueues nsteps passes of every live scenario (asynchronous); a scenario
 * whose loop condition fails does nothing in a pass.  Each run of 16 passes
 * replays one CUDA graph, captured on the batch stream after a change of
 * layout; the passes left over are launched one by one.  Before returning,
 * the call captures (without running it) the graph the next call starts
 * from, if the layout changed.  Inside the caller's own capture of the
 * stream every pass is launched one by one (see dampm_batch_tune). */
int dampm_batch_step(dampm_batch* b, int nsteps);
int dampm_batch_sync(dampm_batch* b);

/* Tuning, for an autotuner: P2G units per CTA of the unit plan and the
 * weight (in particles) of a column in it, and whether dampm_batch_step
 * replays its passes as a CUDA graph (captured after each change of layout;
 * 1 by default).  0 (or -1 for use_graphs) keeps a setting.  None of these
 * changes any result. */
int dampm_batch_tune(dampm_batch* b, int units_per_cta, int col_weight,
                     int use_graphs);

/* Loop state of one scenario (synchronises): iteration, time, last dt,
 * whether its loop condition still holds, particle count. */
int dampm_batch_query(dampm_batch* b, int handle, int* it, double* t,
                      double* dt_last, int* running, long long* np);

/* The loop state of every live scenario in one synchronising call: handle,
 * running (1: its loop condition still holds; 0: finished; -1: stopped by
 * its status word -- its state diverged, see the conventions above; the
 * other scenarios are unaffected), iteration, time.  cap is the length of
 * the arrays; *count receives the live count. */
int dampm_batch_states(dampm_batch* b, int cap, int* handles, int* running,
                       int* its, double* ts, int* count);

/* One particle field of one scenario, reference index order: x, y, vpx, vpy,
 * hp, F_11, F_12 (= F_21), F_22, Mp, Vp, H, mom_px, mom_py. */
int dampm_batch_download(dampm_batch* b, int handle, const char* field,
                         double* out);
int dampm_batch_ledgers(dampm_batch* b, int handle, double out[9]);

/* {live scenarios, removed scenarios awaiting compaction, particles held,
 *  particle capacity, nodes held, node capacity, scenario slots, kernel
 *  launches so far}: what an admission policy needs. */
int dampm_batch_usage(dampm_batch* b, long long out[8]);
const char* dampm_batch_last_error(dampm_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* DAMPM_CUDA_H */
