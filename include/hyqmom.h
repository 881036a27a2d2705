/* C-ABI of libhyqmom_b200.so: the HyQMOM explicit time step on one B200.
 *
 * Drop-in boundary for the reference's time loop.  The reference
 * (HyQMOM.jl) has no FFI; these entry points replace the body of
 * simulation_runner (src/simulation_runner.jl:346-560, one rank):
 *   hyq_create        <- parameter unpacking + allocation (:63-185)
 *   hyq_set_state     <- IC fill of M (:187-271), done by the caller's IC code
 *   hyq_advance       <- `while t < tmax && nn < nnmax` step loop (:346-560)
 *   hyq_get_state     <- gather_M of the interior (:745-752)
 *   hyq_get_SC        <- compute_standardized_field / compute_central_field
 *                        (src/utils/compute_standardized_field.jl:16-66)
 *   hyq_stats         <- vmax / dt diagnostics printed by the loop (:402-433)
 * State buffers are Julia column-major (Nx, Ny, Nz, 35) Float64 arrays
 * (moment-major SoA), passed as plain pointers.
 *
 * Conventions: every call returns 0 on success or a negative HYQ_E* code;
 * hyq_last_error(ctx) describes the last failure.  The library owns device
 * memory; the caller owns host buffers.  A context is not thread-safe.
 */
#ifndef HYQMOM_B200_H
#define HYQMOM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HYQ_ABI_VERSION 2

#define HYQ_OK 0
#define HYQ_EINVAL -1      /* invalid argument or parameter */
#define HYQ_ECUDA -2       /* CUDA runtime error */
#define HYQ_ENONFINITE -3  /* non-finite state found (opt-in check) */
#define HYQ_ETIMEOUT -4    /* a bounded device wait ran out */
#define HYQ_ENOMEM -5      /* device allocation failed */

/* Eigenvalue path of a context (hyq_params.mode).
 * HYQ_MODE_PLAIN: every flux-Jacobian eigen-solve follows the reference's
 *   LAPACK path (eigvals), bit for bit.
 * HYQ_MODE_LEARNED: the learned wave-speed path.  After the first closure of
 *   each step a small network (35 standardized moments -> 6 standardized
 *   extreme speeds, BF16 tensor-core kernels) predicts each cell's extreme
 *   x/y/z wave speeds; they seed a certified solve of each Jacobian's
 *   characteristic polynomial, which proves all six eigenvalues real and
 *   distinct and converges the extremes to full FP64 precision.  Jacobians it
 *   cannot certify (and the usual pattern-1 Jacobians, which are cheap) take
 *   the LAPACK path, so the speeds agree with the plain path to round-off and
 *   every complex-eigenvalue decision is the reference's.  Needs the network
 *   (hyq_set_wavespeed_net) before the first step.
 * HYQ_MODE_CERTIFIED: the same certified solve started from bounds instead of
 *   predicted speeds (the learned path without its network). */
#define HYQ_MODE_PLAIN 0
#define HYQ_MODE_LEARNED 1
#define HYQ_MODE_CERTIFIED 2

/* Fields read by simulation_runner (src/simulation_runner.jl:74-129). */
typedef struct hyq_params {
  int32_t Nx, Ny, Nz;
  int32_t flag2D;      /* params.flag2D */
  int32_t positivity;  /* params.positivity (default true, :87-91) */
  int32_t device;      /* CUDA device ordinal */
  int64_t nnmax;       /* params.nnmax */
  double tmax, Kn, Ma, CFL, dtmax;
  double xmin, xmax, ymin, ymax, zmin, zmax; /* domain extents (:123-129) */
  int32_t mode;        /* HYQ_MODE_* (0 = plain, the reference's path) */
  int32_t symmetry_check_interval; /* params.symmetry_check_interval: MaxDiff
                                    * every this many steps and at step 1
                                    * (:562-637); 0 = never */
} hyq_params;

typedef struct hyq_stats {
  double t, dt, vmax;  /* time, last dt, last CFL wave speed (:402-433) */
  int64_t nn;          /* steps taken */
  int32_t done;        /* 1 once t >= tmax or nn >= nnmax */
  int32_t status;      /* 0 = ok; k > 0: step k met a non-finite wave speed */
  /* learned / certified modes, summed since hyq_set_state or
   * hyq_reset_counters: cells of the certified eigenvalue stages (five per
   * step: x, y, z before the flux, x, y after it) and those of them that fell
   * back to the LAPACK path (a Jacobian not certified).  0 in plain mode. */
  int64_t stage_cells, fallback_cells;
  /* eigenvalue stages (bit q: A x, y, z, E x, y) running dense at this step:
   * their general eigen-solve takes every cell directly because the stage
   * listed most of its cells recently */
  int32_t dense_mask;
  /* first-step diagnostics (:404-470): the largest |wave speed| along x, y
   * and z at step 1, and the cell (c = i + Nx (j + Ny k)) and direction
   * (0 x, 1 y, 2 z) of the largest one */
  int32_t worst_dir;
  double vmax_first[3];
  int64_t worst_cell;
  /* the diagonal symmetry measure MaxDiff (:562-637) of the state after step
   * maxdiff_step (the last step with nn % symmetry_check_interval == 0 or
   * nn == 1; -1 before any) */
  double maxdiff;
  int64_t maxdiff_step;
} hyq_stats;

typedef struct hyq_ctx hyq_ctx;

int hyq_abi_version(void);
/* Grids need Nx >= 2, Ny >= 2, Nz >= 1 and fewer than 2^29 cells (the step's
 * cell lists hold 32-bit entries); anything else gets HYQ_EINVAL before any
 * CUDA call. */
int hyq_create(const hyq_params* p, hyq_ctx** out);
void hyq_destroy(hyq_ctx* ctx);
const char* hyq_last_error(const hyq_ctx* ctx);

/* ---- a domain decomposed into z-slabs (one context per slab) -------------
 * No reference counterpart as an API: replaces the rank-local parts of the
 * reference's MPI step (src/mpi/halo_exchange_3d.jl:26-122, the dt
 * all-reduce at src/simulation_runner.jl:403).  A slab context holds its
 * own z-layers plus two ghost layers on each side that has a neighbour, and
 * steps in two halves around the CFL reduction:
 *   hyq_step_begin: phase [A] on every local layer (ghosts included: their
 *     inputs are the neighbour's pre-step layers, so they reproduce the
 *     neighbour's results bit for bit) and the local max |speed|, written to
 *     the device buffer *xchg = {max |speed| over non-NaN cells, NaN flag};
 *     the caller reduces it with MAX over the slabs in place (e.g. an NCCL
 *     all-reduce on the context's stream, hyq_stream) before
 *   hyq_step_end: dt from the global value, then the HLL sweeps (each owned
 *     layer is at least two layers from the local ends, so the serial
 *     boundary rules there touch only ghosts), phases [E]+[F].
 * The slabs' owned layers then equal the single-domain step bit for bit.
 * hyq_copy_layers copies z-layers [k0, k0 + nk) of all 35 moment planes
 * between the state and a packed device buffer (35 planes of nk Nx Ny
 * doubles; into_state = 1 writes the state), on the context's stream, for
 * the ghost exchange.  hyq_set_spacing overrides dx, dy, dz (the slab's
 * extents then need not divide exactly). */
int hyq_step_begin(hyq_ctx* ctx, double* xchg);
int hyq_step_end(hyq_ctx* ctx, const double* xchg);
int hyq_copy_layers(hyq_ctx* ctx, int32_t k0, int32_t nk, double* buf, int32_t into_state);
int hyq_set_spacing(hyq_ctx* ctx, double dx, double dy, double dz);

/* Host (Nx,Ny,Nz,35) column-major buffers; time and step count reset to 0
 * by hyq_set_state (simulation_runner's t = 0.0; nn = 0, :333-334). */
int hyq_set_state(hyq_ctx* ctx, const double* M);
int hyq_get_state(hyq_ctx* ctx, double* M);
/* Device-pointer variants (same layout, device memory of ctx's device).
 * Both copy on the context's stream (hyq_stream), a non-blocking stream that
 * is not ordered against the caller's streams (nor the legacy default
 * stream), and return before the copy has finished.  A caller that writes dM
 * on its own stream must finish that work before hyq_set_state_device, and
 * must order any use of dM after hyq_get_state_device behind the context's
 * stream (hyq_synchronize, or an event recorded on hyq_stream). */
int hyq_set_state_device(hyq_ctx* ctx, const double* dM);
int hyq_get_state_device(hyq_ctx* ctx, double* dM);
/* The initial condition generated on the device (no host state, no upload):
 * the reference's region fill of initialize_moment_field_mpi
 * (src/initial_conditions.jl:152-217, cell_overlaps_cube :281-302) and of the
 * runner's built-in cubes (src/simulation_runner.jl:200-271).  Every cell
 * gets bg[35], then, region by region in order, the region's moments where
 * the region covers the cell:
 *   kind 0, a box [lo, hi] in coordinates (lo = center - width/2, hi =
 *     center + width/2 as the reference forms them): the cell with centre
 *     (xm[i], ym[j], zm[k]) and widths (dx, dy, dz) overlaps it when
 *     max(x - d/2, lo) < min(x + d/2, hi) on every axis (strict, as the
 *     reference), or everywhere when `everywhere` is set (infinite width);
 *   kind 1, an index box: i0 <= i <= i1, j0 <= j <= j1, k0 <= k <= k1
 *     (0-based, inclusive).
 * xm, ym, zm: the cell centres (Nx, Ny, Nz doubles, Julia range values);
 * moments: 35 * nregions doubles.  Time and step count reset to 0. */
typedef struct hyq_ic_region {
  int32_t kind, everywhere;
  double lo[3], hi[3];
  int32_t i0, i1, j0, j1, k0, k1;
} hyq_ic_region;
int hyq_set_state_ic(hyq_ctx* ctx, const double* xm, const double* ym, const double* zm, double dx, double dy, double dz,
                     const double* bg, int32_t nregions, const hyq_ic_region* regions, const double* moments);

/* Set the loop clock (t, nn) without touching the state. */
int hyq_set_clock(hyq_ctx* ctx, double t, int64_t nn);
/* Zero the fallback counters of hyq_stats. */
int hyq_reset_counters(hyq_ctx* ctx);

/* The wave-speed network of HYQ_MODE_LEARNED (no reference counterpart: it
 * replaces nothing, it only seeds the certified solve of
 * compute_jacobian_eigenvalues, src/numerics/compute_jacobian_eigenvalues.jl:18-50).
 * w: HYQ_NET_PARAMS floats, the FP32 parameters in this order (row-major,
 * out x in): W1 (128 x 35), b1 (128), W2 (128 x 128), b2 (128),
 * W3 (128 x 128), b3 (128), W4 (6 x 128), b4 (6); SiLU between layers.
 * Inputs: the cell's 35 standardized moments (M2CS4_35's S); outputs: the
 * extreme eigenvalues of the x, y and z flux Jacobians as (lam - u_a) /
 * sqrt(C_aa), in the order x min, x max, y min, y max, z min, z max.
 * margin: normalised distance by which the seeds are moved outward.  The
 * weights are stored as BF16 on the device. */
#define HYQ_NET_PARAMS 38406
int hyq_set_wavespeed_net(hyq_ctx* ctx, const float* w, double margin);

/* ---- the wave-speed network's own kernels (device pointers) ---------------
 * No reference counterpart: these train and evaluate the network of
 * HYQ_MODE_LEARNED with hand-written tcgen05 (BF16 x BF16 -> FP32) kernels.
 * All pointers are device memory of the current device; every call is
 * asynchronous on `stream` (a cudaStream_t, NULL for the legacy stream).
 * Kernel waits are bounded: a wait that runs out sets *err (device int) to a
 * nonzero value instead of hanging; check it after synchronising.
 *   image: hyq_net_image_bytes() bytes, the BF16 weight image (hyq_net_pack).
 *   X: training inputs, ceil(n / 128) tiles of hyq_net_tile_bytes() bytes
 *      (hyq_net_features of the moments, stride n).
 *   T: targets, n rows of 8 floats (the 6 outputs, 2 unused).
 *   order: the tiles of one batch (ntiles indices into X).
 *   partial: nparts * HYQ_NET_PARAMS floats of per-CTA gradients (nparts
 *      CTAs run the batch); ds_scratch: hyq_net_scratch_bytes(nparts) bytes.
 *   loss: += the batch's sum of squared errors; the gradient is that of
 *      dscale / 2 * (sum of squared errors), dscale = 2 / (rows * 6) for the
 *      mean square error.
 *   hyq_net_adam sums the partials (into gout, when not NULL) and, with
 *   lr > 0, takes one Adam step (decoupled weight decay wd) on w. */
int64_t hyq_net_image_bytes(void);
int64_t hyq_net_tile_bytes(void);
int64_t hyq_net_scratch_bytes(int32_t nparts);
int hyq_net_pack(const float* w, void* image, void* stream);
int hyq_net_features(const double* M, int64_t n, void* X, void* stream);
/* out: [6][n] FP32, the standardized extreme speeds of moments M (stride n) */
int hyq_net_forward(const void* image, const double* M, int64_t n, float* out, int32_t* err, void* stream);
int hyq_net_train_batch(const void* image, const void* X, const float* T, int64_t n, const int32_t* order, int32_t ntiles,
                        float dscale, void* ds_scratch, float* partial, int32_t nparts, float* loss, int32_t* err, void* stream);
int hyq_net_adam(float* w, float* m, float* v, const float* partial, int32_t nparts, float lr, float beta1, float beta2, float eps,
                 float wd, int32_t step, float* gout, void* stream);
/* Training targets of n cells (moments M, stride n): the plain path's
 * extreme eigenvalues of the x, y and z flux Jacobians of the realized
 * moments, standardized as the network outputs; T: n rows of 8 floats (NaN
 * where a speed is not finite); Mr (may be NULL): the realized moments. */
int hyq_cells_wavespeed_targets(const double* M, int64_t n, int32_t flag2D, double Ma, int32_t positivity, float* T, double* Mr,
                                void* stream);

/* Run up to max_steps steps of the reference loop, stopping on the device
 * once t >= tmax or nn >= nnmax.  Outputs may be NULL.  Returns
 * HYQ_ENONFINITE (outputs still filled) once a step met a non-finite CFL wave
 * speed: the reference's eigvals throws at that point; here t becomes NaN
 * and the loop predicate stops further steps. */
int hyq_advance(hyq_ctx* ctx, int64_t max_steps, double* t, int64_t* nn, int32_t* done);
/* Same, asynchronous on the context's stream (no host synchronization). */
int hyq_advance_async(hyq_ctx* ctx, int64_t max_steps);
int hyq_synchronize(hyq_ctx* ctx);
int hyq_stats_get(hyq_ctx* ctx, hyq_stats* out);

/* One step of the reference loop on a host state, the host<->device copies
 * overlapped with the per-cell phases: the state goes up in `nslabs` chunks
 * of whole 128-cell blocks while phase [A] runs on the chunks already there,
 * and comes back chunk by chunk as phases [E]+[F] finish them (the CFL
 * reduction and the HLL sweep need every cell and run in between).  The
 * chunks are graded: the uploads grow and the downloads shrink, so that only
 * a small first upload and a small last download are not hidden.  M_in and
 * M_out are host (Nx,Ny,Nz,35) column-major buffers and may be the same; in
 * pinned memory the copies run asynchronously.  The step uses the context's
 * clock (t, nn) like hyq_advance(ctx, 1, ...), with the same outputs and
 * return codes; the device state is left equal to M_out. */
int hyq_step_host(hyq_ctx* ctx, const double* M_in, double* M_out, int32_t nslabs, double* t, int64_t* nn, int32_t* done);

/* Standardized and central moment fields of the current state, host
 * (Nx,Ny,Nz,35) buffers (either may be NULL). */
int hyq_get_SC(hyq_ctx* ctx, double* S, double* C);

/* cudaStream_t of the context, for callers that order their own work. */
void* hyq_stream(hyq_ctx* ctx);

/* Run `steps` steps launching the step kernels individually (not the graph)
 * with CUDA events around each on the context stream; ms[HYQ_TIMED_SLOTS]
 * receives the summed device time of each kernel, in launch order:
 * A1 closure, A2 x eigenvalues, A3 y eigenvalues, A4 z eigenvalues (each
 * with its passes over the cells it listed: general eigen-solve, correction),
 * A5 closure with fluxes and speeds, CFL reduction, HLL sweep,
 * E1 closure, E2 x eigenvalues, E3 y eigenvalues (each with its pass that
 * decides and corrects the listed cells), E4 closure + BGK.
 * For profiling; results equal hyq_advance. */
#define HYQ_TIMED_SLOTS 11
int hyq_advance_timed(hyq_ctx* ctx, int64_t steps, float* ms);

/* ---- batched independent domains ------------------------------------------
 * The reference runs one simulation per simulation_runner call; a sweep of
 * many small domains (uneven grids, each with its own Ma, Kn, CFL, tmax,
 * nnmax and dt) leaves most of a B200 idle when run one at a time.  A batch
 * owns one ordinary context per member (hyq_batch_member returns it, for
 * hyq_set_state / hyq_get_state / hyq_stats_get) and one CUDA graph per step
 * in one of two schedules:
 *   HYQ_BATCH_FUSED (default when all members share hyq_params.mode): one
 *     launch per kernel of the step for ALL members; each block finds its
 *     member in a table (constants, device clock, buffers) and works on that
 *     member's cells, so a step is the same ~24 launches however many members
 *     there are, and the block scheduler balances the (member, cell block)
 *     queue of each launch;
 *   HYQ_BATCH_BRANCHES: every member's own step graph as an independent
 *     branch of the batch graph.
 * Each replay advances every member that is not done by one step with its
 * own dt.  Members stop on the device at their own tmax / nnmax or at a
 * non-finite wave speed (their stats status > 0); that is not an error of
 * the batch call.  Both schedules give every member the bits of its own
 * hyq_advance.  Batch calls report failures through hyq_last_error(NULL). */
#define HYQ_BATCH_BRANCHES 0
#define HYQ_BATCH_FUSED 1
typedef struct hyq_batch hyq_batch;
int hyq_batch_create(const hyq_params* p, int32_t n, hyq_batch** out);  /* p[n], one device, n <= 4096 */
void hyq_batch_destroy(hyq_batch* b);
int32_t hyq_batch_size(const hyq_batch* b);
hyq_ctx* hyq_batch_member(hyq_batch* b, int32_t i);  /* NULL when out of range */
void* hyq_batch_stream(hyq_batch* b);                /* cudaStream_t of the replays */
/* HYQ_EINVAL for a fused schedule over members of different modes. */
int hyq_batch_set_schedule(hyq_batch* b, int32_t schedule);
int32_t hyq_batch_schedule(const hyq_batch* b);
/* Queue max_steps replays (after waiting for the members' own streams).
 * Each member's stream is then made to wait for the replays, so a later
 * member call (hyq_get_state, hyq_stats_get, hyq_set_state) sees the state
 * after them.  A member whose constants changed since the last replay
 * (hyq_set_spacing, hyq_set_wavespeed_net, hyq_set_variant) is picked up by
 * capturing the batch graph again. */
int hyq_batch_advance_async(hyq_batch* b, int64_t max_steps);
/* Same, then wait; ndone / nfailed (may be NULL) count members that are done
 * and members that met a non-finite wave speed. */
int hyq_batch_advance(hyq_batch* b, int64_t max_steps, int32_t* ndone, int32_t* nfailed);

/* ---- launch variants (for the autotuner) ----------------------------------
 * Kernels with more than one launch shape; every variant gives the same bits,
 * only the time differs.  hyqmom/autotune.py times them on the caller's own
 * workload and keeps the choice per device.
 *   HYQ_KERNEL_HLL: cells per block x moment groups of the HLL sweep
 *     (0: 256 x 1, 1: 256 x 5, 2: 256 x 7, 3: 128 x 5, 4: 128 x 7, 5: 128 x 1;
 *     6: 256 x 7 and 7: 256 x 5 with fewer registers for more resident blocks;
 *     8, 9: 32 x 8 and 32 x 4 cell tiles of a layer staged in shared memory,
 *     7 groups of 5 moments);
 *     per context (hyq_set_variant) or for every member of a batch.
 *   HYQ_KERNEL_CORR: blocks per member of a fused batch's correction passes
 *     (0: 64, 1: 16, 2: 4, 3: 592); batches only. */
#define HYQ_KERNEL_HLL 0
#define HYQ_KERNEL_CORR 1
#define HYQ_CORR_VARIANTS 4
int32_t hyq_variant_count(int32_t kernel);
int hyq_set_variant(hyq_ctx* ctx, int32_t kernel, int32_t variant);
int hyq_batch_set_variant(hyq_batch* b, int32_t kernel, int32_t variant);

/* ---- allocation-free step ------------------------------------------------
 * No counterpart in the reference (its Julia loop allocates freely); added
 * for callers that must not allocate device memory while they step: a host
 * program that passes in a buffer from its own pool under a fixed memory
 * budget, or a loop that cannot take the device-wide synchronisation that
 * cudaMalloc/cudaFree may cause.  hyq_step_noalloc runs one step of the same
 * kernels as hyq_advance on M (device pointer, 35*N doubles, the moment-major
 * layout of hyq_set_state_device), updated in place.  stats: in, t and nn of
 * the state; out, t, dt, vmax, nn, done and status after the step (no step is
 * taken once t >= tmax or nn >= nnmax).  It returns after the step finished
 * on `stream` (a cudaStream_t, NULL = default stream).
 * Its work arrays live in one fixed scratch array in the library's device
 * image (about 19 MB), sized for at most HYQ_NOALLOC_MAX_CELLS cells; larger
 * grids get HYQ_EINVAL.  All calls on a device share that scratch, so calls
 * that overlap on one device (other host threads, unordered streams) race
 * and corrupt each other's step.  The first call on each device looks up the
 * scratch address (and may load the module); make it before any stream
 * capture on that device. */
#define HYQ_NOALLOC_MAX_CELLS 16384
int hyq_step_noalloc(const hyq_params* p, double* M, hyq_stats* stats, void* stream);

/* ---- per-cell entry points on device arrays (SoA, stride n) ------------
 * Used by parity tests and by callers composing their own loops.  `stream`
 * is a cudaStream_t (NULL = default stream).  Arrays are device pointers. */
/* Flux_closure35_and_realizable_3D (src/numerics/Flux_closure35_and_realizable_3D.jl:33). */
int hyq_cells_flux_closure(const double* M, int64_t n, int32_t flag2D, double Ma, double* Fx, double* Fy, double* Fz,
                           double* Mr, void* stream);
/* eigenvalues6_hyperbolic_3D (axis 1, 2) and eigenvalues6z_hyperbolic_3D (axis 3):
 * v[2n] = (vmin, vmax) pairs, Mr the corrected moments
 * (src/numerics/eigenvalues6_hyperbolic_3D.jl:22, eigenvalues6z_hyperbolic_3D.jl:23). */
int hyq_cells_eigenvalues(const double* M, int64_t n, int32_t axis, int32_t flag2D, double Ma, int32_t positivity,
                          double* v, double* Mr, void* stream);
/* closure_and_eigenvalues on 5 moments per cell (src/numerics/closure_and_eigenvalues.jl:76):
 * mom[5n] SoA, v[2n] = (vmin, vmax). */
int hyq_cells_closure_eigs(const double* mom, int64_t n, double* v, void* stream);
/* collision35 (src/numerics/collision35.jl:154). */
int hyq_cells_collision(const double* M, int64_t n, double dt, double Kn, int32_t positivity, double* out, void* stream);
/* Phase [A] of the step (src/simulation_runner.jl:357-379): fluxes, realizable
 * moments and the six wave-speed arrays vp[6n] = (xmin,xmax,ymin,ymax,zmin,zmax).
 * Runs as a chain of per-function kernels on `stream` that keep their
 * intermediate states in the output arrays, so M must not overlap them. */
int hyq_cells_phase_A(const double* M, int64_t n, int32_t flag2D, double Ma, int32_t positivity, double* Fx, double* Fy,
                      double* Fz, double* Mr, double* vp, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HYQMOM_B200_H */
