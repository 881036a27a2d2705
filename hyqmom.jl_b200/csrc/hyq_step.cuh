// Shared definitions of the step kernels, split over several translation
// units so that ptxas compiles the large per-cell kernels in parallel.
#pragma once
#include <cuda_runtime.h>

namespace hyqk {

// Device-side loop clock of one simulation (t, dt, nn live on the GPU).
struct DevClock {
  double t, dt, vmax;
  long long nn;
  int active;  // 1 while the current step runs
  int status;
  // per eigenvalue stage (A x, y, z, E x, y): runs left in which the general
  // eigen-solve takes every cell directly (set when a stage listed most of its
  // cells; 0: the pattern-1 kernel first)
  int dense[5];
  // learned wave-speed path: cells whose Jacobians the certified solve could
  // not certify (they fell back to the LAPACK path), and cells the certified
  // stages processed, summed over stages and steps since the last reset
  unsigned long long fb_cells, stage_cells;
  // first-step diagnostics: per-direction max |speed| (bit patterns, for
  // atomicMax), the worst cell and its direction
  unsigned long long vdir_bits[3];
  unsigned long long worst_cell;
  int worst_dir;
  // MaxDiff of the state after step maxdiff_nn (-1: none yet)
  double maxdiff;
  long long maxdiff_nn;
};

// Eigenvalue path of a context (hyq_params.mode).
enum StepMode { MODE_PLAIN = 0, MODE_LEARNED = 1, MODE_CERTIFIED = 2 };

// Per-context constants of the step.
struct StepConst {
  long long N;
  int Nx, Ny, Nz, flag2D, positivity;
  long long nnmax;
  double tmax, Kn, Ma, CFL, dtmax, dx, dy, dz;
  int nblocksA;
  // MODE_PLAIN: the LAPACK-path eigen-solve of the reference for every
  // Jacobian.  MODE_CERTIFIED: the certified characteristic-polynomial solve
  // (hyq_charpoly.cuh) for every Jacobian it can certify, from bound starts.
  // MODE_LEARNED: the same, started from the wave-speed network's predicted
  // speeds, which the network kernel writes to `seeds` after the first
  // closure of each step.
  int mode;
  int symmetry_check_interval;
  // predicted standardized extreme speeds, SoA [6][N] (x lo, x hi, y lo,
  // y hi, z lo, z hi): lam = u + sqrt(C_aa) * s; NULL unless MODE_LEARNED
  float* seeds;
  double seed_margin;  // normalised outward shift of the seeds
};

// Minimum resident blocks per SM requested from ptxas for the per-cell
// kernels (bounds their registers): the closure kernels run best at 4 blocks
// of 128 threads (128 registers), the eigenvalue kernels at 8 (64 registers);
// measured on the 160x160x80 crossing-jets step.
#ifndef HQ_MINB_CLOSURE
#define HQ_MINB_CLOSURE 4
#endif
// The closures without fluxes (A1, E1) run best at 3 blocks (168 registers),
// measured on step 151 of the 128x128x64 crossing-jets run.
#ifndef HQ_MINB_REALIZE
#define HQ_MINB_REALIZE 3
#endif
#ifndef HQ_MINB_EIG
#define HQ_MINB_EIG 8
#endif
// The passes over listed cells (complete eigen-solve, corrections) run at the
// eigenvalue kernels' occupancy (fewer resident blocks with more registers
// were slower), one thread per possible entry of the list, so that the block
// scheduler balances the uneven per-cell cost (a persistent grid striding
// over a long list was 1.5x slower).
#ifndef HQ_MINB_FIX
#define HQ_MINB_FIX 8
#endif
constexpr int MINB_CLOSURE = HQ_MINB_CLOSURE;
constexpr int MINB_REALIZE = HQ_MINB_REALIZE;
constexpr int MINB_EIG = HQ_MINB_EIG;
constexpr int MINB_FIX = HQ_MINB_FIX;
// Eigen-solve code of those passes (hyq::JacMode; 2 = the general code only)
#ifndef HQ_FIX_MODE
#define HQ_FIX_MODE 2
#endif
constexpr int FIX_MODE = HQ_FIX_MODE;
// Eigen-solve code of the eigenvalue kernels themselves (hyq::JacMode; 1 =
// the pattern-1 register path, the rest left to the passes above)
#ifndef HQ_EIG_MODE
#define HQ_EIG_MODE 1
#endif
constexpr int EIG_MODE = HQ_EIG_MODE;
// A stage that listed more than 3/4 of its cells runs dense for the next
// DENSE_RUNS runs, then tries the pattern-1 kernel again.
constexpr int DENSE_RUNS = 16;
// The correction passes (few cells, or none) stride over their list with at
// most one wave of blocks of CORR_BS threads: one warp per block, so that a
// short list spreads one cell per SM-resident warp and each lone lane's work
// arrays stay in L1 (a lone lane touches a separate cache line per word of
// its local memory).
constexpr int CORR_BLOCKS = 148 * 4;
constexpr int CORR_BS = 32;
constexpr int CORR_SPLIT = 128 / CORR_BS;  // blocks per 128-cell block of the grid

constexpr int BS_A = 128;
constexpr int BS_EF = 128;
constexpr int BS_HLL = 256;
constexpr int BS_CELLS = 128;

inline int grid_of(long long n, int bs) { return int((n + bs - 1) / bs); }

// The HLL kernel's launch shapes: cells per block and moment groups (the 35
// moments split over that many blocks of the same cells).
// Variants 6 and 7 trade registers for occupancy (6 and 5 blocks of 256
// per SM instead of 4); 8 and 9 stage 32 x 8 and 32 x 4 cell tiles of a
// layer in shared memory, seven groups of five moments (their grids count
// tiles: hll_blocks).
constexpr int HLL_VARIANTS = 10;
inline void hll_shape(int variant, int& bs, int& groups) {
  static const int tab[HLL_VARIANTS][2] = {{256, 1}, {256, 5}, {256, 7}, {128, 5}, {128, 7}, {128, 1}, {256, 7}, {256, 5}, {256, 7}, {128, 7}};
  const int v = (variant >= 0 && variant < HLL_VARIANTS) ? variant : 0;
  bs = tab[v][0];
  groups = tab[v][1];
}
// ---- fused batches: many independent domains in one launch per kernel ----
// A member as the fused kernels see it: its constants, clock and buffers.
enum DomBuf { DB_M = 0, DB_MTMP, DB_FX, DB_FY, DB_FZ, DB_VP, DB_BMAX, DB_NBUF };
struct Dom {
  StepConst sc;
  DevClock* clk;
  double* buf[DB_NBUF];
};
// Launch shapes of the fused kernels; a launch of kind K gives member m the
// blocks [blk0[K][m], blk0[K][m + 1]) of its grid.
enum DomKind { DK_CELLS = 0, DK_CORR, DK_HLL, DK_ONE, DK_DIAG, DK_NKIND };
constexpr int DK_MAX_MEMBERS = 4096;
// The block counts of member m's launch of each kind (hll_g: the HLL
// kernel's moment groups; corr_cap: the correction passes' blocks per member).
// The HLL kernel's blocks for a grid: cell blocks x moment groups, or for
// the tiled variants (8, 9) 32 x 8 or 32 x 4 tiles per layer x layers x groups.
inline int hll_blocks(int variant, int Nx, int Ny, int Nz) {
  int bs, g;
  hll_shape(variant, bs, g);
  if (variant == 8) return ((Nx + 31) / 32) * ((Ny + 7) / 8) * Nz * g;
  if (variant == 9) return ((Nx + 31) / 32) * ((Ny + 3) / 4) * Nz * g;
  return grid_of((long long)Nx * Ny * Nz, bs) * g;
}
inline void dom_blocks(int Nx, int Ny, int Nz, int hll_variant, int corr_cap, int* nb) {
  const long long N = (long long)Nx * Ny * Nz;
  const int g = grid_of(N, BS_A);
  nb[DK_CELLS] = g;
  nb[DK_CORR] = (g < corr_cap ? g : corr_cap) * CORR_SPLIT;
  nb[DK_HLL] = hll_blocks(hll_variant, Nx, Ny, Nz);
  nb[DK_ONE] = 1;
  const int gd = grid_of(N, 256);
  nb[DK_DIAG] = gd < 64 ? gd : 64;
}
// What the fused kernels of one launch get: the member table and the block
// prefix of the launch's kind (device arrays owned by the batch).
struct Batch {
  const Dom* dom;
  const int* blk0;  // n + 1 entries
  int n;
};
// Host-side view of a fused batch: device tables and total blocks per kind.
struct BatchPlan {
  const Dom* dom;
  const int* blk0[DK_NKIND];
  int nblk[DK_NKIND];
  int n;
  int hll_variant;
  Batch of(int kind) const { return Batch{dom, blk0[kind], n}; }
};

// launch wrappers (defined in k_phase_A.cu, k_phase_EF.cu, k_cells.cu)
// Phase [A] in place on M; Mtmp, Fx, Fy, Fz carry its intermediate states,
// and on completion Fx, Fy, Fz hold the fluxes (Mtmp is left as scratch).
// vp: 7N + 16 doubles, the six wave-speed arrays and the lists of cells left
// to the later parts of the eigenvalue stages.  ev (optional): five events
// recorded after A1, A2, A3, A4 (each with its passes over listed cells) and
// A5.  [c0, c1):
// the cells to process (default all; c0 a multiple of BS_A).
// The wave-speed network of MODE_LEARNED on the device: its BF16 weight
// image (k_mlp.cu layout) and an error word set when a bounded wait of its
// kernel ran out.
struct WaveNet {
  unsigned char* image;
  int* err;
};
// net: the wave-speed network (MODE_LEARNED only).
void launch_phase_A(const StepConst& sc, double* M, double* Mtmp, double* Fx, double* Fy, double* Fz, double* vp, double* blockmax,
                    DevClock* clk, cudaStream_t s, cudaEvent_t* ev = nullptr, long long c0 = 0, long long c1 = -1,
                    const WaveNet* net = nullptr);
// Phases [E]+[F] from Min to Mout; Fx, Fy, Fz are overwritten and vp (6N
// doubles, dead after the HLL sweep) holds the correction lists.
// ev (optional): four events recorded after E1, E2, E3 and E4.
void launch_phase_EF(const StepConst& sc, const double* Min, double* Mout, double* Fx, double* Fy, double* Fz, double* vp,
                     DevClock* clk, cudaStream_t s, cudaEvent_t* ev = nullptr, long long c0 = 0, long long c1 = -1);
void launch_cells_phase_A(const double* M, long long n, int flag2D, double Ma, int positivity, double* Fx, double* Fy, double* Fz,
                          double* Mr, double* vp, cudaStream_t s);
void launch_cells_flux(const double* M, long long n, int flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr, cudaStream_t s);
void launch_cells_eig(const double* M, long long n, int axis, int flag2D, double Ma, int positivity, double* v, double* Mr, cudaStream_t s);
void launch_cells_closure_eigs(const double* mom, long long n, double* v, cudaStream_t s);
void launch_cells_collision(const double* M, long long n, double dt, double Kn, int positivity, double* out, cudaStream_t s);
void launch_std_central(const double* M, long long n, double* S, double* C, cudaStream_t s);
void launch_cells_targets(const double* M, long long n, int flag2D, double Ma, int positivity, float* T, double* Mr, cudaStream_t s);
// (defined in hyq_b200.cu) the CFL, HLL and clock-reset launches of one step,
// and the thread-local error text read by hyq_last_error(NULL)
void launch_cfl(const double* blockmax, const StepConst& sc, DevClock* clk, cudaStream_t s);
// the first-step diagnostics (after the CFL reduction, on the six speed
// arrays vp) and MaxDiff (after the step, on M); both return at once on
// the steps they do not measure
void launch_diagnostics_speeds(const double* vp, const StepConst& sc, DevClock* clk, cudaStream_t s);
void launch_maxdiff(const double* M, const StepConst& sc, DevClock* clk, cudaStream_t s);
// variant: the HLL kernel's launch shape (hll_shape); all variants give the
// same bits
void launch_hll(const double* M, const double* Fx, const double* Fy, const double* Fz, const double* vp, double* Mout, const StepConst& sc,
                const DevClock* clk, cudaStream_t s, int variant = 0);
// Fused batches (one launch per kernel for all members of the plan):
// phase [A] (after_a1, when set, runs after the first closure: the learned
// path's per-member network launches), the CFL reduction, the diagnostics and
// the HLL sweep, phases [E]+[F] and MaxDiff; mode: the members' common
// eigenvalue path.
void launch_phase_A_batch(const BatchPlan& bp, int mode, cudaStream_t s, void (*after_a1)(void*, cudaStream_t), void* arg);
void launch_mid_batch(const BatchPlan& bp, cudaStream_t s);
void launch_phase_EF_batch(const BatchPlan& bp, int mode, cudaStream_t s);
void launch_maxdiff_batch(const BatchPlan& bp, cudaStream_t s);
void launch_set_clock(DevClock* clk, double t, long long nn, cudaStream_t s);
int report_error(int code, const char* msg);
// (defined in k_mlp.cu) the wave-speed network on the realized moments of
// phase [A]'s first closure (moment-major, stride N, cells [c0, c1)): writes
// sc.seeds for those cells.  net_set_smem raises the kernels' shared-memory
// limit (call before the first launch on a device).
cudaError_t net_set_smem();
void launch_wavespeed_seeds(const StepConst& sc, const double* Mr, const WaveNet* net, float* seeds, const DevClock* clk, cudaStream_t s,
                            long long c0, long long c1);

}  // namespace hyqk

#if defined(__CUDACC__) && defined(HQ_SEEDS)
namespace hyqk {
// The learned path's seeds of plane Jacobians along `axis` for cell c: the
// network's standardized extreme speeds mapped back with the stage input's
// mean velocity and variance along the axis (NaN seeds when there are none).
__device__ __forceinline__ hyq::Seeds stage_seeds(const double* in, long long c, int axis, const StepConst& sc) {
  if (!sc.seeds) return hyq::no_seeds();
  const long long N = sc.N;
  const int iu = axis == 1 ? 1 : (axis == 2 ? 5 : 15), i2 = axis == 1 ? 2 : (axis == 2 ? 9 : 19);
  const double m0 = in[c], mu = in[c + N * iu] / m0;
  const double var = in[c + N * i2] / m0 - mu * mu;
  const double sd = sqrt(var > 0.0 ? var : 0.0);
  const float* sp = sc.seeds + 2 * (axis - 1) * N + c;
  hyq::Seeds s;
  s.lo = mu + sd * (double)sp[0];
  s.hi = mu + sd * (double)sp[N];
  s.margin = sc.seed_margin;
  return s;
}

}  // namespace hyqk
#endif

#ifdef __CUDACC__
namespace hyqk {
// The member whose blocks contain block `blk` of a fused launch.
__device__ __forceinline__ int member_of(const Batch& b, int blk) {
  int lo = 0, hi = b.n;  // b.blk0[lo] <= blk < b.blk0[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(b.blk0 + mid) <= blk) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ double nanmax(double a, double b) { return (a != a) ? a : ((b != b) ? b : fmax(a, b)); }

__device__ __forceinline__ double warp_nanmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// NaN-propagating block max (Julia `maximum` semantics).
template <int BS> __device__ double block_nanmax(double v) {
  __shared__ double red[BS / 32];
  v = warp_nanmax(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = (threadIdx.x < BS / 32) ? red[threadIdx.x] : 0.0;
    w = warp_nanmax(w);
    if (threadIdx.x == 0) red[0] = w;
  }
  __syncthreads();
  return red[0];
}
}  // namespace hyqk
#endif
