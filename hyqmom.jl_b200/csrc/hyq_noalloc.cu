// hyq_step_noalloc: one explicit time step on a caller-owned device state
// that allocates no device memory.
//
// Who needs it: callers that must not allocate while they step, e.g. a host
// program that hands the library a device buffer from its own memory pool
// and runs under a fixed device-memory budget, or a loop that cannot afford
// the device-wide synchronisation cudaMalloc/cudaFree may cause.  The
// context API (hyq_create) allocates five state-sized work arrays per
// context; this entry point instead uses one fixed scratch array that is part
// of the library's device image, so no call allocates.
//
// The scratch array holds the fluxes, the realized state, the wave speeds
// with the step's lists of cells left to a second pass, the per-block maxima
// and the device clock of ONE step of at most
// HYQ_NOALLOC_MAX_CELLS cells.  Every call on a device shares it: calls that
// overlap on one device (two host threads, or two streams without ordering
// between them) race on the scratch and give wrong results.  Nothing in it
// has to start at zero: each call writes the clock from the caller's t and nn
// first, and every other region is written in full before it is read within
// the same step.
//
// The first call on each device (and the first after a device reset, which
// replaces the context) looks up the scratch address with
// cudaGetSymbolAddress (which may load this module); make that first call
// before any stream capture on that device.
#include <cuda.h>
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "hyq_step.cuh"
#include "../../include/hyqmom.h"

using namespace hyqk;

namespace {

// Layout in doubles; each region starts on a 256-byte boundary.
constexpr long long kMax = HYQ_NOALLOC_MAX_CELLS;
constexpr long long kClock = 0;                                   // DevClock (<= 256 B)
constexpr long long kBlockmax = 32;                               // ceil(kMax / BS_A) maxima
constexpr long long kBlockmaxLen = ((kMax + BS_A - 1) / BS_A + 31) / 32 * 32;
constexpr long long kVp = kBlockmax + kBlockmaxLen;               // 6 * kMax wave speeds + cell lists
constexpr long long kFx = kVp + 7 * kMax + 32;                    // 35 * kMax each
constexpr long long kFy = kFx + 35 * kMax;
constexpr long long kFz = kFy + 35 * kMax;
constexpr long long kMtmp = kFz + 35 * kMax;
constexpr long long kTotal = kMtmp + 35 * kMax;
static_assert(sizeof(DevClock) <= 32 * sizeof(double), "clock region");
static_assert(kMax % 32 == 0, "regions stay 256-byte aligned");

static __device__ __align__(256) double g_noalloc_scratch[kTotal];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
// Per device: the scratch address and the id of the CUDA context it was
// looked up in.  A device reset (cudaDeviceReset) or a new primary context
// reloads this module, which moves the scratch, so the address is looked up
// again whenever the current context's id differs from the cached one.
struct ScratchAddr {
  unsigned long long ctx_id = 0;
  double* ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

// The driver's cuCtxGetCurrent and cuCtxGetId, fetched through the runtime
// (the library does not link libcuda directly).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

cudaError_t current_ctx_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* a = nullptr;
    void* b = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault);
    if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault);
    if (e != cudaSuccess) return e;
    if (!a || !b) return cudaErrorSymbolNotFound;
    get_current = reinterpret_cast<CtxGetCurrentFn>(a);
    get_id = reinterpret_cast<CtxGetIdFn>(b);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  return cudaSuccess;
}

// Device address of the scratch on `dev` (the current device, whose primary
// context the caller's cudaSetDevice has made current), looked up once per
// context.
cudaError_t scratch_for(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  unsigned long long id = 0;
  // cudaSetDevice (called before) initialises the device's primary context
  // and makes it current
  cudaError_t e = current_ctx_id(&id);
  if (e != cudaSuccess) return e;
  ScratchAddr& s = g_scratch[dev];
  if (!s.ptr || s.ctx_id != id) {
    void* p = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_noalloc_scratch)) != cudaSuccess) return e;
    s.ptr = static_cast<double*>(p);
    s.ctx_id = id;
  }
  *out = s.ptr;
  return cudaSuccess;
}

int cuda_error(cudaError_t e, const char* what) {
  return report_error(HYQ_ECUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

}  // namespace

extern "C" int hyq_step_noalloc(const hyq_params* p, double* M, hyq_stats* stats, void* stream) {
  if (!p || !M || !stats) return report_error(HYQ_EINVAL, "null argument");
  if (p->Nx < 2 || p->Ny < 2 || p->Nz < 1)
    return report_error(HYQ_EINVAL, "grid must have Nx >= 2, Ny >= 2, Nz >= 1 (pas_HLL needs two cells per row)");
  if (!(p->CFL > 0) || !(p->Kn > 0) || !(p->dtmax > 0)) return report_error(HYQ_EINVAL, "CFL, Kn and dtmax must be positive");
  if (p->device < 0 || p->device >= kMaxDevices) return report_error(HYQ_EINVAL, "device index out of range");
  if (p->mode != HYQ_MODE_PLAIN) return report_error(HYQ_EINVAL, "hyq_step_noalloc runs the plain eigenvalue path only (mode 0)");
  const long long N = (long long)p->Nx * p->Ny * p->Nz;
  if (N > kMax)
    return report_error(HYQ_EINVAL, ("grid has " + std::to_string(N) + " cells; hyq_step_noalloc supports at most " +
                                     std::to_string(kMax) + " (HYQ_NOALLOC_MAX_CELLS); use hyq_create/hyq_advance for larger grids")
                                        .c_str());
  cudaError_t e = cudaSetDevice(p->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  double* base = nullptr;
  if ((e = scratch_for(p->device, &base)) != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress");

  StepConst sc;
  sc.N = N; sc.Nx = p->Nx; sc.Ny = p->Ny; sc.Nz = p->Nz; sc.flag2D = p->flag2D; sc.positivity = p->positivity;
  sc.nnmax = p->nnmax; sc.tmax = p->tmax; sc.Kn = p->Kn; sc.Ma = p->Ma; sc.CFL = p->CFL; sc.dtmax = p->dtmax;
  sc.dx = (p->xmax - p->xmin) / p->Nx; sc.dy = (p->ymax - p->ymin) / p->Ny; sc.dz = (p->zmax - p->zmin) / p->Nz;
  sc.nblocksA = grid_of(N, BS_A);
  sc.mode = MODE_PLAIN;
  sc.symmetry_check_interval = 0;
  sc.seeds = nullptr;
  sc.seed_margin = 0.0;

  DevClock* clk = reinterpret_cast<DevClock*>(base + kClock);
  double* blockmax = base + kBlockmax;
  double* vp = base + kVp;  // vp[c + N*q]: six arrays of stride N inside the region
  double* Fx = base + kFx;
  double* Fy = base + kFy;
  double* Fz = base + kFz;
  double* Mtmp = base + kMtmp;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  launch_set_clock(clk, stats->t, (long long)stats->nn, s);
  launch_phase_A(sc, M, Mtmp, Fx, Fy, Fz, vp, blockmax, clk, s);
  launch_cfl(blockmax, sc, clk, s);
  launch_hll(M, Fx, Fy, Fz, vp, Mtmp, sc, clk, s);
  launch_phase_EF(sc, Mtmp, M, Fx, Fy, Fz, vp, clk, s);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "launch");

  DevClock h;
  if ((e = cudaMemcpyAsync(&h, clk, sizeof(DevClock), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_error(e, "clock copy");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "cudaStreamSynchronize");
  stats->t = h.t; stats->dt = h.dt; stats->vmax = h.vmax; stats->nn = h.nn; stats->status = h.status;
  stats->stage_cells = 0; stats->fallback_cells = 0; stats->dense_mask = 0; stats->worst_dir = -1;
  stats->vmax_first[0] = stats->vmax_first[1] = stats->vmax_first[2] = 0.0; stats->worst_cell = -1;
  stats->maxdiff = 0.0; stats->maxdiff_step = -1;
  stats->done = (h.t < p->tmax && h.nn < p->nnmax) ? 0 : 1;
  if (h.status > 0)
    return report_error(HYQ_ENONFINITE, ("non-finite CFL wave speed at step " + std::to_string(h.status) +
                                         " (a flux Jacobian with Inf/NaN entries; the reference's eigvals throws there)")
                                            .c_str());
  return HYQ_OK;
}
