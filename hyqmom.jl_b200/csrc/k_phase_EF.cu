// Phases [E] realizability and [F] BGK collision of the step
// (src/simulation_runner.jl:526-557), per cell, out of place.
#include "hyq_eigen.cuh"
#define HQ_SEEDS
#include "hyq_step.cuh"

using namespace hyq;

namespace hyqk {
namespace {


// Phases [E]+[F] run as per-function kernels (small code per kernel);
// intermediate states go through a flux buffer, dead after the HLL sweep:
//   Mtmp -E1-> Fx -E2, E3 (in place: only corrected moments are written)-> Fx -E4-> M.
// E2/E3 copy the moments, list the cells whose Jacobians have complex
// eigenvalues for the correction, and list the cells with a Jacobian outside
// the usual permutation (pattern 1, the only one their 64-register code
// solves) for k_E_fix, which decides them with the general eigen-solve and
// lists those that need the correction; k_E_corr corrects the cells of its
// list, so that each kernel keeps small code and a few such cells no longer
// hold every lane of their warps.  The lists live in the wave-speed buffer
// vp, dead after the HLL sweep: the cells to decide at vp[0..N) (64-bit
// entries cell << 2), four 32-bit counters at vp + N (to decide: x, y; to
// correct: x, y), the cells to correct from vp + N + 8 ((cell << 2) | planes).
// A stage that listed most of its cells runs dense for a while
// (DevClock::dense): k_E_eig only copies and k_E_fix decides every cell,
// listing those to correct.
__device__ __forceinline__ unsigned int* fix_counters(double* vp, long long N) { return reinterpret_cast<unsigned int*>(vp + N); }
__device__ __forceinline__ unsigned long long* corr_list_ef(double* vp, long long N) { return reinterpret_cast<unsigned long long*>(vp + N + 8); }
// Append a cell to the correction list of stage `which`.
__device__ __forceinline__ void list_corr_ef(double* vp, long long N, int which, long long c, int planes) {
  corr_list_ef(vp, N)[atomicAdd(fix_counters(vp, N) + 2 + which, 1u)] = ((unsigned long long)c << 2) | (unsigned long long)planes;
}

// E1: Flux_closure35_and_realizable_3D; also resets the list counters
__device__ __forceinline__ void E1_body(const double* __restrict__ in, double* __restrict__ out, double* vp, const StepConst& sc,
                                        const DevClock* clk, long long c0, long long c1, int bid) {
  if (!clk->active) return;
  const long long N = sc.N, c = c0 + (long long)bid * BS_EF + threadIdx.x;
  if (c == c0) { unsigned int* cnt = fix_counters(vp, N); cnt[0] = 0; cnt[1] = 0; cnt[2] = 0; cnt[3] = 0; }
  if (c >= c1) return;
  flux_closure35(in + c, sc.flag2D, sc.Ma, nullptr, nullptr, nullptr, out + c, N, N);
}
__global__ void __launch_bounds__(BS_EF, MINB_REALIZE) k_E1_closure(const double* __restrict__ in, double* __restrict__ out, double* vp,
                                                                const StepConst sc, const DevClock* clk, long long c0, long long c1) {
  E1_body(in, out, vp, sc, clk, c0, c1, blockIdx.x);
}
// The fused-batch form of each kernel: the block's member from the table,
// then the same body on that member's buffers over all its cells.
__global__ void __launch_bounds__(BS_EF, MINB_REALIZE) k_E1_closure_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  E1_body(d.buf[DB_MTMP], d.buf[DB_FX], d.buf[DB_VP], sc, d.clk, 0, sc.N, blockIdx.x - __ldg(bt.blk0 + m));
}

// Warp-aggregated count of the calling threads with `flag` set, added to *ctr.
__device__ __forceinline__ void count_flag_ef(bool flag, unsigned long long* ctr) {
  const unsigned int act = __activemask();
  const unsigned int m = __ballot_sync(act, flag);
  if (m && (int)(threadIdx.x & 31) == __ffs(act) - 1) atomicAdd(ctr, (unsigned long long)__popc(m));
}

// E2/E3: eigenvalues6_hyperbolic_3D along x or y: copy, and list the cells
// that need the correction or the complete eigen-solve (counter `which`).
// JM = EIG_MODE: the pattern-1 register path; JM = JAC_CP (certified and
// learned paths): that path or the certified solve, which decides a Jacobian
// without its eigenvalues; the cells it leaves to the LAPACK path are counted.
template <int JM>
__device__ __forceinline__ void E_eig_body(const double* in, double* out, double* vp, int axis, int which, const StepConst& sc, DevClock* clk,
                                           long long c0, long long c1, int bid) {
  if (!clk->active) return;
  const bool dense = clk->dense[3 + which] != 0;
  if (JM == JAC_CP && bid == 0 && threadIdx.x == 0) {
    atomicAdd(&clk->stage_cells, (unsigned long long)(c1 - c0));
    if (dense) atomicAdd(&clk->fb_cells, (unsigned long long)(c1 - c0));
  }
  const long long N = sc.N, c = c0 + (long long)bid * BS_EF + threadIdx.x;
  if (c >= c1) return;
  // the learned path seeds the certified solve with the network's speeds of
  // this step (predicted in phase [A]; a poor seed only costs evaluations)
  const int planes = dense ? 0 : eigenvalues6_flags_t<JM>(in + c, axis, N, JM == JAC_CP ? stage_seeds(in, c, axis, sc) : no_seeds());
  if (JM == JAC_CP && !dense) count_flag_ef(planes < 0, &clk->fb_cells);
  if (out != in) {
#pragma unroll
    for (int n = 0; n < 35; ++n) out[c + N * n] = in[c + N * n];
  }
  if (planes > 0) {
    list_corr_ef(vp, N, which, c, planes);
  } else if (planes < 0) {
    const unsigned int slot = atomicAdd(fix_counters(vp, N) + which, 1u);
    reinterpret_cast<unsigned long long*>(vp)[slot] = (unsigned long long)c << 2;
  }
}
template <int JM>
__global__ void __launch_bounds__(BS_EF, MINB_EIG) k_E_eig(const double* in, double* out, double* vp, int axis,
                                                           int which, const StepConst sc, DevClock* clk, long long c0, long long c1) {
  E_eig_body<JM>(in, out, vp, axis, which, sc, clk, c0, c1, blockIdx.x);
}
template <int JM>
__global__ void __launch_bounds__(BS_EF, MINB_EIG) k_E_eig_b(const Batch bt, int axis, int which) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  E_eig_body<JM>(d.buf[DB_FX], d.buf[DB_FX], d.buf[DB_VP], axis, which, sc, d.clk, 0, sc.N, blockIdx.x - __ldg(bt.blk0 + m));
}

// The undecided listed cells (dense: every cell of the range): their planes
// from the general eigen-solve, written back into the entry (dense: listed).
// One thread per possible entry.
__device__ __forceinline__ void E_fix_body(const double* __restrict__ in, double* vp, int axis, int which, const StepConst& sc,
                                           const DevClock* clk, long long c0, long long c1, int bid, int nblk) {
  if (!clk->active) return;
  const long long N = sc.N;
  unsigned long long* list = reinterpret_cast<unsigned long long*>(vp);
  if (clk->dense[3 + which]) {
    const long long c = c0 + (long long)bid * BS_EF + threadIdx.x;
    if (c >= c1) return;
    const int planes = eigenvalues6_flags_t<FIX_MODE>(in + c, axis, N);
    if (planes) list_corr_ef(vp, N, which, c, planes);
    return;
  }
  const unsigned int count = reinterpret_cast<const unsigned int*>(vp + N)[which];
  for (unsigned int e = bid * BS_EF + threadIdx.x; e < count; e += nblk * BS_EF) {
    const long long c = (long long)(list[e] >> 2);
    const int planes = eigenvalues6_flags_t<FIX_MODE>(in + c, axis, N);
    if (planes) list_corr_ef(vp, N, which, c, planes);
  }
}
__global__ void __launch_bounds__(BS_EF, MINB_FIX) k_E_fix(const double* __restrict__ in, double* vp, int axis, int which,
                                                           const StepConst sc, const DevClock* clk, long long c0, long long c1) {
  E_fix_body(in, vp, axis, which, sc, clk, c0, c1, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(BS_EF, MINB_FIX) k_E_fix_b(const Batch bt, int axis, int which) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  const int b0 = __ldg(bt.blk0 + m);
  E_fix_body(d.buf[DB_FX], d.buf[DB_VP], axis, which, sc, d.clk, 0, sc.N, blockIdx.x - b0, __ldg(bt.blk0 + m + 1) - b0);
}

// The correction of the listed cells that need it
// (correct_moments_for_real_eigenvalues, as in eigenvalues6); the first thread
// then decides whether the stage runs dense next time
__device__ __forceinline__ void E_corr_body(const double* in, double* out, const double* vp, int axis, int which, const StepConst& sc,
                                            DevClock* clk, long long c0, long long c1, int bid, int nblk) {
  if (!clk->active) return;
  const long long N = sc.N;
  const unsigned int count = reinterpret_cast<const unsigned int*>(vp + N)[2 + which];
  const unsigned long long* list = reinterpret_cast<const unsigned long long*>(vp + N + 8);
  if (bid == 0 && threadIdx.x == 0) {
    int& d = clk->dense[3 + which];
    const long long listed = (long long)reinterpret_cast<const unsigned int*>(vp + N)[which] + count;
    if (d > 0) d = d - 1;
    else if (listed * 4 > (c1 - c0) * 3) d = DENSE_RUNS;
  }
  // one cell per warp for a short list, one per thread for a long one (as
  // the phase-A correction passes)
  const bool sparse = (unsigned long long)count * 32ull <= (unsigned long long)nblk * CORR_BS;
  if (sparse && (threadIdx.x & 31)) return;
  const unsigned int e0 = sparse ? (bid * CORR_BS + threadIdx.x) >> 5 : bid * CORR_BS + threadIdx.x;
  const unsigned int es = sparse ? (unsigned int)(nblk * CORR_BS) >> 5 : (unsigned int)(nblk * CORR_BS);
  for (unsigned int e = e0; e < count; e += es) {
    const unsigned long long v = list[e];
    const int planes = int(v & 3ull);
    const long long c = (long long)(v >> 2);
    double Ml[35], Mc[35];
    for (int n = 0; n < 35; ++n) Ml[n] = in[c + N * n];
    correct_for_real(Ml, 0, 1, axis == 1 ? 0 : 1, 2, planes, sc.flag2D, sc.Ma, Mc);
    for (int n = 0; n < 35; ++n) out[c + N * n] = Mc[n];
  }
}
__global__ void __launch_bounds__(CORR_BS, MINB_CLOSURE * CORR_SPLIT) k_E_corr(const double* in, double* out, const double* vp,
                                                                int axis, int which, const StepConst sc, DevClock* clk, long long c0,
                                                                long long c1) {
  E_corr_body(in, out, vp, axis, which, sc, clk, c0, c1, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(CORR_BS, MINB_CLOSURE * CORR_SPLIT) k_E_corr_b(const Batch bt, int axis, int which) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  const int b0 = __ldg(bt.blk0 + m);
  E_corr_body(d.buf[DB_FX], d.buf[DB_FX], d.buf[DB_VP], axis, which, sc, d.clk, 0, sc.N, blockIdx.x - b0, __ldg(bt.blk0 + m + 1) - b0);
}

// E4: Flux_closure35_and_realizable_3D, then collision35 with the step's dt
__device__ __forceinline__ void E4_body(const double* __restrict__ in, double* __restrict__ Mout, const StepConst& sc, const DevClock* clk,
                                        long long c0, long long c1, int bid) {
  if (!clk->active) return;
  const long long N = sc.N, c = c0 + (long long)bid * BS_EF + threadIdx.x;
  if (c >= c1) return;
  double a[35];
  flux_closure35(in + c, sc.flag2D, sc.Ma, nullptr, nullptr, nullptr, a, N, 1);
  collision35(a, clk->dt, sc.Kn, sc.positivity);
#pragma unroll
  for (int n = 0; n < 35; ++n) Mout[c + N * n] = a[n];
}
__global__ void __launch_bounds__(BS_EF, MINB_CLOSURE) k_E4_closure_bgk(const double* __restrict__ in, double* __restrict__ Mout, const StepConst sc,
                                                                    const DevClock* clk, long long c0, long long c1) {
  E4_body(in, Mout, sc, clk, c0, c1, blockIdx.x);
}
__global__ void __launch_bounds__(BS_EF, MINB_CLOSURE) k_E4_closure_bgk_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  E4_body(d.buf[DB_FX], d.buf[DB_M], sc, d.clk, 0, sc.N, blockIdx.x - __ldg(bt.blk0 + m));
}

}  // namespace

void launch_phase_EF(const StepConst& sc, const double* Min, double* Mout, double* Fx, double* Fy, double* Fz, double* vp,
                     DevClock* clk, cudaStream_t s, cudaEvent_t* ev, long long c0, long long c1) {
  if (c1 < 0) c1 = sc.N;
  const int g = grid_of(c1 - c0, BS_EF);
  const int gfix = g;  // one thread per possible list entry: blocks past the count exit at once
  const int gcorr = (g < CORR_BLOCKS ? g : CORR_BLOCKS) * CORR_SPLIT;
  k_E1_closure<<<g, BS_EF, 0, s>>>(Min, Fx, vp, sc, clk, c0, c1);
  if (ev) cudaEventRecord(ev[0], s);
  if (sc.mode == MODE_PLAIN) k_E_eig<EIG_MODE><<<g, BS_EF, 0, s>>>(Fx, Fx, vp, 1, 0, sc, clk, c0, c1);
  else k_E_eig<JAC_CP><<<g, BS_EF, 0, s>>>(Fx, Fx, vp, 1, 0, sc, clk, c0, c1);
  k_E_fix<<<gfix, BS_EF, 0, s>>>(Fx, vp, 1, 0, sc, clk, c0, c1);
  k_E_corr<<<gcorr, CORR_BS, 0, s>>>(Fx, Fx, vp, 1, 0, sc, clk, c0, c1);
  if (ev) cudaEventRecord(ev[1], s);
  if (sc.mode == MODE_PLAIN) k_E_eig<EIG_MODE><<<g, BS_EF, 0, s>>>(Fx, Fx, vp, 2, 1, sc, clk, c0, c1);
  else k_E_eig<JAC_CP><<<g, BS_EF, 0, s>>>(Fx, Fx, vp, 2, 1, sc, clk, c0, c1);
  k_E_fix<<<gfix, BS_EF, 0, s>>>(Fx, vp, 2, 1, sc, clk, c0, c1);
  k_E_corr<<<gcorr, CORR_BS, 0, s>>>(Fx, Fx, vp, 2, 1, sc, clk, c0, c1);
  if (ev) cudaEventRecord(ev[2], s);
  k_E4_closure_bgk<<<g, BS_EF, 0, s>>>(Fx, Mout, sc, clk, c0, c1);
  if (ev) cudaEventRecord(ev[3], s);
}

void launch_phase_EF_batch(const BatchPlan& bp, int mode, cudaStream_t s) {
  const Batch cells = bp.of(DK_CELLS), corr = bp.of(DK_CORR);
  const int g = bp.nblk[DK_CELLS], gc = bp.nblk[DK_CORR];
  k_E1_closure_b<<<g, BS_EF, 0, s>>>(cells);
  for (int which = 0; which < 2; ++which) {
    const int axis = which + 1;
    if (mode == MODE_PLAIN) k_E_eig_b<EIG_MODE><<<g, BS_EF, 0, s>>>(cells, axis, which);
    else k_E_eig_b<JAC_CP><<<g, BS_EF, 0, s>>>(cells, axis, which);
    k_E_fix_b<<<g, BS_EF, 0, s>>>(cells, axis, which);
    k_E_corr_b<<<gc, CORR_BS, 0, s>>>(corr, axis, which);
  }
  k_E4_closure_bgk_b<<<g, BS_EF, 0, s>>>(cells);
}

}  // namespace hyqk
