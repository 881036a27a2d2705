// Phase [A] of the step (src/simulation_runner.jl:352-383): per cell, the
// closure + realizability, x/y/z flux-Jacobian eigenvalues with their
// corrections, the closure of the realized moments (fluxes Fx, Fy, Fz) and the
// 1-D closure speeds; a NaN-propagating block max of |speed| feeds the CFL
// reduction.
#include "hyq_eigen.cuh"
#define HQ_SEEDS
#include "hyq_step.cuh"

using namespace hyq;

namespace hyqk {
namespace {


// Phase [A] runs as five kernels, one per-cell function each, so that every
// kernel's code stays small (one kernel for the whole phase was bound by
// instruction fetch); the intermediate states go through buffers that are
// dead during phase A:  M -A1-> Fx -A2, A3 (in place)-> Fx -A4-> Mtmp -A5-> M,
// with the Jacobian speeds of A2-A4 parked in vp and combined in A5 (A2 and A3
// write only the moments they correct).
// Each eigenvalue stage A2-A4 runs in three parts, each with small code: the
// kernel itself solves pattern-1 Jacobians on its 64-register path and lists
// every other cell; k_A_fix runs the general eigen-solve on the listed cells
// (packed densely into warps) and marks those that need the correction of
// complex eigenvalues; k_A_corr finishes those cells (rare) from the planes
// to correct.  Two lists live in the seventh plane of vp (from vp + 6N, as
// 32-bit words, one pair per stage in turn): the cells to solve (entries
// cell << 3, N of them, then the three counters at N + axis - 1) and, from
// word N + 16, the cells to correct (entries (cell << 3) | code, code 1-3 =
// the planes to correct, 4 = the complete function; counters at
// N + 4 + axis - 1), so that the correction pass only reads its own cells.
// Late in a developed flow nearly every cell is listed; a stage then runs
// dense for a while (DevClock::dense): k_A_eig returns at once and k_A_fix
// takes every cell of the range, listing only those to correct.
__device__ __forceinline__ bool phase_A_active(const StepConst& sc, const DevClock* clk) {
  return (clk->t < sc.tmax) && (clk->nn < sc.nnmax);
}
__device__ __forceinline__ unsigned int* defer_list(double* vp, long long N) { return reinterpret_cast<unsigned int*>(vp + 6 * N); }
__device__ __forceinline__ unsigned int* corr_list(double* vp, long long N) { return defer_list(vp, N) + N + 16; }
__device__ __forceinline__ unsigned int* corr_count(double* vp, long long N, int axis) { return defer_list(vp, N) + N + 4 + (axis - 1); }
// Append a cell to the correction list of its stage.
__device__ __forceinline__ void list_corr(double* vp, long long N, int axis, long long c, unsigned int code) {
  corr_list(vp, N)[atomicAdd(corr_count(vp, N, axis), 1u)] = ((unsigned int)c << 3) | code;
}

// A1: Flux_closure35_and_realizable_3D (realized moments only); also resets
// the list counters
__device__ __forceinline__ void A1_body(const double* __restrict__ M, double* __restrict__ out, double* vp, const StepConst& sc,
                                        const DevClock* clk, long long c0, long long c1, int bid) {
  if (!phase_A_active(sc, clk)) return;
  const long long N = sc.N, c = c0 + (long long)bid * BS_A + threadIdx.x;
  if (c == c0) {
    unsigned int* cnt = defer_list(vp, N) + N;
    for (int q = 0; q < 8; ++q) cnt[q] = 0;
  }
  if (c >= c1) return;
  flux_closure35(M + c, sc.flag2D, sc.Ma, nullptr, nullptr, nullptr, out + c, N, N);
}
__global__ void __launch_bounds__(BS_A, MINB_REALIZE) k_A1_closure(const double* __restrict__ M, double* __restrict__ out, double* vp,
                                                              const StepConst sc, const DevClock* clk, long long c0, long long c1) {
  A1_body(M, out, vp, sc, clk, c0, c1, blockIdx.x);
}
// The fused-batch form of each kernel: the block's member from the table,
// then the same body on that member's buffers over all its cells.
__global__ void __launch_bounds__(BS_A, MINB_REALIZE) k_A1_closure_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  A1_body(d.buf[DB_M], d.buf[DB_FX], d.buf[DB_VP], sc, d.clk, 0, sc.N, blockIdx.x - __ldg(bt.blk0 + m));
}

// eigenvalues6_hyperbolic_3D along x (axis 1) or y (axis 2), and
// eigenvalues6z_hyperbolic_3D (axis 3), as a part (MODE, CORR) for cell c; a
// cell left for the correction gets its list code in *code.  The y stage
// parks its VW-plane speeds in the z stage's speed slots (vp[4N + c],
// vp[5N + c], which the z stage reads and then overwrites); every part of the
// y stage that finishes a cell parks, so no stale pair survives.
template <int MODE, bool CORR>
__device__ __forceinline__ int eig_stage(const double* in, double* out, double* vp, long long c, int axis, const StepConst& sc,
                                         double& lo, double& hi, unsigned int* code = nullptr) {
  const long long N = sc.N;
  int planes = 0;
  double* park = vp + 4 * N + c;
  const Seeds sd = (MODE == JAC_CP) ? stage_seeds(in, c, axis, sc) : no_seeds();
  const int st = axis == 3 ? eigenvalues6z_s<MODE, CORR>(in + c, sc.flag2D, sc.Ma, sc.positivity, lo, hi, out + c, N, N, &planes, park, N, sd)
                           : eigenvalues6_s<MODE, CORR>(in + c, axis, sc.flag2D, sc.Ma, lo, hi, out + c, N, N, &planes,
                                                        axis == 2 ? park : nullptr, N, sd);
  if (code) *code = st == EIG_NEEDS_FIX ? (planes ? (unsigned int)planes : 4u) : 0u;
  return st;
}

// Warp-aggregated count of the calling threads with `flag` set, added to *ctr.
__device__ __forceinline__ void count_flag(bool flag, unsigned long long* ctr) {
  const unsigned int act = __activemask();
  const unsigned int m = __ballot_sync(act, flag);
  if (m && (int)(threadIdx.x & 31) == __ffs(act) - 1) atomicAdd(ctr, (unsigned long long)__popc(m));
}

// A2/A3/A4: the pattern-1 part (JM = EIG_MODE) or, on the certified and
// learned paths, the pattern-1 part and the certified solve (JM = JAC_CP);
// cells left go to the list, marked when they need the correction.  JAC_CP
// counts the cells it had to leave to the LAPACK path (list code 0).
template <int JM>
__device__ __forceinline__ void A_eig_body(const double* in, double* out, double* vp, int axis, const StepConst& sc, DevClock* clk,
                                           long long c0, long long c1, int bid) {
  if (!phase_A_active(sc, clk)) return;
  const bool dense = clk->dense[axis - 1] != 0;
  if (JM == JAC_CP && bid == 0 && threadIdx.x == 0) {
    atomicAdd(&clk->stage_cells, (unsigned long long)(c1 - c0));
    if (dense) atomicAdd(&clk->fb_cells, (unsigned long long)(c1 - c0));  // every cell to the LAPACK path
  }
  if (dense) return;
  const long long N = sc.N, c = c0 + (long long)bid * BS_A + threadIdx.x;
  if (c >= c1) return;
  double lo, hi;
  unsigned int code;
  const int st = eig_stage<JM, false>(in, out, vp, c, axis, sc, lo, hi, &code);
  if (JM == JAC_CP) count_flag(st == EIG_DEFERRED, &clk->fb_cells);
  if (st == EIG_DONE) {
    double* v = vp + 2 * (axis - 1) * N;
    v[c] = lo; v[c + N] = hi;
  } else if (code) {
    list_corr(vp, N, axis, c, code);
  } else {
    unsigned int* list = defer_list(vp, N);
    list[atomicAdd(list + N + (axis - 1), 1u)] = (unsigned int)c << 3;
  }
}
template <int JM>
__global__ void __launch_bounds__(BS_A, MINB_EIG) k_A_eig(const double* in, double* out, double* vp,
                                                         int axis, const StepConst sc, DevClock* clk, long long c0, long long c1) {
  A_eig_body<JM>(in, out, vp, axis, sc, clk, c0, c1, blockIdx.x);
}
template <int JM>
__global__ void __launch_bounds__(BS_A, MINB_EIG) k_A_eig_b(const Batch bt, int r_in, int r_out, int axis) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  A_eig_body<JM>(d.buf[r_in], d.buf[r_out], d.buf[DB_VP], axis, sc, d.clk, 0, sc.N, blockIdx.x - __ldg(bt.blk0 + m));
}

// The general eigen-solve on the unmarked listed cells (dense: on every cell
// of the range); marks (lists) the ones that need the correction.  One thread
// per possible entry.
__device__ __forceinline__ void A_fix_body(const double* in, double* out, double* vp, int axis, const StepConst& sc, const DevClock* clk,
                                           long long c0, long long c1, int bid, int nblk) {
  if (!phase_A_active(sc, clk)) return;
  const long long N = sc.N;
  unsigned int* list = defer_list(vp, N);
  double* v = vp + 2 * (axis - 1) * N;
  double lo, hi;
  unsigned int code;
  if (clk->dense[axis - 1]) {
    const long long c = c0 + (long long)bid * BS_A + threadIdx.x;
    if (c >= c1) return;
    if (eig_stage<FIX_MODE, false>(in, out, vp, c, axis, sc, lo, hi, &code) == EIG_DONE) { v[c] = lo; v[c + N] = hi; }
    else list_corr(vp, N, axis, c, code);
    return;
  }
  const unsigned int count = list[N + (axis - 1)];
  for (unsigned int e = bid * BS_A + threadIdx.x; e < count; e += nblk * BS_A) {
    const long long c = list[e] >> 3;
    if (eig_stage<FIX_MODE, false>(in, out, vp, c, axis, sc, lo, hi, &code) == EIG_DONE) { v[c] = lo; v[c + N] = hi; }
    else list_corr(vp, N, axis, c, code);
  }
}
__global__ void __launch_bounds__(BS_A, MINB_FIX) k_A_fix(const double* in, double* out, double* vp, int axis,
                                                         const StepConst sc, const DevClock* clk, long long c0, long long c1) {
  A_fix_body(in, out, vp, axis, sc, clk, c0, c1, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(BS_A, MINB_FIX) k_A_fix_b(const Batch bt, int r_in, int r_out, int axis) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  const int b0 = __ldg(bt.blk0 + m);
  A_fix_body(d.buf[r_in], d.buf[r_out], d.buf[DB_VP], axis, sc, d.clk, 0, sc.N, blockIdx.x - b0, __ldg(bt.blk0 + m + 1) - b0);
}

// The marked listed cells: the correction from the recorded planes (code
// 1-3), or the complete function (code 4, a z-stage re-realization); the first
// thread then decides whether the stage runs dense next time
__device__ __forceinline__ void A_corr_body(const double* in, double* out, double* vp, int axis, const StepConst& sc, DevClock* clk,
                                            long long c0, long long c1, int bid, int nblk) {
  if (!phase_A_active(sc, clk)) return;
  const long long N = sc.N;
  const unsigned int* list = corr_list(vp, N);
  const unsigned int count = *corr_count(vp, N, axis);
  double* v = vp + 2 * (axis - 1) * N;
  if (bid == 0 && threadIdx.x == 0) {
    int& d = clk->dense[axis - 1];
    const long long listed = (long long)defer_list(vp, N)[N + (axis - 1)] + count;
    if (d > 0) d = d - 1;
    else if (listed * 4 > (c1 - c0) * 3) d = DENSE_RUNS;
  }
  // A short list (the usual case) gets one cell per warp: the correction's
  // long serial chain then runs without the other lanes' divergent branches,
  // spread over more SMs; a long one gets one cell per thread.
  const bool sparse = (unsigned long long)count * 32ull <= (unsigned long long)nblk * CORR_BS;
  if (sparse && (threadIdx.x & 31)) return;
  const unsigned int e0 = sparse ? (bid * CORR_BS + threadIdx.x) >> 5 : bid * CORR_BS + threadIdx.x;
  const unsigned int es = sparse ? (unsigned int)(nblk * CORR_BS) >> 5 : (unsigned int)(nblk * CORR_BS);
  for (unsigned int e = e0; e < count; e += es) {
    const unsigned int entry = list[e];
    const int code = int(entry & 7u);
    const long long c = entry >> 3;
    double lo, hi;
    if (code == 4) eig_stage<FIX_MODE, true>(in, out, vp, c, axis, sc, lo, hi);
    else if (axis == 3) eigenvalues6z_corrected<FIX_MODE>(in + c, code, sc.flag2D, sc.Ma, lo, hi, out + c, N, N);
    else eigenvalues6_corrected<FIX_MODE>(in + c, axis, code, sc.flag2D, sc.Ma, lo, hi, out + c, N, N,
                                          axis == 2 ? vp + 4 * N + c : nullptr, N);
    v[c] = lo; v[c + N] = hi;
  }
}
__global__ void __launch_bounds__(CORR_BS, MINB_CLOSURE * CORR_SPLIT) k_A_corr(const double* in, double* out, double* vp,
                                                              int axis, const StepConst sc, DevClock* clk, long long c0, long long c1) {
  A_corr_body(in, out, vp, axis, sc, clk, c0, c1, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(CORR_BS, MINB_CLOSURE * CORR_SPLIT) k_A_corr_b(const Batch bt, int r_in, int r_out, int axis) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  const int b0 = __ldg(bt.blk0 + m);
  A_corr_body(d.buf[r_in], d.buf[r_out], d.buf[DB_VP], axis, sc, d.clk, 0, sc.N, blockIdx.x - b0, __ldg(bt.blk0 + m + 1) - b0);
}

// A5: closure of the realized moments with fluxes, 1-D closure speeds, the
// six wave speeds and the NaN-propagating block max of |speed|
__device__ __forceinline__ void A5_body(const double* __restrict__ in, double* __restrict__ M, double* __restrict__ Fx,
                                        double* __restrict__ Fy, double* __restrict__ Fz, double* __restrict__ vp,
                                        double* __restrict__ blockmax, const StepConst& sc, const DevClock* clk, long long c0, long long c1,
                                        int bid) {
  if (!phase_A_active(sc, clk)) return;
  const long long N = sc.N, c = c0 + (long long)bid * BS_A + threadIdx.x;
  double local = 0.0;
  if (c < c1) {
    flux_closure35(in + c, sc.flag2D, sc.Ma, Fx + c, Fy + c, Fz + c, M + c, N, N, N);
    const double* mr = M + c;  // the realized moments this thread just wrote, stride N
    double v5[6];
    closure_eigs(mr[0], mr[1 * N], mr[2 * N], mr[3 * N], mr[4 * N], v5[0], v5[1]);
    closure_eigs(mr[0], mr[5 * N], mr[9 * N], mr[12 * N], mr[14 * N], v5[2], v5[3]);
    closure_eigs(mr[0], mr[15 * N], mr[19 * N], mr[22 * N], mr[24 * N], v5[4], v5[5]);
#pragma unroll
    for (int q = 0; q < 6; q += 2) {
      const double lo = jmin(v5[q], vp[c + N * q]), hi = jmax(v5[q + 1], vp[c + N * (q + 1)]);
      vp[c + N * q] = lo; vp[c + N * (q + 1)] = hi;
      local = nanmax(local, fabs(lo));
      local = nanmax(local, fabs(hi));
    }
  }
  const double bm = block_nanmax<BS_A>(local);
  if (threadIdx.x == 0) blockmax[c0 / BS_A + bid] = bm;  // c0 is a multiple of BS_A
}
__global__ void __launch_bounds__(BS_A, MINB_CLOSURE) k_A5_flux(const double* __restrict__ in, double* __restrict__ M, double* __restrict__ Fx,
                                                           double* __restrict__ Fy, double* __restrict__ Fz, double* __restrict__ vp,
                                                           double* __restrict__ blockmax, const StepConst sc, const DevClock* clk,
                                                           long long c0, long long c1) {
  A5_body(in, M, Fx, Fy, Fz, vp, blockmax, sc, clk, c0, c1, blockIdx.x);
}
__global__ void __launch_bounds__(BS_A, MINB_CLOSURE) k_A5_flux_b(const Batch bt) {
  const int m = member_of(bt, blockIdx.x);
  const Dom& d = bt.dom[m];
  const StepConst sc = d.sc;
  A5_body(d.buf[DB_MTMP], d.buf[DB_M], d.buf[DB_FX], d.buf[DB_FY], d.buf[DB_FZ], d.buf[DB_VP], d.buf[DB_BMAX], sc, d.clk, 0, sc.N,
          blockIdx.x - __ldg(bt.blk0 + m));
}

// The last part of the per-cell phase [A]: the closure with fluxes of the
// z stage's output (read from Fz, which it then overwrites: each thread reads
// its cell's 35 moments before it writes any output), the 1-D closure speeds,
// and the six wave speeds from the Jacobian speeds parked in vp.
__global__ void __launch_bounds__(BS_CELLS) k_cells_phase_A_end(long long n, int flag2D, double Ma, double* Fx, double* Fy, double* Fz,
                                                                 double* Mr, double* vp) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35], fx[35], fy[35], fz[35], r[35];
  for (int q = 0; q < 35; ++q) m[q] = Fz[c + n * q];
  flux_closure35(m, flag2D, Ma, fx, fy, fz, r);
  double v5[6];
  closure_eigs(r[0], r[1], r[2], r[3], r[4], v5[0], v5[1]);
  closure_eigs(r[0], r[5], r[9], r[12], r[14], v5[2], v5[3]);
  closure_eigs(r[0], r[15], r[19], r[22], r[24], v5[4], v5[5]);
  for (int q = 0; q < 6; q += 2) {
    vp[c + n * q] = jmin(v5[q], vp[c + n * q]);
    vp[c + n * (q + 1)] = jmax(v5[q + 1], vp[c + n * (q + 1)]);
  }
  for (int q = 0; q < 35; ++q) { Fx[c + n * q] = fx[q]; Fy[c + n * q] = fy[q]; Fz[c + n * q] = fz[q]; Mr[c + n * q] = r[q]; }
}

}  // namespace

void launch_phase_A(const StepConst& sc, double* M, double* Mtmp, double* Fx, double* Fy, double* Fz, double* vp, double* blockmax,
                    DevClock* clk, cudaStream_t s, cudaEvent_t* ev, long long c0, long long c1, const WaveNet* net) {
  const long long N = sc.N;
  if (c1 < 0) c1 = N;
  const int g = grid_of(c1 - c0, BS_A);
  const int gfix = g;  // one thread per possible list entry: blocks past the count exit at once
  const int gcorr = (g < CORR_BLOCKS ? g : CORR_BLOCKS) * CORR_SPLIT;
  k_A1_closure<<<g, BS_A, 0, s>>>(M, Fx, vp, sc, clk, c0, c1);
  if (sc.mode == MODE_LEARNED) launch_wavespeed_seeds(sc, Fx, net, sc.seeds, clk, s, c0, c1);
  if (ev) cudaEventRecord(ev[0], s);
  double* const ins[3] = {Fx, Fx, Fx};
  double* const outs[3] = {Fx, Fx, Mtmp};  // x and y in place
  for (int axis = 1; axis <= 3; ++axis) {
    if (sc.mode == MODE_PLAIN) k_A_eig<EIG_MODE><<<g, BS_A, 0, s>>>(ins[axis - 1], outs[axis - 1], vp, axis, sc, clk, c0, c1);
    else k_A_eig<JAC_CP><<<g, BS_A, 0, s>>>(ins[axis - 1], outs[axis - 1], vp, axis, sc, clk, c0, c1);
    k_A_fix<<<gfix, BS_A, 0, s>>>(ins[axis - 1], outs[axis - 1], vp, axis, sc, clk, c0, c1);
    k_A_corr<<<gcorr, CORR_BS, 0, s>>>(ins[axis - 1], outs[axis - 1], vp, axis, sc, clk, c0, c1);
    if (ev) cudaEventRecord(ev[axis], s);
  }
  k_A5_flux<<<g, BS_A, 0, s>>>(Mtmp, M, Fx, Fy, Fz, vp, blockmax, sc, clk, c0, c1);
  if (ev) cudaEventRecord(ev[4], s);
}
void launch_phase_A_batch(const BatchPlan& bp, int mode, cudaStream_t s, void (*after_a1)(void*, cudaStream_t), void* arg) {
  const Batch cells = bp.of(DK_CELLS), corr = bp.of(DK_CORR);
  const int g = bp.nblk[DK_CELLS], gc = bp.nblk[DK_CORR];
  k_A1_closure_b<<<g, BS_A, 0, s>>>(cells);
  if (after_a1) after_a1(arg, s);
  const int ins[3] = {DB_FX, DB_FX, DB_FX};
  const int outs[3] = {DB_FX, DB_FX, DB_MTMP};  // x and y in place
  for (int axis = 1; axis <= 3; ++axis) {
    if (mode == MODE_PLAIN) k_A_eig_b<EIG_MODE><<<g, BS_A, 0, s>>>(cells, ins[axis - 1], outs[axis - 1], axis);
    else k_A_eig_b<JAC_CP><<<g, BS_A, 0, s>>>(cells, ins[axis - 1], outs[axis - 1], axis);
    k_A_fix_b<<<g, BS_A, 0, s>>>(cells, ins[axis - 1], outs[axis - 1], axis);
    k_A_corr_b<<<gc, CORR_BS, 0, s>>>(corr, ins[axis - 1], outs[axis - 1], axis);
  }
  k_A5_flux_b<<<g, BS_A, 0, s>>>(cells);
}
// The per-cell phase [A] (the step's phase A for independent cells, without
// the HLL neighbours) as a chain of per-function kernels, with the caller's
// outputs as the intermediate states: closure M -> Mr, x stage Mr -> Fx, y
// stage Fx -> Mr, z stage Mr -> Fz (Jacobian speeds into vp), then the
// closure with fluxes.  Small kernels, as in the step: one kernel calling the
// whole chain per thread faulted on the GPU.
void launch_cells_phase_A(const double* M, long long n, int flag2D, double Ma, int positivity, double* Fx, double* Fy, double* Fz,
                          double* Mr, double* vp, cudaStream_t s) {
  launch_cells_flux(M, n, flag2D, Ma, nullptr, nullptr, nullptr, Mr, s);
  launch_cells_eig(Mr, n, 1, flag2D, Ma, positivity, vp, Fx, s);
  launch_cells_eig(Fx, n, 2, flag2D, Ma, positivity, vp + 2 * n, Mr, s);
  launch_cells_eig(Mr, n, 3, flag2D, Ma, positivity, vp + 4 * n, Fz, s);
  k_cells_phase_A_end<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(n, flag2D, Ma, Fx, Fy, Fz, Mr, vp);
}

}  // namespace hyqk
