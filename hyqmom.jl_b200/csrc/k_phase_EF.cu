// Phases [E] realizability and [F] BGK collision of the step
// (src/simulation_runner.jl:526-557), per cell, out of place.
#include "hyq_eigen.cuh"
#include "hyq_step.cuh"

using namespace hyq;

namespace hyqk {
namespace {


// Phases [E]+[F] run as four kernels, one per-cell function each (small code
// per kernel); intermediate states go through the flux buffers, dead after
// the HLL sweep:  Mtmp -E1-> Fx -E2-> Fy -E3-> Fz -E4-> M.
// E1: Flux_closure35_and_realizable_3D
__global__ void __launch_bounds__(BS_EF, MINB_CLOSURE) k_E1_closure(const double* __restrict__ in, double* __restrict__ out, const StepConst sc,
                                                                const DevClock* clk) {
  if (!clk->active) return;
  const long long N = sc.N, c = (long long)blockIdx.x * BS_EF + threadIdx.x;
  if (c >= N) return;
  flux_closure35(in + c, sc.flag2D, sc.Ma, nullptr, nullptr, nullptr, out + c, N, N);
}

// E2/E3: eigenvalues6_hyperbolic_3D along x or y (corrected moments only)
__global__ void __launch_bounds__(BS_EF, MINB_EIG) k_E_eig(const double* __restrict__ in, double* __restrict__ out, int axis, const StepConst sc,
                                                           const DevClock* clk) {
  if (!clk->active) return;
  const long long N = sc.N, c = (long long)blockIdx.x * BS_EF + threadIdx.x;
  if (c >= N) return;
  double v0, v1;
  eigenvalues6(in + c, axis, sc.flag2D, sc.Ma, v0, v1, out + c, N, N);
}

// E4: Flux_closure35_and_realizable_3D, then collision35 with the step's dt
__global__ void __launch_bounds__(BS_EF, MINB_CLOSURE) k_E4_closure_bgk(const double* __restrict__ in, double* __restrict__ Mout, const StepConst sc,
                                                                    const DevClock* clk) {
  if (!clk->active) return;
  const long long N = sc.N, c = (long long)blockIdx.x * BS_EF + threadIdx.x;
  if (c >= N) return;
  double a[35];
  flux_closure35(in + c, sc.flag2D, sc.Ma, nullptr, nullptr, nullptr, a, N, 1);
  collision35(a, clk->dt, sc.Kn, sc.positivity);
#pragma unroll
  for (int n = 0; n < 35; ++n) Mout[c + N * n] = a[n];
}

}  // namespace

void launch_phase_EF(const StepConst& sc, const double* Min, double* Mout, double* Fx, double* Fy, double* Fz, const DevClock* clk,
                     cudaStream_t s, cudaEvent_t* ev) {
  const int g = grid_of(sc.N, BS_EF);
  k_E1_closure<<<g, BS_EF, 0, s>>>(Min, Fx, sc, clk);
  if (ev) cudaEventRecord(ev[0], s);
  k_E_eig<<<g, BS_EF, 0, s>>>(Fx, Fy, 1, sc, clk);
  if (ev) cudaEventRecord(ev[1], s);
  k_E_eig<<<g, BS_EF, 0, s>>>(Fy, Fz, 2, sc, clk);
  if (ev) cudaEventRecord(ev[2], s);
  k_E4_closure_bgk<<<g, BS_EF, 0, s>>>(Fz, Mout, sc, clk);
  if (ev) cudaEventRecord(ev[3], s);
}

}  // namespace hyqk
