// Phases [E] realizability and [F] BGK collision of the step
// (src/simulation_runner.jl:526-557), per cell, out of place.
#include "hyq_eigen.cuh"
#include "hyq_step.cuh"

using namespace hyq;

namespace hyqk {
namespace {

__device__ __noinline__ void cell_phase_EF(double* m, int flag2D, double Ma, int positivity, double dt, double Kn) {
  double a[35], b[35];
  double v0, v1;
  flux_closure35(m, flag2D, Ma, nullptr, nullptr, nullptr, a);
  eigenvalues6(a, 1, flag2D, Ma, v0, v1, b);
  eigenvalues6(b, 2, flag2D, Ma, v0, v1, a);
  flux_closure35(a, flag2D, Ma, nullptr, nullptr, nullptr, m);
  collision35(m, dt, Kn, positivity);
}

__global__ void __launch_bounds__(BS_EF) k_phase_EF(const double* __restrict__ Min, double* __restrict__ Mout, const StepConst sc,
                                                     const DevClock* clk) {
  if (!clk->active) return;
  const long long N = sc.N;
  const long long c = (long long)blockIdx.x * BS_EF + threadIdx.x;
  if (c >= N) return;
  double m[35];
#pragma unroll
  for (int n = 0; n < 35; ++n) m[n] = Min[c + N * n];
  cell_phase_EF(m, sc.flag2D, sc.Ma, sc.positivity, clk->dt, sc.Kn);
#pragma unroll
  for (int n = 0; n < 35; ++n) Mout[c + N * n] = m[n];
}

}  // namespace

void launch_phase_EF(const StepConst& sc, const double* Min, double* Mout, const DevClock* clk, cudaStream_t s) {
  k_phase_EF<<<grid_of(sc.N, BS_EF), BS_EF, 0, s>>>(Min, Mout, sc, clk);
}

}  // namespace hyqk
