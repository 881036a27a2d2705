// Phase [A] of the step (src/simulation_runner.jl:352-383): per cell, the
// closure + realizability, x/y/z flux-Jacobian eigenvalues with their
// corrections, the closure of the realized moments (fluxes Fx, Fy, Fz) and the
// 1-D closure speeds; a NaN-propagating block max of |speed| feeds the CFL
// reduction.
#include "hyq_eigen.cuh"
#include "hyq_step.cuh"

using namespace hyq;

namespace hyqk {
namespace {

// One cell: in m[35]; out Fx, Fy, Fz, Mr (35 each) and vp[6].
__device__ __noinline__ void cell_phase_A(const double* m, int flag2D, double Ma, int positivity, double* Fx, double* Fy, double* Fz, double* Mr,
                                          double* vp) {
  double a[35], b[35];
  flux_closure35(m, flag2D, Ma, nullptr, nullptr, nullptr, a);
  double v6xmin, v6xmax, v6ymin, v6ymax, v6zmin, v6zmax;
  eigenvalues6(a, 1, flag2D, Ma, v6xmin, v6xmax, b);
  eigenvalues6(b, 2, flag2D, Ma, v6ymin, v6ymax, a);
  eigenvalues6z(a, flag2D, Ma, positivity, v6zmin, v6zmax, b);
  flux_closure35(b, flag2D, Ma, Fx, Fy, Fz, Mr);
  double v5xmin, v5xmax, v5ymin, v5ymax, v5zmin, v5zmax;
  closure_eigs(Mr[0], Mr[1], Mr[2], Mr[3], Mr[4], v5xmin, v5xmax);
  closure_eigs(Mr[0], Mr[5], Mr[9], Mr[12], Mr[14], v5ymin, v5ymax);
  closure_eigs(Mr[0], Mr[15], Mr[19], Mr[22], Mr[24], v5zmin, v5zmax);
  vp[0] = jmin(v5xmin, v6xmin); vp[1] = jmax(v5xmax, v6xmax);
  vp[2] = jmin(v5ymin, v6ymin); vp[3] = jmax(v5ymax, v6ymax);
  vp[4] = jmin(v5zmin, v6zmin); vp[5] = jmax(v5zmax, v6zmax);
}

__global__ void __launch_bounds__(BS_A) k_phase_A(double* __restrict__ M, double* __restrict__ Fx, double* __restrict__ Fy,
                                                   double* __restrict__ Fz, double* __restrict__ vp, double* __restrict__ blockmax,
                                                   const StepConst sc, DevClock* clk) {
  const bool active = (clk->t < sc.tmax) && (clk->nn < sc.nnmax);
  if (!active) return;
  const long long N = sc.N;
  const long long c = (long long)blockIdx.x * BS_A + threadIdx.x;
  double local = 0.0;
  if (c < N) {
    double m[35], fx[35], fy[35], fz[35], mr[35], v[6];
#pragma unroll
    for (int n = 0; n < 35; ++n) m[n] = M[c + N * n];
    cell_phase_A(m, sc.flag2D, sc.Ma, sc.positivity, fx, fy, fz, mr, v);
#pragma unroll
    for (int n = 0; n < 35; ++n) {
      Fx[c + N * n] = fx[n]; Fy[c + N * n] = fy[n]; Fz[c + N * n] = fz[n]; M[c + N * n] = mr[n];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) { vp[c + N * q] = v[q]; local = nanmax(local, fabs(v[q])); }
  }
  const double bm = block_nanmax<BS_A>(local);
  if (threadIdx.x == 0) blockmax[blockIdx.x] = bm;
}

__global__ void __launch_bounds__(BS_CELLS) k_cells_phase_A(const double* __restrict__ M, long long n, int flag2D, double Ma, int positivity,
                                                             double* Fx, double* Fy, double* Fz, double* Mr, double* vp) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35], fx[35], fy[35], fz[35], r[35], v[6];
  for (int q = 0; q < 35; ++q) m[q] = M[c + n * q];
  cell_phase_A(m, flag2D, Ma, positivity, fx, fy, fz, r, v);
  for (int q = 0; q < 35; ++q) { Fx[c + n * q] = fx[q]; Fy[c + n * q] = fy[q]; Fz[c + n * q] = fz[q]; Mr[c + n * q] = r[q]; }
  for (int q = 0; q < 6; ++q) vp[c + n * q] = v[q];
}

}  // namespace

void launch_phase_A(const StepConst& sc, double* M, double* Fx, double* Fy, double* Fz, double* vp, double* blockmax, DevClock* clk,
                    cudaStream_t s) {
  k_phase_A<<<sc.nblocksA, BS_A, 0, s>>>(M, Fx, Fy, Fz, vp, blockmax, sc, clk);
}
void launch_cells_phase_A(const double* M, long long n, int flag2D, double Ma, int positivity, double* Fx, double* Fy, double* Fz,
                          double* Mr, double* vp, cudaStream_t s) {
  k_cells_phase_A<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(M, n, flag2D, Ma, positivity, Fx, Fy, Fz, Mr, vp);
}

}  // namespace hyqk
