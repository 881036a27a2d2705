// Per-cell entry points on device arrays (SoA, stride n): the reference's
// per-cell functions, exposed for parity tests and for callers that compose
// their own loops.
#include "hyq_eigen.cuh"
#include "hyq_step.cuh"

using namespace hyq;

namespace hyqk {
namespace {

__device__ __forceinline__ float qnan_f() { return __int_as_float(0x7fc00000); }

__global__ void __launch_bounds__(BS_CELLS) k_cells_flux(const double* __restrict__ M, long long n, int flag2D, double Ma, double* Fx, double* Fy,
                                                          double* Fz, double* Mr) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35], fx[35], fy[35], fz[35], r[35];
  for (int q = 0; q < 35; ++q) m[q] = M[c + n * q];
  flux_closure35(m, flag2D, Ma, fx, fy, fz, r);
  for (int q = 0; q < 35; ++q) {
    if (Fx) Fx[c + n * q] = fx[q];
    if (Fy) Fy[c + n * q] = fy[q];
    if (Fz) Fz[c + n * q] = fz[q];
    if (Mr) Mr[c + n * q] = r[q];
  }
}

__global__ void __launch_bounds__(BS_CELLS) k_cells_eig(const double* __restrict__ M, long long n, int axis, int flag2D, double Ma, int positivity,
                                                         double* v, double* Mr) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35], r[35];
  for (int q = 0; q < 35; ++q) m[q] = M[c + n * q];
  double a, b;
  if (axis == 3) eigenvalues6z(m, flag2D, Ma, positivity, a, b, r);
  else eigenvalues6(m, axis, flag2D, Ma, a, b, r);
  v[c] = a; v[c + n] = b;
  for (int q = 0; q < 35; ++q) Mr[c + n * q] = r[q];
}

__global__ void __launch_bounds__(BS_CELLS) k_cells_closure_eigs(const double* __restrict__ mom, long long n, double* v) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double a, b;
  closure_eigs(mom[c], mom[c + n], mom[c + 2 * n], mom[c + 3 * n], mom[c + 4 * n], a, b);
  v[c] = a; v[c + n] = b;
}

__global__ void __launch_bounds__(BS_CELLS) k_cells_collision(const double* __restrict__ M, long long n, double dt, double Kn, int positivity,
                                                               double* out) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35];
  for (int q = 0; q < 35; ++q) m[q] = M[c + n * q];
  collision35(m, dt, Kn, positivity);
  for (int q = 0; q < 35; ++q) out[c + n * q] = m[q];
}

// compute_standardized_field / compute_central_field
// (src/utils/compute_standardized_field.jl:16-66): M2CS4_35 per cell.
__global__ void __launch_bounds__(BS_CELLS) k_std_central(const double* __restrict__ M, long long n, double* S, double* C) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35], cc[35], ss[35];
  for (int q = 0; q < 35; ++q) m[q] = M[c + n * q];
  raw_to_central(m, cc);
  central_to_std(cc, ss);
  for (int q = 0; q < 35; ++q) {
    if (S) S[c + n * q] = ss[q];
    if (C) C[c + n * q] = cc[q];
  }
}

// Training targets of the wave-speed network: phase [A]'s first closure,
// then the x, y and z eigenvalue functions (the plain path, with their
// corrections) as the step runs them; the six extreme speeds standardized by
// the realized moments' mean velocity and variance along each axis.
__global__ void __launch_bounds__(BS_CELLS) k_cells_targets(const double* __restrict__ M, long long n, int flag2D, double Ma, int positivity,
                                                             float* __restrict__ T, double* __restrict__ Mr) {
  const long long c = (long long)blockIdx.x * BS_CELLS + threadIdx.x;
  if (c >= n) return;
  double m[35], a[35], b[35];
  for (int q = 0; q < 35; ++q) m[q] = M[c + n * q];
  flux_closure35(m, flag2D, Ma, nullptr, nullptr, nullptr, a);
  if (Mr) for (int q = 0; q < 35; ++q) Mr[c + n * q] = a[q];
  double v[6];
  eigenvalues6(a, 1, flag2D, Ma, v[0], v[1], b);
  eigenvalues6(b, 2, flag2D, Ma, v[2], v[3], m);
  eigenvalues6z(m, flag2D, Ma, positivity, v[4], v[5], b);
  const int iu[3] = {1, 5, 15}, i2[3] = {2, 9, 19};
  for (int d = 0; d < 3; ++d) {
    const double mu = a[iu[d]] / a[0], var = a[i2[d]] / a[0] - mu * mu;
    const double sd = sqrt(var);
    for (int q = 0; q < 2; ++q) {
      const double s = (v[2 * d + q] - mu) / sd;
      T[c * 8 + 2 * d + q] = isfinite(s) ? (float)s : qnan_f();
    }
  }
  T[c * 8 + 6] = 0.0f;
  T[c * 8 + 7] = 0.0f;
}

}  // namespace

void launch_cells_targets(const double* M, long long n, int flag2D, double Ma, int positivity, float* T, double* Mr, cudaStream_t s) {
  k_cells_targets<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(M, n, flag2D, Ma, positivity, T, Mr);
}

void launch_cells_flux(const double* M, long long n, int flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr, cudaStream_t s) {
  k_cells_flux<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(M, n, flag2D, Ma, Fx, Fy, Fz, Mr);
}
void launch_cells_eig(const double* M, long long n, int axis, int flag2D, double Ma, int positivity, double* v, double* Mr, cudaStream_t s) {
  k_cells_eig<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(M, n, axis, flag2D, Ma, positivity, v, Mr);
}
void launch_cells_closure_eigs(const double* mom, long long n, double* v, cudaStream_t s) {
  k_cells_closure_eigs<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(mom, n, v);
}
void launch_cells_collision(const double* M, long long n, double dt, double Kn, int positivity, double* out, cudaStream_t s) {
  k_cells_collision<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(M, n, dt, Kn, positivity, out);
}
void launch_std_central(const double* M, long long n, double* S, double* C, cudaStream_t s) {
  k_std_central<<<grid_of(n, BS_CELLS), BS_CELLS, 0, s>>>(M, n, S, C);
}

}  // namespace hyqk
