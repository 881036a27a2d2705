// Per-cell FP64 physics of the HyQMOM explicit step, device code for sm_100a.
//
// One thread owns one cell; the closure, realizability projection,
// eigen-solves and BGK relaxation run as straight FP64 code.  Work arrays
// that are indexed with compile-time constants (the moment transforms of the
// closure, the leading-minor determinants, the usual case of the 6x6
// eigen-solve) stay in registers; the rest lives in thread-local memory.
//
// Reference functions restated here (HyQMOM.jl):
//   src/numerics/Flux_closure35_and_realizable_3D.jl:33-234
//   src/moments/{M2CS4_35,enforce_univariate,hyqmom_3D,InitializeM4_35}.jl
//   src/realizability/*.jl, src/utils/diagnostics.jl:128-187
//   src/autogen/*.jl (derived from their mathematics, see below)
//   src/numerics/{eigenvalues6_hyperbolic_3D,eigenvalues6z_hyperbolic_3D,
//                 compute_jacobian_eigenvalues,closure_and_eigenvalues,
//                 collision35}.jl
// Generated closed forms of the reference are computed from their
// definitions: delta2star3D is the Schur complement M22 - M21 M11^-1 M12 of
// the standardized moment matrix (basis {1,x,y,z} | {x2,xy,xz,y2,yz,z2});
// lower_bound_S220 and bound_minor1 are entries of M21 M11^-1 M12;
// delta2starchol_L3 = (1 - s11^2) det of the 2-D Schur complement; rootsR and
// rootsR_X_Y are the Cardano roots of determinant cubics (real fast-math sqrt,
// so three real roots give NaN exactly like the reference); jacobian6 is the
// Jacobian of the closed 2-D x-fluxes (m32, m23, m14) with respect to
// (m02, m12, m22, m03, m13, m04), in a closed form generated symbolically
// (gen_jacobian6.inc).
#pragma once
#include <cstdint>
#include <cmath>

namespace hyq {

#define HQD __device__ __forceinline__
#define HQN static __device__ __noinline__

constexpr double EPS = 2.220446049250313e-16;

// Julia max/min: NaN-propagating.
HQD double jmax(double a, double b) { return (a != a) ? a : ((b != b) ? b : (a < b ? b : a)); }
HQD double jmin(double a, double b) { return (a != a) ? a : ((b != b) ? b : (b < a ? b : a)); }
HQD double jsign(double x) { return (x != x) ? x : (x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0)); }
HQD double fm_sqrt(double x) { return x < 0.0 ? __longlong_as_double(0x7ff8000000000000LL) : sqrt(x); }
HQD double sq(double x) { return x * x; }
HQD double cube(double x) { return x * x * x; }
HQD double pow4(double x) { double y = x * x; return y * y; }
HQD double pow5(double x) { double y = x * x; return y * y * x; }
HQD double qnan() { return __longlong_as_double(0x7ff8000000000000LL); }

// exp(x) written here (Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, the
// Taylor series of exp(r) to degree 14 by Horner, scaling by 2^k), so that
// the device code and the CPU oracle round identically; accuracy ~1 ulp.
HQD double hexp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return __longlong_as_double(0x7ff0000000000000LL);
  if (x < -745.1332191019412) return 0.0;
  const double k = rint(x * 1.4426950408889634);
  const double r = (x - k * 0.6931471803691238) - k * 1.9082149292705877e-10;
  double p = 1.1470745597729725e-11;
  p = p * r + 1.6059043836821613e-10;
  p = p * r + 2.08767569878681e-09;
  p = p * r + 2.505210838544172e-08;
  p = p * r + 2.755731922398589e-07;
  p = p * r + 2.7557319223985893e-06;
  p = p * r + 2.48015873015873e-05;
  p = p * r + 0.0001984126984126984;
  p = p * r + 0.001388888888888889;
  p = p * r + 0.008333333333333333;
  p = p * r + 0.041666666666666664;
  p = p * r + 0.16666666666666666;
  p = p * r + 0.5;
  p = p * r + 1.0;
  p = p * r + 1.0;
  return ldexp(p, (int)k);
}

// Real cube root written here (exponent split into a multiple of 3, Newton
// iterations on the mantissa), identical on device and in the oracle.
HQD double hcbrt(double x) {
  if (x == 0.0 || x != x || isinf(x)) return x;
  int e;
  double m = frexp(fabs(x), &e);
  int rr = e % 3;
  if (rr < 0) rr += 3;
  m = ldexp(m, rr);
  e -= rr;
  double y = 0.7 + 0.25 * m;
  for (int it = 0; it < 7; ++it) y = y - (y * y * y - m) / (3.0 * y * y);
  y = ldexp(y, e / 3);
  return x < 0.0 ? -y : y;
}

// a / d when the reciprocal r = 1.0 / d (IEEE-rounded) is already known, as
// in the HLL star state where the same d divides all 35 moments: q = a r
// is within an ulp of a / d, the remainder a - q d is exact with one fused
// multiply-add, and q + (a - q d) r rounds to the correctly rounded quotient
// (Markstein's correction step, IBM J. Res. Dev. 34(1), 1990).  A zero a
// gives the signed zero a r (the sign of a / d); outside the normal range of
// the quotient (and for Inf/NaN) it falls back to a / d.  The result equals
// a / d bit for bit; tests/test_device_code_on_host.py checks that on random
// operands.
HQD double div_by(double a, double d, double r) {
  const double q = a * r;
  if (fabs(q) > 1e-290 && fabs(q) < 1e290) {
    const double e = fma(-q, d, a);
    return fma(e, r, q);
  }
  if (a == 0.0) return q;
  return a / d;
}

// 35-moment order (src/utils/moment_idx.jl:73-76) as exponent tables.
__device__ constexpr int T_EXI[35] = {0,1,2,3,4,0,1,2,3,0,1,2,0,1,0,0,1,2,3,0,1,2,0,1,0,0,1,2,0,1,0,0,1,0,0};
__device__ constexpr int T_EXJ[35] = {0,0,0,0,0,1,1,1,1,2,2,2,3,3,4,0,0,0,0,0,0,0,0,0,0,1,1,1,2,2,3,1,1,1,2};
__device__ constexpr int T_EXK[35] = {0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,1,1,1,1,2,2,2,3,3,4,1,1,1,1,1,1,2,2,3,2};
__device__ constexpr int T_BIN[49] = {1,0,0,0,0,0,0, 1,1,0,0,0,0,0, 1,2,1,0,0,0,0, 1,3,3,1,0,0,0, 1,4,6,4,1,0,0, 1,5,10,10,5,1,0, 1,6,15,20,15,6,1};
// Compile-time lookup tables, flattened [i][j][k] over 0..5 (i*36 + j*6 + k).
__device__ constexpr int T_IDX35[216] = {0,15,19,22,24,-1,5,25,31,33,-1,-1,9,28,34,-1,-1,-1,12,30,-1,-1,-1,-1,14,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,1,16,20,23,-1,-1,6,26,32,-1,-1,-1,10,29,-1,-1,-1,-1,13,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,2,17,21,-1,-1,-1,7,27,-1,-1,-1,-1,11,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,3,18,-1,-1,-1,-1,8,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,4,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
__device__ constexpr int T_S28[216] = {-1,-1,-1,15,17,-1,-1,18,24,26,-1,-1,-1,21,27,-1,-1,-1,7,23,-1,-1,-1,-1,9,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,10,13,16,-1,-1,2,19,25,-1,-1,-1,5,22,-1,-1,-1,-1,8,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,11,14,-1,-1,-1,3,20,-1,-1,-1,-1,6,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,0,12,-1,-1,-1,-1,4,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
__device__ constexpr int T_F5[216] = {-1,-1,-1,-1,-1,20,-1,-1,-1,-1,19,-1,-1,-1,-1,18,-1,-1,-1,-1,17,-1,-1,-1,-1,16,-1,-1,-1,-1,15,-1,-1,-1,-1,-1,-1,-1,-1,-1,8,-1,-1,-1,-1,13,-1,-1,-1,-1,14,-1,-1,-1,-1,11,-1,-1,-1,-1,4,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,7,-1,-1,-1,-1,12,-1,-1,-1,-1,10,-1,-1,-1,-1,3,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,6,-1,-1,-1,-1,9,-1,-1,-1,-1,2,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,5,-1,-1,-1,-1,1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,0,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
HQD int ex_i(int n) { return T_EXI[n]; }
HQD int ex_j(int n) { return T_EXJ[n]; }
HQD int ex_k(int n) { return T_EXK[n]; }
// index of moment (i,j,k), order <= 4, in the 35-vector; -1 if absent
HQD int idx35(int i, int j, int k) { return T_IDX35[i * 36 + j * 6 + k]; }
HQD int binom(int n, int k) { return T_BIN[n * 7 + k]; }

// ------------------------------------------------------------ conversions
// 56-entry moment storage (order <= 5): the 35 moments of order <= 4 in the
// reference order, then the 21 fifth-order moments in the closure order.
__device__ constexpr unsigned char T_EX56I[56] = {0,1,2,3,4,0,1,2,3,0,1,2,0,1,0,0,1,2,3,0,1,2,0,1,0,0,1,2,0,1,0,0,1,0,0,5,4,3,2,1,4,3,2,1,3,2,1,2,1,1,0,0,0,0,0,0};
__device__ constexpr unsigned char T_EX56J[56] = {0,0,0,0,0,1,1,1,1,2,2,2,3,3,4,0,0,0,0,0,0,0,0,0,0,1,1,1,2,2,3,1,1,1,2,0,1,2,3,4,0,0,0,0,1,2,3,1,1,2,5,4,3,2,1,0};
__device__ constexpr unsigned char T_EX56K[56] = {0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,1,1,1,1,2,2,2,3,3,4,1,1,1,1,1,1,2,2,3,2,0,0,0,0,0,1,2,3,4,1,1,1,2,3,2,0,1,2,3,4,5};
__device__ constexpr signed char T_IDX56[216] = {0,15,19,22,24,55,5,25,31,33,54,-1,9,28,34,53,-1,-1,12,30,52,-1,-1,-1,14,51,-1,-1,-1,-1,50,-1,-1,-1,-1,-1,1,16,20,23,43,-1,6,26,32,48,-1,-1,10,29,49,-1,-1,-1,13,46,-1,-1,-1,-1,39,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,2,17,21,42,-1,-1,7,27,47,-1,-1,-1,11,45,-1,-1,-1,-1,38,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,3,18,41,-1,-1,-1,8,44,-1,-1,-1,-1,37,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,4,40,-1,-1,-1,-1,36,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,35,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
// pass orders of the separable shift transforms (exponent of the axis descending)
__device__ constexpr unsigned char T_L35X[35] = {4,3,8,18,2,7,11,17,21,27,1,6,10,13,16,20,23,26,29,32,0,5,9,12,14,15,19,22,24,25,28,30,31,33,34};
__device__ constexpr unsigned char T_L35Y[35] = {14,12,13,30,9,10,11,28,29,34,5,6,7,8,25,26,27,31,32,33,0,1,2,3,4,15,16,17,18,19,20,21,22,23,24};
__device__ constexpr unsigned char T_L35Z[35] = {24,22,23,33,19,20,21,31,32,34,15,16,17,18,25,26,27,28,29,30,0,1,2,3,4,5,6,7,8,9,10,11,12,13,14};
__device__ constexpr unsigned char T_L56X[56] = {35,4,36,40,3,8,18,37,41,44,2,7,11,17,21,27,38,42,45,47,1,6,10,13,16,20,23,26,29,32,39,43,46,48,49,0,5,9,12,14,15,19,22,24,25,28,30,31,33,34,50,51,52,53,54,55};
__device__ constexpr unsigned char T_L56Y[56] = {50,14,39,51,12,13,30,38,46,52,9,10,11,28,29,34,37,45,49,53,5,6,7,8,25,26,27,31,32,33,36,44,47,48,54,0,1,2,3,4,15,16,17,18,19,20,21,22,23,24,35,40,41,42,43,55};
__device__ constexpr unsigned char T_L56Z[56] = {55,24,43,54,22,23,33,42,48,53,19,20,21,31,32,34,41,47,49,52,15,16,17,18,25,26,27,28,29,30,40,44,45,46,51,0,1,2,3,4,5,6,7,8,9,10,11,12,13,14,35,36,37,38,39,50};
// 28-set index of each stored moment (-1: order 0, 1, diagonal 2, or 5)
__device__ constexpr signed char T_S28OF56[56] = {-1,-1,-1,0,1,-1,2,3,4,-1,5,6,7,8,9,-1,10,11,12,-1,13,14,15,16,17,18,19,20,21,22,23,24,25,26,27,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
// storage index of the x/y/z flux moment of each of the 35 moments
__device__ constexpr unsigned char T_FX[35] = {1,2,3,4,35,6,7,8,36,10,11,37,13,38,39,16,17,18,40,20,21,41,23,42,43,26,27,44,29,45,46,32,47,48,49};
__device__ constexpr unsigned char T_FY[35] = {5,6,7,8,36,9,10,11,37,12,13,38,14,39,50,25,26,27,44,31,32,47,33,48,54,28,29,45,30,46,51,34,49,53,52};
__device__ constexpr unsigned char T_FZ[35] = {15,16,17,18,40,25,26,27,44,28,29,45,30,46,51,19,20,21,41,22,23,42,24,43,55,31,32,47,34,49,52,33,48,54,53};

// Separable binomial shift of stored moments along one axis (n = 35: order
// <= 4, n = 56: order <= 5):  A_ijk <- sum_{a <= i} C(i,a) s^(i-a) A_ajk
// (x axis shown).  Entries are visited with the axis exponent descending, so
// the update is in place.  Raw <-> central conversions are three such passes,
// one per axis, instead of the full triple sums.
HQN void shift_axis(double* A, int n, int axis, double sh) {
  double pw[6];
  pw[0] = 1.0;
  for (int q = 1; q < 6; ++q) pw[q] = pw[q - 1] * sh;
  const unsigned char* L = (n == 35) ? (axis == 0 ? T_L35X : axis == 1 ? T_L35Y : T_L35Z) : (axis == 0 ? T_L56X : axis == 1 ? T_L56Y : T_L56Z);
  const int stride = axis == 0 ? 36 : axis == 1 ? 6 : 1;
  for (int t = 0; t < n; ++t) {
    const int q = L[t];
    const int e = axis == 0 ? T_EX56I[q] : axis == 1 ? T_EX56J[q] : T_EX56K[q];
    if (e == 0) continue;
    const int base = T_EX56I[q] * 36 + T_EX56J[q] * 6 + T_EX56K[q] - e * stride;
    double acc = 0.0;
    for (int a = 0; a <= e; ++a) acc = acc + (double(T_BIN[e * 7 + a]) * pw[e - a]) * A[T_IDX56[base + a * stride]];
    A[q] = acc;
  }
}

// shift_axis with the store size and axis fixed at compile time and every
// loop unrolled, so that a store held in a local array of the caller can stay
// in registers; same operations in the same order as shift_axis.
template <int N, int AXIS> HQD void shift_axis_r(double (&A)[N], double sh) {
  double pw[6];
  pw[0] = 1.0;
#pragma unroll
  for (int q = 1; q < 6; ++q) pw[q] = pw[q - 1] * sh;
  const unsigned char* L = (N == 35) ? (AXIS == 0 ? T_L35X : AXIS == 1 ? T_L35Y : T_L35Z) : (AXIS == 0 ? T_L56X : AXIS == 1 ? T_L56Y : T_L56Z);
  constexpr int stride = AXIS == 0 ? 36 : AXIS == 1 ? 6 : 1;
#pragma unroll
  for (int t = 0; t < N; ++t) {
    const int q = L[t];
    const int e = AXIS == 0 ? T_EX56I[q] : AXIS == 1 ? T_EX56J[q] : T_EX56K[q];
    if (e == 0) continue;
    const int base = T_EX56I[q] * 36 + T_EX56J[q] * 6 + T_EX56K[q] - e * stride;
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a <= 5; ++a)
      if (a <= e) acc = acc + (double(T_BIN[e * 7 + a]) * pw[e - a]) * A[T_IDX56[base + a * stride]];
    A[q] = acc;
  }
}

// Central moments C (35-order, C000=1, first order 0) of raw M
// (M4toC4_3D, src/autogen/M4toC4_3D.jl:42-55).
HQD void raw_to_central(const double* M, double* C) {
  const double inv = 1.0 / M[0];
  const double u = M[1] * inv, v = M[5] * inv, w = M[15] * inv;
  for (int n = 0; n < 35; ++n) C[n] = M[n] * inv;
  shift_axis(C, 35, 0, -u);
  shift_axis(C, 35, 1, -v);
  shift_axis(C, 35, 2, -w);
  C[0] = 1.0; C[1] = 0.0; C[5] = 0.0; C[15] = 0.0;
}

// Raw moments from density, mean and central moments, in place on the store
// A (n = 35 or 56 entries; A[0] = 1 and first order 0 on entry)
// (C4toM4_3D / C5toM5_3D, src/autogen/C4toM4_3D.jl:64-118, C5toM5_3D.jl:16-28).
HQD void central_to_raw(double M000, double u, double v, double w, double* A, int n) {
  shift_axis(A, n, 0, u);
  shift_axis(A, n, 1, v);
  shift_axis(A, n, 2, w);
  for (int q = 0; q < n; ++q) A[q] = M000 * A[q];
}

// raw_to_central / central_to_raw on caller-held arrays (register path).
// (M[n * st]: the moments may be read straight from a moment-major field)
HQD void raw_to_central_r(const double* M, long long st, double (&C)[35]) {
  const double inv = 1.0 / M[0];
  const double u = M[1 * st] * inv, v = M[5 * st] * inv, w = M[15 * st] * inv;
#pragma unroll
  for (int n = 0; n < 35; ++n) C[n] = M[n * st] * inv;
  shift_axis_r<35, 0>(C, -u);
  shift_axis_r<35, 1>(C, -v);
  shift_axis_r<35, 2>(C, -w);
  C[0] = 1.0; C[1] = 0.0; C[5] = 0.0; C[15] = 0.0;
}
template <int N> HQD void central_to_raw_r(double M000, double u, double v, double w, double (&A)[N]) {
  shift_axis_r<N, 0>(A, u);
  shift_axis_r<N, 1>(A, v);
  shift_axis_r<N, 2>(A, w);
#pragma unroll
  for (int q = 0; q < N; ++q) A[q] = M000 * A[q];
}

// Standardized moments S (35-order) from central C (M2CS4_35,
// src/moments/M2CS4_35.jl:15-98).
HQD void central_to_std(const double* C, double* S) {
  const double s1 = sqrt(jmax(C[2], EPS)), s2 = sqrt(jmax(C[9], EPS)), s3 = sqrt(jmax(C[19], EPS));
  double p1[5], p2[5], p3[5];
  p1[0] = p2[0] = p3[0] = 1.0;
  p1[1] = s1; p2[1] = s2; p3[1] = s3;
  p1[2] = s1 * s1; p2[2] = s2 * s2; p3[2] = s3 * s3;
  p1[3] = s1 * s1 * s1; p2[3] = s2 * s2 * s2; p3[3] = s3 * s3 * s3;
  p1[4] = pow4(s1); p2[4] = pow4(s2); p3[4] = pow4(s3);
#pragma unroll
  for (int n = 0; n < 35; ++n) {
    const int i = ex_i(n), j = ex_j(n), k = ex_k(n);
    const int o = i + j + k;
    if (o == 0 || (o == 2 && (i == 2 || j == 2 || k == 2))) { S[n] = 1.0; continue; }
    if (o == 1) { S[n] = 0.0; continue; }
    double d;
    if (i) { d = p1[i]; if (j) d = d * p2[j]; if (k) d = d * p3[k]; }
    else if (j) { d = p2[j]; if (k) d = d * p3[k]; }
    else d = p3[k];
    S[n] = C[n] / d;
  }
}

// ------------------------------------------------------------ univariate
HQD void enforce_univariate(double& S3, double& S4, double h2min, double s3max, double& H) {
  H = S4 - S3 * S3 - 1.0;
  if (H <= h2min) { H = h2min; S4 = H + S3 * S3 + 1.0; }
  if (S3 < -s3max) { S3 = -s3max; S4 = H + S3 * S3 + 1.0; }
  else if (S3 > s3max) { S3 = s3max; S4 = H + S3 * S3 + 1.0; }
}

HQD double realizablity_S220(double S110, double S220, double A220) {
  double r = S220;
  const double mn = jmax(S110 * S110, 1.0 - A220), mx = 1.0 + A220;
  if (S220 < mn) r = mn; else if (S220 > mx) r = mx;
  return r;
}

// realizability_S2 + bisection (src/realizability/realizability_S2.jl:18-66)
HQD void realizability_S2(double& S110, double& S101, double& S011, double& S2r) {
  const double S2 = 1.0 + 2.0 * S110 * S101 * S011 - (S110 * S110 + S101 * S101 + S011 * S011);
  double xr = 1.0;
  if (S2 < 0.0) {
    const double c3 = 2.0 * S110 * S101 * S011, c2 = (S110 * S110 + S101 * S101 + S011 * S011);
    double a = 0.0, b = 1.0;
    double fa = 1.0 + c3 * (a * a * a) - c2 * (a * a);
    bool done = false;
    for (int it = 0; it < 100; ++it) {
      const double c = (a + b) / 2.0;
      const double fc = 1.0 + c3 * (c * c * c) - c2 * (c * c);
      if (fabs(fc) < 1e-12 || (b - a) / 2.0 < 1e-12) { xr = c; done = true; break; }
      if (jsign(fc) == jsign(fa)) { a = c; fa = fc; } else { b = c; }
    }
    if (!done) xr = (a + b) / 2.0;
  }
  xr = 0.9999 * xr;
  S110 = xr * S110; S101 = xr * S101; S011 = xr * S011;
  S2r = 1.0 + 2.0 * S110 * S101 * S011 - (S110 * S110 + S101 * S101 + S011 * S011);
}

// det of a 2x2 with Julia semantics (triangular shortcut, else LU).
HQD double det2(double a, double b, double c, double d) {
  if (b == 0.0 || c == 0.0) return a * d;
  if (fabs(c) > fabs(a)) {  // pivot swap
    const double l = a * (1.0 / c);
    const double u = b - l * d;
    return -(c * u);
  }
  if (a == 0.0) return 0.0;
  const double l = c * (1.0 / a);
  const double u = d - l * b;
  return a * u;
}

// realizability_S210 (src/realizability/realizability_S210.jl:86-110):
// matrix square root of the 2x2 D1 via its closed-form eigen decomposition.
HQD void realizability_S210(double S110, double S101, double S011, double S300, double& S210, double& S201, double H200, double beta) {
  double xr = 1.0;
  const double X0 = S210 - S110 * S300, X1 = S201 - S101 * S300;
  const double a = 1.0 - S101 * S101, b = S101 * S110 - S011, d = 1.0 - S110 * S110;
  double U00, U01, U11;
  {
    const double tr = (a + d) / 2.0, df = (a - d) / 2.0;
    const double r = sqrt(df * df + b * b);
    const double l1 = tr + r, l2 = tr - r;
    const double lmax = jmax(fabs(l1), fabs(l2));
    const double tol = -(2.0 * EPS) * lmax;
    const double s1 = l1 >= tol ? sqrt(jmax(0.0, l1)) : 0.0;
    const double s2 = l2 >= tol ? sqrt(jmax(0.0, l2)) : 0.0;
    if (b == 0.0) {
      U00 = sqrt(jmax(0.0, a)); U11 = sqrt(jmax(0.0, d)); U01 = 0.0;
    } else {
      double vx = b, vy = l1 - a;
      double nv = sqrt(vx * vx + vy * vy);
      if (nv == 0.0) { vx = l1 - d; vy = b; nv = sqrt(vx * vx + vy * vy); }
      vx = vx / nv; vy = vy / nv;
      U00 = s1 * vx * vx + s2 * vy * vy;
      U01 = s1 * vx * vy - s2 * vx * vy;
      U11 = s1 * vy * vy + s2 * vx * vx;
    }
  }
  const double V0 = U00 * X0 + U01 * X1, V1 = U01 * X0 + U11 * X1;
  const double L = jmax(0.0, V0 * V0 + V1 * V1);
  const double dD1 = jmax(0.0, det2(a, b, b, d));
  const double R = H200 * dD1;
  if (R <= 0.0 || X0 * X0 + X1 * X1 < 1000.0 * EPS) xr = 0.0;
  else if (L > R) xr = sqrt(R / L);
  const double Vr0 = beta * xr * V0, Vr1 = beta * xr * V1;
  // Xr = U \ Vr, LU with partial pivoting
  double x0, x1;
  {
    double A00 = U00, A01 = U01, A10 = U01, A11 = U11, r0 = Vr0, r1 = Vr1;
    if (fabs(A10) > fabs(A00)) { double t; t = A00; A00 = A10; A10 = t; t = A01; A01 = A11; A11 = t; t = r0; r0 = r1; r1 = t; }
    const double l = A10 * (1.0 / A00);
    const double u11 = A11 - l * A01;
    const double y1 = r1 - l * r0;
    x1 = y1 / u11;
    x0 = (r0 - A01 * x1) / A00;
  }
  S210 = x0 + S110 * S300;
  S201 = x1 + S101 * S300;
}

HQD double realizability_S111(double S110, double S101, double S011, double S210, double S201, double S120, double S021, double S102, double S012, double S111) {
  double r = S111;
  const double A110 = ((S101 - S011 * S110) * S210 + (S011 - S101 * S110) * S120) / (1.0 - S110 * S110);
  const double A101 = ((S110 - S011 * S101) * S201 + (S011 - S110 * S101) * S102) / (1.0 - S101 * S101);
  const double A011 = ((S110 - S101 * S011) * S021 + (S101 - S110 * S011) * S012) / (1.0 - S011 * S011);
  const double Rmin = jmin(jmin(A110, A101), A011), Rmax = jmax(jmax(A110, A101), A011);
  if (S111 > Rmax) r = Rmax; else if (S111 < Rmin) r = Rmin;
  return r;
}

HQD double realizability_S211(double e11, double e22, double e33, double e12, double e13, double d23, double S211, double beta) {
  double r = S211;
  const double b211 = e12 * e13;
  const double G = jmax(0.0, (e11 * e22 - e13 * e13) * (e11 * e33 - e12 * e12));
  const double sG = beta * fm_sqrt(G);
  const double mn = d23 + (b211 - sG) / e11, mx = d23 + (b211 + sG) / e11;
  if (S211 <= mn) r = mn; else if (S211 >= mx) r = mx;
  return r;
}

// quadratic form V2^T D2 V2 shared by realizability_S310 / _S310_220
HQD double l2_form(double S110, double S101, double S011, double V0, double V1, double V2) {
  const double d00 = 1.0 - S011 * S011, d01 = S011 * S101 - S110, d02 = S011 * S110 - S101;
  const double d11 = 1.0 - S101 * S101, d12 = S101 * S110 - S011, d22 = 1.0 - S110 * S110;
  const double r0 = d00 * V0 + d01 * V1 + d02 * V2;
  const double r1 = d01 * V0 + d11 * V1 + d12 * V2;
  const double r2 = d02 * V0 + d12 * V1 + d22 * V2;
  double q = 0.0;
  q = q + V0 * r0; q = q + V1 * r1; q = q + V2 * r2;
  return q;
}

HQD double realizability_S310(double S110, double S101, double S011, double S300, double S210, double S201, double S120, double S111, double S310, double S220, double H200, double beta) {
  double r = S310;
  const double b310 = S111 * ((1.0 - S110 * S110) * S201 + (S101 * S110 - S011) * S210 + (S011 * S110 - S101) * S300) +
                      S120 * ((1.0 - S101 * S101) * S210 + (S011 * S101 - S110) * S300 + (S101 * S110 - S011) * S201) +
                      S210 * ((1.0 - S011 * S011) * S300 + (S011 * S101 - S110) * S210 + (S011 * S110 - S101) * S201);
  const double a = 1.0 - S101 * S101, b = S101 * S110 - S011, d = 1.0 - S110 * S110;
  const double dD1 = det2(a, b, b, d);
  const double V0 = S210 - S110 * S300, V1 = S201 - S101 * S300;
  const double w0 = a * V0 + b * V1, w1 = b * V0 + d * V1;
  const double L1 = (V0 * w0 + V1 * w1) / dD1;
  double G310b = H200 - L1;
  if (G310b < 0.0) G310b = 0.0;
  const double L2 = l2_form(S110, S101, S011, S210, S120, S111) / dD1;
  double G310a = S220 - S110 * S110 - L2 + 1000.0 * EPS;
  if (G310a < 0.0 || L2 < 0.0) G310a = 0.0;
  const double sG = beta * fm_sqrt(G310a * G310b);
  const double mn = S110 + b310 / dD1 - sG, mx = S110 + b310 / dD1 + sG;
  if (S310 <= mn) r = mn; else if (S310 >= mx) r = mx;
  return r;
}

HQD double realizability_S310_220(double S110, double S101, double S011, double S210, double S120, double S111, double S220) {
  double r = S220;
  const double a = 1.0 - S101 * S101, b = S101 * S110 - S011, d = 1.0 - S110 * S110;
  const double dD1 = det2(a, b, b, d);
  const double L2 = l2_form(S110, S101, S011, S210, S120, S111) / dD1;
  const double mn = S110 * S110 + L2 + 1000.0 * EPS;
  if (mn > r) r = mn;
  return r;
}

// ---------------------------------------------------- standardized set
// The 28 standardized moments of realizable_3D, addressable by index so a
// coordinate permutation is an index remap.
enum : int {
  s300, s400, s110, s210, s310, s120, s220, s030, s130, s040, s101, s201, s301, s102, s202, s003, s103, s004, s011, s111,
  s211, s021, s121, s031, s012, s112, s013, s022, NS
};

// delta2star3D_permutation (src/autogen/delta2star3D_permutation.jl:26-61):
// argument lists of the 6 permutations, as indices into the 28-set.
__device__ constexpr int PERM[6][28] = {
    {s300, s400, s110, s210, s310, s120, s220, s030, s130, s040, s101, s201, s301, s102, s202, s003, s103, s004, s011, s111, s211, s021, s121, s031, s012, s112, s013, s022},
    {s300, s400, s101, s201, s301, s102, s202, s003, s103, s004, s110, s210, s310, s120, s220, s030, s130, s040, s011, s111, s211, s012, s112, s013, s021, s121, s031, s022},
    {s030, s040, s110, s120, s130, s210, s220, s300, s310, s400, s011, s021, s031, s012, s022, s003, s013, s004, s101, s111, s121, s201, s211, s301, s102, s112, s103, s202},
    {s003, s004, s101, s102, s103, s201, s202, s300, s301, s400, s011, s012, s013, s021, s022, s030, s031, s040, s110, s111, s112, s210, s211, s310, s120, s121, s130, s220},
    {s030, s040, s011, s021, s031, s012, s022, s003, s013, s004, s110, s120, s130, s210, s220, s300, s310, s400, s101, s111, s121, s102, s112, s103, s201, s211, s301, s202},
    {s003, s004, s011, s012, s013, s021, s022, s030, s031, s040, s101, s102, s103, s201, s202, s300, s301, s400, s110, s111, s112, s120, s121, s130, s210, s211, s310, s220}};

// Projection Q = M21 M11^-1 M12 (6x6 symmetric, upper triangle in q[21])
// and the Schur complement E = M22 - Q, for the moments g[] of one
// permutation.  M11 = 1 (+) R, R the 3x3 correlation matrix; R^-1 by
// cofactors.  Basis order {x2, xy, xz, y2, yz, z2}.
// Only the entries the realizability check reads are kept (12 of each
// triangle): E on the leading 4x4 block and the last two diagonal entries,
// Q at the diagonal lower bounds and the bound_minor1 values.  The tables
// give each (a, b) its slot, -1 for an entry that is not kept (never read).
struct Delta {
  double e[12];
  double q[12];
};
__device__ constexpr int TRI_E[6][6] = {{0, 1, 2, 3, -1, -1}, {1, 4, 5, 6, -1, -1}, {2, 5, 7, 8, -1, -1},
                                        {3, 6, 8, 9, -1, -1}, {-1, -1, -1, -1, 10, -1}, {-1, -1, -1, -1, -1, 11}};
__device__ constexpr int TRI_Q[6][6] = {{-1, 0, 1, -1, 2, -1}, {0, 3, -1, 4, -1, 5}, {1, -1, 6, 7, -1, 8},
                                        {-1, 4, 7, -1, 9, -1}, {2, -1, -1, 9, 10, 11}, {-1, 5, 8, -1, 11, -1}};

HQN void delta2star_p(const double* s, int P, Delta& D) {
  // arguments of delta2star3D for permutation P (named by the argument slot)
  const int* pm = PERM[P];
  const double g300 = s[pm[0]], g400 = s[pm[1]], g110 = s[pm[2]], g210 = s[pm[3]], g310 = s[pm[4]], g120 = s[pm[5]], g220 = s[pm[6]],
               g030 = s[pm[7]], g130 = s[pm[8]], g040 = s[pm[9]], g101 = s[pm[10]], g201 = s[pm[11]], g301 = s[pm[12]], g102 = s[pm[13]],
               g202 = s[pm[14]], g003 = s[pm[15]], g103 = s[pm[16]], g004 = s[pm[17]], g011 = s[pm[18]], g111 = s[pm[19]], g211 = s[pm[20]],
               g021 = s[pm[21]], g121 = s[pm[22]], g031 = s[pm[23]], g012 = s[pm[24]], g112 = s[pm[25]], g013 = s[pm[26]], g022 = s[pm[27]];
  // R^-1 (symmetric) of R = [1 g110 g101; g110 1 g011; g101 g011 1]
  const double c00 = 1.0 - g011 * g011, c01 = g101 * g011 - g110, c02 = g110 * g011 - g101;
  const double c11 = 1.0 - g101 * g101, c12 = g110 * g101 - g011, c22 = 1.0 - g110 * g110;
  const double det = c00 + g110 * c01 + g101 * c02;
  const double id = 1.0 / det;
  const double r00 = c00 * id, r01 = c01 * id, r02 = c02 * id, r11 = c11 * id, r12 = c12 * id, r22 = c22 * id;
  // mean (order-2 moment) of each basis function and its third-order vector
  const double mu[6] = {1.0, g110, g101, 1.0, g011, 1.0};
  const double w[6][3] = {{g300, g210, g201}, {g210, g120, g111}, {g201, g111, g102},
                          {g120, g030, g021}, {g111, g021, g012}, {g102, g012, g003}};
  double z[6][3];
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    z[a][0] = r00 * w[a][0] + r01 * w[a][1] + r02 * w[a][2];
    z[a][1] = r01 * w[a][0] + r11 * w[a][1] + r12 * w[a][2];
    z[a][2] = r02 * w[a][0] + r12 * w[a][1] + r22 * w[a][2];
  }
  // fourth-order block M22
  const double m22[21] = {g400, g310, g301, g220, g211, g202, g220, g211, g130, g121, g112,
                          g202, g121, g112, g103, g040, g031, g022, g022, g013, g004};
#pragma unroll
  for (int a = 0; a < 6; ++a)
#pragma unroll
    for (int b = a; b < 6; ++b) {
      if (TRI_E[a][b] < 0 && TRI_Q[a][b] < 0) continue;
      const double qv = mu[a] * mu[b] + (w[a][0] * z[b][0] + w[a][1] * z[b][1] + w[a][2] * z[b][2]);
      if (TRI_Q[a][b] >= 0) D.q[TRI_Q[a][b]] = qv;
      if (TRI_E[a][b] >= 0) D.e[TRI_E[a][b]] = m22[a * 6 + b - a * (a + 1) / 2] - qv;
    }
}

HQD double E_(const Delta& D, int a, int b) { return D.e[TRI_E[a][b]]; }
HQD double Q_(const Delta& D, int a, int b) { return D.q[TRI_Q[a][b]]; }

// Leading K x K minor determinant with Julia det semantics (triangular
// shortcut, else LU with partial pivoting and reciprocal row scaling); K is
// fixed at compile time and every loop unrolled (row swaps through
// compile-time selects), so the K x K block stays in registers.
template <int K> HQD double lead_det_k(const Delta& D) {
  double A[K][K];
#pragma unroll
  for (int i = 0; i < K; ++i)
#pragma unroll
    for (int j = 0; j < K; ++j) A[i][j] = E_(D, i, j);
  bool triu = true, tril = true;
#pragma unroll
  for (int i = 0; i < K; ++i)
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (i > j && A[i][j] != 0.0) triu = false;
      if (i < j && A[i][j] != 0.0) tril = false;
    }
  if (triu || tril) {
    double p = 1.0;
#pragma unroll
    for (int i = 0; i < K; ++i) p = p * A[i][i];
    return p;
  }
  int swaps = 0;
  bool singular = false;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    int p = k;
    double amax = fabs(A[k][k]);
#pragma unroll
    for (int i = k + 1; i < K; ++i)
      if (fabs(A[i][k]) > amax) { amax = fabs(A[i][k]); p = i; }
    if (p != k) {
#pragma unroll
      for (int i = k + 1; i < K; ++i)
        if (p == i) {
#pragma unroll
          for (int j = 0; j < K; ++j) { const double t = A[k][j]; A[k][j] = A[i][j]; A[i][j] = t; }
        }
      ++swaps;
    }
    if (A[k][k] == 0.0) { singular = true; continue; }
    const double r = 1.0 / A[k][k];
#pragma unroll
    for (int i = k + 1; i < K; ++i) A[i][k] = A[i][k] * r;
#pragma unroll
    for (int i = k + 1; i < K; ++i)
#pragma unroll
      for (int j = k + 1; j < K; ++j) A[i][j] = A[i][j] - A[i][k] * A[k][j];
  }
  if (singular) return 0.0;
  double P = 1.0;
#pragma unroll
  for (int i = 0; i < K; ++i) P = P * A[i][i];
  return (swaps & 1) ? -P : P;
}


// --------------------------------------------------- cubic (Cardano) roots
// Reference form (rootsR / rootsR_X_Y): for c3 X^3 + c2 X^2 + c1 X + c0,
// shift + C + p/C and the pair shift - (C + p/C)/2 +- i sqrt(3)/2 (C - p/C),
// C = cbrt(q + sqrt(q^2 - p^3)) with the real fast-math sqrt.
struct Roots3 { double re[3], im[3]; };
HQD Roots3 cardano(double c3, double c2, double c1, double c0) {
  const double B = -c2 / c3, Cc = c1 / c3, Dd = -c0 / c3;
  const double p = B * B / 9.0 - Cc / 3.0;
  const double q = B * B * B / 27.0 - B * Cc / 6.0 + Dd / 2.0;
  const double disc = q * q - p * p * p;
  const double sd = fm_sqrt(disc);
  Roots3 R;
  if (sd != sd) {
#pragma unroll
    for (int i = 0; i < 3; ++i) { R.re[i] = sd; R.im[i] = i == 0 ? 0.0 : sd; }
    return R;
  }
  const double C = hcbrt(q + sd);
  const double pc = p / C;
  const double sh = B / 3.0;
  const double s3 = 1.7320508075688772;  // sqrt(3)
  R.re[0] = sh + C + pc; R.im[0] = 0.0;
  R.re[1] = sh - C / 2.0 - pc / 2.0; R.im[1] = s3 * (C - pc) / 2.0;
  R.re[2] = R.re[1]; R.im[2] = -R.im[1];
  return R;
}
HQD void sort3(double (&r)[3]) {
  auto lt = [](double a, double b) { return (a != a) ? false : ((b != b) ? true : a < b); };
  if (lt(r[1], r[0])) { double t = r[0]; r[0] = r[1]; r[1] = t; }
  if (lt(r[2], r[1])) { double t = r[1]; r[1] = r[2]; r[2] = t; }
  if (lt(r[1], r[0])) { double t = r[0]; r[0] = r[1]; r[1] = t; }
}
HQD double imag_ratio(const Roots3& R) {
  double mi = fabs(R.im[0]), ma = sqrt(R.re[0] * R.re[0] + R.im[0] * R.im[0]);
#pragma unroll
  for (int i = 1; i < 3; ++i) { mi = jmax(mi, fabs(R.im[i])); ma = jmax(ma, sqrt(R.re[i] * R.re[i] + R.im[i] * R.im[i])); }
  return mi / ma;
}

// det of [[a00, a01, a02, ex+X],[a01, X, a12, a13],[a02, a12, Y, a23],[ex+X, a13, a23, a33]]
// as a cubic in X (rootsR_X_Y, src/autogen/rootsR_X_Y.jl:6-77).
HQD Roots3 roots_X_Y(double Y, double e11, double e12, double e13, double e23, double e24, double e34, double e44, double ex) {
  // Expand along the structure: entries affine in X are (1,1)->X, (0,3),(3,0)->ex+X.
  // det = sum over permutations; computed as polynomial by cofactor expansion.
  // Polynomials as (c0,c1,c2,c3).
  struct P { double c[4]; };
  auto mk = [](double a, double b) { P p; p.c[0] = a; p.c[1] = b; p.c[2] = 0.0; p.c[3] = 0.0; return p; };
  auto mul = [](const P& a, const P& b) {
    P r; r.c[0] = r.c[1] = r.c[2] = r.c[3] = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; i + j < 4; ++j) r.c[i + j] = r.c[i + j] + a.c[i] * b.c[j];
    return r;
  };
  auto add = [](const P& a, const P& b, double s) { P r; for (int i = 0; i < 4; ++i) r.c[i] = a.c[i] + s * b.c[i]; return r; };
  P A[4][4] = {{mk(e11, 0), mk(e12, 0), mk(e13, 0), mk(ex, 1)},
               {mk(e12, 0), mk(0, 1), mk(e23, 0), mk(e24, 0)},
               {mk(e13, 0), mk(e23, 0), mk(Y, 0), mk(e34, 0)},
               {mk(ex, 1), mk(e24, 0), mk(e34, 0), mk(e44, 0)}};
  P det = mk(0, 0);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    P S[3][3];
#pragma unroll
    for (int i = 1; i < 4; ++i) {
      int cc = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j != c) { S[i - 1][cc] = A[i][j]; ++cc; }
    }
    P t0 = add(mul(S[1][1], S[2][2]), mul(S[1][2], S[2][1]), -1.0);
    P t1 = add(mul(S[1][0], S[2][2]), mul(S[1][2], S[2][0]), -1.0);
    P t2 = add(mul(S[1][0], S[2][1]), mul(S[1][1], S[2][0]), -1.0);
    P m = mul(S[0][0], t0);
    m = add(m, mul(S[0][1], t1), -1.0);
    m = add(m, mul(S[0][2], t2), 1.0);
    det = add(det, mul(A[0][c], m), (c & 1) ? -1.0 : 1.0);
  }
  return cardano(det.c[3], det.c[2], det.c[1], det.c[0]);
}

// ------------------------------------------------------------ 2-D pieces
// 2-D Schur complement (basis {1,x,y} | {x2,xy,y2}); returns 3x3 symmetric.
HQD void delta2D(double s30, double s40, double s11, double s21, double s31, double s12, double s22, double s03, double s13, double s04,
                 double (&D)[3][3]) {
  // M11 = [1 0 0; 0 1 s11; 0 s11 1], inverse of the 2x2 part
  const double dt = 1.0 - s11 * s11;
  const double i00 = 1.0 / dt, i01 = -s11 / dt;
  const double mu[3] = {1.0, s11, 1.0};
  const double w[3][2] = {{s30, s21}, {s21, s12}, {s12, s03}};
  const double m22[3][3] = {{s40, s31, s22}, {s31, s22, s13}, {s22, s13, s04}};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double z0 = i00 * w[b][0] + i01 * w[b][1], z1 = i01 * w[b][0] + i00 * w[b][1];
      D[a][b] = m22[a][b] - (mu[a] * mu[b] + (w[a][0] * z0 + w[a][1] * z1));
    }
}
HQD double det3(const double (&D)[3][3]) {
  return D[0][0] * (D[1][1] * D[2][2] - D[1][2] * D[2][1]) - D[0][1] * (D[1][0] * D[2][2] - D[1][2] * D[2][0]) +
         D[0][2] * (D[1][0] * D[2][1] - D[1][1] * D[2][0]);
}

// realizable_2D (src/realizability/realizable_2D.jl:24-118)
HQD void realizable_2D(double S30, double S40, double S11, double& S21, double& S31, double& S12, double& S22, double S03, double& S13, double S04) {
  const double Del1 = jmax(0.0, 1.0 - S11 * S11);
  const double H20 = jmax(EPS, S40 - S30 * S30 - 1.0);
  const double H02 = jmax(EPS, S04 - S03 * S03 - 1.0);
  double G1 = sqrt(Del1 * H02);
  const double s12min = S11 * S03 - G1, s12max = S11 * S03 + G1;
  if (S12 <= s12min) S12 = s12min; else if (S12 >= s12max) S12 = s12max;
  G1 = sqrt(Del1 * H20);
  const double s21min = S11 * S30 - G1, s21max = S11 * S30 + G1;
  if (S21 <= s21min) S21 = s21min; else if (S21 >= s21max) S21 = s21max;
  const double G22 = sqrt((H20 + S30 * S30) * (H02 + S03 * S03));
  const double s22min = jmax(S11 * S11, 1.0 - G22), s22max = 1.0 + G22;
  if (S22 < s22min) S22 = s22min; else if (S22 > s22max) S22 = s22max;
  const double common = Del1 * S22 - Del1 * S11 * S11 - S12 * S12 + 2.0 * S11 * S12 * S21 - S21 * S21;
  double G31 = common * (Del1 * H20 - sq(S21 - S11 * S30));
  double G13 = common * (Del1 * H02 - sq(S12 - S11 * S03));
  if (G31 < 0.0 || G13 < 0.0) { G31 = 0.0; G13 = 0.0; } else { G13 = sqrt(G13); G31 = sqrt(G31); }
  const double den = Del1 + EPS;
  const double b31 = S12 * S21 + S21 * S30 - S11 * S21 * S21 - S11 * S12 * S30;
  const double s31min = S11 + (b31 - G31) / den, s31max = S11 + (b31 + G31) / den;
  if (S31 <= s31min) S31 = s31min; else if (S31 >= s31max) S31 = s31max;
  const double b13 = S12 * S21 + S12 * S03 - S11 * S12 * S12 - S11 * S21 * S03;
  const double s13min = S11 + (b13 - G13) / den, s13max = S11 + (b13 + G13) / den;
  if (S13 <= s13min) S13 = s13min; else if (S13 >= s13max) S13 = s13max;
  double D[3][3];
  const double S40e = S40, S04e = S04;
  delta2D(S30, S40e, S11, S21, S31, S12, S22, S03, S13, S04e, D);
  const double L3 = (1.0 - S11 * S11) * det3(D);
  if (L3 < 0.0) {
    // rootsR: det of the 2-D Schur complement as a cubic in S22
    const double s40 = H20 + S30 * S30 + 1.0, s04 = H02 + S03 * S03 + 1.0;
    double D0[3][3];
    delta2D(S30, s40, S11, S21, S31, S12, 0.0, S03, S13, s04, D0);
    // entries (0,2),(2,0),(1,1) carry +X
    const double a = D0[0][0], b = D0[0][1], c = D0[0][2], d = D0[1][1], e = D0[1][2], f = D0[2][2];
    // det [[a, b, c+X],[b, d+X, e],[c+X, e, f]]
    // = a((d+X)f - e^2) - b(b f - e(c+X)) + (c+X)(b e - (d+X)(c+X))
    const double k0 = a * (d * f - e * e) - b * (b * f - e * c) + c * (b * e - d * c);
    const double k1 = a * f + b * e + (b * e - d * c) - c * (d + c);
    const double k2 = -(d + c) - c;
    const double k3 = -1.0;
    Roots3 R = cardano(k3, k2, k1, k0);
    double Rr[3] = {R.re[0], R.re[1], R.re[2]};
    sort3(Rr);
    const double s22maxr = jmin(s22max, Rr[2]);
    double s22minr = jmax(s22min, Rr[1]);
    if (s22maxr < s22minr) s22minr = s22maxr;
    double S22a = S22;
    if (S22 > s22maxr) S22a = s22maxr; else if (S22 < s22minr) S22a = s22minr;
    if (!(imag_ratio(R) > 1000.0 * EPS)) S22 = S22a;
  }
}

// check2D (src/utils/diagnostics.jl:128-153)
HQD void check2D(double& S30, double& S40, double& S11, double& S21, double& S31, double& S12, double& S22, double& S03, double& S13, double& S04) {
  const double h2min = 1000.0 * EPS;
  if (fabs(S11) >= 1.0) {
    S11 = jsign(S11);
    const double s3m = sqrt(fabs(S30 * S03));
    double s4m = sqrt(S40 * S04);
    const double H2m = jmax(h2min, s4m - s3m * s3m - 1.0);
    s4m = H2m + s3m * s3m + 1.0;
    S30 = jsign(S30) * s3m;
    S03 = S11 * S30;
    S40 = s4m; S04 = s4m;
    S12 = S11 * S03; S21 = S11 * S30; S13 = S11 * S04; S31 = S11 * S40; S22 = s4m;
  } else {
    realizable_2D(S30, S40, S11, S21, S31, S12, S22, S03, S13, S04);
  }
}

}  // namespace hyq
