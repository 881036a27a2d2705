// HyQMOM explicit-step ORACLE: a scalar CPU restatement of HyQMOM.jl's
// serial time step, used only as the checker for the CUDA path (tests,
// smoke, and the bench's CPU baseline).  It is test infrastructure, not the
// product.  Every function cites the reference file:line it restates.
//
// Semantics kept from the reference (Julia):
//   * min/max/maximum propagate NaN; sort puts NaN last;
//   * `sqrt` inside @fastmath blocks of a negative number is NaN;
//   * det() of a general matrix is LU with partial pivoting, except that a
//     triangular matrix returns the product of its diagonal;
//   * eigvals() of a real nonsymmetric matrix follows the LAPACK path
//     (balance 'B' -> Householder Hessenberg -> double-shift QR with the
//     standardized 2x2 Schur form).
// Closed forms that the reference generated with MATLAB Symbolic are derived
// here from their defining mathematics:
//   * delta2star3D  = Schur complement M22 - M21 M11^{-1} M12 of the
//     standardized moment matrix, basis {1,x,y,z} | {x2,xy,xz,y2,yz,z2};
//   * lower_bound_S220 / bound_minor1 = entries of M21 M11^{-1} M12;
//   * delta2starchol_L3 = (1 - s11^2) * det(2-D Schur complement);
//   * rootsR / rootsR_X_Y = Cardano roots of the determinant cubics;
//   * jacobian6 = d(m32,m23,m14)/d(m02,m12,m22,m03,m13,m04) of the 2-D
//     HyQMOM closure, evaluated by forward-mode differentiation.
// All arithmetic is templated on the real type T so that an op-counting type
// can measure the algorithmic FP64 work per cell-step.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>

namespace hyqo {

// Branch-hit counters (test instrumentation): built only into the
// -DHYQO_BRANCHES variant of the library, which the tests use to show which
// rare branches of the reference's algorithm a set of states takes.
enum Branch {
  BR_FACES = 0,         // realizable_3D faces case, S2 <= S2min (src/realizability/realizable_3D.jl:79-142)
  BR_EDGE_CORNER = 1,   // edge_corner_correction (src/realizability/edge_corner_correction.jl:24-110)
  BR_FLAG220 = 2,       // a repeat of realizable_3D while flag220 (src/numerics/Flux_closure35_and_realizable_3D.jl:134-143)
  BR_COMPLEX_XY = 3,    // complex Jacobian eigenvalues corrected, x or y (eigenvalues6_hyperbolic_3D.jl:35)
  BR_COMPLEX_Z = 4,     // the same along z (eigenvalues6z_hyperbolic_3D.jl)
  BR_ROOTSR_NAN = 5,    // rootsR three real roots -> NaN under fast-math sqrt (src/autogen/rootsR.jl:275)
  BR_ROOTSRXY_NAN = 6,  // rootsR_X_Y the same (src/autogen/rootsR_X_Y.jl:64)
  BR_REREALIZE_Z = 7,   // eigenvalues6z negative-variance re-realization (eigenvalues6z_hyperbolic_3D.jl:63-104)
  BR_COUNT = 8
};
#ifdef HYQO_BRANCHES
extern long long g_branch_hits[BR_COUNT];
inline void hit(int b) {
#pragma omp atomic
  g_branch_hits[b] += 1;
}
#else
inline void hit(int) {}
#endif

constexpr double EPS = 2.220446049250313e-16;  // Julia eps()

// ---------------------------------------------------------------- indexing
// 35-moment order of the reference (src/utils/moment_idx.jl:73-76).
static const int E35[35][3] = {
    {0,0,0},{1,0,0},{2,0,0},{3,0,0},{4,0,0},{0,1,0},{1,1,0},{2,1,0},{3,1,0},
    {0,2,0},{1,2,0},{2,2,0},{0,3,0},{1,3,0},{0,4,0},{0,0,1},{1,0,1},{2,0,1},
    {3,0,1},{0,0,2},{1,0,2},{2,0,2},{0,0,3},{1,0,3},{0,0,4},{0,1,1},{1,1,1},
    {2,1,1},{0,2,1},{1,2,1},{0,3,1},{0,1,2},{1,1,2},{0,1,3},{0,2,2}};

inline int t3(int i, int j, int k) { return i + 6 * j + 36 * k; }  // 6x6x6 cube

// --------------------------------------------------------- scalar helpers
template <class T> inline T jmax(T a, T b) {  // Julia max: NaN-propagating
  if (a != a) return a;
  if (b != b) return b;
  return a < b ? b : a;
}
template <class T> inline T jmin(T a, T b) {
  if (a != a) return a;
  if (b != b) return b;
  return b < a ? b : a;
}
template <class T> inline T jsign(T x) {
  if (x != x) return x;
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0));
}
template <class T> inline T fm_sqrt(T x) {  // @fastmath sqrt
  if (x < T(0)) return T(std::numeric_limits<double>::quiet_NaN());
  using std::sqrt;
  return sqrt(x);
}
template <class T> inline T sq(T x) { return x * x; }
template <class T> inline T cube(T x) { return x * x * x; }
template <class T> inline T pow4(T x) { T y = x * x; return y * y; }
template <class T> inline T pow5(T x) { T y = x * x; return y * y * x; }

// exp(x) written here (Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, the
// Taylor series of exp(r) to degree 14 by Horner, scaling by 2^k), so that
// the device code and the CPU oracle round identically; accuracy ~1 ulp.
inline double hexp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return std::numeric_limits<double>::infinity();
  if (x < -745.1332191019412) return 0.0;
  const double k = std::rint(x * 1.4426950408889634);
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
  return std::ldexp(p, (int)k);
}

// Real cube root written here (exponent split into a multiple of 3, Newton
// iterations on the mantissa), identical on device and in the oracle.
inline double hcbrt(double x) {
  if (x == 0.0 || x != x || std::isinf(x)) return x;
  int e;
  double m = std::frexp(std::fabs(x), &e);
  int rr = e % 3;
  if (rr < 0) rr += 3;
  m = std::ldexp(m, rr);
  e -= rr;
  double y = 0.7 + 0.25 * m;
  for (int it = 0; it < 7; ++it) y = y - (y * y * y - m) / (3.0 * y * y);
  y = std::ldexp(y, e / 3);
  return x < 0.0 ? -y : y;
}

// the real type may be an op counter: exp/cbrt of T go through these
template <class T> inline T hexpT(T x) { using std::exp; return exp(x); }
template <> inline double hexpT<double>(double x) { return hexp(x); }
template <class T> inline T hcbrtT(T x) { using std::cbrt; return cbrt(x); }
template <> inline double hcbrtT<double>(double x) { return hcbrt(x); }

template <class T> inline T ipow(T x, int n) {
  T r = T(1);
  for (int i = 0; i < n; ++i) r = r * x;
  return r;
}

inline int binom(int n, int k) {
  static const int B[6][6] = {{1, 0, 0, 0, 0, 0}, {1, 1, 0, 0, 0, 0},
                              {1, 2, 1, 0, 0, 0}, {1, 3, 3, 1, 0, 0},
                              {1, 4, 6, 4, 1, 0}, {1, 5, 10, 10, 5, 1}};
  return B[n][k];
}

// 56-entry moment storage (order <= 5): the 35 moments of order <= 4 in the
// reference order, then the 21 fifth-order moments in the closure order.
static const unsigned char T_EX56I[56] = {0,1,2,3,4,0,1,2,3,0,1,2,0,1,0,0,1,2,3,0,1,2,0,1,0,0,1,2,0,1,0,0,1,0,0,5,4,3,2,1,4,3,2,1,3,2,1,2,1,1,0,0,0,0,0,0};
static const unsigned char T_EX56J[56] = {0,0,0,0,0,1,1,1,1,2,2,2,3,3,4,0,0,0,0,0,0,0,0,0,0,1,1,1,2,2,3,1,1,1,2,0,1,2,3,4,0,0,0,0,1,2,3,1,1,2,5,4,3,2,1,0};
static const unsigned char T_EX56K[56] = {0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,1,1,1,1,2,2,2,3,3,4,1,1,1,1,1,1,2,2,3,2,0,0,0,0,0,1,2,3,4,1,1,1,2,3,2,0,1,2,3,4,5};
static const signed char T_IDX56[216] = {0,15,19,22,24,55,5,25,31,33,54,-1,9,28,34,53,-1,-1,12,30,52,-1,-1,-1,14,51,-1,-1,-1,-1,50,-1,-1,-1,-1,-1,1,16,20,23,43,-1,6,26,32,48,-1,-1,10,29,49,-1,-1,-1,13,46,-1,-1,-1,-1,39,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,2,17,21,42,-1,-1,7,27,47,-1,-1,-1,11,45,-1,-1,-1,-1,38,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,3,18,41,-1,-1,-1,8,44,-1,-1,-1,-1,37,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,4,40,-1,-1,-1,-1,36,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,35,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
// pass orders of the separable shift transforms (exponent of the axis descending)
static const unsigned char T_L35X[35] = {4,3,8,18,2,7,11,17,21,27,1,6,10,13,16,20,23,26,29,32,0,5,9,12,14,15,19,22,24,25,28,30,31,33,34};
static const unsigned char T_L35Y[35] = {14,12,13,30,9,10,11,28,29,34,5,6,7,8,25,26,27,31,32,33,0,1,2,3,4,15,16,17,18,19,20,21,22,23,24};
static const unsigned char T_L35Z[35] = {24,22,23,33,19,20,21,31,32,34,15,16,17,18,25,26,27,28,29,30,0,1,2,3,4,5,6,7,8,9,10,11,12,13,14};
static const unsigned char T_L56X[56] = {35,4,36,40,3,8,18,37,41,44,2,7,11,17,21,27,38,42,45,47,1,6,10,13,16,20,23,26,29,32,39,43,46,48,49,0,5,9,12,14,15,19,22,24,25,28,30,31,33,34,50,51,52,53,54,55};
static const unsigned char T_L56Y[56] = {50,14,39,51,12,13,30,38,46,52,9,10,11,28,29,34,37,45,49,53,5,6,7,8,25,26,27,31,32,33,36,44,47,48,54,0,1,2,3,4,15,16,17,18,19,20,21,22,23,24,35,40,41,42,43,55};
static const unsigned char T_L56Z[56] = {55,24,43,54,22,23,33,42,48,53,19,20,21,31,32,34,41,47,49,52,15,16,17,18,25,26,27,28,29,30,40,44,45,46,51,0,1,2,3,4,5,6,7,8,9,10,11,12,13,14,35,36,37,38,39,50};
// 28-set index of each stored moment (-1: order 0, 1, diagonal 2, or 5)
static const signed char T_S28OF56[56] = {-1,-1,-1,0,1,-1,2,3,4,-1,5,6,7,8,9,-1,10,11,12,-1,13,14,15,16,17,18,19,20,21,22,23,24,25,26,27,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1,-1};
// storage index of the x/y/z flux moment of each of the 35 moments
static const unsigned char T_FX[35] = {1,2,3,4,35,6,7,8,36,10,11,37,13,38,39,16,17,18,40,20,21,41,23,42,43,26,27,44,29,45,46,32,47,48,49};
static const unsigned char T_FY[35] = {5,6,7,8,36,9,10,11,37,12,13,38,14,39,50,25,26,27,44,31,32,47,33,48,54,28,29,45,30,46,51,34,49,53,52};
static const unsigned char T_FZ[35] = {15,16,17,18,40,25,26,27,44,28,29,45,30,46,51,19,20,21,41,22,23,42,24,43,55,31,32,47,34,49,52,33,48,54,53};
static const int BIN7[49] = {1,0,0,0,0,0,0, 1,1,0,0,0,0,0, 1,2,1,0,0,0,0, 1,3,3,1,0,0,0, 1,4,6,4,1,0,0, 1,5,10,10,5,1,0, 1,6,15,20,15,6,1};

// Separable binomial shift along one axis on the 56-entry moment store
// (first n entries; n = 35: order <= 4, 56: order <= 5):
// A_ijk <- sum_{a<=i} C(i,a) sh^(i-a) A_ajk (x shown); raw <-> central
// conversions are three passes, one per axis.
template <class T> void shift_axis(T* A, int n, int axis, T sh) {
  T pw[6];
  pw[0] = T(1);
  for (int q = 1; q < 6; ++q) pw[q] = pw[q - 1] * sh;
  const unsigned char* L = (n == 35) ? (axis == 0 ? T_L35X : axis == 1 ? T_L35Y : T_L35Z) : (axis == 0 ? T_L56X : axis == 1 ? T_L56Y : T_L56Z);
  const int stride = axis == 0 ? 36 : axis == 1 ? 6 : 1;
  for (int t = 0; t < n; ++t) {
    const int q = L[t];
    const int e = axis == 0 ? T_EX56I[q] : axis == 1 ? T_EX56J[q] : T_EX56K[q];
    if (e == 0) continue;
    const int base = T_EX56I[q] * 36 + T_EX56J[q] * 6 + T_EX56K[q] - e * stride;
    T acc = T(0);
    for (int a = 0; a <= e; ++a) acc = acc + (T(double(BIN7[e * 7 + a])) * pw[e - a]) * A[T_IDX56[base + a * stride]];
    A[q] = acc;
  }
}

// Central moments (35-order, C000=1, first order 0) of raw M
// (M4toC4_3D, src/autogen/M4toC4_3D.jl:42-55).
template <class T> void raw_to_central35(const T* M, T* C) {
  T inv = T(1) / M[0];
  T u = M[1] * inv, v = M[5] * inv, w = M[15] * inv;
  for (int n = 0; n < 35; ++n) C[n] = M[n] * inv;
  shift_axis(C, 35, 0, T(-u));
  shift_axis(C, 35, 1, T(-v));
  shift_axis(C, 35, 2, T(-w));
  C[0] = T(1); C[1] = T(0); C[5] = T(0); C[15] = T(0);
}

// Raw moments from density, mean and central moments, in place on the
// store A (n = 35 or 56; A[0] = 1, first order 0)
// (C4toM4_3D / C5toM5_3D, src/autogen/C4toM4_3D.jl:64-118, C5toM5_3D.jl:16-28).
template <class T> void central_to_raw(T M000, T u, T v, T w, T* A, int n) {
  shift_axis(A, n, 0, u);
  shift_axis(A, n, 1, v);
  shift_axis(A, n, 2, w);
  for (int q = 0; q < n; ++q) A[q] = M000 * A[q];
}

// ------------------------------------------------------------ small dense LA
// det() with Julia semantics (LinearAlgebra det -> istriu/istril shortcut,
// else LU with partial pivoting, row scaling by the reciprocal pivot).
template <class T, int N> T det_lu(const T (&Ain)[N][N]) {
  T A[N][N];
  bool triu = true, tril = true;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      A[i][j] = Ain[i][j];
      if (i > j && !(Ain[i][j] == T(0))) triu = false;
      if (i < j && !(Ain[i][j] == T(0))) tril = false;
    }
  if (triu || tril) {
    T p = T(1);
    for (int i = 0; i < N; ++i) p = p * A[i][i];
    return p;
  }
  int swaps = 0;
  bool singular = false;
  for (int k = 0; k < N; ++k) {
    int p = k;
    using std::fabs;
    T amax = fabs(A[k][k]);
    for (int i = k + 1; i < N; ++i)
      if (fabs(A[i][k]) > amax) { amax = fabs(A[i][k]); p = i; }
    if (p != k) {
      for (int j = 0; j < N; ++j) std::swap(A[k][j], A[p][j]);
      ++swaps;
    }
    if (A[k][k] == T(0)) { singular = true; continue; }
    T r = T(1) / A[k][k];
    for (int i = k + 1; i < N; ++i) A[i][k] = A[i][k] * r;
    for (int i = k + 1; i < N; ++i)
      for (int j = k + 1; j < N; ++j) A[i][j] = A[i][j] - A[i][k] * A[k][j];
  }
  if (singular) return T(0);  // issuccess(F) == false -> zero(T)
  T P = T(1);
  for (int i = 0; i < N; ++i) P = P * A[i][i];
  return (swaps & 1) ? -P : P;
}

// Solve A x = b, LU with partial pivoting (Julia `\` on a square Matrix).
template <class T, int N> void solve_lu(const T (&Ain)[N][N], const T (&b)[N], T (&x)[N]) {
  T A[N][N];
  for (int i = 0; i < N; ++i) { x[i] = b[i]; for (int j = 0; j < N; ++j) A[i][j] = Ain[i][j]; }
  for (int k = 0; k < N; ++k) {
    int p = k;
    using std::fabs;
    for (int i = k + 1; i < N; ++i) if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
    if (p != k) { for (int j = 0; j < N; ++j) std::swap(A[k][j], A[p][j]); std::swap(x[k], x[p]); }
    T r = T(1) / A[k][k];
    for (int i = k + 1; i < N; ++i) {
      A[i][k] = A[i][k] * r;
      for (int j = k + 1; j < N; ++j) A[i][j] = A[i][j] - A[i][k] * A[k][j];
      x[i] = x[i] - A[i][k] * x[k];
    }
  }
  for (int k = N - 1; k >= 0; --k) {
    T s = x[k];
    for (int j = k + 1; j < N; ++j) s = s - A[k][j] * x[j];
    x[k] = s / A[k][k];
  }
}

// ------------------------------------------------ raw <-> central moments
// M4toC4_3D (src/autogen/M4toC4_3D.jl:42-55): central moments of order <= 4
// as a 6x6x6 cube.
template <class T> void m4_to_c4(const T* M, T* C /*216 cube*/) {
  T C35[35];
  raw_to_central35(M, C35);
  for (int i = 0; i < 216; ++i) C[i] = T(0);
  for (int n = 0; n < 35; ++n) C[t3(E35[n][0], E35[n][1], E35[n][2])] = C35[n];
}

// C4toM4_3D / C5toM5_3D on 6x6x6 cubes (C000=1, first order zero), for all
// i+j+k <= order (4 or 5), through the 56-entry store.
template <class T> void c_to_m(T M000, T u, T v, T w, const T* C /*216*/, T* Mout /*216*/, int order) {
  const int n = order == 4 ? 35 : 56;
  T A[56];
  for (int q = 0; q < n; ++q) A[q] = C[t3(T_EX56I[q], T_EX56J[q], T_EX56K[q])];
  A[0] = T(1); A[1] = T(0); A[5] = T(0); A[15] = T(0);
  central_to_raw(M000, u, v, w, A, n);
  for (int i = 0; i < 216; ++i) Mout[i] = T(0);
  for (int q = 0; q < n; ++q) Mout[t3(T_EX56I[q], T_EX56J[q], T_EX56K[q])] = A[q];
}

// Symmetric 3x3 principal square root (Julia sqrt(::Matrix) on symmetric
// input -> Hermitian eigen path; eigenvalues slightly below zero within
// eps*n*max|lambda| are clamped to zero).  Jacobi rotations.
template <class T> void sym3_sqrt(const T (&A)[3][3], T (&R)[3][3]) {
  T a[3][3], V[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { a[i][j] = A[i][j]; V[i][j] = T(i == j ? 1 : 0); }
  using std::fabs; using std::sqrt;
  for (int sweep = 0; sweep < 50; ++sweep) {
    T off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
    if (off == T(0)) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == T(0)) continue;
        T theta = (a[q][q] - a[p][p]) / (T(2) * a[p][q]);
        T t = jsign(theta) / (fabs(theta) + sqrt(theta * theta + T(1)));
        if (theta == T(0)) t = T(1);
        T c = T(1) / sqrt(t * t + T(1)), s = t * c;
        for (int k = 0; k < 3; ++k) {
          T akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq; a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          T apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk; a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          T vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq; V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  T lam[3];
  T lmax = T(0);
  for (int i = 0; i < 3; ++i) { lam[i] = a[i][i]; lmax = jmax(lmax, T(fabs(lam[i]))); }
  for (int i = 0; i < 3; ++i) lam[i] = lam[i] >= -T(3 * EPS) * lmax ? sqrt(jmax(T(0), lam[i])) : T(0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T s = T(0);
      for (int k = 0; k < 3; ++k) s = s + V[i][k] * lam[k] * V[j][k];
      R[i][j] = s;
    }
}

// S4toC4_3D_r (src/autogen/S4toC4_3D_r.jl:19-80): central moments of X = A Z
// where A = sqrt(C2) and Z has the given standardized moments of order 3-4
// (first order 0, second order identity).  Diagonal covariance keeps the
// product order of the reference's expansion (A_ii^2 squared).
template <class T> void s4_to_c4_r(T C200, T C110, T C101, T C020, T C011, T C002, const T* Scube /*216*/, T* Ccube) {
  for (int i = 0; i < 216; ++i) Ccube[i] = T(0);
  if (C110 == T(0) && C101 == T(0) && C011 == T(0)) {
    using std::sqrt;
    // Hermitian eigen path of a diagonal matrix is exact: A = diag(sqrt(Cii)).
    T a1 = sqrt(C200), a2 = sqrt(C020), a3 = sqrt(C002);
    T p1[5], p2[5], p3[5];
    p1[0] = p2[0] = p3[0] = T(1);
    p1[1] = a1; p2[1] = a2; p3[1] = a3;
    p1[2] = a1 * a1; p2[2] = a2 * a2; p3[2] = a3 * a3;
    p1[3] = a1 * a1 * a1; p2[3] = a2 * a2 * a2; p3[3] = a3 * a3 * a3;
    p1[4] = p1[2] * p1[2]; p2[4] = p2[2] * p2[2]; p3[4] = p3[2] * p3[2];
    for (int n = 0; n < 35; ++n) {
      int i = E35[n][0], j = E35[n][1], k = E35[n][2];
      int ord = i + j + k;
      T s;
      if (ord == 0) s = T(1);
      else if (ord == 1) s = T(0);
      else if (ord == 2) s = (i == 2 || j == 2 || k == 2) ? T(1) : T(0);
      else s = Scube[t3(i, j, k)];
      Ccube[t3(i, j, k)] = s * p1[i] * p2[j] * p3[k];
    }
    Ccube[t3(1, 1, 0)] = T(0); Ccube[t3(1, 0, 1)] = T(0); Ccube[t3(0, 1, 1)] = T(0);
    return;
  }
  T C2[3][3] = {{C200, C110, C101}, {C110, C020, C011}, {C101, C011, C002}};
  T A[3][3];
  sym3_sqrt(C2, A);
  // full standardized tensor of Z up to order 4
  T Sz[216];
  for (int i = 0; i < 216; ++i) Sz[i] = Scube[i];
  Sz[t3(0, 0, 0)] = T(1);
  Sz[t3(1, 0, 0)] = Sz[t3(0, 1, 0)] = Sz[t3(0, 0, 1)] = T(0);
  Sz[t3(2, 0, 0)] = Sz[t3(0, 2, 0)] = Sz[t3(0, 0, 2)] = T(1);
  Sz[t3(1, 1, 0)] = Sz[t3(1, 0, 1)] = Sz[t3(0, 1, 1)] = T(0);
  // E[prod_r X_r^{n_r}] with X = A Z: expand each X_r as sum_s A_rs Z_s.
  for (int n = 0; n < 35; ++n) {
    int e[3] = {E35[n][0], E35[n][1], E35[n][2]};
    int ord = e[0] + e[1] + e[2];
    int rows[4], m = 0;
    for (int r = 0; r < 3; ++r) for (int q = 0; q < e[r]; ++q) rows[m++] = r;
    T s = T(0);
    int tot = 1;
    for (int q = 0; q < ord; ++q) tot *= 3;
    for (int code = 0; code < tot; ++code) {
      int c = code, cnt[3] = {0, 0, 0};
      T coef = T(1);
      for (int q = 0; q < ord; ++q) { int col = c % 3; c /= 3; cnt[col]++; coef = coef * A[rows[q]][col]; }
      s = s + coef * Sz[t3(cnt[0], cnt[1], cnt[2])];
    }
    Ccube[t3(e[0], e[1], e[2])] = ord == 0 ? T(1) : s;
  }
}

// InitializeM4_35 (src/moments/InitializeM4_35.jl:204-266).
template <class T> void initialize_m4_35(T M000, T u, T v, T w, T C200, T C110, T C101, T C020, T C011, T C002, T* M) {
  T S[216];
  for (int i = 0; i < 216; ++i) S[i] = T(0);
  S[t3(4, 0, 0)] = S[t3(0, 4, 0)] = S[t3(0, 0, 4)] = T(3);
  S[t3(2, 2, 0)] = S[t3(2, 0, 2)] = S[t3(0, 2, 2)] = T(1);
  T C[216], Mc[216];
  s4_to_c4_r(C200, C110, C101, C020, C011, C002, S, C);
  c_to_m(M000, u, v, w, C, Mc, 4);
  for (int n = 0; n < 35; ++n) M[n] = Mc[t3(E35[n][0], E35[n][1], E35[n][2])];
}

// M2CS4_35 (src/moments/M2CS4_35.jl:15-98): central C4 and standardized S4.
template <class T> void m2cs4_35(const T* M, T* C4, T* S4) {
  T C[216];
  m4_to_c4(M, C);
  using std::sqrt;
  T s1 = sqrt(jmax(C[t3(2, 0, 0)], T(EPS)));
  T s2 = sqrt(jmax(C[t3(0, 2, 0)], T(EPS)));
  T s3 = sqrt(jmax(C[t3(0, 0, 2)], T(EPS)));
  for (int n = 0; n < 35; ++n) {
    int i = E35[n][0], j = E35[n][1], k = E35[n][2];
    T c = C[t3(i, j, k)];
    C4[n] = c;
    int ord = i + j + k;
    if (ord == 0 || (ord == 2 && (i == 2 || j == 2 || k == 2))) { S4[n] = T(1); continue; }
    if (ord == 1) { S4[n] = T(0); continue; }
    // denominator sC200^i * sC020^j * sC002^k (Julia literal powers)
    T d = T(1);
    bool first = true;
    T f[3] = {s1, s2, s3};
    int ex[3] = {i, j, k};
    for (int r = 0; r < 3; ++r) {
      if (ex[r] == 0) continue;
      T p = ex[r] == 4 ? pow4(f[r]) : ipow(f[r], ex[r]);
      d = first ? p : d * p;
      first = false;
    }
    S4[n] = c / d;
  }
}

// ------------------------------------------------------------ univariate
// enforce_univariate (src/moments/enforce_univariate.jl:19-39).
template <class T> void enforce_univariate(T& S3, T& S4, T h2min, T s3max, T& H) {
  H = S4 - S3 * S3 - T(1);
  if (H <= h2min) { H = h2min; S4 = H + S3 * S3 + T(1); }
  if (S3 < -s3max) { S3 = -s3max; S4 = H + S3 * S3 + T(1); }
  else if (S3 > s3max) { S3 = s3max; S4 = H + S3 * S3 + T(1); }
}

// realizablity_S220 (src/realizability/realizablity_S220.jl:19-31).
template <class T> T realizablity_S220(T S110, T S220, T A220) {
  T S220r = S220;
  T mn = jmax(S110 * S110, T(1) - A220);
  T mx = T(1) + A220;
  if (S220 < mn) S220r = mn;
  else if (S220 > mx) S220r = mx;
  return S220r;
}

// realizability_S2 + bisection (src/realizability/realizability_S2.jl:18-66).
template <class T> void realizability_S2(T S110, T S101, T S011, T& o110, T& o101, T& o011, T& S2r) {
  T S2 = T(1) + T(2) * S110 * S101 * S011 - (S110 * S110 + S101 * S101 + S011 * S011);
  T xr = T(1);
  if (S2 < T(0)) {
    auto Y = [&](T x) {
      return T(1) + T(2) * S110 * S101 * S011 * (x * x * x) - (S110 * S110 + S101 * S101 + S011 * S011) * (x * x);
    };
    T a = T(0), b = T(1);
    T fa = Y(a);
    bool done = false;
    using std::fabs;
    for (int it = 0; it < 100; ++it) {
      T c = (a + b) / T(2);
      T fc = Y(c);
      if (fabs(fc) < T(1e-12) || (b - a) / T(2) < T(1e-12)) { xr = c; done = true; break; }
      if (jsign(fc) == jsign(fa)) { a = c; fa = fc; } else { b = c; }
    }
    if (!done) xr = (a + b) / T(2);
  }
  xr = T(0.9999) * xr;
  o110 = xr * S110; o101 = xr * S101; o011 = xr * S011;
  S2r = T(1) + T(2) * o110 * o101 * o011 - (o110 * o110 + o101 * o101 + o011 * o011);
}

// 2x2 symmetric principal square root via the closed-form eigen
// decomposition (Julia sqrt(::Matrix) Hermitian path).
template <class T> void sym2_sqrt(T a, T b, T d, T (&U)[2][2]) {
  using std::sqrt; using std::fabs;
  T tr = (a + d) / T(2), df = (a - d) / T(2);
  T r = sqrt(df * df + b * b);
  T l1 = tr + r, l2 = tr - r;
  T lmax = jmax(T(fabs(l1)), T(fabs(l2)));
  T tol = -T(2 * EPS) * lmax;
  T s1 = l1 >= tol ? sqrt(jmax(T(0), l1)) : T(0);
  T s2 = l2 >= tol ? sqrt(jmax(T(0), l2)) : T(0);
  if (b == T(0)) {
    U[0][0] = sqrt(jmax(T(0), a)); U[1][1] = sqrt(jmax(T(0), d)); U[0][1] = U[1][0] = T(0);
    return;
  }
  // eigenvector of l1: (b, l1 - a) normalized
  T vx = b, vy = l1 - a;
  T nv = sqrt(vx * vx + vy * vy);
  if (nv == T(0)) { vx = l1 - d; vy = b; nv = sqrt(vx * vx + vy * vy); }
  vx = vx / nv; vy = vy / nv;
  // U = s1 v v^T + s2 w w^T, w = (-vy, vx)
  U[0][0] = s1 * vx * vx + s2 * vy * vy;
  U[0][1] = s1 * vx * vy - s2 * vx * vy;
  U[1][0] = U[0][1];
  U[1][1] = s1 * vy * vy + s2 * vx * vx;
}

// realizability_S210 (src/realizability/realizability_S210.jl:86-110).
template <class T> void realizability_S210(T S110, T S101, T S011, T S300, T S210, T S201, T H200, T beta, T& o210, T& o201) {
  T xr = T(1);
  T X[2] = {S210 - S110 * S300, S201 - S101 * S300};
  T D1[2][2] = {{T(1) - S101 * S101, S101 * S110 - S011}, {S101 * S110 - S011, T(1) - S110 * S110}};
  T U[2][2];
  sym2_sqrt(D1[0][0], D1[0][1], D1[1][1], U);
  T V[2] = {U[0][0] * X[0] + U[0][1] * X[1], U[1][0] * X[0] + U[1][1] * X[1]};
  T L = jmax(T(0), V[0] * V[0] + V[1] * V[1]);
  T dD1 = jmax(T(0), det_lu<T, 2>(D1));
  T R = H200 * dD1;
  if (R <= T(0) || X[0] * X[0] + X[1] * X[1] < T(1000 * EPS)) xr = T(0);
  else if (L > R) { using std::sqrt; xr = sqrt(R / L); }
  T Vr[2] = {beta * xr * V[0], beta * xr * V[1]};
  T Xr[2];
  solve_lu<T, 2>(U, Vr, Xr);
  o210 = Xr[0] + S110 * S300;
  o201 = Xr[1] + S101 * S300;
}

// realizability_S111 (src/realizability/realizability_S111.jl:128-146).
template <class T> T realizability_S111(T S110, T S101, T S011, T S210, T S201, T S120, T S021, T S102, T S012, T S111) {
  T S111r = S111;
  T A110 = ((S101 - S011 * S110) * S210 + (S011 - S101 * S110) * S120) / (T(1) - S110 * S110);
  T A101 = ((S110 - S011 * S101) * S201 + (S011 - S110 * S101) * S102) / (T(1) - S101 * S101);
  T A011 = ((S110 - S101 * S011) * S021 + (S101 - S110 * S011) * S012) / (T(1) - S011 * S011);
  T Rmin = jmin(jmin(A110, A101), A011);
  T Rmax = jmax(jmax(A110, A101), A011);
  if (S111 > Rmax) S111r = Rmax;
  else if (S111 < Rmin) S111r = Rmin;
  return S111r;
}

// realizability_S211 (src/realizability/realizability_S211.jl:165-180).
template <class T> T realizability_S211(T e11, T e22, T e33, T e12, T e13, T d23, T S211, T beta) {
  T S211r = S211;
  T b211 = e12 * e13;
  T G211 = jmax(T(0), (e11 * e22 - e13 * e13) * (e11 * e33 - e12 * e12));
  T sG = beta * fm_sqrt(G211);
  T mn = d23 + (b211 - sG) / e11;
  T mx = d23 + (b211 + sG) / e11;
  if (S211 <= mn) S211r = mn;
  else if (S211 >= mx) S211r = mx;
  return S211r;
}

// realizability_S310 (src/realizability/realizability_S310.jl:200-249).
template <class T> void realizability_S310(T S110, T S101, T S011, T S300, T S210, T S201, T S120, T S111, T S310, T S220,
                                           T H200, T beta, T& o310, T& o220) {
  T S310r = S310;
  T b310 = S111 * ((T(1) - S110 * S110) * S201 + (S101 * S110 - S011) * S210 + (S011 * S110 - S101) * S300) +
           S120 * ((T(1) - S101 * S101) * S210 + (S011 * S101 - S110) * S300 + (S101 * S110 - S011) * S201) +
           S210 * ((T(1) - S011 * S011) * S300 + (S011 * S101 - S110) * S210 + (S011 * S110 - S101) * S201);
  T D1[2][2] = {{T(1) - S101 * S101, S101 * S110 - S011}, {S101 * S110 - S011, T(1) - S110 * S110}};
  T dD1 = det_lu<T, 2>(D1);
  T V1[2] = {S210 - S110 * S300, S201 - S101 * S300};
  T D1V1[2] = {D1[0][0] * V1[0] + D1[0][1] * V1[1], D1[1][0] * V1[0] + D1[1][1] * V1[1]};
  T L1 = (V1[0] * D1V1[0] + V1[1] * D1V1[1]) / dD1;
  T G310b = H200 - L1;
  if (G310b < T(0)) G310b = T(0);
  T D2[3][3] = {{T(1) - S011 * S011, S011 * S101 - S110, S011 * S110 - S101},
                {S011 * S101 - S110, T(1) - S101 * S101, S101 * S110 - S011},
                {S011 * S110 - S101, S101 * S110 - S011, T(1) - S110 * S110}};
  T V2[3] = {S210, S120, S111};
  T q = T(0);
  for (int i = 0; i < 3; ++i) {
    T r = D2[i][0] * V2[0] + D2[i][1] * V2[1] + D2[i][2] * V2[2];
    q = q + V2[i] * r;
  }
  T L2 = q / dD1;
  T G310a = S220 - S110 * S110 - L2 + T(1000 * EPS);
  if (G310a < T(0) || L2 < T(0)) G310a = T(0);
  T G310 = G310a * G310b;
  T sG = beta * fm_sqrt(G310);
  T mn = S110 + b310 / dD1 - sG;
  T mx = S110 + b310 / dD1 + sG;
  if (S310 <= mn) S310r = mn;
  else if (S310 >= mx) S310r = mx;
  o310 = S310r;
  o220 = S220;
}

// realizability_S310_220 (src/realizability/realizability_S310_220.jl:267-286).
template <class T> T realizability_S310_220(T S110, T S101, T S011, T S210, T S120, T S111, T S220) {
  T S220r = S220;
  T D1[2][2] = {{T(1) - S101 * S101, S101 * S110 - S011}, {S101 * S110 - S011, T(1) - S110 * S110}};
  T dD1 = det_lu<T, 2>(D1);
  T D2[3][3] = {{T(1) - S011 * S011, S011 * S101 - S110, S011 * S110 - S101},
                {S011 * S101 - S110, T(1) - S101 * S101, S101 * S110 - S011},
                {S011 * S110 - S101, S101 * S110 - S011, T(1) - S110 * S110}};
  T V2[3] = {S210, S120, S111};
  T q = T(0);
  for (int i = 0; i < 3; ++i) {
    T r = D2[i][0] * V2[0] + D2[i][1] * V2[1] + D2[i][2] * V2[2];
    q = q + V2[i] * r;
  }
  T L2 = q / dD1;
  T mn = S110 * S110 + L2 + T(1000 * EPS);
  if (mn > S220r) S220r = mn;
  return S220r;
}

// ---------------------------------------------------- Delta2* and bounds
// Standardized moments of one coordinate permutation, named as the
// reference's 28-argument lists (s300 ... s022).
template <class T> struct S28 {
  T s300, s400, s110, s210, s310, s120, s220, s030, s130, s040, s101, s201, s301, s102, s202, s003, s103, s004, s011,
      s111, s211, s021, s121, s031, s012, s112, s013, s022;
};

// Standardized moment lookup with second-order diagonal = 1.
template <class T> inline T sget(const S28<T>& s, int i, int j, int k) {
  int key = 100 * i + 10 * j + k;
  switch (key) {
    case 0: return T(1);
    case 100: case 10: case 1: return T(0);
    case 200: case 20: case 2: return T(1);
    case 110: return s.s110; case 101: return s.s101; case 11: return s.s011;
    case 300: return s.s300; case 210: return s.s210; case 201: return s.s201; case 120: return s.s120;
    case 111: return s.s111; case 102: return s.s102; case 30: return s.s030; case 21: return s.s021;
    case 12: return s.s012; case 3: return s.s003;
    case 400: return s.s400; case 310: return s.s310; case 301: return s.s301; case 220: return s.s220;
    case 211: return s.s211; case 202: return s.s202; case 130: return s.s130; case 121: return s.s121;
    case 112: return s.s112; case 103: return s.s103; case 40: return s.s040; case 31: return s.s031;
    case 22: return s.s022; case 13: return s.s013; case 4: return s.s004;
  }
  return T(0);
}

static const int B1[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
static const int B2[6][3] = {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}};

// Q = M21 M11^{-1} M12 (6x6 symmetric), the projection part of the Schur
// complement.  M11 = 1 (+) R with R the correlation matrix; R^{-1} by
// cofactors; Q(a,b) = mu_a mu_b + w_a . R^{-1} w_b for a <= b, mirrored.
template <class T> void delta_projection(const S28<T>& s, T (&Q)[6][6]) {
  const T c00 = T(1) - s.s011 * s.s011, c01 = s.s101 * s.s011 - s.s110, c02 = s.s110 * s.s011 - s.s101;
  const T c11 = T(1) - s.s101 * s.s101, c12 = s.s110 * s.s101 - s.s011, c22 = T(1) - s.s110 * s.s110;
  const T det = c00 + s.s110 * c01 + s.s101 * c02;
  const T id = T(1) / det;
  const T r00 = c00 * id, r01 = c01 * id, r02 = c02 * id, r11 = c11 * id, r12 = c12 * id, r22 = c22 * id;
  const T mu[6] = {T(1), s.s110, s.s101, T(1), s.s011, T(1)};
  const T w[6][3] = {{s.s300, s.s210, s.s201}, {s.s210, s.s120, s.s111}, {s.s201, s.s111, s.s102},
                     {s.s120, s.s030, s.s021}, {s.s111, s.s021, s.s012}, {s.s102, s.s012, s.s003}};
  T z[6][3];
  for (int a = 0; a < 6; ++a) {
    z[a][0] = r00 * w[a][0] + r01 * w[a][1] + r02 * w[a][2];
    z[a][1] = r01 * w[a][0] + r11 * w[a][1] + r12 * w[a][2];
    z[a][2] = r02 * w[a][0] + r12 * w[a][1] + r22 * w[a][2];
  }
  for (int a = 0; a < 6; ++a)
    for (int b = a; b < 6; ++b) {
      const T qv = mu[a] * mu[b] + (w[a][0] * z[b][0] + w[a][1] * z[b][1] + w[a][2] * z[b][2]);
      Q[a][b] = qv;
      Q[b][a] = qv;
    }
}

// delta2star3D (src/autogen/delta2star3D.jl:11-296).
template <class T> void delta2star3D(const S28<T>& s, T (&E)[6][6]) {
  T Q[6][6];
  delta_projection(s, Q);
  for (int a = 0; a < 6; ++a)
    for (int b = a; b < 6; ++b) {
      const T e = sget(s, B2[a][0] + B2[b][0], B2[a][1] + B2[b][1], B2[a][2] + B2[b][2]) - Q[a][b];
      E[a][b] = e;
      E[b][a] = e;
    }
}

// lower_bound_S220 (src/autogen/lower_bound_S220.jl:14-37): {Q(xy,xy), Q(xz,xz), Q(yz,yz)}.
template <class T> void lower_bound_S220(const S28<T>& s, T (&out)[3]) {
  T Q[6][6];
  delta_projection(s, Q);
  out[0] = Q[1][1]; out[1] = Q[2][2]; out[2] = Q[4][4];
}

// bound_minor1 (src/autogen/bound_minor1.jl:14-60).
template <class T> void bound_minor1(const S28<T>& s, T (&out)[12]) {
  T Q[6][6];
  delta_projection(s, Q);
  // x2=0 xy=1 xz=2 y2=3 yz=4 z2=5
  out[0] = Q[0][1]; out[1] = Q[0][2]; out[2] = Q[1][3]; out[3] = Q[2][5]; out[4] = Q[3][4]; out[5] = Q[4][5];
  out[6] = Q[0][3]; out[7] = Q[0][5]; out[8] = Q[3][5]; out[9] = Q[0][4]; out[10] = Q[2][3]; out[11] = Q[1][5];
}

// ------------------------------------------------------------ 2-D pieces
// 2-D Delta2* (basis {1,x,y} | {x2,xy,y2}) as a 3x3 matrix; M11 =
// [1 0 0; 0 1 s11; 0 s11 1] inverted in closed form.
template <class T> void delta2star2D(T s30, T s40, T s11, T s21, T s31, T s12, T s22, T s03, T s13, T s04, T (&D)[3][3]) {
  const T dt = T(1) - s11 * s11;
  const T i00 = T(1) / dt, i01 = -s11 / dt;
  const T mu[3] = {T(1), s11, T(1)};
  const T w[3][2] = {{s30, s21}, {s21, s12}, {s12, s03}};
  const T m22[3][3] = {{s40, s31, s22}, {s31, s22, s13}, {s22, s13, s04}};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const T z0 = i00 * w[b][0] + i01 * w[b][1], z1 = i01 * w[b][0] + i00 * w[b][1];
      D[a][b] = m22[a][b] - (mu[a] * mu[b] + (w[a][0] * z0 + w[a][1] * z1));
    }
}

template <class T> T det3(const T (&D)[3][3]) {
  return D[0][0] * (D[1][1] * D[2][2] - D[1][2] * D[2][1]) - D[0][1] * (D[1][0] * D[2][2] - D[1][2] * D[2][0]) +
         D[0][2] * (D[1][0] * D[2][1] - D[1][1] * D[2][0]);
}

// delta2starchol_L3 (src/autogen/delta2starchol_L3.jl:6-37).
template <class T> T delta2starchol_L3(T s03, T s04, T s11, T s12, T s13, T s21, T s22, T s30, T s31, T s40) {
  T D[3][3];
  delta2star2D(s30, s40, s11, s21, s31, s12, s22, s03, s13, s04, D);
  return (T(1) - s11 * s11) * det3(D);
}

// Polynomial (degree <= 3) helpers for determinant cubics.
template <class T> struct P3 { T c[4]; };
template <class T> P3<T> pmul(const P3<T>& a, const P3<T>& b) {
  P3<T> r; for (int i = 0; i < 4; ++i) r.c[i] = T(0);
  for (int i = 0; i < 4; ++i) for (int j = 0; i + j < 4; ++j) r.c[i + j] = r.c[i + j] + a.c[i] * b.c[j];
  return r;
}
template <class T> P3<T> padd(const P3<T>& a, const P3<T>& b, T sb) {
  P3<T> r; for (int i = 0; i < 4; ++i) r.c[i] = a.c[i] + sb * b.c[i];
  return r;
}
template <class T> P3<T> pconst(T v, T lin = T(0)) { P3<T> r; r.c[0] = v; r.c[1] = lin; r.c[2] = r.c[3] = T(0); return r; }

// Determinant of an NxN matrix of linear polynomials (Laplace expansion).
template <class T> P3<T> pdet3(const P3<T> (&A)[3][3]) {
  P3<T> t0 = padd(pmul(A[1][1], A[2][2]), pmul(A[1][2], A[2][1]), T(-1));
  P3<T> t1 = padd(pmul(A[1][0], A[2][2]), pmul(A[1][2], A[2][0]), T(-1));
  P3<T> t2 = padd(pmul(A[1][0], A[2][1]), pmul(A[1][1], A[2][0]), T(-1));
  P3<T> r = pmul(A[0][0], t0);
  r = padd(r, pmul(A[0][1], t1), T(-1));
  r = padd(r, pmul(A[0][2], t2), T(1));
  return r;
}
template <class T> P3<T> pdet4(const P3<T> (&A)[4][4]) {
  P3<T> r = pconst(T(0));
  for (int c = 0; c < 4; ++c) {
    P3<T> sub[3][3];
    for (int i = 1; i < 4; ++i) { int cc = 0; for (int j = 0; j < 4; ++j) if (j != c) sub[i - 1][cc++] = A[i][j]; }
    P3<T> d = pdet3(sub);
    r = padd(r, pmul(A[0][c], d), (c & 1) ? T(-1) : T(1));
  }
  return r;
}

// Cardano roots of c3 X^3 + c2 X^2 + c1 X + c0 in the reference's form:
// shift + C + p/C and shift - (C + p/C)/2 +- i sqrt(3)/2 (C - p/C), with the
// real (fast-math) square root of q^2 - p^3, so three real roots give NaN.
// Returned as (re[3], im[3]).
template <class T> void cardano(const P3<T>& P, T (&re)[3], T (&im)[3]) {
  T a = P.c[3];
  T B = -P.c[2] / a, C = P.c[1] / a, D = -P.c[0] / a;  // X^3 - B X^2 + C X - D
  T p = B * B / T(9) - C / T(3);
  T q = B * B * B / T(27) - B * C / T(6) + D / T(2);
  T disc = q * q - p * p * p;
  T sd = fm_sqrt(disc);
  using std::sqrt;
  T Cc = hcbrtT(T(q + sd));
  T pc = p / Cc;
  T sh = B / T(3);
  T s3 = sqrt(T(3));
  re[0] = sh + Cc + pc; im[0] = T(0);
  re[1] = sh - Cc / T(2) - pc / T(2); im[1] = s3 * (Cc - pc) / T(2);
  re[2] = re[1]; im[2] = -im[1];
  if (sd != sd) { for (int i = 0; i < 3; ++i) { re[i] = sd; im[i] = (i == 0) ? T(0) : sd; } }
}

// rootsR (src/autogen/rootsR.jl:7-292): roots in S22 of det(2-D Delta2*(S22)).
// The Schur complement is affine in S22 with slope 1 at (x2,y2), (y2,x2),
// (xy,xy): det [a b c+X; b d+X e; c+X e f] expanded as a cubic in X.
template <class T> void rootsR(T Del1, T H02, T H20, T s03, T s11, T s12, T s13, T s21, T s30, T s31, T (&re)[3], T (&im)[3]) {
  (void)Del1;
  T s40 = H20 + s30 * s30 + T(1), s04 = H02 + s03 * s03 + T(1);
  T D0[3][3];
  delta2star2D(s30, s40, s11, s21, s31, s12, T(0), s03, s13, s04, D0);
  const T a = D0[0][0], b = D0[0][1], c = D0[0][2], d = D0[1][1], e = D0[1][2], f = D0[2][2];
  const T k0 = a * (d * f - e * e) - b * (b * f - e * c) + c * (b * e - d * c);
  const T k1 = a * f + b * e + (b * e - d * c) - c * (d + c);
  const T k2 = -(d + c) - c;
  P3<T> P;
  P.c[0] = k0; P.c[1] = k1; P.c[2] = k2; P.c[3] = T(-1);
  cardano(P, re, im);
  if (re[0] != re[0]) hit(BR_ROOTSR_NAN);
}

// rootsR_X_Y (src/autogen/rootsR_X_Y.jl:6-77): roots in X of
// det([e11 e12 e13 ex+X; e12 X e23 e24; e13 e23 Y e34; ex+X e24 e34 e44]).
template <class T> void rootsR_X_Y(T Y, T e11, T e12, T e13, T e23, T e24, T e34, T e44, T ex, T (&re)[3], T (&im)[3]) {
  P3<T> A[4][4] = {{pconst(e11), pconst(e12), pconst(e13), pconst(ex, T(1))},
                   {pconst(e12), pconst(T(0), T(1)), pconst(e23), pconst(e24)},
                   {pconst(e13), pconst(e23), pconst(Y), pconst(e34)},
                   {pconst(ex, T(1)), pconst(e24), pconst(e34), pconst(e44)}};
  P3<T> P = pdet4(A);
  cardano(P, re, im);
  if (re[0] != re[0]) hit(BR_ROOTSRXY_NAN);
}

// Julia `sort(real(R))` with NaN last, and the complex-root ratio test
// maximum(abs.(imag(R))) / maximum(abs.(R)).
template <class T> void sort3_nan_last(T (&r)[3]) {
  auto lt = [](T a, T b) { if (a != a) return false; if (b != b) return true; return a < b; };
  for (int i = 0; i < 3; ++i) for (int j = 0; j + 1 < 3 - i; ++j) if (lt(r[j + 1], r[j])) std::swap(r[j], r[j + 1]);
}
template <class T> T imag_ratio(const T (&re)[3], const T (&im)[3]) {
  using std::fabs; using std::sqrt;
  T mi = T(0), ma = T(0);
  for (int i = 0; i < 3; ++i) {
    T ai = fabs(im[i]);
    T ab = sqrt(re[i] * re[i] + im[i] * im[i]);
    mi = i == 0 ? ai : jmax(mi, ai);
    ma = i == 0 ? ab : jmax(ma, ab);
  }
  return mi / ma;
}

// realizable_2D (src/realizability/realizable_2D.jl:24-118).
template <class T> void realizable_2D(T S30, T S40, T S11, T& S21, T& S31, T& S12, T& S22, T S03, T& S13, T S04) {
  using std::sqrt;
  T Del1 = jmax(T(0), T(1) - S11 * S11);
  T H20 = jmax(T(EPS), S40 - S30 * S30 - T(1));
  T H02 = jmax(T(EPS), S04 - S03 * S03 - T(1));
  T G1 = sqrt(Del1 * H02);
  T s12min = S11 * S03 - G1, s12max = S11 * S03 + G1;
  if (S12 <= s12min) S12 = s12min; else if (S12 >= s12max) S12 = s12max;
  G1 = sqrt(Del1 * H20);
  T s21min = S11 * S30 - G1, s21max = S11 * S30 + G1;
  if (S21 <= s21min) S21 = s21min; else if (S21 >= s21max) S21 = s21max;
  T G22 = sqrt((H20 + S30 * S30) * (H02 + S03 * S03));
  T s22min = jmax(S11 * S11, T(1) - G22), s22max = T(1) + G22;
  if (S22 < s22min) S22 = s22min; else if (S22 > s22max) S22 = s22max;
  T common = Del1 * S22 - Del1 * S11 * S11 - S12 * S12 + T(2) * S11 * S12 * S21 - S21 * S21;
  T G31 = common * (Del1 * H20 - sq(S21 - S11 * S30));
  T G13 = common * (Del1 * H02 - sq(S12 - S11 * S03));
  if (G31 < T(0) || G13 < T(0)) { G31 = T(0); G13 = T(0); }
  else { G13 = sqrt(G13); G31 = sqrt(G31); }
  T den = Del1 + T(EPS);
  T b31 = S12 * S21 + S21 * S30 - S11 * S21 * S21 - S11 * S12 * S30;
  T s31min = S11 + (b31 - G31) / den, s31max = S11 + (b31 + G31) / den;
  if (S31 <= s31min) S31 = s31min; else if (S31 >= s31max) S31 = s31max;
  T b13 = S12 * S21 + S12 * S03 - S11 * S12 * S12 - S11 * S21 * S03;
  T s13min = S11 + (b13 - G13) / den, s13max = S11 + (b13 + G13) / den;
  if (S13 <= s13min) S13 = s13min; else if (S13 >= s13max) S13 = s13max;
  T L3 = delta2starchol_L3(S03, S04, S11, S12, S13, S21, S22, S30, S31, S40);
  if (L3 < T(0)) {
    T re[3], im[3];
    rootsR(Del1, H02, H20, S03, S11, S12, S13, S21, S30, S31, re, im);
    T Rr[3] = {re[0], re[1], re[2]};
    sort3_nan_last(Rr);
    T s22maxr = jmin(s22max, Rr[2]);
    T s22minr = jmax(s22min, Rr[1]);
    if (s22maxr < s22minr) s22minr = s22maxr;
    T S22a = S22;
    if (S22 > s22maxr) S22a = s22maxr;
    else if (S22 < s22minr) S22a = s22minr;
    if (imag_ratio(re, im) > T(1000 * EPS)) {
      // complex roots: S22 unchanged
    } else {
      S22 = S22a;
    }
  }
}

// check2D (src/utils/diagnostics.jl:128-153); returns the 10 moments in place.
template <class T> void check2D(T& S30, T& S40, T& S11, T& S21, T& S31, T& S12, T& S22, T& S03, T& S13, T& S04) {
  using std::fabs; using std::sqrt;
  T h2min = T(1000 * EPS);
  if (fabs(S11) >= T(1)) {
    S11 = jsign(S11);
    T s3m = sqrt(fabs(S30 * S03));
    T s4m = sqrt(S40 * S04);
    T H2m = jmax(h2min, s4m - s3m * s3m - T(1));
    s4m = H2m + s3m * s3m + T(1);
    S30 = jsign(S30) * s3m;
    S03 = S11 * S30;
    S40 = s4m; S04 = s4m;
    S12 = S11 * S03; S21 = S11 * S30; S13 = S11 * S04; S31 = S11 * S40; S22 = s4m;
  } else {
    realizable_2D(S30, S40, S11, S21, S31, S12, S22, S03, S13, S04);
  }
}

}  // namespace hyqo
