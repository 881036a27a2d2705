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
// from raw moments, by the binomial expansion about the mean.
template <class T> void m4_to_c4(const T* M, T* C /*216 cube*/) {
  T Mc[216];
  for (int i = 0; i < 216; ++i) { Mc[i] = T(0); C[i] = T(0); }
  for (int n = 0; n < 35; ++n) Mc[t3(E35[n][0], E35[n][1], E35[n][2])] = M[n];
  T inv = T(1) / M[0];
  T u = M[1] * inv, v = M[5] * inv, w = M[15] * inv;
  T pu[5], pv[5], pw[5];
  pu[0] = pv[0] = pw[0] = T(1);
  for (int i = 1; i < 5; ++i) { pu[i] = pu[i - 1] * (-u); pv[i] = pv[i - 1] * (-v); pw[i] = pw[i - 1] * (-w); }
  for (int n = 0; n < 35; ++n) {
    int i = E35[n][0], j = E35[n][1], k = E35[n][2];
    T s = T(0);
    for (int a = 0; a <= i; ++a)
      for (int b = 0; b <= j; ++b)
        for (int c = 0; c <= k; ++c) {
          T term = T(double(binom(i, a) * binom(j, b) * binom(k, c))) * (Mc[t3(a, b, c)] * inv) *
                   (pu[i - a] * pv[j - b] * pw[k - c]);
          s = s + term;
        }
    C[t3(i, j, k)] = s;
  }
  C[t3(0, 0, 0)] = T(1);
  C[t3(1, 0, 0)] = T(0);
  C[t3(0, 1, 0)] = T(0);
  C[t3(0, 0, 1)] = T(0);
}

// C4toM4_3D / C5toM5_3D (src/autogen/C4toM4_3D.jl:64-118,
// src/autogen/C5toM5_3D.jl:16-28): raw moments from density, mean velocity
// and central moments (C000=1, first order zero), for all i+j+k <= order.
template <class T> void c_to_m(T M000, T u, T v, T w, const T* C /*216*/, T* Mout /*216*/, int order) {
  T pu[6], pv[6], pw[6];
  pu[0] = pv[0] = pw[0] = T(1);
  for (int i = 1; i < 6; ++i) { pu[i] = pu[i - 1] * u; pv[i] = pv[i - 1] * v; pw[i] = pw[i - 1] * w; }
  for (int i = 0; i < 216; ++i) Mout[i] = T(0);
  for (int i = 0; i <= order; ++i)
    for (int j = 0; i + j <= order; ++j)
      for (int k = 0; i + j + k <= order; ++k) {
        T s = T(0);
        for (int a = 0; a <= i; ++a)
          for (int b = 0; b <= j; ++b)
            for (int c = 0; c <= k; ++c) {
              int ord = a + b + c;
              if (ord == 1) continue;
              T cm = ord == 0 ? T(1) : C[t3(a, b, c)];
              s = s + T(double(binom(i, a) * binom(j, b) * binom(k, c))) * cm * (pu[i - a] * pv[j - b] * pw[k - c]);
            }
        Mout[t3(i, j, k)] = M000 * s;
      }
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

// Q = M21 M11^{-1} M12 (6x6), the projection part of the Schur complement.
template <class T> void delta_projection(const S28<T>& s, T (&Q)[6][6]) {
  T M11[4][4], M12[4][6];
  for (int a = 0; a < 4; ++a) {
    for (int b = 0; b < 4; ++b)
      M11[a][b] = sget(s, B1[a][0] + B1[b][0], B1[a][1] + B1[b][1], B1[a][2] + B1[b][2]);
    for (int b = 0; b < 6; ++b)
      M12[a][b] = sget(s, B1[a][0] + B2[b][0], B1[a][1] + B2[b][1], B1[a][2] + B2[b][2]);
  }
  T X[4][6];
  for (int b = 0; b < 6; ++b) {
    T rhs[4] = {M12[0][b], M12[1][b], M12[2][b], M12[3][b]}, x[4];
    solve_lu<T, 4>(M11, rhs, x);
    for (int a = 0; a < 4; ++a) X[a][b] = x[a];
  }
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) {
      T q = T(0);
      for (int r = 0; r < 4; ++r) q = q + M12[r][a] * X[r][b];
      Q[a][b] = q;
    }
}

// delta2star3D (src/autogen/delta2star3D.jl:11-296).
template <class T> void delta2star3D(const S28<T>& s, T (&E)[6][6]) {
  T Q[6][6];
  delta_projection(s, Q);
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b)
      E[a][b] = sget(s, B2[a][0] + B2[b][0], B2[a][1] + B2[b][1], B2[a][2] + B2[b][2]) - Q[a][b];
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
// 2-D Delta2* (basis {1,x,y} | {x2,xy,y2}) as a 3x3 matrix.
template <class T> void delta2star2D(T s30, T s40, T s11, T s21, T s31, T s12, T s22, T s03, T s13, T s04, T (&D)[3][3]) {
  // standardized 2-D moments m(i,j)
  auto m = [&](int i, int j) -> T {
    int key = 10 * i + j;
    switch (key) {
      case 0: return T(1); case 10: case 1: return T(0); case 20: case 2: return T(1);
      case 11: return s11; case 30: return s30; case 21: return s21; case 12: return s12; case 3: return s03;
      case 40: return s40; case 31: return s31; case 22: return s22; case 13: return s13; case 4: return s04;
    }
    return T(0);
  };
  static const int b1[3][2] = {{0, 0}, {1, 0}, {0, 1}};
  static const int b2[3][2] = {{2, 0}, {1, 1}, {0, 2}};
  T A[3][3], Bm[3][3];
  for (int a = 0; a < 3; ++a) {
    for (int b = 0; b < 3; ++b) A[a][b] = m(b1[a][0] + b1[b][0], b1[a][1] + b1[b][1]);
    for (int b = 0; b < 3; ++b) Bm[a][b] = m(b1[a][0] + b2[b][0], b1[a][1] + b2[b][1]);
  }
  T X[3][3];
  for (int b = 0; b < 3; ++b) {
    T rhs[3] = {Bm[0][b], Bm[1][b], Bm[2][b]}, x[3];
    solve_lu<T, 3>(A, rhs, x);
    for (int a = 0; a < 3; ++a) X[a][b] = x[a];
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      T q = T(0);
      for (int r = 0; r < 3; ++r) q = q + Bm[r][a] * X[r][b];
      D[a][b] = m(b2[a][0] + b2[b][0], b2[a][1] + b2[b][1]) - q;
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
  using std::cbrt; using std::sqrt;
  T Cc = cbrt(q + sd);
  T pc = p / Cc;
  T sh = B / T(3);
  T s3 = sqrt(T(3));
  re[0] = sh + Cc + pc; im[0] = T(0);
  re[1] = sh - Cc / T(2) - pc / T(2); im[1] = s3 * (Cc - pc) / T(2);
  re[2] = re[1]; im[2] = -im[1];
  if (sd != sd) { for (int i = 0; i < 3; ++i) { re[i] = sd; im[i] = (i == 0) ? T(0) : sd; } }
}

// rootsR (src/autogen/rootsR.jl:7-292): roots in S22 of det(2-D Delta2*(S22)).
template <class T> void rootsR(T Del1, T H02, T H20, T s03, T s11, T s12, T s13, T s21, T s30, T s31, T (&re)[3], T (&im)[3]) {
  (void)Del1;
  T s40 = H20 + s30 * s30 + T(1), s04 = H02 + s03 * s03 + T(1);
  // entries of the 2-D Schur complement are affine in S22: evaluate at 0 and 1
  T D0[3][3], D1m[3][3];
  delta2star2D(s30, s40, s11, s21, s31, s12, T(0), s03, s13, s04, D0);
  delta2star2D(s30, s40, s11, s21, s31, s12, T(1), s03, s13, s04, D1m);
  P3<T> A[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = pconst(D0[i][j], D1m[i][j] - D0[i][j]);
  // exact affine structure: only (xy,xy) and (x2,y2) depend on S22 with slope 1
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j].c[1] = T(0);
  A[1][1].c[1] = T(1); A[0][2].c[1] = T(1); A[2][0].c[1] = T(1);
  P3<T> P = pdet3(A);
  cardano(P, re, im);
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
