// ORACLE (test infrastructure): flux-Jacobian eigenvalues, 1-D closure
// eigenvalues, BGK collision and HLL sweeps.  Restates the reference files
// cited per function; see hyq_oracle.hpp for the conventions.
// The eigenvalue routines in this file restate the steps of LAPACK's DGEBAL,
// DGEHD2, DLARFG, DLAHQR and DLANV2 (needed for branch-identical results with
// the reference's eigvals).  LAPACK is distributed under the following
// licence, reproduced as it requires:
//
//   Copyright (c) 1992-2013 The University of Tennessee and The University
//                           of Tennessee Research Foundation.  All rights
//                           reserved.
//   Copyright (c) 2000-2013 The University of California Berkeley.  All
//                           rights reserved.
//   Copyright (c) 2006-2013 The University of Colorado Denver.  All rights
//                           reserved.
//
//   Redistribution and use in source and binary forms, with or without
//   modification, are permitted provided that the following conditions are
//   met:
//   - Redistributions of source code must retain the above copyright
//     notice, this list of conditions and the following disclaimer.
//   - Redistributions in binary form must reproduce the above copyright
//     notice, this list of conditions and the following disclaimer listed
//     in this license in the documentation and/or other materials
//     provided with the distribution.
//   - Neither the name of the copyright holders nor the names of its
//     contributors may be used to endorse or promote products derived from
//     this software without specific prior written permission.
//
//   The copyright holders provide no reassurances that the source code
//   provided does not infringe any patent, copyright, or any other
//   intellectual property rights of third parties.  The copyright holders
//   disclaim any liability to any recipient for claims brought against
//   recipient by a third party for infringement of that parties
//   intellectual property rights.
//
//   THIS SOFTWARE IS PROVIDED BY THE COPYRIGHT HOLDERS AND CONTRIBUTORS
//   "AS IS" AND ANY EXPRESS OR IMPLIED WARRANTIES, INCLUDING, BUT NOT
//   LIMITED TO, THE IMPLIED WARRANTIES OF MERCHANTABILITY AND FITNESS FOR
//   A PARTICULAR PURPOSE ARE DISCLAIMED. IN NO EVENT SHALL THE COPYRIGHT
//   OWNER OR CONTRIBUTORS BE LIABLE FOR ANY DIRECT, INDIRECT, INCIDENTAL,
//   SPECIAL, EXEMPLARY, OR CONSEQUENTIAL DAMAGES (INCLUDING, BUT NOT
//   LIMITED TO, PROCUREMENT OF SUBSTITUTE GOODS OR SERVICES; LOSS OF USE,
//   DATA, OR PROFITS; OR BUSINESS INTERRUPTION) HOWEVER CAUSED AND ON ANY
//   THEORY OF LIABILITY, WHETHER IN CONTRACT, STRICT LIABILITY, OR TORT
//   (INCLUDING NEGLIGENCE OR OTHERWISE) ARISING IN ANY WAY OUT OF THE USE
//   OF THIS SOFTWARE, EVEN IF ADVISED OF THE POSSIBILITY OF SUCH DAMAGE.
//
#pragma once
#include "hyq_oracle_closure.hpp"

namespace hyqo {

// ------------------------------------------- jacobian6 by forward-mode AD
// jacobian6 (src/autogen/jacobian6.jl:14-59) is the Jacobian of the x-fluxes
// (m12, m22, m32, m13, m23, m14) of W = (m02, m12, m22, m03, m13, m04) for
// the 2-D HyQMOM closure of (m32, m23, m14); m_ab = E[x^a y^b], x the flux
// direction.  jacobian6_ad evaluates it with 6-component dual numbers and
// is kept as an independent check of the closed form below.
template <class T> struct D6 {
  T v, d[6];
  D6() {}
  explicit D6(T x) : v(x) { for (int i = 0; i < 6; ++i) d[i] = T(0); }
};
template <class T> D6<T> operator+(const D6<T>& a, const D6<T>& b) { D6<T> r; r.v = a.v + b.v; for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <class T> D6<T> operator-(const D6<T>& a, const D6<T>& b) { D6<T> r; r.v = a.v - b.v; for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <class T> D6<T> operator-(const D6<T>& a) { D6<T> r; r.v = -a.v; for (int i = 0; i < 6; ++i) r.d[i] = -a.d[i]; return r; }
template <class T> D6<T> operator*(const D6<T>& a, const D6<T>& b) { D6<T> r; r.v = a.v * b.v; for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <class T> D6<T> operator/(const D6<T>& a, const D6<T>& b) {
  D6<T> r; r.v = a.v / b.v;
  for (int i = 0; i < 6; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
  return r;
}
template <class T> D6<T> dsqrt(const D6<T>& a) {
  using std::sqrt;
  D6<T> r; r.v = sqrt(a.v);
  for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] / (T(2) * r.v);
  return r;
}
template <class T> D6<T> dc(double x) { return D6<T>(T(x)); }

template <class T> void jacobian6_ad(const T (&m)[15], T (&J)[6][6]) {
  // argument order (m00,m01,m02,m03,m04,m10,m11,m12,m13,m20,m21,m22,m30,m31,m40)
  static const int ab[15][2] = {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {0, 4}, {1, 0}, {1, 1}, {1, 2}, {1, 3}, {2, 0}, {2, 1}, {2, 2}, {3, 0}, {3, 1}, {4, 0}};
  static const int seed[15] = {-1, -1, 0, 3, 5, -1, -1, 1, 4, -1, -1, 2, -1, -1, -1};
  D6<T> R[5][5];
  for (int a = 0; a < 5; ++a) for (int b = 0; b < 5; ++b) R[a][b] = dc<T>(0);
  for (int n = 0; n < 15; ++n) {
    D6<T> x(m[n]);
    if (seed[n] >= 0) x.d[seed[n]] = T(1);
    R[ab[n][0]][ab[n][1]] = x;
  }
  D6<T> m00 = R[0][0];
  D6<T> u = R[1][0] / m00, v = R[0][1] / m00;
  // central moments C_ab (a+b <= 4): binomial shift along x, then along y
  D6<T> Cc[5][5];
  for (int a = 0; a < 5; ++a) for (int b = 0; a + b < 5; ++b) Cc[a][b] = R[a][b] / m00;
  D6<T> nu = -u, nv = -v;
  static const int PX[15][2] = {{4, 0}, {3, 0}, {3, 1}, {2, 0}, {2, 1}, {2, 2}, {1, 0}, {1, 1}, {1, 2}, {1, 3}, {0, 0}, {0, 1}, {0, 2}, {0, 3}, {0, 4}};
  static const int PY[15][2] = {{0, 4}, {0, 3}, {1, 3}, {0, 2}, {1, 2}, {2, 2}, {0, 1}, {1, 1}, {2, 1}, {3, 1}, {0, 0}, {1, 0}, {2, 0}, {3, 0}, {4, 0}};
  for (int t = 0; t < 15; ++t) {
    const int a = PX[t][0], b = PX[t][1];
    if (a == 0) continue;
    D6<T> pw = dc<T>(1), acc = dc<T>(0), terms[5];
    for (int q = 0; q <= a; ++q) { terms[q] = pw; pw = pw * nu; }
    for (int p = 0; p <= a; ++p) acc = acc + (dc<T>(double(binom(a, p))) * terms[a - p]) * Cc[p][b];
    Cc[a][b] = acc;
  }
  for (int t = 0; t < 15; ++t) {
    const int a = PY[t][0], b = PY[t][1];
    if (b == 0) continue;
    D6<T> pw = dc<T>(1), acc = dc<T>(0), terms[5];
    for (int q = 0; q <= b; ++q) { terms[q] = pw; pw = pw * nv; }
    for (int p = 0; p <= b; ++p) acc = acc + (dc<T>(double(binom(b, p))) * terms[b - p]) * Cc[a][p];
    Cc[a][b] = acc;
  }
  D6<T> sx = dsqrt(Cc[2][0]), sy = dsqrt(Cc[0][2]);
  auto S = [&](int a, int b) {
    D6<T> d = dc<T>(1);
    for (int i = 0; i < a; ++i) d = d * sx;
    for (int i = 0; i < b; ++i) d = d * sy;
    return Cc[a][b] / d;
  };
  D6<T> S30 = S(3, 0), S40 = S(4, 0), S03 = S(0, 3), S04 = S(0, 4), S11 = S(1, 1), S21 = S(2, 1), S12 = S(1, 2), S31 = S(3, 1), S13 = S(1, 3), S22 = S(2, 2);
  D6<T> one = dc<T>(1), two = dc<T>(2), three = dc<T>(3);
  auto c32 = [&](D6<T> Sj3, D6<T> Si3, D6<T> Si4, D6<T> Sij, D6<T> Sijj, D6<T> Siij, D6<T> Siijj, D6<T> Siiij) {
    return ((Sj3 * Si3 * Si3) / two - Sj3 + Sj3 * (Si3 * Si3 - Si4 + one)) * Sij + (Si4 - (three * Si3 * Si3) / two) * Sijj +
           (-(three * Sj3 * Si3) / two) * Siij + ((three * Si3) / two) * Siijj + Sj3 * Siiij - Si3 / two;
  };
  D6<T> S32 = c32(S03, S30, S40, S11, S12, S21, S22, S31);
  D6<T> S23 = c32(S30, S03, S04, S11, S21, S12, S22, S13);
  D6<T> S14 = (S03 - two * S03 * S04 + (dc<T>(9) * S03 * S03 * S03) / dc<T>(4)) * S11 +
              ((dc<T>(5) * S04) / two - (dc<T>(15) * S03 * S03) / dc<T>(4) - dc<T>(1.5)) * S12 + (two * S03) * S13;
  // full central table with the three closures, C00=1 and first order zero
  D6<T> Ct[6][6];
  for (int a = 0; a < 6; ++a) for (int b = 0; b < 6; ++b) Ct[a][b] = dc<T>(0);
  for (int a = 0; a < 5; ++a) for (int b = 0; a + b < 5; ++b) Ct[a][b] = Cc[a][b];
  Ct[0][0] = dc<T>(1); Ct[1][0] = dc<T>(0); Ct[0][1] = dc<T>(0);
  auto scl = [&](D6<T> s, int a, int b) { for (int i = 0; i < a; ++i) s = s * sx; for (int i = 0; i < b; ++i) s = s * sy; return s; };
  Ct[3][2] = scl(S32, 3, 2); Ct[2][3] = scl(S23, 2, 3); Ct[1][4] = scl(S14, 1, 4);
  D6<T> qu[6], qv[6];
  qu[0] = qv[0] = dc<T>(1);
  for (int i = 1; i < 6; ++i) { qu[i] = qu[i - 1] * u; qv[i] = qv[i - 1] * v; }
  auto raw = [&](int a, int b) {
    D6<T> s = dc<T>(0);
    for (int p = 0; p <= a; ++p)
      for (int q = 0; q <= b; ++q) {
        if (p + q == 1) continue;
        s = s + dc<T>(double(binom(a, p) * binom(b, q))) * Ct[p][q] * (qu[a - p] * qv[b - q]);
      }
    return m00 * s;
  };
  D6<T> m32 = raw(3, 2), m23 = raw(2, 3), m14 = raw(1, 4);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) J[i][j] = T(0);
  J[0][1] = T(1); J[1][2] = T(1); J[3][4] = T(1);
  for (int j = 0; j < 6; ++j) { J[2][j] = m32.d[j]; J[4][j] = m23.d[j]; J[5][j] = m14.d[j]; }
}

// jacobian6 in closed form: d(m32,m23,m14)/dC derived symbolically from the
// same closure (hyqmom.jl_b200/codegen/gen_jacobian6.py), chained with dC/dW.
template <class T> void jacobian6(const T (&m)[15], T (&J)[6][6]) {
  typedef T R;
  T r3[6], r5[6], r6[6];
#include "gen_jacobian6.inc"
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) J[i][j] = T(0);
  J[0][1] = T(1); J[1][2] = T(1); J[3][4] = T(1);
  for (int j = 0; j < 6; ++j) { J[2][j] = r3[j]; J[4][j] = r5[j]; J[5][j] = r6[j]; }
}

// ------------------------------------- LAPACK-path nonsymmetric eigenvalues
// Julia eigvals(::Matrix{Float64}) -> LAPACK geevx('B','N','N','N'):
// dgebal (permute + scale by powers of 2), dgehd2, dhseqr -> dlahqr (n < 75),
// with dlanv2 for the standardized 2x2 blocks.  Written from the published
// LAPACK algorithms; N <= 6.
constexpr double ULP = 2.220446049250313e-16;      // dlamch('P')
constexpr double SAFMIN = 2.2250738585072014e-308; // dlamch('S')

template <class T> T lsign(T a, T b) { using std::fabs; T x = fabs(a); return std::signbit(double(b)) ? -x : x; }
template <class T> T dlapy2(T x, T y) {
  using std::fabs; using std::sqrt;
  T xa = fabs(x), ya = fabs(y);
  T w = jmax(xa, ya), z = jmin(xa, ya);
  if (z == T(0) || w > T(1.79769313486231571e308)) return w;
  T r = z / w;
  return w * sqrt(T(1) + r * r);
}
// Euclidean norm.  OpenBLAS (Julia's BLAS) forms the plain sum of squares
// and its square root; this does the same in FP64 and falls back to the
// scaled LAPACK dnrm2 recurrence when that sum would lose range (over- or
// underflow, NaN).
template <class T> T nrm2(const T* x, int n, int inc) {
  using std::fabs; using std::sqrt;
  T sq = T(0);
  for (int i = 0; i < n; ++i) sq = sq + x[i * inc] * x[i * inc];
  if (sq >= T(1e-280) && sq <= T(1.7976931348623157e308)) return sqrt(sq);
  T scale = T(0), ssq = T(1);
  for (int i = 0; i < n; ++i) {
    T xi = x[i * inc];
    if (xi != T(0)) {
      T a = fabs(xi);
      if (scale < a) { T r = scale / a; ssq = T(1) + ssq * r * r; scale = a; }
      else { T r = a / scale; ssq = ssq + r * r; }
    }
  }
  return scale * sqrt(ssq);
}
// dlarfg: alpha in/out, x[1..n-1] in/out (stride inc); returns tau.
template <class T> T dlarfg(int n, T& alpha, T* x, int inc) {
  if (n <= 1) return T(0);
  T xnorm = nrm2(x, n - 1, inc);
  if (xnorm == T(0)) return T(0);
  T beta = -lsign(dlapy2(alpha, xnorm), alpha);
  T tau = (beta - alpha) / beta;
  T sc = T(1) / (alpha - beta);
  for (int i = 0; i < n - 1; ++i) x[i * inc] = x[i * inc] * sc;
  alpha = beta;
  return tau;
}

// dlanv2: standardized Schur factorization of a real 2x2 block; returns the
// eigenvalues (rt1r, rt1i), (rt2r, rt2i).
template <class T> void dlanv2(T a, T b, T c, T d, T& rt1r, T& rt1i, T& rt2r, T& rt2i) {
  using std::fabs; using std::sqrt;
  const T multpl = T(4);
  const T eps = T(ULP);
  const T safmn2 = T(std::ldexp(1.0, -485));  // radix^int(log(safmin/eps)/log(radix)/2)
  const T safmx2 = T(1) / safmn2;
  if (c == T(0)) {
  } else if (b == T(0)) {
    T tmp = d; d = a; a = tmp; b = -c; c = T(0);
  } else if ((a - d) == T(0) && lsign(T(1), b) != lsign(T(1), c)) {
  } else {
    T temp = a - d;
    T p = T(0.5) * temp;
    T bcmax = jmax(T(fabs(b)), T(fabs(c)));
    T bcmis = jmin(T(fabs(b)), T(fabs(c))) * lsign(T(1), b) * lsign(T(1), c);
    T scale = jmax(T(fabs(p)), bcmax);
    T z = (p / scale) * p + (bcmax / scale) * bcmis;
    if (z >= multpl * eps) {
      z = p + lsign(T(sqrt(scale) * sqrt(z)), p);
      a = d + z;
      d = d - (bcmax / z) * bcmis;
      b = b - c;
      c = T(0);
    } else {
      int count = 0;
      T sigma = b + c;
      for (;;) {
        ++count;
        scale = jmax(T(fabs(temp)), T(fabs(sigma)));
        if (scale >= safmx2) { sigma = sigma * safmn2; temp = temp * safmn2; if (count <= 20) continue; }
        if (scale <= safmn2) { sigma = sigma * safmx2; temp = temp * safmx2; if (count <= 20) continue; }
        break;
      }
      p = T(0.5) * temp;
      T tau = dlapy2(sigma, temp);
      T cs = sqrt(T(0.5) * (T(1) + fabs(sigma) / tau));
      T sn = -(p / (tau * cs)) * lsign(T(1), sigma);
      T aa = a * cs + b * sn, bb = -a * sn + b * cs, cc = c * cs + d * sn, dd = -c * sn + d * cs;
      a = aa * cs + cc * sn; b = bb * cs + dd * sn; c = -aa * sn + cc * cs; d = -bb * sn + dd * cs;
      temp = T(0.5) * (a + d);
      a = temp; d = temp;
      if (c != T(0)) {
        if (b != T(0)) {
          if (lsign(T(1), b) == lsign(T(1), c)) {
            T sab = sqrt(fabs(b)), sac = sqrt(fabs(c));
            p = lsign(T(sab * sac), c);
            a = temp + p; d = temp - p;
            b = b - c; c = T(0);
          }
        } else {
          b = -c; c = T(0);
        }
      }
    }
  }
  rt1r = a; rt2r = d;
  if (c == T(0)) { rt1i = T(0); rt2i = T(0); }
  else { rt1i = sqrt(fabs(b)) * sqrt(fabs(c)); rt2i = -rt1i; }
}

// Eigenvalues of a real N x N matrix (row-major A[i][j]).  Returns 0 on
// success, >0 if the QR iteration did not converge.
template <class T, int N> int eig_real(const T (&Ain)[N][N], T (&wr)[N], T (&wi)[N]) {
  using std::fabs;
  T A[N][N];
  for (int i = 0; i < N; ++i) for (int j = 0; j < N; ++j) A[i][j] = Ain[i][j];
  for (int i = 0; i < N; ++i) { wr[i] = T(0); wi[i] = T(0); }
  // ---- dgebal: permutation
  int k = 0, l = N - 1;
  auto swapij = [&](int j, int m) {
    if (j == m) return;
    for (int r = 0; r <= l; ++r) std::swap(A[r][j], A[r][m]);
    for (int c = k; c < N; ++c) std::swap(A[j][c], A[m][c]);
  };
  bool found = true;
  while (found && l >= 0) {  // rows isolating an eigenvalue -> bottom
    found = false;
    if (l == 0) break;
    for (int j = l; j >= 0; --j) {
      bool zero = true;
      for (int i = 0; i <= l; ++i) { if (i == j) continue; if (A[j][i] != T(0)) { zero = false; break; } }
      if (zero) { swapij(j, l); --l; found = true; break; }
    }
  }
  found = true;
  while (found) {  // columns isolating an eigenvalue -> left
    found = false;
    for (int j = k; j <= l; ++j) {
      bool zero = true;
      for (int i = k; i <= l; ++i) { if (i == j) continue; if (A[i][j] != T(0)) { zero = false; break; } }
      if (zero) { swapij(j, k); ++k; found = true; break; }
    }
  }
  // ---- dgebal: scaling
  {
    const T radix = T(2), factor = T(0.95);
    const T sfmin1 = T(SAFMIN / ULP), sfmax1 = T(1) / sfmin1, sfmin2 = sfmin1 * radix, sfmax2 = T(1) / sfmin2;
    T scal[N];
    for (int i = 0; i < N; ++i) scal[i] = T(1);
    bool noconv = true;
    int guard = 0;
    while (noconv && guard++ < 1000) {
      noconv = false;
      for (int i = k; i <= l; ++i) {
        T col[N], row[N];
        for (int r = k; r <= l; ++r) col[r - k] = A[r][i];
        for (int c2 = k; c2 <= l; ++c2) row[c2 - k] = A[i][c2];
        T c = nrm2(col, l - k + 1, 1), r = nrm2(row, l - k + 1, 1);
        T ca = T(0), ra = T(0);
        for (int rr = 0; rr <= l; ++rr) ca = jmax(ca, T(fabs(A[rr][i])));
        for (int cc = k; cc < N; ++cc) ra = jmax(ra, T(fabs(A[i][cc])));
        if (c == T(0) || r == T(0)) continue;
        if (!std::isfinite(double(c + ca + r + ra))) return -1;  // LAPACK dgebal: NaN -> error return
        T g = r / radix, f = T(1), s = c + r;
        for (int guard2 = 0; guard2 < 2200 && !(c >= g || jmax(jmax(f, c), ca) >= sfmax2 || jmin(jmin(r, g), ra) <= sfmin2); ++guard2) {
          f = f * radix; c = c * radix; ca = ca * radix; r = r / radix; g = g / radix; ra = ra / radix;
        }
        g = c / radix;
        for (int guard3 = 0; guard3 < 2200 && !(g < r || jmax(r, ra) >= sfmax2 || jmin(jmin(jmin(f, c), g), ca) <= sfmin2); ++guard3) {
          f = f / radix; c = c / radix; g = g / radix; ca = ca / radix; r = r * radix; ra = ra * radix;
        }
        if ((c + r) >= factor * s) continue;
        if (f < T(1) && scal[i] < T(1)) if (f * scal[i] <= sfmin1) continue;
        if (f > T(1) && scal[i] > T(1)) if (scal[i] >= sfmax1 / f) continue;
        g = T(1) / f;
        scal[i] = scal[i] * f;
        noconv = true;
        for (int cc = k; cc < N; ++cc) A[i][cc] = A[i][cc] * g;
        for (int rr = 0; rr <= l; ++rr) A[rr][i] = A[rr][i] * f;
      }
    }
  }
  const int ilo = k, ihi = l;
  // isolated eigenvalues
  for (int i = 0; i < ilo; ++i) { wr[i] = A[i][i]; wi[i] = T(0); }
  for (int i = ihi + 1; i < N; ++i) { wr[i] = A[i][i]; wi[i] = T(0); }
  if (ilo > ihi) return 0;
  if (ilo == ihi) { wr[ilo] = A[ilo][ilo]; wi[ilo] = T(0); return 0; }
  // ---- dgehd2
  for (int i = ilo; i < ihi; ++i) {
    int nr = ihi - i;  // reflector length
    T v[N];
    T alpha = A[i + 1][i];
    for (int r = 0; r < nr - 1; ++r) v[r + 1] = A[i + 2 + r][i];
    T tau = dlarfg(nr, alpha, &v[1], 1);
    v[0] = T(1);
    if (tau != T(0)) {
      // right: A(0:ihi, i+1:ihi) -= tau * (A v) v^T
      for (int r = 0; r <= ihi; ++r) {
        T w = T(0);
        for (int c = 0; c < nr; ++c) w = w + A[r][i + 1 + c] * v[c];
        for (int c = 0; c < nr; ++c) A[r][i + 1 + c] = A[r][i + 1 + c] - tau * w * v[c];
      }
      // left: A(i+1:ihi, i+1:N) -= tau * v (v^T A)
      for (int c = i + 1; c < N; ++c) {
        T w = T(0);
        for (int r = 0; r < nr; ++r) w = w + A[i + 1 + r][c] * v[r];
        for (int r = 0; r < nr; ++r) A[i + 1 + r][c] = A[i + 1 + r][c] - tau * v[r] * w;
      }
    }
    A[i + 1][i] = alpha;
    for (int r = i + 2; r < N; ++r) A[r][i] = T(0);
  }
  // ---- dlahqr (wantt = wantz = false)
  T (&H)[N][N] = A;
  const int nh = ihi - ilo + 1;
  const T smlnum = T(SAFMIN) * (T(double(nh)) / T(ULP));
  const T ulp = T(ULP);
  const int itmax = 30 * std::max(10, nh);
  const int kexsh = 10;
  const T dat1 = T(0.75), dat2 = T(-0.4375);
  int kdefl = 0;
  int i = ihi;
  while (i >= ilo) {
    int lq = ilo;
    bool converged = false;
    for (int its = 0; its <= itmax; ++its) {
      int kk;
      for (kk = i; kk > lq; --kk) {
        if (fabs(H[kk][kk - 1]) <= smlnum) break;
        T tst = fabs(H[kk - 1][kk - 1]) + fabs(H[kk][kk]);
        if (tst == T(0)) {
          if (kk - 2 >= ilo) tst = tst + fabs(H[kk - 1][kk - 2]);
          if (kk + 1 <= ihi) tst = tst + fabs(H[kk + 1][kk]);
        }
        if (fabs(H[kk][kk - 1]) <= ulp * tst) {
          T ab = jmax(T(fabs(H[kk][kk - 1])), T(fabs(H[kk - 1][kk])));
          T ba = jmin(T(fabs(H[kk][kk - 1])), T(fabs(H[kk - 1][kk])));
          T aa = jmax(T(fabs(H[kk][kk])), T(fabs(H[kk - 1][kk - 1] - H[kk][kk])));
          T bb = jmin(T(fabs(H[kk][kk])), T(fabs(H[kk - 1][kk - 1] - H[kk][kk])));
          T s = aa + ab;
          if (ba * (ab / s) <= jmax(smlnum, T(ulp * (bb * (aa / s))))) break;
        }
      }
      lq = kk;
      if (lq > ilo) H[lq][lq - 1] = T(0);
      if (lq >= i - 1) { converged = true; break; }
      ++kdefl;
      const int i1 = lq, i2 = i;
      T h11, h12, h21, h22;
      if (kdefl % (2 * kexsh) == 0) {
        T s = fabs(H[i][i - 1]) + fabs(H[i - 1][i - 2]);
        h11 = dat1 * s + H[i][i]; h12 = dat2 * s; h21 = s; h22 = h11;
      } else if (kdefl % kexsh == 0) {
        T s = fabs(H[lq + 1][lq]) + fabs(H[lq + 2][lq + 1]);
        h11 = dat1 * s + H[lq][lq]; h12 = dat2 * s; h21 = s; h22 = h11;
      } else {
        h11 = H[i - 1][i - 1]; h21 = H[i][i - 1]; h12 = H[i - 1][i]; h22 = H[i][i];
      }
      T s = fabs(h11) + fabs(h12) + fabs(h21) + fabs(h22);
      T rt1r, rt1i, rt2r, rt2i;
      if (s == T(0)) { rt1r = rt1i = rt2r = rt2i = T(0); }
      else {
        h11 = h11 / s; h21 = h21 / s; h12 = h12 / s; h22 = h22 / s;
        T tr = (h11 + h22) / T(2);
        T det = (h11 - tr) * (h22 - tr) - h12 * h21;
        using std::sqrt;
        T rtdisc = sqrt(fabs(det));
        if (det >= T(0)) { rt1r = tr * s; rt2r = rt1r; rt1i = rtdisc * s; rt2i = -rt1i; }
        else {
          rt1r = tr + rtdisc; rt2r = tr - rtdisc;
          if (fabs(rt1r - h22) <= fabs(rt2r - h22)) { rt1r = rt1r * s; rt2r = rt1r; }
          else { rt2r = rt2r * s; rt1r = rt2r; }
          rt1i = rt2i = T(0);
        }
      }
      int m;
      T v[3];
      for (m = i - 2; m >= lq; --m) {
        T h21s = H[m + 1][m];
        T s2 = fabs(H[m][m] - rt2r) + fabs(rt2i) + fabs(h21s);
        h21s = H[m + 1][m] / s2;
        v[0] = h21s * H[m][m + 1] + (H[m][m] - rt1r) * ((H[m][m] - rt2r) / s2) - rt1i * (rt2i / s2);
        v[1] = h21s * (H[m][m] + H[m + 1][m + 1] - rt1r - rt2r);
        v[2] = h21s * H[m + 2][m + 1];
        s2 = fabs(v[0]) + fabs(v[1]) + fabs(v[2]);
        v[0] = v[0] / s2; v[1] = v[1] / s2; v[2] = v[2] / s2;
        if (m == lq) break;
        T h00 = fabs(H[m][m - 1]) * (fabs(v[1]) + fabs(v[2]));
        T h11b = fabs(v[0]) * (fabs(H[m - 1][m - 1]) + fabs(H[m][m]) + fabs(H[m + 1][m + 1]));
        if (h00 <= ulp * h11b) break;
      }
      for (int kq = m; kq <= i - 1; ++kq) {
        int nr = std::min(3, i - kq + 1);
        if (kq > m) for (int r = 0; r < nr; ++r) v[r] = H[kq + r][kq - 1];
        T t1 = dlarfg(nr, v[0], &v[1], 1);
        if (kq > m) {
          H[kq][kq - 1] = v[0];
          H[kq + 1][kq - 1] = T(0);
          if (kq < i - 1) H[kq + 2][kq - 1] = T(0);
        } else if (m > lq) {
          H[kq][kq - 1] = H[kq][kq - 1] * (T(1) - t1);
        }
        T v2 = v[1], t2 = t1 * v2;
        if (nr == 3) {
          T v3 = v[2], t3v = t1 * v3;
          for (int j = kq; j <= i2; ++j) {
            T sum = H[kq][j] + v2 * H[kq + 1][j] + v3 * H[kq + 2][j];
            H[kq][j] = H[kq][j] - sum * t1; H[kq + 1][j] = H[kq + 1][j] - sum * t2; H[kq + 2][j] = H[kq + 2][j] - sum * t3v;
          }
          for (int j = i1; j <= std::min(kq + 3, i); ++j) {
            T sum = H[j][kq] + v2 * H[j][kq + 1] + v3 * H[j][kq + 2];
            H[j][kq] = H[j][kq] - sum * t1; H[j][kq + 1] = H[j][kq + 1] - sum * t2; H[j][kq + 2] = H[j][kq + 2] - sum * t3v;
          }
        } else if (nr == 2) {
          for (int j = kq; j <= i2; ++j) {
            T sum = H[kq][j] + v2 * H[kq + 1][j];
            H[kq][j] = H[kq][j] - sum * t1; H[kq + 1][j] = H[kq + 1][j] - sum * t2;
          }
          for (int j = i1; j <= i; ++j) {
            T sum = H[j][kq] + v2 * H[j][kq + 1];
            H[j][kq] = H[j][kq] - sum * t1; H[j][kq + 1] = H[j][kq + 1] - sum * t2;
          }
        }
      }
    }
    if (!converged) return i + 1;
    if (lq == i) { wr[i] = H[i][i]; wi[i] = T(0); }
    else if (lq == i - 1) dlanv2(H[i - 1][i - 1], H[i - 1][i], H[i][i - 1], H[i][i], wr[i - 1], wi[i - 1], wr[i], wi[i]);
    kdefl = 0;
    i = lq - 1;
  }
  return 0;
}

// ------------------------------------------------ eigenvalue driver pieces
// compute_jacobian_eigenvalues (src/numerics/compute_jacobian_eigenvalues.jl:18-50).
template <class T> void jac_eigs(const T (&ma)[15], T& vmin, T& vmax, T& imaxabs) {
  T J[6][6];
  jacobian6(ma, J);
  bool finite = true;
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) if (!std::isfinite(double(J[i][j]))) finite = false;
  T nan = T(std::numeric_limits<double>::quiet_NaN());
  if (!finite) { vmin = nan; vmax = nan; imaxabs = nan; return; }
  T wr[6], wi[6];
  eig_real<T, 6>(J, wr, wi);
  T r[6];
  for (int i = 0; i < 6; ++i) r[i] = wr[i];
  // sort(real(lam)) with NaN last, take first / last
  auto lt = [](T a, T b) { if (a != a) return false; if (b != b) return true; return a < b; };
  std::sort(r, r + 6, lt);
  vmin = r[0]; vmax = r[5];
  using std::fabs;
  imaxabs = fabs(wi[0]);
  for (int i = 1; i < 6; ++i) imaxabs = jmax(imaxabs, T(fabs(wi[i])));
}

// axis_moment_slice (src/utils/axis_moment_slice.jl:31-54), 0-based.
static const int SLICE[4][15] = {{0, 5, 9, 12, 14, 1, 6, 10, 13, 2, 7, 11, 3, 8, 4},
                                 {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14},
                                 {0, 15, 19, 22, 24, 1, 16, 20, 23, 2, 17, 21, 3, 18, 4},
                                 {0, 15, 19, 22, 24, 5, 25, 31, 33, 9, 28, 34, 12, 30, 14}};

template <class T> void slice15(const T* M, int axis, T (&o)[15]) {
  for (int n = 0; n < 15; ++n) o[n] = M[SLICE[axis - 1][n]];
}

// correct_*_plane helpers (src/numerics/eigenvalues6_hyperbolic_3D.jl:181-252)
// applied on the 216-cube of central moments.
template <class T> void correct_plane(T* Cc, int i, int j, T Sij, T Si3, T Sj3, T Si4, T Sj4, T Sii_jj, T Cii, T Cjj, T* Sii_jj_out) {
  using std::sqrt;
  T Sijj = Sij * Sj3, Siij = Sij * Si3, Sijjj = Sij * Sj4, Siiij = Sij * Si4;
  T s22min = (T(2) + T(5) * Sj3 * Sij * Si3) / T(6);
  if (Sii_jj < s22min) Sii_jj = s22min;
  T si = sqrt(jmax(T(EPS), Cii)), sj = sqrt(jmax(T(EPS), Cjj));
  auto at = [&](int a, int b) {
    int e[3] = {0, 0, 0};
    e[i] += a; e[j] += b;
    return t3(e[0], e[1], e[2]);
  };
  Cc[at(2, 1)] = Siij * (si * si) * sj;
  Cc[at(1, 2)] = Sijj * si * (sj * sj);
  Cc[at(3, 1)] = Siiij * (si * si * si) * sj;
  Cc[at(1, 3)] = Sijjj * si * (sj * sj * sj);
  Cc[at(2, 2)] = Sii_jj * (si * si) * (sj * sj);
  if (Sii_jj_out) *Sii_jj_out = Sii_jj;
}

template <class T> void cube_to_35(const T* cube, T* v) { for (int n = 0; n < 35; ++n) v[n] = cube[t3(E35[n][0], E35[n][1], E35[n][2])]; }

// correct_moments_for_real_eigenvalues (src/numerics/eigenvalues6_hyperbolic_3D.jl:81-155).
template <class T> void correct_for_real(const T* M, int axis, bool fixa, bool fixb, int flag2D, T Ma, T* Mout) {
  T M000 = M[0];
  T u = M[1] / M000, v = M[5] / M000, w = M[15] / M000;
  T C4[35], S4[35];
  m2cs4_35(M, C4, S4);
  T Cc[216];
  for (int q = 0; q < 216; ++q) Cc[q] = T(0);
  for (int n = 0; n < 35; ++n) Cc[t3(E35[n][0], E35[n][1], E35[n][2])] = C4[n];
  T C200 = C4[2], C020 = C4[9], C002 = C4[19];
  T S110 = S4[6], S300 = S4[3], S030 = S4[12], S400 = S4[4], S220 = S4[11], S040 = S4[14];
  T S101 = S4[16], S202 = S4[21], S003 = S4[22], S004 = S4[24], S011 = S4[25], S022 = S4[34];
  if (fixa) correct_plane(Cc, 0, 1, S110, S300, S030, S400, S040, S220, C200, C020, (T*)nullptr);
  if (fixb) {
    if (axis == 1) correct_plane(Cc, 0, 2, S101, S300, S003, S400, S004, S202, C200, C002, (T*)nullptr);
    else correct_plane(Cc, 1, 2, S011, S030, S003, S040, S004, S022, C020, C002, (T*)nullptr);
  }
  Cc[t3(0, 0, 0)] = T(1);
  T Mc[216], Mh[35];
  c_to_m(M000, u, v, w, Cc, Mc, 4);
  cube_to_35(Mc, Mh);
  T Fx[35], Fy[35], Fz[35];
  flux_closure35(Mh, flag2D, Ma, Fx, Fy, Fz, Mout);
}

// eigenvalues6_hyperbolic_3D (src/numerics/eigenvalues6_hyperbolic_3D.jl:22-56).
template <class T> void eigenvalues6_hyperbolic_3D(const T* M, int axis, int flag2D, T Ma, T& v6min, T& v6max, T* Mr) {
  const int a1 = axis == 1 ? 1 : 2, a2 = axis == 1 ? 3 : 4;
  T sa[15], sb[15];
  slice15(M, a1, sa); slice15(M, a2, sb);
  T mn_a, mx_a, ia, mn_b, mx_b, ib;
  jac_eigs(sa, mn_a, mx_a, ia);
  jac_eigs(sb, mn_b, mx_b, ib);
  // v6min/v6max combination of compute_jacobian_eigenvalues: the second
  // Jacobian is skipped when non-finite.
  auto combine = [&](T& vmn, T& vmx) {
    vmn = mn_a; vmx = mx_a;
    if (mn_b == mn_b || mx_b == mx_b) { vmn = jmin(vmn, mn_b); vmx = jmax(vmx, mx_b); }
  };
  combine(v6min, v6max);
  for (int n = 0; n < 35; ++n) Mr[n] = M[n];
  const T thr = T(1000 * EPS);
  bool ca = ia > thr, cb = ib > thr;
  if (ca || cb) {
    hit(BR_COMPLEX_XY);
    T Mc[35];
    correct_for_real(M, axis, ca, cb, flag2D, Ma, Mc);
    slice15(Mc, a1, sa); slice15(Mc, a2, sb);
    jac_eigs(sa, mn_a, mx_a, ia);
    jac_eigs(sb, mn_b, mx_b, ib);
    combine(v6min, v6max);
    for (int n = 0; n < 35; ++n) Mr[n] = Mc[n];
  }
}

// eigenvalues6z_hyperbolic_3D (src/numerics/eigenvalues6z_hyperbolic_3D.jl:23-365).
template <class T> void eigenvalues6z_hyperbolic_3D(const T* M, int flag2D, T Ma, bool positivity, T& v6min, T& v6max, T* Mr) {
  for (int n = 0; n < 35; ++n) Mr[n] = M[n];
  if (positivity && M[0] <= T(0)) Mr[0] = jmax(M[0], T(1e-14));
  T Mw[35];
  for (int n = 0; n < 35; ++n) Mw[n] = M[n];
  Mw[0] = Mr[0];
  if (positivity && Mw[0] > T(1e-15)) {
    T m000 = Mw[0];
    T vx = M[2] / m000 - sq(M[1] / m000);
    T vy = M[9] / m000 - sq(M[5] / m000);
    T vz = M[19] / m000 - sq(M[15] / m000);
    if (vx < T(0) || vy < T(0) || vz < T(0)) {
      hit(BR_REREALIZE_Z);
      T Fx[35], Fy[35], Fz[35];
      flux_closure35(M, flag2D, Ma, Fx, Fy, Fz, Mr);
      for (int n = 0; n < 35; ++n) Mw[n] = Mr[n];
    }
  }
  // WU: jacobian6(m000,m100,m200,m300,m400,m001,m101,m201,m301,m002,m102,m202,m003,m103,m004)
  static const int WU[15] = {0, 1, 2, 3, 4, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24};
  static const int WV[15] = {0, 15, 19, 22, 24, 5, 25, 31, 33, 9, 28, 34, 12, 30, 14};
  T sa[15], sb[15];
  for (int n = 0; n < 15; ++n) { sa[n] = Mw[WU[n]]; sb[n] = Mw[WV[n]]; }
  T mn_a, mx_a, ia, mn_b, mx_b, ib;
  jac_eigs(sa, mn_a, mx_a, ia);
  jac_eigs(sb, mn_b, mx_b, ib);
  v6min = jmin(mn_a, mn_b);
  v6max = jmax(mx_a, mx_b);
  const T thr = T(1000 * EPS);
  bool ca = ia > thr, cb = ib > thr;
  if (ca || cb) {
    hit(BR_COMPLEX_Z);
    T M000 = M[0];
    T u = M[1] / M000, v = M[5] / M000, w = M[15] / M000;
    T C4[35], S4[35];
    m2cs4_35(M, C4, S4);
    T Cc[216];
    for (int q = 0; q < 216; ++q) Cc[q] = T(0);
    for (int n = 0; n < 35; ++n) Cc[t3(E35[n][0], E35[n][1], E35[n][2])] = C4[n];
    T C200 = C4[2], C020 = C4[9], C002 = C4[19];
    T S101 = S4[16], S300 = S4[3], S003 = S4[22], S400 = S4[4], S202 = S4[21], S004 = S4[24];
    T S011 = S4[25], S030 = S4[12], S022 = S4[34], S040 = S4[14];
    if (ca) correct_plane(Cc, 0, 2, S101, S300, S003, S400, S004, S202, C200, C002, (T*)nullptr);
    if (cb) correct_plane(Cc, 1, 2, S011, S030, S003, S040, S004, S022, C020, C002, (T*)nullptr);
    Cc[t3(0, 0, 0)] = T(1);
    T Mc[216], Mh[35];
    c_to_m(M000, u, v, w, Cc, Mc, 4);
    cube_to_35(Mc, Mh);
    T Fx[35], Fy[35], Fz[35];
    flux_closure35(Mh, flag2D, Ma, Fx, Fy, Fz, Mr);
    for (int n = 0; n < 15; ++n) { sa[n] = Mr[WU[n]]; sb[n] = Mr[WV[n]]; }
    jac_eigs(sa, mn_a, mx_a, ia);
    jac_eigs(sb, mn_b, mx_b, ib);
    v6min = jmin(mn_a, mn_b);
    v6max = jmax(mx_a, mx_b);
  }
}

// ------------------------------------------ closure_and_eigenvalues (N = 2)
// (src/numerics/closure_and_eigenvalues.jl:76-137).  The eigenvalues of the
// 3x3 Jacobi matrix z (off-diagonals sqrt(Complex(b))) are those of the real
// matrix [a1 b2 0; 1 a2 b3; 0 1 a3] (same characteristic polynomial); when
// both b >= 0 z is real symmetric and the symmetric eigenvalues are used.
template <class T> void closure_and_eigenvalues(const T (&mom)[5], T& Mp, T& vpmin, T& vpmax) {
  T sig[4][7];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 7; ++j) sig[i][j] = T(0);
  T a[3] = {T(0), T(0), T(0)}, b[4] = {T(0), T(0), T(0), T(0)};
  for (int i = 1; i <= 5; ++i) sig[1][i] = mom[i - 1];
  a[0] = mom[1] / mom[0];
  // k = 3 (1-based) -> row index 2
  for (int l = 2; l <= 4; ++l) sig[2][l] = sig[1][l + 1] - a[0] * sig[1][l] - b[0] * sig[0][l];
  a[1] = sig[2][3] / sig[2][2] - sig[1][2] / sig[1][1];
  b[1] = sig[2][2] / sig[1][1];
  sig[3][3] = sig[2][4] - a[1] * sig[2][3] - b[1] * sig[1][3];
  b[2] = sig[3][3] / sig[2][2];
  a[2] = (a[0] + a[1]) / T(2);
  sig[3][4] = sig[3][3] * (a[2] + sig[2][3] / sig[2][2]);
  sig[2][5] = sig[3][4] + a[1] * sig[2][4] + b[1] * sig[1][4];
  sig[1][6] = sig[2][5] + a[0] * sig[1][5] + b[0] * sig[0][5];
  Mp = sig[1][6];
  b[2] = b[2] * T(5) / T(2);
  T nan = T(std::numeric_limits<double>::quiet_NaN());
  // finiteness of z = [a1 sqrt(b2) 0; . a2 sqrt(b3); . . a3]
  bool fin = std::isfinite(double(a[0])) && std::isfinite(double(a[1])) && std::isfinite(double(a[2])) &&
             std::isfinite(double(b[1])) && std::isfinite(double(b[2]));
  if (!fin) { vpmin = nan; vpmax = nan; return; }
  if (b[1] >= T(0) && b[2] >= T(0)) {
    using std::sqrt;
    T S3[3][3] = {{a[0], sqrt(b[1]), T(0)}, {sqrt(b[1]), a[1], sqrt(b[2])}, {T(0), sqrt(b[2]), a[2]}};
    // symmetric eigenvalues by cyclic Jacobi rotation; from the fourth sweep
    // on, an off-diagonal entry too small to change either diagonal entry
    // (|d| + 100|e| == |d|) is set to zero (Rutishauser's threshold rule), so
    // the sweeps end after a few iterations instead of hunting round-off
    T A[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = S3[i][j];
    using std::fabs;
    for (int sweep = 0; sweep < 60; ++sweep) {
      T off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
      if (off == T(0)) break;
      for (int p = 0; p < 2; ++p)
        for (int q = p + 1; q < 3; ++q) {
          if (A[p][q] == T(0)) continue;
          if (sweep >= 3) {
            const T g = T(100) * fabs(A[p][q]);
            if (fabs(A[p][p]) + g == fabs(A[p][p]) && fabs(A[q][q]) + g == fabs(A[q][q])) {
              A[p][q] = T(0); A[q][p] = T(0);
              continue;
            }
          }
          T theta = (A[q][q] - A[p][p]) / (T(2) * A[p][q]);
          T t = jsign(theta) / (fabs(theta) + sqrt(theta * theta + T(1)));
          if (theta == T(0)) t = T(1);
          T c = T(1) / sqrt(t * t + T(1)), s = t * c;
          for (int k = 0; k < 3; ++k) { T akp = A[k][p], akq = A[k][q]; A[k][p] = c * akp - s * akq; A[k][q] = s * akp + c * akq; }
          for (int k = 0; k < 3; ++k) { T apk = A[p][k], aqk = A[q][k]; A[p][k] = c * apk - s * aqk; A[q][k] = s * apk + c * aqk; }
        }
    }
    vpmin = jmin(jmin(A[0][0], A[1][1]), A[2][2]);
    vpmax = jmax(jmax(A[0][0], A[1][1]), A[2][2]);
    return;
  }
  T R[3][3] = {{a[0], b[1], T(0)}, {T(1), a[1], b[2]}, {T(0), T(1), a[2]}};
  T wr[3], wi[3];
  eig_real<T, 3>(R, wr, wi);
  vpmin = jmin(jmin(wr[0], wr[1]), wr[2]);
  vpmax = jmax(jmax(wr[0], wr[1]), wr[2]);
}

// ---------------------------------------------------------------- collision
// collision35 (src/numerics/collision35.jl:154-182).
template <class T> void collision35(const T* M, T dt, T Kn, bool positivity, T* Mout) {
  using std::sqrt; using std::exp;
  T rho = M[0];
  T u = M[1] / rho, v = M[5] / rho, w = M[15] / rho;
  T C200 = M[2] / rho - u * u, C020 = M[9] / rho - v * v, C002 = M[19] / rho - w * w;
  T Theta = (C200 + C020 + C002) / T(3);
  if (positivity) Theta = jmax(Theta, T(1e-14));
  T tc = Kn / (rho * sqrt(Theta) * T(2));
  T MG[35];
  initialize_m4_35(rho, u, v, w, Theta, T(0), T(0), Theta, T(0), Theta, MG);
  T e = hexpT(T(-dt / tc));
  for (int n = 0; n < 35; ++n) Mout[n] = MG[n] - e * (MG[n] - M[n]);
}

// ------------------------------------------------------------------ HLL row
// pas_HLL + flux_HLL with physical BCs on both ends
// (src/numerics/pas_HLL.jl:238-298, src/numerics/flux_HLL.jl:318-330).
// Row of Np cells, moment stride `ms` between the 35 moments, cell stride cs.
template <class T> void pas_HLL_row(int Np, const T* M, const T* F, int cs, int ms, const T* vmin, const T* vmax, int vs,
                                    T dt, T dx, T* Mp) {
  using std::fabs;
  // lleft/lright, with 0 at j = 1 (index 0) and at Np
  T* ll = new T[Np];
  T* lr = new T[Np];
  T* Ws = new T[Np * 35];
  T* Fm = new T[Np * 35];
  T* Fl = new T[(Np - 1) * 35];
  for (int j = 0; j < Np; ++j) { ll[j] = T(0); lr[j] = T(0); }
  for (int j = 0; j < Np * 35; ++j) Ws[j] = T(0);
  for (int j = 0; j < Np; ++j) for (int n = 0; n < 35; ++n) Fm[j * 35 + n] = F[j * cs + n * ms];
  for (int j = 1; j <= Np - 2; ++j) {
    ll[j] = jmin(vmin[j * vs], vmin[(j + 1) * vs]);
    lr[j] = jmax(vmax[j * vs], vmax[(j + 1) * vs]);
    if (fabs(ll[j] - lr[j]) > T(1e-10)) {
      for (int n = 0; n < 35; ++n) {
        T mj = M[j * cs + n * ms], mj1 = M[(j + 1) * cs + n * ms];
        Ws[j * 35 + n] = (ll[j] * mj - lr[j] * mj1) / (ll[j] - lr[j]) - (Fm[j * 35 + n] - Fm[(j + 1) * 35 + n]) / (ll[j] - lr[j]);
      }
    }
  }
  for (int n = 0; n < 35; ++n) {
    Ws[n] = Ws[35 + n];
    Ws[(Np - 1) * 35 + n] = Ws[(Np - 2) * 35 + n];
    Fm[n] = Fm[35 + n];
    Fm[(Np - 1) * 35 + n] = Fm[(Np - 2) * 35 + n];
  }
  for (int j = 0; j < Np - 1; ++j)
    for (int n = 0; n < 35; ++n) {
      T w = Ws[j * 35 + n];
      Fl[j * 35 + n] = T(0.5) * (Fm[j * 35 + n] + Fm[(j + 1) * 35 + n]) -
                       T(0.5) * (fabs(ll[j]) * (w - M[j * cs + n * ms]) - fabs(lr[j]) * (w - M[(j + 1) * cs + n * ms]));
    }
  T r = dt / dx;
  for (int j = 0; j < Np; ++j)
    for (int n = 0; n < 35; ++n) Mp[j * cs + n * ms] = M[j * cs + n * ms];
  for (int j = 1; j <= Np - 2; ++j)
    for (int n = 0; n < 35; ++n)
      Mp[j * cs + n * ms] = M[j * cs + n * ms] - r * (Fl[j * 35 + n] - Fl[(j - 1) * 35 + n]);
  for (int n = 0; n < 35; ++n) {
    Mp[n * ms] = Mp[cs + n * ms];
    Mp[(Np - 1) * cs + n * ms] = Mp[(Np - 2) * cs + n * ms];
  }
  delete[] ll; delete[] lr; delete[] Ws; delete[] Fm; delete[] Fl;
}

}  // namespace hyqo
