// Wave speeds and BGK relaxation (device code): jacobian6, the LAPACK-path
// nonsymmetric eigenvalue solve, eigenvalues6_hyperbolic_3D (x, y),
// eigenvalues6z_hyperbolic_3D, closure_and_eigenvalues and collision35.
// Restates src/numerics/{eigenvalues6_hyperbolic_3D.jl:22-252,
// eigenvalues6z_hyperbolic_3D.jl:23-365, compute_jacobian_eigenvalues.jl:18-50,
// closure_and_eigenvalues.jl:76-137, collision35.jl:154-182},
// src/utils/axis_moment_slice.jl:31-54 and src/autogen/jacobian6.jl:14-59.
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
#include "hyq_closure.cuh"

namespace hyq {

// ------------------------------------------------------------ jacobian6
// m[15] in jacobian6 argument order (m00,m01,m02,m03,m04,m10,m11,m12,m13,
// m20,m21,m22,m30,m31,m40); m_ab = E[x^a y^b], x = flux direction.
// Output: rows 3, 5, 6 of the Jacobian (rows 1, 2, 4 are unit rows e2, e3, e5).
// The body is the closed form d(m32,m23,m14)/dC chained with dC/dW, derived
// symbolically from the 2-D HyQMOM closure by codegen/gen_jacobian6.py; the
// CPU oracle includes the same generated body.
HQD void jacobian6_rows(const double* m, double* r3, double* r5, double* r6) {
  typedef double R;
#include "gen_jacobian6.inc"
}

// ------------------------------------------- LAPACK-path eigenvalues, N <= 6
// Julia eigvals(::Matrix{Float64}) -> geevx('B'): dgebal (permute + power-of-2
// scaling), dgehd2 Householder Hessenberg reduction, dlahqr double-shift QR
// (eigenvalues only) with dlanv2 standardization of 2x2 blocks.
constexpr double ULP = 2.220446049250313e-16;
constexpr double SAFMIN = 2.2250738585072014e-308;

HQD double lsign(double a, double b) { return signbit(b) ? -fabs(a) : fabs(a); }
HQD double dlapy2(double x, double y) {
  const double xa = fabs(x), ya = fabs(y);
  const double w = jmax(xa, ya), z = jmin(xa, ya);
  if (z == 0.0 || w > 1.79769313486231571e308) return w;
  const double r = z / w;
  return w * sqrt(1.0 + r * r);
}
// Euclidean norm: the plain sum of squares and its square root (as
// OpenBLAS computes it), with the scaled LAPACK dnrm2 recurrence when that
// sum would lose range (over- or underflow, NaN).
HQD double nrm2(const double* x, int n, int inc) {
  double sq = 0.0;
  for (int i = 0; i < n; ++i) sq = sq + x[i * inc] * x[i * inc];
  if (sq >= 1e-280 && sq <= 1.7976931348623157e308) return sqrt(sq);
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; ++i) {
    const double xi = x[i * inc];
    if (xi != 0.0) {
      const double a = fabs(xi);
      if (scale < a) { const double r = scale / a; ssq = 1.0 + ssq * r * r; scale = a; }
      else { const double r = a / scale; ssq = ssq + r * r; }
    }
  }
  return scale * sqrt(ssq);
}
HQD double dlarfg(int n, double& alpha, double* x, int inc) {
  if (n <= 1) return 0.0;
  const double xnorm = nrm2(x, n - 1, inc);
  if (xnorm == 0.0) return 0.0;
  const double beta = -lsign(dlapy2(alpha, xnorm), alpha);
  const double tau = (beta - alpha) / beta;
  const double sc = 1.0 / (alpha - beta);
  for (int i = 0; i < n - 1; ++i) x[i * inc] = x[i * inc] * sc;
  alpha = beta;
  return tau;
}
HQD void dlanv2(double a, double b, double c, double d, double& rt1r, double& rt1i, double& rt2r, double& rt2i) {
  const double eps = ULP;
  const double safmn2 = 1.0010415475915505e-146;  // 2^-485
  const double safmx2 = 1.0 / safmn2;
  if (c == 0.0) {
  } else if (b == 0.0) {
    const double t = d; d = a; a = t; b = -c; c = 0.0;
  } else if ((a - d) == 0.0 && lsign(1.0, b) != lsign(1.0, c)) {
  } else {
    double temp = a - d;
    double p = 0.5 * temp;
    const double bcmax = jmax(fabs(b), fabs(c));
    const double bcmis = jmin(fabs(b), fabs(c)) * lsign(1.0, b) * lsign(1.0, c);
    double scale = jmax(fabs(p), bcmax);
    double z = (p / scale) * p + (bcmax / scale) * bcmis;
    if (z >= 4.0 * eps) {
      z = p + lsign(sqrt(scale) * sqrt(z), p);
      a = d + z;
      d = d - (bcmax / z) * bcmis;
      b = b - c;
      c = 0.0;
    } else {
      int count = 0;
      double sigma = b + c;
      for (;;) {
        ++count;
        scale = jmax(fabs(temp), fabs(sigma));
        if (scale >= safmx2) { sigma = sigma * safmn2; temp = temp * safmn2; if (count <= 20) continue; }
        if (scale <= safmn2) { sigma = sigma * safmx2; temp = temp * safmx2; if (count <= 20) continue; }
        break;
      }
      p = 0.5 * temp;
      const double tau = dlapy2(sigma, temp);
      const double cs = sqrt(0.5 * (1.0 + fabs(sigma) / tau));
      const double sn = -(p / (tau * cs)) * lsign(1.0, sigma);
      const double aa = a * cs + b * sn, bb = -a * sn + b * cs, cc = c * cs + d * sn, dd = -c * sn + d * cs;
      a = aa * cs + cc * sn; b = bb * cs + dd * sn; c = -aa * sn + cc * cs; d = -bb * sn + dd * cs;
      temp = 0.5 * (a + d);
      a = temp; d = temp;
      if (c != 0.0) {
        if (b != 0.0) {
          if (lsign(1.0, b) == lsign(1.0, c)) {
            const double sab = sqrt(fabs(b)), sac = sqrt(fabs(c));
            p = lsign(sab * sac, c);
            a = temp + p; d = temp - p;
            b = b - c; c = 0.0;
          }
        } else {
          b = -c; c = 0.0;
        }
      }
    }
  }
  rt1r = a; rt2r = d;
  if (c == 0.0) { rt1i = 0.0; rt2i = 0.0; }
  else { rt1i = sqrt(fabs(b)) * sqrt(fabs(c)); rt2i = -rt1i; }
}

// Loops of the general eigen-solve below stay rolled on the device: its
// passes over listed cells wait mostly on instruction fetch, and the compact
// code made them 1.3x faster on late crossing-jet states than the unrolled.
#ifndef HQ_GEN_ROLLED
#define HQ_GEN_ROLLED 1
#endif
#if defined(__CUDACC__) && HQ_GEN_ROLLED
#define HQ_ROLLED _Pragma("unroll 1")
#else
#define HQ_ROLLED
#endif

// Eigenvalues of the N x N row-major matrix A (overwritten).  Returns 0 on
// success, > 0 when the QR iteration limit was reached.
template <int N>
HQN int eig_real(double (&A)[N][N], double (&wr)[N], double (&wi)[N]) {
  HQ_ROLLED for (int i = 0; i < N; ++i) { wr[i] = 0.0; wi[i] = 0.0; }
  int k = 0, l = N - 1;
  auto swapij = [&](int j, int m) {
    if (j == m) return;
    HQ_ROLLED for (int r = 0; r <= l; ++r) { const double t = A[r][j]; A[r][j] = A[r][m]; A[r][m] = t; }
    HQ_ROLLED for (int c = k; c < N; ++c) { const double t = A[j][c]; A[j][c] = A[m][c]; A[m][c] = t; }
  };
  bool found = true;
  while (found && l >= 0) {
    found = false;
    if (l == 0) break;
    HQ_ROLLED for (int j = l; j >= 0; --j) {
      bool zero = true;
      HQ_ROLLED for (int i = 0; i <= l; ++i) { if (i == j) continue; if (A[j][i] != 0.0) { zero = false; break; } }
      if (zero) { swapij(j, l); --l; found = true; break; }
    }
  }
  found = true;
  while (found) {
    found = false;
    HQ_ROLLED for (int j = k; j <= l; ++j) {
      bool zero = true;
      HQ_ROLLED for (int i = k; i <= l; ++i) { if (i == j) continue; if (A[i][j] != 0.0) { zero = false; break; } }
      if (zero) { swapij(j, k); ++k; found = true; break; }
    }
  }
  {
    const double radix = 2.0, factor = 0.95;
    const double sfmin1 = SAFMIN / ULP, sfmax1 = 1.0 / sfmin1, sfmin2 = sfmin1 * radix, sfmax2 = 1.0 / sfmin2;
    double scal[N];
    HQ_ROLLED for (int i = 0; i < N; ++i) scal[i] = 1.0;
    bool noconv = true;
    int guard = 0;
    while (noconv && guard++ < 1000) {
      noconv = false;
      HQ_ROLLED for (int i = k; i <= l; ++i) {
        double col[N], row[N];
        HQ_ROLLED for (int r = k; r <= l; ++r) col[r - k] = A[r][i];
        HQ_ROLLED for (int c2 = k; c2 <= l; ++c2) row[c2 - k] = A[i][c2];
        double c = nrm2(col, l - k + 1, 1), r = nrm2(row, l - k + 1, 1);
        double ca = 0.0, ra = 0.0;
        HQ_ROLLED for (int rr = 0; rr <= l; ++rr) ca = jmax(ca, fabs(A[rr][i]));
        HQ_ROLLED for (int cc = k; cc < N; ++cc) ra = jmax(ra, fabs(A[i][cc]));
        if (c == 0.0 || r == 0.0) continue;
        if (!isfinite(c + ca + r + ra)) return -1;  // LAPACK dgebal: NaN -> error return
        double g = r / radix, f = 1.0;
        const double s = c + r;
        HQ_ROLLED for (int guard2 = 0; guard2 < 2200 && !(c >= g || jmax(jmax(f, c), ca) >= sfmax2 || jmin(jmin(r, g), ra) <= sfmin2); ++guard2) {
          f = f * radix; c = c * radix; ca = ca * radix; r = r / radix; g = g / radix; ra = ra / radix;
        }
        g = c / radix;
        HQ_ROLLED for (int guard3 = 0; guard3 < 2200 && !(g < r || jmax(r, ra) >= sfmax2 || jmin(jmin(jmin(f, c), g), ca) <= sfmin2); ++guard3) {
          f = f / radix; c = c / radix; g = g / radix; ca = ca / radix; r = r * radix; ra = ra * radix;
        }
        if ((c + r) >= factor * s) continue;
        if (f < 1.0 && scal[i] < 1.0) if (f * scal[i] <= sfmin1) continue;
        if (f > 1.0 && scal[i] > 1.0) if (scal[i] >= sfmax1 / f) continue;
        g = 1.0 / f;
        scal[i] = scal[i] * f;
        noconv = true;
        HQ_ROLLED for (int cc = k; cc < N; ++cc) A[i][cc] = A[i][cc] * g;
        HQ_ROLLED for (int rr = 0; rr <= l; ++rr) A[rr][i] = A[rr][i] * f;
      }
    }
  }
  const int ilo = k, ihi = l;
  HQ_ROLLED for (int i = 0; i < ilo; ++i) { wr[i] = A[i][i]; wi[i] = 0.0; }
  HQ_ROLLED for (int i = ihi + 1; i < N; ++i) { wr[i] = A[i][i]; wi[i] = 0.0; }
  if (ilo > ihi) return 0;
  if (ilo == ihi) { wr[ilo] = A[ilo][ilo]; wi[ilo] = 0.0; return 0; }
  HQ_ROLLED for (int i = ilo; i < ihi; ++i) {
    const int nr = ihi - i;
    double v[N];
    double alpha = A[i + 1][i];
    HQ_ROLLED for (int r = 0; r < nr - 1; ++r) v[r + 1] = A[i + 2 + r][i];
    const double tau = dlarfg(nr, alpha, &v[1], 1);
    v[0] = 1.0;
    if (tau != 0.0) {
      HQ_ROLLED for (int r = 0; r <= ihi; ++r) {
        double w = 0.0;
        HQ_ROLLED for (int c = 0; c < nr; ++c) w = w + A[r][i + 1 + c] * v[c];
        HQ_ROLLED for (int c = 0; c < nr; ++c) A[r][i + 1 + c] = A[r][i + 1 + c] - tau * w * v[c];
      }
      HQ_ROLLED for (int c = i + 1; c < N; ++c) {
        double w = 0.0;
        HQ_ROLLED for (int r = 0; r < nr; ++r) w = w + A[i + 1 + r][c] * v[r];
        HQ_ROLLED for (int r = 0; r < nr; ++r) A[i + 1 + r][c] = A[i + 1 + r][c] - tau * v[r] * w;
      }
    }
    A[i + 1][i] = alpha;
    HQ_ROLLED for (int r = i + 2; r < N; ++r) A[r][i] = 0.0;
  }
  double (&H)[N][N] = A;
  const int nh = ihi - ilo + 1;
  const double smlnum = SAFMIN * (double(nh) / ULP);
  const double ulp = ULP;
  const int itmax = 30 * (nh > 10 ? nh : 10);
  const double dat1 = 0.75, dat2 = -0.4375;
  int kdefl = 0;
  int i = ihi;
  while (i >= ilo) {
    int lq = ilo;
    bool converged = false;
    HQ_ROLLED for (int its = 0; its <= itmax; ++its) {
      int kk;
      HQ_ROLLED for (kk = i; kk > lq; --kk) {
        if (fabs(H[kk][kk - 1]) <= smlnum) break;
        double tst = fabs(H[kk - 1][kk - 1]) + fabs(H[kk][kk]);
        if (tst == 0.0) {
          if (kk - 2 >= ilo) tst = tst + fabs(H[kk - 1][kk - 2]);
          if (kk + 1 <= ihi) tst = tst + fabs(H[kk + 1][kk]);
        }
        if (fabs(H[kk][kk - 1]) <= ulp * tst) {
          const double ab = jmax(fabs(H[kk][kk - 1]), fabs(H[kk - 1][kk]));
          const double ba = jmin(fabs(H[kk][kk - 1]), fabs(H[kk - 1][kk]));
          const double aa = jmax(fabs(H[kk][kk]), fabs(H[kk - 1][kk - 1] - H[kk][kk]));
          const double bb = jmin(fabs(H[kk][kk]), fabs(H[kk - 1][kk - 1] - H[kk][kk]));
          const double s = aa + ab;
          if (ba * (ab / s) <= jmax(smlnum, ulp * (bb * (aa / s)))) break;
        }
      }
      lq = kk;
      if (lq > ilo) H[lq][lq - 1] = 0.0;
      if (lq >= i - 1) { converged = true; break; }
      ++kdefl;
      const int i1 = lq, i2 = i;
      double h11, h12, h21, h22;
      if (kdefl % 20 == 0) {
        const double s = fabs(H[i][i - 1]) + fabs(H[i - 1][i - 2]);
        h11 = dat1 * s + H[i][i]; h12 = dat2 * s; h21 = s; h22 = h11;
      } else if (kdefl % 10 == 0) {
        const double s = fabs(H[lq + 1][lq]) + fabs(H[lq + 2][lq + 1]);
        h11 = dat1 * s + H[lq][lq]; h12 = dat2 * s; h21 = s; h22 = h11;
      } else {
        h11 = H[i - 1][i - 1]; h21 = H[i][i - 1]; h12 = H[i - 1][i]; h22 = H[i][i];
      }
      const double s = fabs(h11) + fabs(h12) + fabs(h21) + fabs(h22);
      double rt1r, rt1i, rt2r, rt2i;
      if (s == 0.0) { rt1r = rt1i = rt2r = rt2i = 0.0; }
      else {
        h11 = h11 / s; h21 = h21 / s; h12 = h12 / s; h22 = h22 / s;
        const double tr = (h11 + h22) / 2.0;
        const double det = (h11 - tr) * (h22 - tr) - h12 * h21;
        const double rtdisc = sqrt(fabs(det));
        if (det >= 0.0) { rt1r = tr * s; rt2r = rt1r; rt1i = rtdisc * s; rt2i = -rt1i; }
        else {
          rt1r = tr + rtdisc; rt2r = tr - rtdisc;
          if (fabs(rt1r - h22) <= fabs(rt2r - h22)) { rt1r = rt1r * s; rt2r = rt1r; }
          else { rt2r = rt2r * s; rt1r = rt2r; }
          rt1i = rt2i = 0.0;
        }
      }
      int m;
      double v[3];
      HQ_ROLLED for (m = i - 2; m >= lq; --m) {
        double h21s = H[m + 1][m];
        double s2 = fabs(H[m][m] - rt2r) + fabs(rt2i) + fabs(h21s);
        h21s = H[m + 1][m] / s2;
        v[0] = h21s * H[m][m + 1] + (H[m][m] - rt1r) * ((H[m][m] - rt2r) / s2) - rt1i * (rt2i / s2);
        v[1] = h21s * (H[m][m] + H[m + 1][m + 1] - rt1r - rt2r);
        v[2] = h21s * H[m + 2][m + 1];
        s2 = fabs(v[0]) + fabs(v[1]) + fabs(v[2]);
        v[0] = v[0] / s2; v[1] = v[1] / s2; v[2] = v[2] / s2;
        if (m == lq) break;
        const double h00 = fabs(H[m][m - 1]) * (fabs(v[1]) + fabs(v[2]));
        const double h11b = fabs(v[0]) * (fabs(H[m - 1][m - 1]) + fabs(H[m][m]) + fabs(H[m + 1][m + 1]));
        if (h00 <= ulp * h11b) break;
      }
      HQ_ROLLED for (int kq = m; kq <= i - 1; ++kq) {
        const int nr = (i - kq + 1) < 3 ? (i - kq + 1) : 3;
        if (kq > m) HQ_ROLLED for (int r = 0; r < nr; ++r) v[r] = H[kq + r][kq - 1];
        const double t1 = dlarfg(nr, v[0], &v[1], 1);
        if (kq > m) {
          H[kq][kq - 1] = v[0];
          H[kq + 1][kq - 1] = 0.0;
          if (kq < i - 1) H[kq + 2][kq - 1] = 0.0;
        } else if (m > lq) {
          H[kq][kq - 1] = H[kq][kq - 1] * (1.0 - t1);
        }
        const double v2 = v[1], t2 = t1 * v2;
        if (nr == 3) {
          const double v3 = v[2], t3v = t1 * v3;
          HQ_ROLLED for (int j = kq; j <= i2; ++j) {
            const double sum = H[kq][j] + v2 * H[kq + 1][j] + v3 * H[kq + 2][j];
            H[kq][j] = H[kq][j] - sum * t1; H[kq + 1][j] = H[kq + 1][j] - sum * t2; H[kq + 2][j] = H[kq + 2][j] - sum * t3v;
          }
          const int jm = (kq + 3 < i) ? kq + 3 : i;
          HQ_ROLLED for (int j = i1; j <= jm; ++j) {
            const double sum = H[j][kq] + v2 * H[j][kq + 1] + v3 * H[j][kq + 2];
            H[j][kq] = H[j][kq] - sum * t1; H[j][kq + 1] = H[j][kq + 1] - sum * t2; H[j][kq + 2] = H[j][kq + 2] - sum * t3v;
          }
        } else if (nr == 2) {
          HQ_ROLLED for (int j = kq; j <= i2; ++j) {
            const double sum = H[kq][j] + v2 * H[kq + 1][j];
            H[kq][j] = H[kq][j] - sum * t1; H[kq + 1][j] = H[kq + 1][j] - sum * t2;
          }
          HQ_ROLLED for (int j = i1; j <= i; ++j) {
            const double sum = H[j][kq] + v2 * H[j][kq + 1];
            H[j][kq] = H[j][kq] - sum * t1; H[j][kq + 1] = H[j][kq + 1] - sum * t2;
          }
        }
      }
    }
    if (!converged) return i + 1;
    if (lq == i) { wr[i] = H[i][i]; wi[i] = 0.0; }
    else if (lq == i - 1) dlanv2(H[i - 1][i - 1], H[i - 1][i], H[i][i - 1], H[i][i], wr[i - 1], wi[i - 1], wr[i], wi[i]);
    kdefl = 0;
    i = lq - 1;
  }
  return 0;
}

}  // namespace hyq
#include "hyq_eig6.cuh"
#include "hyq_charpoly.cuh"
namespace hyq {

// eig_real<6> of a flux Jacobian: the register-resident path (hyq_eig6.cuh)
// when dgebal's search isolates columns 0 and 5 (pattern 1, the usual case on
// smooth states), else the general code; identical results either way.  No
// isolation at all (pattern 0: round-off-sized entries in the first column,
// common once the flow has developed) also goes to the general code: an
// unrolled register path for it made the step kernels slower through its
// code size, even in a pass over only such cells.
HQD void eig_real_jac(double (&h)[36], double (&wr)[6], double (&wi)[6]) {
  if (e6::pattern(h) != 1) {
    double J[6][6];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < 6; ++c) J[r][c] = h[r * 6 + c];
    eig_real<6>(J, wr, wi);
    return;
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) { wr[i] = 0.0; wi[i] = 0.0; }
  e6::apply_pattern1(h);
  e6::solve<2>(h, wr, wi);
}

// Pattern 1 only: false (nothing computed) for any other permutation, whose
// Jacobians the step kernels leave to a separate pass over listed cells.
HQD bool eig_real_jac_p1(double (&h)[36], double (&wr)[6], double (&wi)[6]) {
  if (e6::pattern(h) != 1) return false;
#pragma unroll
  for (int i = 0; i < 6; ++i) { wr[i] = 0.0; wi[i] = 0.0; }
  e6::apply_pattern1(h);
  e6::solve<2>(h, wr, wi);
  return true;
}

// Which eigen-solve code jac_eigs_t and the functions above it run:
// JAC_ANY the register path for pattern-1 Jacobians and the general code for
// the rest; JAC_P1 pattern-1 Jacobians only (any other defers the cell);
// JAC_GEN the general code for every Jacobian (one compact code path for a
// pass over cells most of whose Jacobians need it).  Identical results.
// JAC_CP (the learned wave-speed path) the register path for pattern-1
// Jacobians and, for the rest, the certified characteristic-polynomial solve
// of hyq_charpoly.cuh seeded by the predicted speeds; a Jacobian it cannot
// certify defers the cell, which then takes the general code (the LAPACK
// path) in the pass over listed cells.
enum JacMode { JAC_ANY = 0, JAC_P1 = 1, JAC_GEN = 2, JAC_CP = 3 };

// Predicted extreme eigenvalues of a plane's Jacobian (NaN: none) and the
// normalised margin by which the certified solve moves them outward.
struct Seeds { double lo, hi, margin; };
HQD Seeds no_seeds() { Seeds s; s.lo = qnan(); s.hi = qnan(); s.margin = 0.0; return s; }

// compute_jacobian_eigenvalues for one 15-moment slice: extreme real parts
// and max |imag|.  A non-finite Jacobian gives NaN (the reference's guard).
// Under JAC_P1 a Jacobian of another pattern sets `deferred` and leaves the
// rest unset.
struct EigOut { double vmin, vmax, imax; bool deferred; };
template <int MODE> HQN EigOut jac_eigs_t(const double* ma, const Seeds sd) {
  double r3[6], r5[6], r6[6];
  jacobian6_rows(ma, r3, r5, r6);
  double h[36];  // the Jacobian, row-major, held in registers
#pragma unroll
  for (int i = 0; i < 36; ++i) h[i] = 0.0;
  h[0 * 6 + 1] = 1.0; h[1 * 6 + 2] = 1.0; h[3 * 6 + 4] = 1.0;
  bool fin = true;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    h[2 * 6 + j] = r3[j]; h[4 * 6 + j] = r5[j]; h[5 * 6 + j] = r6[j];
    fin = fin && isfinite(r3[j]) && isfinite(r5[j]) && isfinite(r6[j]);
  }
  EigOut o;
  o.deferred = false;
  if (!fin) { o.vmin = qnan(); o.vmax = qnan(); o.imax = qnan(); return o; }
  double wr[6], wi[6];
  if (MODE == JAC_P1) {
    if (!eig_real_jac_p1(h, wr, wi)) { o.deferred = true; return o; }
  } else if (MODE == JAC_CP) {
    if (!eig_real_jac_p1(h, wr, wi)) {
      const cp::Extremes e = cp::extremes(r3, r5, r6, sd.lo, sd.hi, sd.margin);
      if (!e.ok) { o.deferred = true; return o; }
      o.vmin = e.vmin;
      o.vmax = e.vmax;
      o.imax = 0.0;
      return o;
    }
  } else if (MODE == JAC_GEN) {
    double J[6][6];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < 6; ++c) J[r][c] = h[r * 6 + c];
    eig_real<6>(J, wr, wi);
  } else {
    eig_real_jac(h, wr, wi);
  }
  // sort(real) with NaN last, first and last
  double mn = wr[0], mx = wr[0];
  bool anynan = (wr[0] != wr[0]);
#pragma unroll
  for (int q = 1; q < 6; ++q) {
    if (wr[q] != wr[q]) { anynan = true; continue; }
    if (mn != mn || wr[q] < mn) mn = wr[q];
    if (mx != mx || wr[q] > mx) mx = wr[q];
  }
  o.vmin = mn;
  o.vmax = anynan ? qnan() : mx;
  double im = fabs(wi[0]);
#pragma unroll
  for (int q = 1; q < 6; ++q) im = jmax(im, fabs(wi[q]));
  o.imax = im;
  return o;
}
template <int MODE> HQD EigOut jac_eigs_t(const double* ma) { return jac_eigs_t<MODE>(ma, no_seeds()); }
HQD EigOut jac_eigs(const double* ma) { return jac_eigs_t<JAC_ANY>(ma); }

// axis_moment_slice (src/utils/axis_moment_slice.jl:31-54), 0-based
__device__ constexpr int SLICE[4][15] = {{0, 5, 9, 12, 14, 1, 6, 10, 13, 2, 7, 11, 3, 8, 4},
                                         {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14},
                                         {0, 15, 19, 22, 24, 1, 16, 20, 23, 2, 17, 21, 3, 18, 4},
                                         {0, 15, 19, 22, 24, 5, 25, 31, 33, 9, 28, 34, 12, 30, 14}};
// eigenvalues6z planes: WU and WV argument orders
__device__ constexpr int WUI[15] = {0, 1, 2, 3, 4, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24};

// Reference correct_{uv,uw,vw}_plane on central moments C (35-order) for the
// coordinate pair (i, j) in {0,1,2}.
HQD void correct_plane(double* C, int i, int j, double Sij, double Si3, double Sj3, double Si4, double Sj4, double Sii_jj, double Cii, double Cjj) {
  const double Sijj = Sij * Sj3, Siij = Sij * Si3, Sijjj = Sij * Sj4, Siiij = Sij * Si4;
  const double s22min = (2.0 + 5.0 * Sj3 * Sij * Si3) / 6.0;
  if (Sii_jj < s22min) Sii_jj = s22min;
  const double si = sqrt(jmax(EPS, Cii)), sj = sqrt(jmax(EPS, Cjj));
  auto at = [&](int a, int b) {
    int e[3] = {0, 0, 0};
    e[i] += a; e[j] += b;
    return idx35(e[0], e[1], e[2]);
  };
  C[at(2, 1)] = Siij * (si * si) * sj;
  C[at(1, 2)] = Sijj * si * (sj * sj);
  C[at(3, 1)] = Siiij * (si * si * si) * sj;
  C[at(1, 3)] = Sijjj * si * (sj * sj * sj);
  C[at(2, 2)] = Sii_jj * (si * si) * (sj * sj);
}

// Moments whose flux-Jacobian eigenvalues are complex are corrected, rebuilt
// and re-realized (correct_moments_for_real_eigenvalues and the eigenvalues6z
// branch).  planes: bit0 = first slice (pair a), bit1 = second slice.
HQN void correct_for_real(const double* M, int pa_i, int pa_j, int pb_i, int pb_j, int planes, int flag2D, double Ma, double* Mout) {
  const double M000 = M[0];
  const double u = M[1] / M000, v = M[5] / M000, w = M[15] / M000;
  double C[35], S[35];
  raw_to_central_r(M, 1, C);
  central_to_std(C, S);
  const double Cd[3] = {C[2], C[9], C[19]};
  const double S3[3] = {S[3], S[12], S[22]}, S4v[3] = {S[4], S[14], S[24]};
  auto corr = [&](int i, int j) {
    const int ij = (i == 0 && j == 1) ? 6 : (i == 0 && j == 2) ? 16 : 25;   // S110, S101, S011
    const int iijj = (i == 0 && j == 1) ? 11 : (i == 0 && j == 2) ? 21 : 34; // S220, S202, S022
    correct_plane(C, i, j, S[ij], S3[i], S3[j], S4v[i], S4v[j], S[iijj], Cd[i], Cd[j]);
  };
  if (planes & 1) corr(pa_i, pa_j);
  if (planes & 2) corr(pb_i, pb_j);
  C[0] = 1.0;
  central_to_raw_r<35>(M000, u, v, w, C);
  flux_closure35(C, flag2D, Ma, nullptr, nullptr, nullptr, Mout);
}

// Outcome of the eigenvalue functions below when run in parts.
enum EigStatus { EIG_DONE = 0, EIG_DEFERRED = 1, EIG_NEEDS_FIX = 2 };

// eigenvalues6_hyperbolic_3D for axis 1 (x) or 2 (y).
// Moment n is read from M[n * ist] and written to Mr[n * ost] (the step
// kernels pass the cell's entry of the moment-major fields, stride N); M and
// Mr either do not overlap or are the same array with the same strides (in
// place: only corrected moments are written).  MODE as jac_eigs_t.  With CORR the whole function
// runs (EIG_DONE, or EIG_DEFERRED under JAC_P1); without it, a cell whose
// Jacobians have complex eigenvalues returns EIG_NEEDS_FIX before the
// correction, whose code (a closure with its realizability) is then not part
// of the caller.  vmin, vmax and Mr are complete only with EIG_DONE.
//
// park (optional): on EIG_DONE, the second Jacobian's (vmin, vmax) go to
// park[0], park[pst] when the moments were not corrected, NaN otherwise.
// Along y that Jacobian is the VW plane, which eigenvalues6z_s solves again
// from the same moments when it neither floors nor re-realizes them.
template <int MODE, bool CORR>
HQN int eigenvalues6_s(const double* M, int axis, int flag2D, double Ma, double& vmin, double& vmax, double* Mr, long long ist,
                       long long ost, int* planes = nullptr, double* park = nullptr, long long pst = 0, const Seeds sd = no_seeds()) {
  const int sa = axis == 1 ? 0 : 1, sb = axis == 1 ? 2 : 3;
  double a[15], b[15];
  for (int n = 0; n < 15; ++n) { a[n] = M[SLICE[sa][n] * ist]; b[n] = M[SLICE[sb][n] * ist]; }
  EigOut ea = jac_eigs_t<MODE>(a, sd);
  if (ea.deferred) return EIG_DEFERRED;
  EigOut eb = jac_eigs_t<MODE>(b, sd);
  if (eb.deferred) return EIG_DEFERRED;
  const double thr = 1000.0 * EPS;
  const bool ca = ea.imax > thr, cb = eb.imax > thr;
  if (!CORR && (ca || cb)) {
    if (planes) *planes = (ca ? 1 : 0) | (cb ? 2 : 0);
    return EIG_NEEDS_FIX;
  }
  auto combine = [&]() {
    vmin = ea.vmin; vmax = ea.vmax;
    if (eb.vmin == eb.vmin || eb.vmax == eb.vmax) { vmin = jmin(vmin, eb.vmin); vmax = jmax(vmax, eb.vmax); }
  };
  combine();
  if (Mr != M) {  // in place (Mr == M, same strides) the moments are already there
#pragma unroll
    for (int n = 0; n < 35; ++n) Mr[n * ost] = M[n * ist];
  }
  if (park) {
    const bool fixed = ca || cb;
    park[0] = fixed ? qnan() : eb.vmin;
    park[pst] = fixed ? qnan() : eb.vmax;
  }
  if constexpr (CORR) {
    if (ca || cb) {
      double Ml[35], Mc[35];
      for (int n = 0; n < 35; ++n) Ml[n] = M[n * ist];
      // pair a is always the UV plane; pair b is UW (x) or VW (y)
      correct_for_real(Ml, 0, 1, axis == 1 ? 0 : 1, 2, (ca ? 1 : 0) | (cb ? 2 : 0), flag2D, Ma, Mc);
      for (int n = 0; n < 15; ++n) { a[n] = Mc[SLICE[sa][n]]; b[n] = Mc[SLICE[sb][n]]; }
      ea = jac_eigs_t<MODE>(a);
      if (ea.deferred) return EIG_DEFERRED;
      eb = jac_eigs_t<MODE>(b);
      if (eb.deferred) return EIG_DEFERRED;
      combine();
      for (int n = 0; n < 35; ++n) Mr[n * ost] = Mc[n];
    }
  }
  return EIG_DONE;
}
HQD void eigenvalues6(const double* M, int axis, int flag2D, double Ma, double& vmin, double& vmax, double* Mr, long long ist = 1,
                      long long ost = 1) {
  eigenvalues6_s<JAC_ANY, true>(M, axis, flag2D, Ma, vmin, vmax, Mr, ist, ost);
}

// The end of eigenvalues6 for a cell whose planes need the correction
// (planes as eigenvalues6_s reported them): the corrected moments and their
// speeds, the same results as the complete function.
template <int MODE>
HQN void eigenvalues6_corrected(const double* M, int axis, int planes, int flag2D, double Ma, double& vmin, double& vmax, double* Mr,
                                long long ist, long long ost, double* park = nullptr, long long pst = 0) {
  if (park) { park[0] = qnan(); park[pst] = qnan(); }
  const int sa = axis == 1 ? 0 : 1, sb = axis == 1 ? 2 : 3;
  double Ml[35], Mc[35], a[15], b[15];
  for (int n = 0; n < 35; ++n) Ml[n] = M[n * ist];
  correct_for_real(Ml, 0, 1, axis == 1 ? 0 : 1, 2, planes, flag2D, Ma, Mc);
  for (int n = 0; n < 15; ++n) { a[n] = Mc[SLICE[sa][n]]; b[n] = Mc[SLICE[sb][n]]; }
  const EigOut ea = jac_eigs_t<MODE>(a), eb = jac_eigs_t<MODE>(b);
  vmin = ea.vmin; vmax = ea.vmax;
  if (eb.vmin == eb.vmin || eb.vmax == eb.vmax) { vmin = jmin(vmin, eb.vmin); vmax = jmax(vmax, eb.vmax); }
  for (int n = 0; n < 35; ++n) Mr[n * ost] = Mc[n];
}

// Which of eigenvalues6's two planes need the complex-eigenvalue correction
// (bit 0: first slice, bit 1: second), from the same Jacobians and the same
// test; phase E only needs the corrected moments, so its kernels decide here
// and leave the corrections to a separate pass over the flagged cells.
// -1 when MODE defers a Jacobian (JAC_P1).
template <int MODE> HQN int eigenvalues6_flags_t(const double* M, int axis, long long ist, const Seeds sd = no_seeds()) {
  const int sa = axis == 1 ? 0 : 1, sb = axis == 1 ? 2 : 3;
  double a[15], b[15];
  for (int n = 0; n < 15; ++n) { a[n] = M[SLICE[sa][n] * ist]; b[n] = M[SLICE[sb][n] * ist]; }
  const EigOut ea = jac_eigs_t<MODE>(a, sd);
  if (ea.deferred) return -1;
  const EigOut eb = jac_eigs_t<MODE>(b, sd);
  if (eb.deferred) return -1;
  const double thr = 1000.0 * EPS;
  return (ea.imax > thr ? 1 : 0) | (eb.imax > thr ? 2 : 0);
}

// eigenvalues6z_hyperbolic_3D (strides, MODE, CORR and the outcome as
// eigenvalues6_s; without CORR the negative-variance re-realization also
// returns EIG_NEEDS_FIX).  parked (optional): the VW-plane speeds that the y
// stage parked for these moments (eigenvalues6_s park); used instead of
// solving that Jacobian again when the moments go in unchanged and the pair
// is not NaN, NaN (the same numbers either way).
template <int MODE, bool CORR>
HQN int eigenvalues6z_s(const double* M, int flag2D, double Ma, int positivity, double& vmin, double& vmax, double* Mr, long long ist,
                        long long ost, int* planes = nullptr, const double* parked = nullptr, long long pst = 0,
                        const Seeds sd = no_seeds()) {
  double Mw[35];
#pragma unroll
  for (int n = 0; n < 35; ++n) Mw[n] = M[n * ist];
  bool same = true;  // Mw equals the input moments
  if (positivity && Mw[0] <= 0.0) { Mw[0] = jmax(Mw[0], 1e-14); same = false; }
  if (positivity && Mw[0] > 1e-15) {
    const double m000 = Mw[0];
    const double vx = M[2 * ist] / m000 - sq(M[1 * ist] / m000), vy = M[9 * ist] / m000 - sq(M[5 * ist] / m000),
                 vz = M[19 * ist] / m000 - sq(M[15 * ist] / m000);
    if (vx < 0.0 || vy < 0.0 || vz < 0.0) {
      same = false;
      if constexpr (CORR) flux_closure35(M, flag2D, Ma, nullptr, nullptr, nullptr, Mw, ist, 1);
      else {
        if (planes) *planes = 0;  // the re-realization: only the complete function
        return EIG_NEEDS_FIX;
      }
    }
  }
  double a[15], b[15];
  for (int n = 0; n < 15; ++n) { a[n] = Mw[WUI[n]]; b[n] = Mw[SLICE[3][n]]; }
  EigOut ea = jac_eigs_t<MODE>(a, sd);
  if (ea.deferred) return EIG_DEFERRED;
  EigOut eb;
  if (parked && same && !(parked[0] != parked[0] && parked[pst] != parked[pst])) {
    // the y stage did not correct these moments, so its VW Jacobian had no
    // eigenvalue with |imag| above the threshold
    eb.vmin = parked[0]; eb.vmax = parked[pst]; eb.imax = 0.0; eb.deferred = false;
  } else {
    eb = jac_eigs_t<MODE>(b, sd);
    if (eb.deferred) return EIG_DEFERRED;
  }
  const double thr = 1000.0 * EPS;
  const bool ca = ea.imax > thr, cb = eb.imax > thr;
  if (!CORR && (ca || cb)) {
    if (planes) *planes = (ca ? 1 : 0) | (cb ? 2 : 0);
    return EIG_NEEDS_FIX;
  }
  // Mr: the input with its density floored or, after the negative-variance
  // re-realization, that closure -- Mw in both cases
#pragma unroll
  for (int n = 0; n < 35; ++n) Mr[n * ost] = Mw[n];
  vmin = jmin(ea.vmin, eb.vmin);
  vmax = jmax(ea.vmax, eb.vmax);
  if constexpr (CORR) {
    if (ca || cb) {
      double Ml[35], Mc[35];
      for (int n = 0; n < 35; ++n) Ml[n] = M[n * ist];
      correct_for_real(Ml, 0, 2, 1, 2, (ca ? 1 : 0) | (cb ? 2 : 0), flag2D, Ma, Mc);
      for (int n = 0; n < 15; ++n) { a[n] = Mc[WUI[n]]; b[n] = Mc[SLICE[3][n]]; }
      ea = jac_eigs_t<MODE>(a);
      if (ea.deferred) return EIG_DEFERRED;
      eb = jac_eigs_t<MODE>(b);
      if (eb.deferred) return EIG_DEFERRED;
      vmin = jmin(ea.vmin, eb.vmin);
      vmax = jmax(ea.vmax, eb.vmax);
      for (int n = 0; n < 35; ++n) Mr[n * ost] = Mc[n];
    }
  }
  return EIG_DONE;
}
HQD void eigenvalues6z(const double* M, int flag2D, double Ma, int positivity, double& vmin, double& vmax, double* Mr, long long ist = 1,
                       long long ost = 1) {
  eigenvalues6z_s<JAC_ANY, true>(M, flag2D, Ma, positivity, vmin, vmax, Mr, ist, ost);
}

// The end of eigenvalues6z for a cell whose planes need the correction
// (the correction starts from the input moments, not the floored ones)
template <int MODE>
HQN void eigenvalues6z_corrected(const double* M, int planes, int flag2D, double Ma, double& vmin, double& vmax, double* Mr,
                                 long long ist, long long ost) {
  double Ml[35], Mc[35], a[15], b[15];
  for (int n = 0; n < 35; ++n) Ml[n] = M[n * ist];
  correct_for_real(Ml, 0, 2, 1, 2, planes, flag2D, Ma, Mc);
  for (int n = 0; n < 15; ++n) { a[n] = Mc[WUI[n]]; b[n] = Mc[SLICE[3][n]]; }
  const EigOut ea = jac_eigs_t<MODE>(a), eb = jac_eigs_t<MODE>(b);
  vmin = jmin(ea.vmin, eb.vmin);
  vmax = jmax(ea.vmax, eb.vmax);
  for (int n = 0; n < 35; ++n) Mr[n * ost] = Mc[n];
}

// closure_and_eigenvalues with N = 2: extreme eigenvalues of the 3x3 Jacobi
// matrix (symmetric tridiagonal when both b >= 0; otherwise through the real
// matrix with the same characteristic polynomial).
HQN void closure_eigs(double m0, double m1, double m2, double m3, double m4, double& vmin, double& vmax) {
  // Chebyshev recurrence
  const double a0 = m1 / m0;
  const double s21 = m0, s22 = m1, s23 = m2, s24 = m3, s25 = m4;
  const double r32 = s23 - a0 * s22, r33 = s24 - a0 * s23, r34 = s25 - a0 * s24;
  const double a1 = r33 / r32 - s22 / s21;
  const double b1 = r32 / s21;
  const double r43 = r34 - a1 * r33 - b1 * s23;
  double b2 = r43 / r32;
  const double a2 = (a0 + a1) / 2.0;
  b2 = b2 * 5.0 / 2.0;
  if (!(isfinite(a0) && isfinite(a1) && isfinite(a2) && isfinite(b1) && isfinite(b2))) { vmin = qnan(); vmax = qnan(); return; }
  if (b1 >= 0.0 && b2 >= 0.0) {
    // cyclic Jacobi; from the fourth sweep on, an off-diagonal entry too small
    // to change either diagonal entry (|d| + 100|e| == |d|) is set to zero
    // (Rutishauser's threshold rule).  p, q and kk are unrolled so that A
    // stays in registers.
    double A[3][3] = {{a0, sqrt(b1), 0.0}, {sqrt(b1), a1, sqrt(b2)}, {0.0, sqrt(b2), a2}};
    for (int sweep = 0; sweep < 60; ++sweep) {
      const double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
      if (off == 0.0) break;
#pragma unroll
      for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = p + 1; q < 3; ++q) {
          if (A[p][q] == 0.0) continue;
          if (sweep >= 3) {
            const double g = 100.0 * fabs(A[p][q]);
            if (fabs(A[p][p]) + g == fabs(A[p][p]) && fabs(A[q][q]) + g == fabs(A[q][q])) {
              A[p][q] = 0.0; A[q][p] = 0.0;
              continue;
            }
          }
          const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
          double t = jsign(theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
          if (theta == 0.0) t = 1.0;
          const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
          for (int kk = 0; kk < 3; ++kk) { const double akp = A[kk][p], akq = A[kk][q]; A[kk][p] = c * akp - s * akq; A[kk][q] = s * akp + c * akq; }
#pragma unroll
          for (int kk = 0; kk < 3; ++kk) { const double apk = A[p][kk], aqk = A[q][kk]; A[p][kk] = c * apk - s * aqk; A[q][kk] = s * apk + c * aqk; }
        }
    }
    vmin = jmin(jmin(A[0][0], A[1][1]), A[2][2]);
    vmax = jmax(jmax(A[0][0], A[1][1]), A[2][2]);
    return;
  }
  double R[3][3] = {{a0, b1, 0.0}, {1.0, a1, b2}, {0.0, 1.0, a2}};
  double wr[3], wi[3];
  eig_real<3>(R, wr, wi);
  vmin = jmin(jmin(wr[0], wr[1]), wr[2]);
  vmax = jmax(jmax(wr[0], wr[1]), wr[2]);
}

// collision35: BGK relaxation toward the isotropic Gaussian.
HQD void collision35(double* M, double dt, double Kn, int positivity) {
  const double rho = M[0];
  const double u = M[1] / rho, v = M[5] / rho, w = M[15] / rho;
  const double C200 = M[2] / rho - u * u, C020 = M[9] / rho - v * v, C002 = M[19] / rho - w * w;
  double Th = (C200 + C020 + C002) / 3.0;
  if (positivity) Th = jmax(Th, 1e-14);
  const double tc = Kn / (rho * sqrt(Th) * 2.0);
  // central moments of the isotropic Gaussian: A = sqrt(Th) I,
  // C_ijk = S_ijk a^i a^j a^k with S the standard-normal moments.
  const double a = sqrt(Th);
  const double p2 = a * a, p3 = a * a * a, p4 = p2 * p2;
  const double pw[5] = {1.0, a, p2, p3, p4};
  double C[35];
#pragma unroll
  for (int n = 0; n < 35; ++n) {
    const int i = ex_i(n), j = ex_j(n), k = ex_k(n);
    const double zi = (i == 0) ? 1.0 : (i == 2) ? 1.0 : (i == 4) ? 3.0 : 0.0;
    const double zj = (j == 0) ? 1.0 : (j == 2) ? 1.0 : (j == 4) ? 3.0 : 0.0;
    const double zk = (k == 0) ? 1.0 : (k == 2) ? 1.0 : (k == 4) ? 3.0 : 0.0;
    C[n] = zi * zj * zk * pw[i] * pw[j] * pw[k];
  }
  C[0] = 1.0;
  central_to_raw_r<35>(rho, u, v, w, C);
  const double e = hexp(-dt / tc);
#pragma unroll
  for (int n = 0; n < 35; ++n) M[n] = C[n] - e * (C[n] - M[n]);
}

}  // namespace hyq
