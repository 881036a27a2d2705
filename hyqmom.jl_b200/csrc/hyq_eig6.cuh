// Register-resident fast path of eig_real<6> for the flux Jacobian.
//
// LAPACK's balancing (dgebal) isolates columns 0 and 5 of almost every
// 6 x 6 flux Jacobian of the closure (their off-diagonal entries are exactly
// zero; measured on the crossing-jets states: 97 % of the Jacobians), which
// leaves the 4 x 4 active block of rows/columns 2..5.  For that case this file
// repeats the operations of eig_real<6> -- the same expressions in the same
// order -- with every matrix index a compile-time constant, so the 36 entries
// stay in registers instead of local memory (solve<K> also covers the
// unpermuted case, K = 0, which the device code leaves to the general path).
// Any other case goes to eig_real<6>.  tests/test_device_code_on_host.py checks the two bit for bit.
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

namespace hyq {
namespace e6 {

// flat index of (r, c); indices of accesses that a runtime guard never
// executes may fall outside the matrix and are folded to 0
__host__ __device__ constexpr int IX(int r, int c) { return (r < 0 || c < 0 || r > 5 || c > 5) ? 0 : r * 6 + c; }
#define H6(r, c) h[IX((r), (c))]

// nrm2 / dlarfg of eig_real with a compile-time length (same operation order)
template <int n> HQD double nrm2_s(const double* x) {
  double sq = 0.0;
#pragma unroll
  for (int i = 0; i < n; ++i) sq = sq + x[i] * x[i];
  if (sq >= 1e-280 && sq <= 1.7976931348623157e308) return sqrt(sq);
  double scale = 0.0, ssq = 1.0;
#pragma unroll
  for (int i = 0; i < n; ++i) {
    const double xi = x[i];
    if (xi != 0.0) {
      const double a = fabs(xi);
      if (scale < a) { const double r = scale / a; ssq = 1.0 + ssq * r * r; scale = a; }
      else { const double r = a / scale; ssq = ssq + r * r; }
    }
  }
  return scale * sqrt(ssq);
}
template <int n> HQD double dlarfg_s(double& alpha, double* x) {
  if (n <= 1) return 0.0;
  const double xnorm = nrm2_s<n - 1>(x);
  if (xnorm == 0.0) return 0.0;
  const double beta = -lsign(dlapy2(alpha, xnorm), alpha);
  const double tau = (beta - alpha) / beta;
  const double sc = 1.0 / (alpha - beta);
#pragma unroll
  for (int i = 0; i < n - 1; ++i) x[i] = x[i] * sc;
  alpha = beta;
  return tau;
}

// Which permutation dgebal's search makes: 1 = columns 0 and 5 isolated
// (swap(0,0), swap(5,1), ilo = 2, ihi = 5), 0 = none (ilo = 0, ihi = 5),
// -1 = anything else.  h is not modified.
HQD int pattern(const double (&h)[36]) {
  // row search with l = 5: a row j whose entries in columns 0..5 (except j)
  // are all zero
#pragma unroll
  for (int j = 5; j >= 0; --j) {
    bool zero = true;
#pragma unroll
    for (int i = 0; i <= 5; ++i)
      if (i != j && H6(j, i) != 0.0) zero = false;
    if (zero) return -1;
  }
  // column search with k = 0
  bool col0 = true;
#pragma unroll
  for (int i = 1; i <= 5; ++i)
    if (H6(i, 0) != 0.0) col0 = false;
  if (!col0) {
#pragma unroll
    for (int j = 1; j <= 5; ++j) {
      bool zero = true;
#pragma unroll
      for (int i = 0; i <= 5; ++i)
        if (i != j && H6(i, j) != 0.0) zero = false;
      if (zero) return -1;
    }
    return 0;
  }
  // k = 1: the first column j in 1..5 whose rows 1..5 (except j) are zero must be 5
#pragma unroll
  for (int j = 1; j <= 4; ++j) {
    bool zero = true;
#pragma unroll
    for (int i = 1; i <= 5; ++i)
      if (i != j && H6(i, j) != 0.0) zero = false;
    if (zero) return -1;
  }
  {
    bool zero = true;
#pragma unroll
    for (int i = 1; i <= 4; ++i)
      if (H6(i, 5) != 0.0) zero = false;
    if (!zero) return -1;
  }
  // after swap(5, 1) with k = 1: no column j in 2..5 may have rows 2..5
  // (except j) all zero.  Rows 1 and 5 exchange in columns 1..5, columns 1
  // and 5 exchange in rows 0..5; entry (i, j) for i, j >= 2 comes from
  // (i', j') with 5 <-> 1 swapped.
#pragma unroll
  for (int j = 2; j <= 5; ++j) {
    bool zero = true;
#pragma unroll
    for (int i = 2; i <= 5; ++i) {
      if (i == j) continue;
      const int si = (i == 5) ? 1 : i, sj = (j == 5) ? 1 : j;
      if (H6(si, sj) != 0.0) zero = false;
    }
    if (zero) return -1;
  }
  return 1;
}

// swap(5, 1) of dgebal with l = 5, k = 1: columns 1 and 5 in rows 0..5, then
// rows 1 and 5 in columns 1..5
HQD void apply_pattern1(double (&h)[36]) {
#pragma unroll
  for (int r = 0; r <= 5; ++r) { const double t = H6(r, 5); H6(r, 5) = H6(r, 1); H6(r, 1) = t; }
#pragma unroll
  for (int c = 1; c < 6; ++c) { const double t = H6(5, c); H6(5, c) = H6(1, c); H6(1, c) = t; }
}

// dgebal scaling over i = K..L (k = K, l = L).  Returns -1 on a non-finite
// norm (as eig_real).
template <int K, int L> HQD int scale(double (&h)[36]) {
  const double radix = 2.0, factor = 0.95;
  const double sfmin1 = SAFMIN / ULP, sfmax1 = 1.0 / sfmin1, sfmin2 = sfmin1 * radix, sfmax2 = 1.0 / sfmin2;
  double scal[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) scal[i] = 1.0;
  bool noconv = true;
  int guard = 0;
  while (noconv && guard++ < 1000) {
    noconv = false;
#pragma unroll
    for (int i = K; i <= L; ++i) {
      double col[6], row[6];
#pragma unroll
      for (int r = K; r <= L; ++r) col[r - K] = H6(r, i);
#pragma unroll
      for (int c2 = K; c2 <= L; ++c2) row[c2 - K] = H6(i, c2);
      double c = nrm2_s<L - K + 1>(col), r = nrm2_s<L - K + 1>(row);
      double ca = 0.0, ra = 0.0;
#pragma unroll
      for (int rr = 0; rr <= L; ++rr) ca = jmax(ca, fabs(H6(rr, i)));
#pragma unroll
      for (int cc = K; cc < 6; ++cc) ra = jmax(ra, fabs(H6(i, cc)));
      if (c == 0.0 || r == 0.0) continue;
      if (!isfinite(c + ca + r + ra)) return -1;
      double g = r / radix, f = 1.0;
      const double s = c + r;
      for (int guard2 = 0; guard2 < 2200 && !(c >= g || jmax(jmax(f, c), ca) >= sfmax2 || jmin(jmin(r, g), ra) <= sfmin2); ++guard2) {
        f = f * radix; c = c * radix; ca = ca * radix; r = r / radix; g = g / radix; ra = ra / radix;
      }
      g = c / radix;
      for (int guard3 = 0; guard3 < 2200 && !(g < r || jmax(r, ra) >= sfmax2 || jmin(jmin(jmin(f, c), g), ca) <= sfmin2); ++guard3) {
        f = f / radix; c = c / radix; g = g / radix; ca = ca / radix; r = r * radix; ra = ra * radix;
      }
      if ((c + r) >= factor * s) continue;
      if (f < 1.0 && scal[i] < 1.0) if (f * scal[i] <= sfmin1) continue;
      if (f > 1.0 && scal[i] > 1.0) if (scal[i] >= sfmax1 / f) continue;
      g = 1.0 / f;
      scal[i] = scal[i] * f;
      noconv = true;
#pragma unroll
      for (int cc = K; cc < 6; ++cc) H6(i, cc) = H6(i, cc) * g;
#pragma unroll
      for (int rr = 0; rr <= L; ++rr) H6(rr, i) = H6(rr, i) * f;
    }
  }
  return 0;
}

// dgehd2 over i = K..L-1 (ilo = K, ihi = L)
template <int K, int L> HQD void hessenberg(double (&h)[36]) {
#pragma unroll
  for (int i = K; i < L; ++i) {
    const int nr = L - i;
    double v[6];
    double alpha = H6(i + 1, i);
#pragma unroll
    for (int r = 0; r < 5; ++r)
      if (r < nr - 1) v[r + 1] = H6(i + 2 + r, i);
    double tau;
    switch (nr) {  // nr is a constant once i is unrolled
      case 1: tau = dlarfg_s<1>(alpha, &v[1]); break;
      case 2: tau = dlarfg_s<2>(alpha, &v[1]); break;
      case 3: tau = dlarfg_s<3>(alpha, &v[1]); break;
      case 4: tau = dlarfg_s<4>(alpha, &v[1]); break;
      default: tau = dlarfg_s<5>(alpha, &v[1]); break;
    }
    v[0] = 1.0;
    if (tau != 0.0) {
#pragma unroll
      for (int r = 0; r <= L; ++r) {
        double w = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c)
          if (c < nr) w = w + H6(r, i + 1 + c) * v[c];
#pragma unroll
        for (int c = 0; c < 5; ++c)
          if (c < nr) H6(r, i + 1 + c) = H6(r, i + 1 + c) - tau * w * v[c];
      }
#pragma unroll
      for (int c = i + 1; c < 6; ++c) {
        double w = 0.0;
#pragma unroll
        for (int r = 0; r < 5; ++r)
          if (r < nr) w = w + H6(i + 1 + r, c) * v[r];
#pragma unroll
        for (int r = 0; r < 5; ++r)
          if (r < nr) H6(i + 1 + r, c) = H6(i + 1 + r, c) - tau * v[r] * w;
      }
    }
    H6(i + 1, i) = alpha;
#pragma unroll
    for (int r = i + 2; r < 6; ++r) H6(r, i) = 0.0;
  }
}

// One deflation window of dlahqr (wantt = false) for the current bottom row
// I, ilo = K, ihi = L: iterate until H(lq, lq-1) is negligible with
// lq >= I-1, store the one or two converged eigenvalues and return lq - 1
// (the next I); return -100 - (I + 1) when the iteration limit is reached.
template <int I, int K, int L> HQD int qr_window(double (&h)[36], double (&wr)[6], double (&wi)[6], int& kdefl) {
  constexpr int nh = L - K + 1;
  const double smlnum = SAFMIN * (double(nh) / ULP);
  const double ulp = ULP;
  constexpr int itmax = 30 * (nh > 10 ? nh : 10);
  const double dat1 = 0.75, dat2 = -0.4375;
  int lq = K;
  bool converged = false;
  for (int its = 0; its <= itmax; ++its) {
    // scan for a negligible subdiagonal entry, kk = I down to lq + 1
    int kk = lq;
    bool found = false;
#pragma unroll
    for (int q = I; q > K; --q) {
      if (!found && q > lq) {
        if (fabs(H6(q, q - 1)) <= smlnum) { kk = q; found = true; }
        else {
          double tst = fabs(H6(q - 1, q - 1)) + fabs(H6(q, q));
          if (tst == 0.0) {
            if (q - 2 >= K) tst = tst + fabs(H6(q - 1, q - 2));
            if (q + 1 <= L) tst = tst + fabs(H6(q + 1, q));
          }
          if (fabs(H6(q, q - 1)) <= ulp * tst) {
            const double ab = jmax(fabs(H6(q, q - 1)), fabs(H6(q - 1, q)));
            const double ba = jmin(fabs(H6(q, q - 1)), fabs(H6(q - 1, q)));
            const double aa = jmax(fabs(H6(q, q)), fabs(H6(q - 1, q - 1) - H6(q, q)));
            const double bb = jmin(fabs(H6(q, q)), fabs(H6(q - 1, q - 1) - H6(q, q)));
            const double s = aa + ab;
            if (ba * (ab / s) <= jmax(smlnum, ulp * (bb * (aa / s)))) { kk = q; found = true; }
          }
        }
      }
    }
    lq = kk;
#pragma unroll
    for (int q = K + 1; q <= I; ++q)
      if (q == lq) H6(q, q - 1) = 0.0;
    if (lq >= I - 1) { converged = true; break; }
    ++kdefl;
    double h11, h12, h21, h22;
    if (kdefl % 20 == 0) {
      const double s = fabs(H6(I, I - 1)) + fabs(H6(I - 1, I - 2));
      h11 = dat1 * s + H6(I, I); h12 = dat2 * s; h21 = s; h22 = h11;
    } else if (kdefl % 10 == 0) {
      double s = 0.0, hll = 0.0;
#pragma unroll
      for (int q = K; q <= I - 2; ++q)
        if (q == lq) { s = fabs(H6(q + 1, q)) + fabs(H6(q + 2, q + 1)); hll = H6(q, q); }
      h11 = dat1 * s + hll; h12 = dat2 * s; h21 = s; h22 = h11;
    } else {
      h11 = H6(I - 1, I - 1); h21 = H6(I, I - 1); h12 = H6(I - 1, I); h22 = H6(I, I);
    }
    const double s = fabs(h11) + fabs(h12) + fabs(h21) + fabs(h22);
    double rt1r, rt1i, rt2r, rt2i;
    if (s == 0.0) { rt1r = rt1i = rt2r = rt2i = 0.0; }
    else {
      // four quotients by s through one reciprocal (div_by: bit-identical)
      const double rs = 1.0 / s;
      h11 = div_by(h11, s, rs); h21 = div_by(h21, s, rs); h12 = div_by(h12, s, rs); h22 = div_by(h22, s, rs);
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
    // m = I-2 down to lq: start of the bulge
    int m = lq;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    bool stop = false;
#pragma unroll
    for (int q = I - 2; q >= K; --q) {
      if (!stop && q >= lq) {
        double h21s = H6(q + 1, q);
        double s2 = fabs(H6(q, q) - rt2r) + fabs(rt2i) + fabs(h21s);
        const double rs2 = 1.0 / s2;
        h21s = div_by(H6(q + 1, q), s2, rs2);
        v0 = h21s * H6(q, q + 1) + (H6(q, q) - rt1r) * div_by(H6(q, q) - rt2r, s2, rs2) - rt1i * div_by(rt2i, s2, rs2);
        v1 = h21s * (H6(q, q) + H6(q + 1, q + 1) - rt1r - rt2r);
        v2 = h21s * H6(q + 2, q + 1);
        s2 = fabs(v0) + fabs(v1) + fabs(v2);
        const double rv = 1.0 / s2;
        v0 = div_by(v0, s2, rv); v1 = div_by(v1, s2, rv); v2 = div_by(v2, s2, rv);
        m = q;
        if (q == lq) stop = true;
        else {
          const double h00 = fabs(H6(q, q - 1)) * (fabs(v1) + fabs(v2));
          const double h11b = fabs(v0) * (fabs(H6(q - 1, q - 1)) + fabs(H6(q, q)) + fabs(H6(q + 1, q + 1)));
          if (h00 <= ulp * h11b) stop = true;
        }
      }
    }
    // double-shift sweep kq = m .. I-1
#pragma unroll
    for (int kq = K; kq <= I - 1; ++kq) {
      if (kq >= m) {
        const int nr = (I - kq + 1) < 3 ? (I - kq + 1) : 3;
        double v[3] = {v0, v1, v2};
        if (kq > m) {
#pragma unroll
          for (int r = 0; r < 3; ++r)
            if (r < nr) v[r] = H6(kq + r, kq - 1);
        }
        const double t1 = (nr == 3) ? dlarfg_s<3>(v[0], &v[1]) : dlarfg_s<2>(v[0], &v[1]);
        if (kq > m) {
          H6(kq, kq - 1) = v[0];
          H6(kq + 1, kq - 1) = 0.0;
          if (kq < I - 1) H6(kq + 2, kq - 1) = 0.0;
        } else if (m > lq) {
          H6(kq, kq - 1) = H6(kq, kq - 1) * (1.0 - t1);
        }
        const double vv2 = v[1], t2 = t1 * vv2;
        if (nr == 3) {
          const double vv3 = v[2], t3v = t1 * vv3;
#pragma unroll
          for (int j = kq; j <= I; ++j) {
            const double sum = H6(kq, j) + vv2 * H6(kq + 1, j) + vv3 * H6(kq + 2, j);
            H6(kq, j) = H6(kq, j) - sum * t1; H6(kq + 1, j) = H6(kq + 1, j) - sum * t2; H6(kq + 2, j) = H6(kq + 2, j) - sum * t3v;
          }
          const int jm = (kq + 3 < I) ? kq + 3 : I;
#pragma unroll
          for (int j = K; j <= 5; ++j) {
            if (j >= lq && j <= jm) {
              const double sum = H6(j, kq) + vv2 * H6(j, kq + 1) + vv3 * H6(j, kq + 2);
              H6(j, kq) = H6(j, kq) - sum * t1; H6(j, kq + 1) = H6(j, kq + 1) - sum * t2; H6(j, kq + 2) = H6(j, kq + 2) - sum * t3v;
            }
          }
        } else {
#pragma unroll
          for (int j = kq; j <= I; ++j) {
            const double sum = H6(kq, j) + vv2 * H6(kq + 1, j);
            H6(kq, j) = H6(kq, j) - sum * t1; H6(kq + 1, j) = H6(kq + 1, j) - sum * t2;
          }
#pragma unroll
          for (int j = K; j <= I; ++j) {
            if (j >= lq) {
              const double sum = H6(j, kq) + vv2 * H6(j, kq + 1);
              H6(j, kq) = H6(j, kq) - sum * t1; H6(j, kq + 1) = H6(j, kq + 1) - sum * t2;
            }
          }
        }
      }
    }
  }
  if (!converged) return -100 - (I + 1);
  if (lq == I) { wr[I] = H6(I, I); wi[I] = 0.0; }
  else if constexpr (I >= 1) {
    if (lq == I - 1) dlanv2(H6(I - 1, I - 1), H6(I - 1, I), H6(I, I - 1), H6(I, I), wr[I - 1], wi[I - 1], wr[I], wi[I]);
  }
  kdefl = 0;
  return lq - 1;
}

// eig_real<6> after a permutation that left ilo = K, ihi = 5 (h already
// permuted); wr, wi zeroed by the caller.  Same return codes as eig_real.
template <int K> HQD int solve(double (&h)[36], double (&wr)[6], double (&wi)[6]) {
  if (scale<K, 5>(h) != 0) return -1;
#pragma unroll
  for (int i = 0; i < K; ++i) { wr[i] = H6(i, i); wi[i] = 0.0; }
  hessenberg<K, 5>(h);
  int kdefl = 0;
  int i = 5;
  while (i >= K) {
    int next;
    switch (i) {
      case 5: next = qr_window<5, K, 5>(h, wr, wi, kdefl); break;
      case 4: next = qr_window<4, K, 5>(h, wr, wi, kdefl); break;
      case 3: next = qr_window<3, K, 5>(h, wr, wi, kdefl); break;
      case 2: next = qr_window<(K <= 2 ? 2 : 5), K, 5>(h, wr, wi, kdefl); break;
      case 1: next = qr_window<(K <= 1 ? 1 : 5), K, 5>(h, wr, wi, kdefl); break;
      default: next = qr_window<(K <= 0 ? 0 : 5), K, 5>(h, wr, wi, kdefl); break;
    }
    if (next <= -100) return -(next + 100);
    i = next;
  }
  return 0;
}

#undef H6
}  // namespace e6
}  // namespace hyq
