// Certified extreme eigenvalues of the 6 x 6 flux Jacobian from its
// characteristic polynomial: the solver of the learned wave-speed path.
//
// The reference takes the wave speeds of a plane as the extreme real parts of
// eigvals(jacobian6(...)) and corrects the moments when any eigenvalue has
// |imag| > 1000 eps (src/numerics/compute_jacobian_eigenvalues.jl:18-50,
// src/numerics/eigenvalues6_hyperbolic_3D.jl:22-56).  jacobian6 has unit rows
// 0, 1 and 3 (J[0][1] = J[1][2] = J[3][4] = 1, src/autogen/jacobian6.jl:52-57),
// so an eigenvector is (v0, lam v0, lam^2 v0, v3, lam v3, v5) and
// det(lam I - J) is the determinant of a 3 x 3 matrix of polynomials in lam
// built from the three remaining rows r3, r5, r6 -- a monic degree-6
// polynomial in about a hundred operations.
//
// The solver centres and scales it (x = (lam - s) / sig, s the mean and sig
// the RMS spread of the roots, both read off its coefficients), finds the two
// extreme roots by Newton's method from outside (monotone for a polynomial
// whose roots are all real) starting from the caller's seeds -- the learned
// network's predicted speeds -- or from a bound, deflates them and finds the
// remaining four, and then CERTIFIES the result: at seven points, one below
// the smallest root, one between each pair of neighbours and one above the
// largest, the polynomial must take the alternating signs + - + - + - + with
// |value| above a rigorous bound on its Horner rounding error plus the
// rounding error of the coefficients themselves (the determinant expansion,
// the shift and the scaling, bounded by evaluating the same expressions on
// absolute values).  By the intermediate value theorem that proves that the
// exact characteristic polynomial of J (the matrix as given) has six
// distinct real roots, one in each gap, so the extremes found are the
// extremes of the spectrum and no eigenvalue is complex.  The five interior sign values must also exceed
// GAP_VAL, which proves neighbouring roots at least 1.26e-6 apart
// (normalised): LAPACK's own rounding then cannot turn a pair complex, so a
// certified Jacobian is one the reference's complex test passes.
// Anything else (double roots, complex pairs, no convergence, non-finite
// data) is NOT certified, and the caller falls back to the LAPACK-path
// eigen-solve, which decides as the reference does.
//
// Arithmetic is FP64 in a fixed order: the Horner, Taylor-shift and
// deflation recurrences use explicit fused multiply-adds (fma, correctly
// rounded on the device and in the host's std::fma), everything else plain
// operations compiled without contraction, so the host build of this header
// gives the device's bits.  (The fused operations are this solve's own: its
// results are compared with the LAPACK path to round-off, not bit for bit.)
#pragma once

namespace hyq {
namespace cp {

constexpr int ITMAX = 40;              // Newton iterations per root
constexpr double NEWTON_TOL = 1e-12;   // extremes: |dx| <= TOL (1 + |x|), then one more step
constexpr double LOOSE_TOL = 1e-2;     // interior roots: only separating points are needed
constexpr double CERT_ERR = 40.0 * 2.220446049250313e-16;  // > gamma_12 of the Horner bound
// Rounding bounds of the coefficients (u = 2^-53): the charpoly expressions
// take at most 12 operations along any path (gamma_16 used), the Taylor
// shift 12 (gamma_16 used), the scaling by r^(6-k) up to 8 (gamma_10 used).
constexpr double G_CP = 16.0 * 1.1102230246251565e-16 / (1.0 - 16.0 * 1.1102230246251565e-16);
constexpr double G_SH = G_CP;
constexpr double G_SC = 10.0 * 1.1102230246251565e-16 / (1.0 - 10.0 * 1.1102230246251565e-16);
constexpr double ROOT_BOUND = 2.25;    // |x| <= sqrt(5) when all roots are real, sum x = 0, sum x^2 = 6
// |b(y)| at a point y between neighbouring roots r_k < y < r_k+1 bounds their
// distance from below: |b(y)| <= |y - r_k| |y - r_k+1| * D with D <= 5^4 the
// product of the other four distances (all roots within +-2.5), so
// |b(y)| >= GAP_VAL certifies r_k+1 - r_k >= sqrt(GAP_VAL / 625) = 1.26e-6
// (normalised).  At that distance LAPACK's rounding (a perturbation of order
// 1e-16 moves a close pair by about its square root, 1e-8) cannot make the
// pair complex.
constexpr double GAP_VAL = 1e-9;
// With converged interior roots, the smallest computed gap accepted
// (normalised): a pair that close stays real under LAPACK's rounding, which
// moves a near-double pair by about sqrt(eps |J|) ~ 1e-8.
constexpr double GAP_MIN = 1e-6;
// The extremes must also be well conditioned: the rounding bound of b at the
// root (Horner's and the coefficients') over |b'| -- the first-order error of
// the computed root -- at most EXT_ERR (normalised), so that the speeds
// differ from the exact extremes by at most 1e-12 of the spread.  An extreme
// in a tight cluster has a small b' and an error far above round-off, in
// this solve and in the LAPACK path alike, so the two would differ by more
// than round-off; such Jacobians go to the LAPACK path.  (The bound is
// pessimistic: on evolved states of the 256 x 256 x 128 run the certified
// extremes differ from the LAPACK path's by at most 9e-15 of the largest
// |eigenvalue|.)
#ifndef HQ_CP_EXT_ERR
#define HQ_CP_EXT_ERR 1e-12
#endif
constexpr double EXT_ERR = HQ_CP_EXT_ERR;

// c[0..6] (c[6] = 1) of det(lam I - J), J given by its rows 2 (r3), 4 (r5)
// and 5 (r6); rows 0, 1, 3 are the unit rows of jacobian6.
//   | A0 A1 A2 |   A0 = lam^3 - r3_2 lam^2 - r3_1 lam - r3_0,  A1 = -(r3_4 lam + r3_3),  A2 = -r3_5
//   | B0 B1 B2 |   B0 = -(r5_2 lam^2 + r5_1 lam + r5_0),     B1 = lam^2 - r5_4 lam - r5_3, B2 = -r5_5
//   | C0 C1 C2 |   C0 = -(r6_2 lam^2 + r6_1 lam + r6_0),     C1 = -(r6_4 lam + r6_3),      C2 = lam - r6_5
HQD void charpoly(const double* r3, const double* r5, const double* r6, double (&c)[7]) {
  // d = B1 C2 - B2 C1 (degree 3)
  const double d0 = (-r5[3]) * (-r6[5]) - (-r5[5]) * (-r6[3]);
  const double d1 = (-r5[3]) + (-r5[4]) * (-r6[5]) - (-r5[5]) * (-r6[4]);
  const double d2 = (-r5[4]) + (-r6[5]);
  const double d3 = 1.0;
  // e = B0 C2 - B2 C0 (degree 3)
  const double e0 = (-r5[0]) * (-r6[5]) - (-r5[5]) * (-r6[0]);
  const double e1 = (-r5[0]) + (-r5[1]) * (-r6[5]) - (-r5[5]) * (-r6[1]);
  const double e2 = (-r5[1]) + (-r5[2]) * (-r6[5]) - (-r5[5]) * (-r6[2]);
  const double e3 = (-r5[2]);
  // f = B0 C1 - B1 C0 (degree 4)
  const double f0 = (-r5[0]) * (-r6[3]) - (-r5[3]) * (-r6[0]);
  const double f1 = (-r5[0]) * (-r6[4]) + (-r5[1]) * (-r6[3]) - ((-r5[3]) * (-r6[1]) + (-r5[4]) * (-r6[0]));
  const double f2 = (-r5[1]) * (-r6[4]) + (-r5[2]) * (-r6[3]) - ((-r5[3]) * (-r6[2]) + (-r5[4]) * (-r6[1]) + (-r6[0]));
  const double f3 = (-r5[2]) * (-r6[4]) - ((-r5[4]) * (-r6[2]) + (-r6[1]));
  const double f4 = -(-r6[2]);
  // p = A0 d - A1 e + A2 f
  const double a0 = -r3[0], a1 = -r3[1], a2 = -r3[2];  // A0 = lam^3 + a2 lam^2 + a1 lam + a0
  const double b0 = -r3[3], b1 = -r3[4];               // A1 = b1 lam + b0
  const double g = -r3[5];                             // A2
  // A0 d (degree 6)
  const double p0 = a0 * d0;
  const double p1 = a0 * d1 + a1 * d0;
  const double p2 = a0 * d2 + a1 * d1 + a2 * d0;
  const double p3 = a0 * d3 + a1 * d2 + a2 * d1 + d0;
  const double p4 = a1 * d3 + a2 * d2 + d1;
  const double p5 = a2 * d3 + d2;
  // A1 e (degree 4)
  const double q0 = b0 * e0;
  const double q1 = b0 * e1 + b1 * e0;
  const double q2 = b0 * e2 + b1 * e1;
  const double q3 = b0 * e3 + b1 * e2;
  const double q4 = b1 * e3;
  c[0] = p0 - q0 + g * f0;
  c[1] = p1 - q1 + g * f1;
  c[2] = p2 - q2 + g * f2;
  c[3] = p3 - q3 + g * f3;
  c[4] = p4 - q4 + g * f4;
  c[5] = p5;
  c[6] = 1.0;
}

// The same expansion on absolute values (every term added): cabs[k] bounds
// the terms that make up c[k], so |computed c[k] - exact c[k]| <= G_CP cabs[k].
HQD void charpoly_abs(const double* r3, const double* r5, const double* r6, double (&cabs)[7]) {
  double R3[6], R5[6], R6[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) { R3[k] = fabs(r3[k]); R5[k] = fabs(r5[k]); R6[k] = fabs(r6[k]); }
  const double d0 = R5[3] * R6[5] + R5[5] * R6[3];
  const double d1 = R5[3] + R5[4] * R6[5] + R5[5] * R6[4];
  const double d2 = R5[4] + R6[5];
  const double e0 = R5[0] * R6[5] + R5[5] * R6[0];
  const double e1 = R5[0] + R5[1] * R6[5] + R5[5] * R6[1];
  const double e2 = R5[1] + R5[2] * R6[5] + R5[5] * R6[2];
  const double e3 = R5[2];
  const double f0 = R5[0] * R6[3] + R5[3] * R6[0];
  const double f1 = R5[0] * R6[4] + R5[1] * R6[3] + R5[3] * R6[1] + R5[4] * R6[0];
  const double f2 = R5[1] * R6[4] + R5[2] * R6[3] + R5[3] * R6[2] + R5[4] * R6[1] + R6[0];
  const double f3 = R5[2] * R6[4] + R5[4] * R6[2] + R6[1];
  const double f4 = R6[2];
  const double a0 = R3[0], a1 = R3[1], a2 = R3[2], b0 = R3[3], b1 = R3[4], g = R3[5];
  cabs[0] = a0 * d0 + b0 * e0 + g * f0;
  cabs[1] = a0 * d1 + a1 * d0 + b0 * e1 + b1 * e0 + g * f1;
  cabs[2] = a0 * d2 + a1 * d1 + a2 * d0 + b0 * e2 + b1 * e1 + g * f2;
  cabs[3] = a0 + a1 * d2 + a2 * d1 + d0 + b0 * e3 + b1 * e2 + g * f3;
  cabs[4] = a1 + a2 * d2 + d1 + b1 * e3 + g * f4;
  cabs[5] = a2 + d2;
  cabs[6] = 0.0;
}

// p(x) and p'(x) of the degree-N polynomial d[0..N] by Horner.
template <int N> HQD void horner2(const double* d, double x, double& p, double& dp) {
  p = d[N];
  dp = 0.0;
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    dp = fma(dp, x, p);
    p = fma(p, x, d[k]);
  }
}

// The monic degree-6 polynomial c centred and scaled: b(x) = c(s + sig x) /
// sig^6 with s = -c5 / 6 (mean root) and sig^2 = (a5^2 - 2 a4) / 6 (mean
// square deviation, a = c shifted to s), so that sum x_i = -b5 ~ 0 and
// sum x_i^2 = 6.  With x = (lam - s) r, r = 1 / sig as rounded, eb[k] bounds
// |b[k] - the exact coefficient| given |c[k] - exact c[k]| <= G_CP cabs[k]
// (the shift's and the scaling's rounding included).  False when the spread
// is not a positive finite number.
HQD bool normalize(const double (&c)[7], const double (&cabs)[7], double& s, double& sig, double (&b)[7], double (&eb)[7]) {
  double a[7], v[7];
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    a[k] = c[k];
    v[k] = G_CP * cabs[k] + G_SH * fabs(c[k]);
  }
  s = -c[5] / 6.0;
  const double as = fabs(s);
  // Taylor shift a(x) = c(x + s), repeated synthetic division; v the same
  // shift of the error terms with |s| (all terms positive)
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int k = 5; k >= i; --k) {
      a[k] = fma(s, a[k + 1], a[k]);
      v[k] = fma(as, v[k + 1], v[k]);
    }
  const double vv = (a[5] * a[5] - 2.0 * a[4]) / 6.0;
  if (!(vv > 0.0) || !(vv < 1.79769313486231571e308)) return false;
  sig = sqrt(vv);
  const double r = 1.0 / sig;
  double pw = 1.0;
  bool fin = true;
  b[6] = 1.0;
  eb[6] = 0.0;
#pragma unroll
  for (int k = 5; k >= 0; --k) {
    pw = pw * r;
    b[k] = a[k] * pw;
    eb[k] = (v[k] * pw + G_SC * fabs(b[k])) * (1.0 + 1e-12);
    fin = fin && isfinite(b[k]) && isfinite(eb[k]);
  }
  return fin;
}

// Newton's method on the degree-N polynomial d from x; true once a step is
// below tol (one more step is then taken), false when it does not converge
// within ITMAX steps or meets a zero / non-finite derivative.
template <int N> HQD bool newton(const double* d, double& x, double tol, int& its) {
#pragma unroll 1
  for (int it = 0; it < ITMAX; ++it) {
    double p, dp;
    horner2<N>(d, x, p, dp);
    ++its;
    if (!(dp != 0.0)) return false;
    const double dx = p / dp;
    x = x - dx;
    if (!(fabs(dx) > tol * (1.0 + fabs(x)))) {
      horner2<N>(d, x, p, dp);
      ++its;
      if (dp != 0.0) x = x - p / dp;
      return isfinite(x);
    }
  }
  return false;
}

// Upper bound of the roots of the monic degree-N polynomial d when they are
// all real: mean + sqrt((N - 1) variance), from the sum and the sum of
// squares of the roots (-d[N-1] and d[N-1]^2 - 2 d[N-2]); slightly inflated.
// NaN when the variance is negative (complex roots), which jmin then skips.
template <int N> HQD double upper_bound(const double* d) {
  const double m = -d[N - 1] / double(N);
  const double s2 = d[N - 1] * d[N - 1] - 2.0 * d[N - 2];
  const double var = s2 / double(N) - m * m;
  return m + sqrt(double(N - 1) * var) * (1.0 + 1e-12) + 1e-12;
}

// One Newton step on the full polynomial b (polishes a root found on a
// deflated polynomial).
HQD double polish(const double (&b)[7], double x, int& its) {
  double p, dp;
  horner2<6>(b, x, p, dp);
  ++its;
  return (dp != 0.0) ? x - p / dp : x;
}

// q = d / (X - x), d of degree N (the remainder is dropped).
template <int N> HQD void deflate(const double* d, double x, double* q) {
  q[N - 1] = d[N];
#pragma unroll
  for (int k = N - 1; k >= 1; --k) q[k - 1] = fma(x, q[k], d[k]);
}

// Sign of the exact normalised polynomial at y, certified from the computed
// b: |b(y)| must exceed its Horner rounding error, the coefficients' error
// bound sum eb[k] |y|^k and the floor `floor_val`: +1 / -1, or 0.
HQD int certified_sign(const double (&b)[7], const double (&eb)[7], double y, double floor_val) {
  double p = b[6], bound = 1.0, ce = eb[6];
  const double ay = fabs(y);
#pragma unroll
  for (int k = 5; k >= 0; --k) {
    p = fma(p, y, b[k]);
    bound = bound * ay + fabs(b[k]);
    ce = ce * ay + eb[k];
  }
  const double err = jmax((CERT_ERR * bound + ce) * (1.0 + 1e-12), floor_val);
  if (p > err) return 1;
  if (p < -err) return -1;
  return 0;
}

HQD void cswap(double& a, double& b) {
  const double lo = a < b ? a : b, hi = a < b ? b : a;
  a = lo;
  b = hi;
}

// Result of a certified solve, in the normalised variable.
struct CpOut {
  double xmin, xmax;
  int its;   // polynomial evaluations spent
  bool ok;   // certified: six distinct real roots, the extremes are xmin and xmax
};

// The six roots of the normalised b, searched from the starting points xhi
// (above the largest root) and xlo (below the smallest), and the certificate.
// The extremes are converged to full precision; the four interior roots only
// need to lie within their gaps (they place the separating points), so their
// Newton iterations stop early and the last two come from the quadratic.
// The four interior roots of b between the extremes x6 < x1 (searched by
// Newton to tolerance `tol`, the last two from the quadratic) and the
// certificate.  tight = false: interior roots only placed (tol loose), the
// interior sign values must exceed GAP_VAL (a rigorous lower bound on every
// gap); tight = true: interior roots converged, their computed gaps must be
// at least GAP_MIN and the signs only beyond the rounding bound.
HQD bool interior_certify(const double (&b)[7], const double (&eb)[7], double x1, double x6, bool tight, int& its) {
  double d5[6], d4[5], d3[4], d2[3];
  deflate<6>(b, x1, d5);
  deflate<5>(d5, x6, d4);
  const double tol = tight ? NEWTON_TOL : LOOSE_TOL;
  // each interior search starts from the upper bound mean + sqrt((n-1) var)
  // of the deflated polynomial's roots (read off its monic coefficients)
  // when that is below the previous root
  double x2 = jmin(x1, upper_bound<4>(d4));
  if (!newton<4>(d4, x2, tol, its)) return false;
  if (tight) x2 = polish(b, x2, its);
  deflate<4>(d4, x2, d3);
  double x3 = jmin(x2, upper_bound<3>(d3));
  if (!newton<3>(d3, x3, tol, its)) return false;
  if (tight) x3 = polish(b, x3, its);
  deflate<3>(d3, x3, d2);
  // the last two from the quadratic, in the cancellation-free form
  const double disc = d2[1] * d2[1] - 4.0 * d2[2] * d2[0];
  if (!(disc > 0.0)) return false;
  const double sq = sqrt(disc);
  const double qq = -0.5 * (d2[1] + (d2[1] < 0.0 ? -sq : sq));
  if (!(qq != 0.0)) return false;
  double x4 = qq / d2[2], x5 = d2[0] / qq;
  if (tight) {
    x4 = polish(b, x4, its);
    x5 = polish(b, x5, its);
  }
  // ascending order of the interior four (a sorting network); the extremes
  // must lie outside them
  double r[6] = {x6, x5, x4, x3, x2, x1};
  cswap(r[1], r[2]); cswap(r[3], r[4]);
  cswap(r[1], r[3]); cswap(r[2], r[4]);
  cswap(r[2], r[3]);
  if (!(r[0] < r[1] && r[4] < r[5])) return false;
  bool ok = true;
  if (tight) {
#pragma unroll
    for (int k = 0; k < 5; ++k) ok = ok && (r[k + 1] - r[k] >= GAP_MIN);
    if (!ok) return false;
  }
  // alternating certified signs at the seven separating points
  double y[7];
  y[0] = r[0] - 0.5 * (r[1] - r[0]);
#pragma unroll
  for (int k = 1; k < 6; ++k) y[k] = 0.5 * (r[k - 1] + r[k]);
  y[6] = r[5] + 0.5 * (r[5] - r[4]);
#pragma unroll
  for (int k = 0; k < 7; ++k)
    ok = ok && (certified_sign(b, eb, y[k], (k == 0 || k == 6 || tight) ? 0.0 : GAP_VAL) == ((k & 1) ? -1 : 1));
  its += 7;
  return ok;
}

HQD CpOut solve(const double (&b)[7], const double (&eb)[7], double xhi, double xlo) {
  CpOut o;
  o.ok = false;
  o.its = 0;
  o.xmin = o.xmax = 0.0;
  double x1 = xhi, x6 = xlo;
  if (!newton<6>(b, x1, NEWTON_TOL, o.its)) return o;
  if (!newton<6>(b, x6, NEWTON_TOL, o.its)) return o;
  if (!(x6 < x1)) return o;
  // interior roots placed loosely first; a cluster (a near-double interior
  // pair, common in nearly Gaussian cells) needs them converged
  if (!interior_certify(b, eb, x1, x6, false, o.its) && !interior_certify(b, eb, x1, x6, true, o.its)) return o;
  // conditioning of the two extremes
  bool ok = true;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const double x = q ? x1 : x6;
    double p = b[6], dp = 0.0, bound = 1.0, ce = eb[6];
    const double ax = fabs(x);
#pragma unroll
    for (int k = 5; k >= 0; --k) {
      dp = fma(dp, x, p);
      p = fma(p, x, b[k]);
      bound = bound * ax + fabs(b[k]);
      ce = ce * ax + eb[k];
    }
    ok = ok && (CERT_ERR * bound + ce <= EXT_ERR * fabs(dp));
  }
  o.its += 2;
  if (!ok) return o;
  o.xmin = x6;
  o.xmax = x1;
  o.ok = true;
  return o;
}

// A seed x (in the normalised variable) is used as the start of the search
// for the largest root when b has no root at or above it: the coefficients of
// b(x + y) as a polynomial in y (the Taylor coefficients b^(k)(x) / k!) are
// all positive, so by Descartes' rule b(x + y) has no positive root.  For the
// smallest root the coefficients of b(x - y) must all be positive.  Otherwise
// (and for NaN seeds) the search starts from the bound, so a poor prediction
// costs a few evaluations and never a wrong start.
HQD bool taylor_signs(const double (&b)[7], double x, bool above) {
  double t[7];
#pragma unroll
  for (int k = 0; k < 7; ++k) t[k] = b[k];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int k = 5; k >= i; --k) t[k] = fma(x, t[k + 1], t[k]);
  bool ok = x == x && fabs(x) < 8.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) ok = ok && ((above || (k & 1) == 0) ? t[k] > 0.0 : t[k] < 0.0);
  return ok;
}
HQD double start_above(const double (&b)[7], double x) { return taylor_signs(b, x, true) ? x : ROOT_BOUND + fabs(b[5]); }
HQD double start_below(const double (&b)[7], double x) { return taylor_signs(b, x, false) ? x : -ROOT_BOUND - fabs(b[5]); }

// Extreme eigenvalues of the flux Jacobian (rows r3, r5, r6) when certified.
// lo_seed, hi_seed: predicted extreme eigenvalues (NaN for none); margin: the
// normalised distance by which the seeds are moved outward.  On success
// vmin, vmax hold the extremes; its counts polynomial evaluations.
struct Extremes {
  double vmin, vmax;
  int its;
  bool ok;
};
HQD Extremes extremes(const double* r3, const double* r5, const double* r6, double lo_seed, double hi_seed, double margin) {
  Extremes e;
  e.ok = false;
  e.its = 0;
  e.vmin = e.vmax = 0.0;
  double c[7], cabs[7], b[7], eb[7], s, sig;
  charpoly(r3, r5, r6, c);
  charpoly_abs(r3, r5, r6, cabs);
  if (!normalize(c, cabs, s, sig, b, eb)) return e;
  const double xhi = start_above(b, (hi_seed - s) / sig + margin);
  const double xlo = start_below(b, (lo_seed - s) / sig - margin);
  const CpOut o = solve(b, eb, xhi, xlo);
  e.its = o.its + 2;
  if (!o.ok) return e;
  e.vmin = s + sig * o.xmin;
  e.vmax = s + sig * o.xmax;
  e.ok = true;
  return e;
}

}  // namespace cp
}  // namespace hyq
