// Host (g++) build of the device per-cell code: the CPU tests compare it bit
// for bit with the oracle, so arithmetic divergence between the CUDA path and
// the checker is caught without a GPU.  Test infrastructure only.
#include <cmath>
#include <cstring>
#include <limits>
using std::sqrt; using std::fabs; using std::isfinite; using std::isinf; using std::signbit; using std::rint; using std::ldexp; using std::frexp; using std::fmax; using std::fma;
static inline double __longlong_as_double(long long x) { double d; std::memcpy(&d, &x, 8); return d; }
#define __device__
#define __forceinline__ inline
#define __noinline__
#define __host__
#include "hyq_eigen.cuh"
using namespace hyq;
extern "C" {
void sh_flux(const double* m, int flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr) { flux_closure35(m, flag2D, Ma, Fx, Fy, Fz, Mr); }
// the realized moments alone (no flux wanted: the variant without the
// fifth-order work)
void sh_realized(const double* m, int flag2D, double Ma, double* Mr) { flux_closure35(m, flag2D, Ma, nullptr, nullptr, nullptr, Mr); }
void sh_eig(const double* m, int axis, int flag2D, double Ma, int pos, double* v, double* Mr) {
  if (axis == 3) eigenvalues6z(m, flag2D, Ma, pos, v[0], v[1], Mr); else eigenvalues6(m, axis, flag2D, Ma, v[0], v[1], Mr);
}
// the parts the step kernels run before the correction pass: gen = 0 the
// pattern-1-only variant, 1 the general code; 0 done, 1 deferred, 2
// correction needed (outputs then incomplete; *planes: the planes to
// correct, 0 = only the complete function)
int sh_eig_part(const double* m, int axis, int flag2D, double Ma, int pos, int gen, double* v, double* Mr, int* planes) {
  if (gen) {
    if (axis == 3) return eigenvalues6z_s<JAC_GEN, false>(m, flag2D, Ma, pos, v[0], v[1], Mr, 1, 1, planes);
    return eigenvalues6_s<JAC_GEN, false>(m, axis, flag2D, Ma, v[0], v[1], Mr, 1, 1, planes);
  }
  if (axis == 3) return eigenvalues6z_s<JAC_P1, false>(m, flag2D, Ma, pos, v[0], v[1], Mr, 1, 1, planes);
  return eigenvalues6_s<JAC_P1, false>(m, axis, flag2D, Ma, v[0], v[1], Mr, 1, 1, planes);
}
// the y stage parking its VW-plane speeds and the z stage reusing them, on
// the y stage's output, against the z stage solving everything (out[0..1]
// and out[2..1+35]: with reuse; out[37..38], out[39..73]: without); returns
// 1 when the parked pair was usable (not NaN, NaN)
int sh_yz_park(const double* m, int pos, double* out) {
  double My[35], park[2], lo, hi;
  eigenvalues6_s<JAC_ANY, true>(m, 2, 0, 0.0, lo, hi, My, 1, 1, nullptr, park, 1);
  eigenvalues6z_s<JAC_ANY, true>(My, 0, 0.0, pos, out[0], out[1], out + 2, 1, 1, nullptr, park, 1);
  eigenvalues6z_s<JAC_ANY, true>(My, 0, 0.0, pos, out[37], out[38], out + 39, 1, 1);
  return (park[0] != park[0] && park[1] != park[1]) ? 0 : 1;
}
// the correction pass from the reported planes
void sh_eig_corrected(const double* m, int axis, int planes, int flag2D, double Ma, double* v, double* Mr) {
  if (axis == 3) eigenvalues6z_corrected<JAC_GEN>(m, planes, flag2D, Ma, v[0], v[1], Mr, 1, 1);
  else eigenvalues6_corrected<JAC_GEN>(m, axis, planes, flag2D, Ma, v[0], v[1], Mr, 1, 1);
}
int sh_eig_flags(const double* m, int axis, int mode) {
  if (mode == 1) return eigenvalues6_flags_t<JAC_P1>(m, axis, 1);
  if (mode == 2) return eigenvalues6_flags_t<JAC_GEN>(m, axis, 1);
  return eigenvalues6_flags_t<JAC_ANY>(m, axis, 1);
}
void sh_closure(const double* mom, double* v) { closure_eigs(mom[0], mom[1], mom[2], mom[3], mom[4], v[0], v[1]); }
void sh_coll(double* m, double dt, double Kn, int pos) { collision35(m, dt, Kn, pos); }
// div_by against plain division on n pseudo-random operand pairs (exponents
// within +-e of 1, significands random or all ones); returns the mismatches
long long sh_div_check(long long n, int e, unsigned long long seed) {
  unsigned long long x = seed | 1ull;
  auto next = [&]() { x ^= x << 13; x ^= x >> 7; x ^= x << 17; return x; };
  auto mk = [&](int mode) {
    unsigned long long m = next() & 0xFFFFFFFFFFFFFull;
    if (mode == 1) m = 0xFFFFFFFFFFFFFull;
    const int ex = int(next() % (unsigned long long)(2 * e + 1)) - e;
    unsigned long long b = ((unsigned long long)(ex + 1023) << 52) | m | ((next() & 1) << 63);
    double v; std::memcpy(&v, &b, 8); return v;
  };
  long long bad = 0;
  for (long long i = 0; i < n; ++i) {
    const double d = mk(int(i & 1));
    double a = mk(int((i >> 1) & 1));
    if ((i & 15) == 3) a = 0.0;
    if ((i & 15) == 7) a = -0.0;
    const double q1 = div_by(a, d, 1.0 / d), q2 = a / d;
    if (std::memcmp(&q1, &q2, 8) != 0) ++bad;
  }
  return bad;
}
// eig_real<6> and the register-resident flux-Jacobian path on the same
// matrix: out[0..11] = general (wr, wi), out[12..23] = fast path, out[24] =
// the permutation pattern the fast path recognised (-1: none, general code).
void sh_eig6_both(const double* A, double* out) {
  double J[6][6], K[6][6], h[36];
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) { J[i][j] = K[i][j] = A[i * 6 + j]; h[i * 6 + j] = A[i * 6 + j]; }
  double wr[6], wi[6];
  eig_real<6>(J, wr, wi);
  for (int i = 0; i < 6; ++i) { out[i] = wr[i]; out[6 + i] = wi[i]; }
  eig_real_jac(h, wr, wi);
  for (int i = 0; i < 6; ++i) { out[12 + i] = wr[i]; out[18 + i] = wi[i]; }
  double h2[36];
  for (int i = 0; i < 36; ++i) h2[i] = A[i];
  out[24] = e6::pattern(h2);
}
// characteristic polynomial of a flux Jacobian (row-major 6 x 6 with the
// unit rows of jacobian6): c[0..6]
void sh_cp_charpoly(const double* A, double* c) {
  double cc[7];
  cp::charpoly(A + 12, A + 24, A + 30, cc);
  for (int k = 0; k < 7; ++k) c[k] = cc[k];
}
// certified extremes: out = {ok, vmin, vmax, its}
void sh_cp_extremes(const double* A, double lo_seed, double hi_seed, double margin, double* out) {
  const cp::Extremes e = cp::extremes(A + 12, A + 24, A + 30, lo_seed, hi_seed, margin);
  out[0] = e.ok ? 1.0 : 0.0; out[1] = e.vmin; out[2] = e.vmax; out[3] = e.its;
}
// the step's own exp and cbrt (hyq_cell.cuh) on n arguments
void sh_hexp_n(const double* x, double* y, long long n) { for (long long i = 0; i < n; ++i) y[i] = hexp(x[i]); }
void sh_hcbrt_n(const double* x, double* y, long long n) { for (long long i = 0; i < n; ++i) y[i] = hcbrt(x[i]); }
// realizable_3D on the 28 standardized moments (enum order), in place
int sh_realizable_3d(double* a28) { return realizable_3D(a28); }
// phase [A] of one cell as the step kernels run it on the plain path
// (cp = 0) or the certified path (cp = 1: the certified solve where it
// certifies, the complete LAPACK-path function for the cells it leaves):
// v[6] the six Jacobian extremes (x, y, z), Mr the stage output
void sh_phaseA_eigs(const double* m, int cp, double* v, double* Mr) {
  double a[35], b[35], c[35];
  for (int n = 0; n < 35; ++n) a[n] = m[n];
  int planes = 0;
  if (!cp || eigenvalues6_s<JAC_CP, false>(a, 1, 0, 1.0, v[0], v[1], b, 1, 1, &planes) != EIG_DONE)
    eigenvalues6(a, 1, 0, 1.0, v[0], v[1], b);
  if (!cp || eigenvalues6_s<JAC_CP, false>(b, 2, 0, 1.0, v[2], v[3], c, 1, 1, &planes) != EIG_DONE)
    eigenvalues6(b, 2, 0, 1.0, v[2], v[3], c);
  if (!cp || eigenvalues6z_s<JAC_CP, false>(c, 0, 1.0, 1, v[4], v[5], Mr, 1, 1, &planes) != EIG_DONE)
    eigenvalues6z(c, 0, 1.0, 1, v[4], v[5], Mr);
}
// the complex-eigenvalue flags of phase [E] along `axis` on the certified
// path (the certified solve, else the general code)
int sh_flags_cp(const double* m, int axis) {
  const int f = eigenvalues6_flags_t<JAC_CP>(m, axis, 1);
  return f >= 0 ? f : eigenvalues6_flags_t<JAC_GEN>(m, axis, 1);
}
}
