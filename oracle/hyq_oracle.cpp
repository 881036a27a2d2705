// C entry points of the HyQMOM ORACLE (test infrastructure only: imported by
// tests/, __graft_entry__.smoke() and the bench's CPU-baseline leg, never by
// the product).  The serial time step restates src/simulation_runner.jl:346-560
// for one rank: phases [A] closure + wave speeds, CFL dt, HLL x/y/z sweeps with
// the copy boundary handling of pas_HLL, the Strang combination, [E]
// realizability and [F] BGK collision.
//
// State layout: Julia column-major (Nx, Ny, Nz, 35), i fastest.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <atomic>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "hyq_oracle_eigen.hpp"

namespace hyqo {

// FP64 operation counter: +,-,*,/ count 1, sqrt/cbrt/exp count 1.
struct Counted {
  double v;
  static thread_local unsigned long long ops;
  Counted() : v(0) {}
  Counted(double x) : v(x) {}
  explicit operator double() const { return v; }
};
thread_local unsigned long long Counted::ops = 0;
inline Counted operator+(Counted a, Counted b) { ++Counted::ops; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++Counted::ops; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++Counted::ops; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++Counted::ops; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }
inline Counted sqrt(Counted a) { ++Counted::ops; return Counted(std::sqrt(a.v)); }
inline Counted cbrt(Counted a) { ++Counted::ops; return Counted(std::cbrt(a.v)); }
inline Counted exp(Counted a) { ++Counted::ops; return Counted(std::exp(a.v)); }
inline Counted fabs(Counted a) { return Counted(std::fabs(a.v)); }
}  // namespace hyqo
namespace std {
inline bool signbit(hyqo::Counted a) { return std::signbit(a.v); }
inline bool isfinite(hyqo::Counted a) { return std::isfinite(a.v); }
}  // namespace std

namespace hyqo {

struct Params {
  int Nx, Ny, Nz, flag2D, positivity;
  double Kn, Ma, CFL, dtmax, tmax, dx, dy, dz;
};

// Phase [A] for one cell (src/simulation_runner.jl:357-379).
template <class T> void phase_A(const T* m, const Params& P, T* Fx, T* Fy, T* Fz, T* Mr, T* vp /*6*/) {
  T a[35], b[35], c[35], fx[35], fy[35], fz[35];
  T Ma = T(P.Ma);
  flux_closure35(m, P.flag2D, Ma, fx, fy, fz, a);
  T v6xmin, v6xmax, v6ymin, v6ymax, v6zmin, v6zmax;
  eigenvalues6_hyperbolic_3D(a, 1, P.flag2D, Ma, v6xmin, v6xmax, b);
  eigenvalues6_hyperbolic_3D(b, 2, P.flag2D, Ma, v6ymin, v6ymax, c);
  eigenvalues6z_hyperbolic_3D(c, P.flag2D, Ma, P.positivity != 0, v6zmin, v6zmax, a);
  flux_closure35(a, P.flag2D, Ma, Fx, Fy, Fz, Mr);
  T mx[5] = {Mr[0], Mr[1], Mr[2], Mr[3], Mr[4]};
  T my[5] = {Mr[0], Mr[5], Mr[9], Mr[12], Mr[14]};
  T mz[5] = {Mr[0], Mr[15], Mr[19], Mr[22], Mr[24]};
  T Mp, v5xmin, v5xmax, v5ymin, v5ymax, v5zmin, v5zmax;
  closure_and_eigenvalues(mx, Mp, v5xmin, v5xmax);
  closure_and_eigenvalues(my, Mp, v5ymin, v5ymax);
  closure_and_eigenvalues(mz, Mp, v5zmin, v5zmax);
  vp[0] = jmin(v5xmin, v6xmin); vp[1] = jmax(v5xmax, v6xmax);
  vp[2] = jmin(v5ymin, v6ymin); vp[3] = jmax(v5ymax, v6ymax);
  vp[4] = jmin(v5zmin, v6zmin); vp[5] = jmax(v5zmax, v6zmax);
}

// Phase [E] for one cell (src/simulation_runner.jl:531-538).
template <class T> void phase_E(const T* m, const Params& P, T* out) {
  T a[35], b[35], c[35], fx[35], fy[35], fz[35];
  T Ma = T(P.Ma);
  T v0, v1;
  flux_closure35(m, P.flag2D, Ma, fx, fy, fz, a);
  eigenvalues6_hyperbolic_3D(a, 1, P.flag2D, Ma, v0, v1, b);
  eigenvalues6_hyperbolic_3D(b, 2, P.flag2D, Ma, v0, v1, c);
  flux_closure35(c, P.flag2D, Ma, fx, fy, fz, out);
}

}  // namespace hyqo

using namespace hyqo;

#ifdef HYQO_BRANCHES
namespace hyqo { long long g_branch_hits[BR_COUNT] = {0}; }
#endif

extern "C" {

int hyqo_abi_version(void) { return 1; }

int hyqo_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Branch-hit counters of the instrumented build (zeros otherwise): out[8]
// (hyqo::Branch order); reset = 1 zeroes them after reading.
void hyqo_branch_counts(long long* out, int reset) {
  for (int b = 0; b < BR_COUNT; ++b) {
#ifdef HYQO_BRANCHES
    out[b] = g_branch_hits[b];
    if (reset) g_branch_hits[b] = 0;
#else
    (void)reset;
    out[b] = 0;
#endif
  }
}

// Threads of the OpenMP loops from now on (1: the serial step).
void hyqo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}

void hyqo_initialize_m4_35(double rho, double u, double v, double w, double C200, double C110, double C101, double C020,
                           double C011, double C002, double* out) {
  initialize_m4_35<double>(rho, u, v, w, C200, C110, C101, C020, C011, C002, out);
}
void hyqo_m2cs4_35(const double* M, double* C4, double* S4) { m2cs4_35<double>(M, C4, S4); }
void hyqo_flux_closure35(const double* M, int flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr) {
  flux_closure35<double>(M, flag2D, Ma, Fx, Fy, Fz, Mr);
}
void hyqo_eigenvalues6(const double* M, int axis, int flag2D, double Ma, double* v, double* Mr) {
  eigenvalues6_hyperbolic_3D<double>(M, axis, flag2D, Ma, v[0], v[1], Mr);
}
void hyqo_eigenvalues6z(const double* M, int flag2D, double Ma, int positivity, double* v, double* Mr) {
  eigenvalues6z_hyperbolic_3D<double>(M, flag2D, Ma, positivity != 0, v[0], v[1], Mr);
}
void hyqo_closure_and_eigenvalues(const double* mom, double* out) {
  double m[5] = {mom[0], mom[1], mom[2], mom[3], mom[4]};
  closure_and_eigenvalues<double>(m, out[0], out[1], out[2]);
}
void hyqo_collision35(const double* M, double dt, double Kn, int positivity, double* out) {
  collision35<double>(M, dt, Kn, positivity != 0, out);
}
// pas_HLL on an (Np, 35) column-major block.
void hyqo_pas_hll(int Np, const double* M, const double* F, double dt, double dx, const double* vpmin, const double* vpmax,
                  double* Mp) {
  pas_HLL_row<double>(Np, M, F, 1, Np, vpmin, vpmax, 1, dt, dx, Mp);
}
void hyqo_realizability_S2(double S110, double S101, double S011, double* out) {
  realizability_S2<double>(S110, S101, S011, out[0], out[1], out[2], out[3]);
}
void hyqo_check2d(double* s10) { check2D<double>(s10[0], s10[1], s10[2], s10[3], s10[4], s10[5], s10[6], s10[7], s10[8], s10[9]); }
void hyqo_realizable_2d(double* s10) {
  realizable_2D<double>(s10[0], s10[1], s10[2], s10[3], s10[4], s10[5], s10[6], s10[7], s10[8], s10[9]);
}

static S28<double> s28_from(const double* a) {
  S28<double> s = {a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], a[12], a[13],
                   a[14], a[15], a[16], a[17], a[18], a[19], a[20], a[21], a[22], a[23], a[24], a[25], a[26], a[27]};
  return s;
}
// 28 arguments in the reference order (s300, s400, s110, ... s022) -> 6x6 row-major.
void hyqo_delta2star3D(const double* a28, double* E) {
  double M[6][6];
  delta2star3D<double>(s28_from(a28), M);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) E[i * 6 + j] = M[i][j];
}
void hyqo_realizable_3d(double* a28, int* flag) {
  S28<double> s = s28_from(a28);
  *flag = realizable_3D<double>(s);
  double* o = a28;
  double v[28] = {s.s300, s.s400, s.s110, s.s210, s.s310, s.s120, s.s220, s.s030, s.s130, s.s040, s.s101, s.s201, s.s301, s.s102,
                  s.s202, s.s003, s.s103, s.s004, s.s011, s.s111, s.s211, s.s021, s.s121, s.s031, s.s012, s.s112, s.s013, s.s022};
  for (int i = 0; i < 28; ++i) o[i] = v[i];
}
// lower_bound_S220(S011,S012,S021,S101,S102,S110,S111,S120,S201,S210)
void hyqo_lower_bound_S220(const double* a, double* out) {
  S28<double> s{};
  s.s011 = a[0]; s.s012 = a[1]; s.s021 = a[2]; s.s101 = a[3]; s.s102 = a[4]; s.s110 = a[5]; s.s111 = a[6]; s.s120 = a[7];
  s.s201 = a[8]; s.s210 = a[9];
  double o[3];
  lower_bound_S220<double>(s, o);
  for (int i = 0; i < 3; ++i) out[i] = o[i];
}
// bound_minor1(S003,S011,S012,S021,S030,S101,S102,S110,S111,S120,S201,S210,S300)
void hyqo_bound_minor1(const double* a, double* out) {
  S28<double> s{};
  s.s003 = a[0]; s.s011 = a[1]; s.s012 = a[2]; s.s021 = a[3]; s.s030 = a[4]; s.s101 = a[5]; s.s102 = a[6]; s.s110 = a[7];
  s.s111 = a[8]; s.s120 = a[9]; s.s201 = a[10]; s.s210 = a[11]; s.s300 = a[12];
  double o[12];
  bound_minor1<double>(s, o);
  for (int i = 0; i < 12; ++i) out[i] = o[i];
}
// delta2starchol_L3(s03, s04, s11, s12, s13, s21, s22, s30, s31, s40)
double hyqo_delta2starchol_L3(const double* a) { return delta2starchol_L3<double>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9]); }
// rootsR(Del1, H02, H20, s03, s11, s12, s13, s21, s30, s31) -> re[3], im[3]
void hyqo_rootsR(const double* a, double* re, double* im) {
  double r[3], i3[3];
  rootsR<double>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], r, i3);
  for (int k = 0; k < 3; ++k) { re[k] = r[k]; im[k] = i3[k]; }
}
// rootsR_X_Y(Y, e11, e12, e13, e23, e24, e34, e44, ex)
void hyqo_rootsR_X_Y(const double* a, double* re, double* im) {
  double r[3], i3[3];
  rootsR_X_Y<double>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], r, i3);
  for (int k = 0; k < 3; ++k) { re[k] = r[k]; im[k] = i3[k]; }
}
// jacobian6(m00..m40) -> 6x6 row-major
void hyqo_jacobian6(const double* m, double* J) {
  double mm[15], JJ[6][6];
  for (int i = 0; i < 15; ++i) mm[i] = m[i];
  jacobian6<double>(mm, JJ);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) J[i * 6 + j] = JJ[i][j];
}
void hyqo_jacobian6_ad(const double* m, double* J) {
  double mm[15], JJ[6][6];
  for (int i = 0; i < 15; ++i) mm[i] = m[i];
  jacobian6_ad<double>(mm, JJ);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) J[i * 6 + j] = JJ[i][j];
}
int hyqo_eig6(const double* A, double* wr, double* wi) {
  double AA[6][6], r[6], im[6];
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) AA[i][j] = A[i * 6 + j];
  int info = eig_real<double, 6>(AA, r, im);
  for (int i = 0; i < 6; ++i) { wr[i] = r[i]; wi[i] = im[i]; }
  return info;
}
// M4toC4_3D on the 35 raw moments -> 35 central moments (35-order)
void hyqo_m4toc4(const double* M, double* C) {
  double cube[216];
  m4_to_c4<double>(M, cube);
  cube_to_35(cube, C);
}
// C5toM5_3D: central moments as a 6x6x6 cube (i + 6j + 36k) -> raw cube
void hyqo_c5tom5(double M000, double u, double v, double w, const double* Ccube, double* Mcube) {
  c_to_m<double>(M000, u, v, w, Ccube, Mcube, 5);
}
// S4toC4_3D_r: standardized cube -> central cube (order <= 4)
void hyqo_s4toc4_r(const double* C2, const double* Scube, double* Ccube) {
  s4_to_c4_r<double>(C2[0], C2[1], C2[2], C2[3], C2[4], C2[5], Scube, Ccube);
}

// ---------------------------------------------------------------- the step
// One serial time step of simulation_runner (src/simulation_runner.jl:346-560).
// M: (Nx,Ny,Nz,35) column-major, updated in place.  t: in/out.  Returns dt.
// vmax_out (optional): the CFL wave speed of the step.
static inline size_t at(const Params& P, int i, int j, int k) { return size_t(i) + size_t(P.Nx) * (size_t(j) + size_t(P.Ny) * size_t(k)); }

// The step in two halves around the CFL reduction (a slab of a decomposed
// domain calls them with the global max |speed| in between): begin runs
// phase [A] and returns the work state and the local NaN-propagating max.
struct StepWork {
  Params P;
  size_t N;
  std::vector<double> Fx, Fy, Fz, vp;
  int stop_after_hll = 0;
};

void* hyqo_step_begin(int Nx, int Ny, int Nz, double* M, double Kn, double Ma, int flag2D, double CFL, double dtmax, double tmax,
                      double dx, double dy, double dz, int positivity, double* vmax_local) {
  StepWork* w = new StepWork{Params{Nx, Ny, Nz, flag2D, positivity, Kn, Ma, CFL, dtmax, tmax, dx, dy, dz}, size_t(Nx) * Ny * Nz, {}, {}, {}, {}, 0};
  const Params& P = w->P;
  const size_t N = w->N;
  w->Fx.resize(N * 35); w->Fy.resize(N * 35); w->Fz.resize(N * 35); w->vp.resize(N * 6);
  std::vector<double> Mnp(N * 35);
#pragma omp parallel for schedule(dynamic, 16)
  for (long long c = 0; c < (long long)N; ++c) {
    double m[35], fx[35], fy[35], fz[35], mr[35], v[6];
    for (int n = 0; n < 35; ++n) m[n] = M[c + N * n];
    phase_A<double>(m, P, fx, fy, fz, mr, v);
    for (int n = 0; n < 35; ++n) { w->Fx[c + N * n] = fx[n]; w->Fy[c + N * n] = fy[n]; w->Fz[c + N * n] = fz[n]; Mnp[c + N * n] = mr[n]; }
    for (int q = 0; q < 6; ++q) w->vp[c + N * q] = v[q];
  }
  for (size_t q = 0; q < N * 35; ++q) M[q] = Mnp[q];
  // vmax = maximum(|vp*|) over all six arrays, NaN-propagating
  double vmax = 0.0;
  bool first = true;
  for (int q = 0; q < 6; ++q)
    for (size_t c = 0; c < N; ++c) {
      double a = std::fabs(w->vp[c + N * q]);
      vmax = first ? a : jmax(vmax, a);
      first = false;
    }
  *vmax_local = vmax;
  return w;
}

// dt from vmax, the HLL sweeps, phases [E]+[F]; frees the work state.
double hyqo_step_end(void* work, double* M, double vmax, double* t) {
  StepWork* w = static_cast<StepWork*>(work);
  const Params& P = w->P;
  const size_t N = w->N;
  const int Nx = P.Nx, Ny = P.Ny, Nz = P.Nz;
  const double dx = P.dx, dy = P.dy, dz = P.dz;
  double dt = jmin(P.CFL * jmin(jmin(dx, dy), dz) / vmax, jmin(P.dtmax, P.Kn));
  dt = jmin(dt, P.tmax - *t);
  *t = *t + dt;
  // HLL sweeps (src/numerics/apply_flux_update_3d.jl:30-213)
  std::vector<double> Mx(M, M + N * 35), My(M, M + N * 35), Mz(M, M + N * 35);
  const int ms = int(N);
  double* vp = w->vp.data();
#pragma omp parallel for schedule(static)
  for (int jk = 0; jk < Ny * Nz; ++jk) {
    int j = jk % Ny, k = jk / Ny;
    size_t o = at(P, 0, j, k);
    pas_HLL_row<double>(Nx, M + o, w->Fx.data() + o, 1, ms, vp + o, vp + N + o, 1, dt, dx, Mx.data() + o);
  }
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < Nx * Nz; ++ik) {
    int i = ik % Nx, k = ik / Nx;
    size_t o = at(P, i, 0, k);
    pas_HLL_row<double>(Ny, M + o, w->Fy.data() + o, Nx, ms, vp + 2 * N + o, vp + 3 * N + o, Nx, dt, dy, My.data() + o);
  }
  if (Nz > 1) {
#pragma omp parallel for schedule(static)
    for (int ij = 0; ij < Nx * Ny; ++ij) {
      int i = ij % Nx, j = ij / Nx;
      size_t o = at(P, i, j, 0);
      pas_HLL_row<double>(Nz, M + o, w->Fz.data() + o, Nx * Ny, ms, vp + 4 * N + o, vp + 5 * N + o, Nx * Ny, dt, dz, Mz.data() + o);
    }
  }
  for (size_t q = 0; q < N * 35; ++q) M[q] = Mx[q] + My[q] + Mz[q] - 2.0 * M[q];
  if (w->stop_after_hll) { delete w; return dt; }
  // [E] realizability and [F] collision
#pragma omp parallel for schedule(dynamic, 16)
  for (long long c = 0; c < (long long)N; ++c) {
    double m[35], r[35], o[35];
    for (int n = 0; n < 35; ++n) m[n] = M[c + N * n];
    phase_E<double>(m, P, r);
    collision35<double>(r, dt, P.Kn, P.positivity != 0, o);
    for (int n = 0; n < 35; ++n) M[c + N * n] = o[n];
  }
  delete w;
  return dt;
}

// The step's end stopped after the HLL combination (M = the state phase [E]
// starts from); frees the work state.
double hyqo_step_end_hll(void* work, double* M, double vmax, double* t) {
  static_cast<StepWork*>(work)->stop_after_hll = 1;
  return hyqo_step_end(work, M, vmax, t);
}

// Phases [E]+[F] alone (src/simulation_runner.jl:526-557) on a state M that
// the HLL combination produced, with the step's dt: the part of the step
// after the wave speeds, for measuring how the reference's step responds to
// round-off in its intermediate state.
void hyqo_phase_EF(int Nx, int Ny, int Nz, double* M, double Kn, double Ma, int flag2D, int positivity, double dt) {
  Params P{Nx, Ny, Nz, flag2D, positivity, Kn, Ma, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const size_t N = (size_t)Nx * Ny * Nz;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long c = 0; c < (long long)N; ++c) {
    double m[35], r[35], o[35];
    for (int n = 0; n < 35; ++n) m[n] = M[c + N * n];
    phase_E<double>(m, P, r);
    collision35<double>(r, dt, P.Kn, P.positivity != 0, o);
    for (int n = 0; n < 35; ++n) M[c + N * n] = o[n];
  }
}

double hyqo_step(int Nx, int Ny, int Nz, double* M, double Kn, double Ma, int flag2D, double CFL, double dtmax, double tmax,
                 double dx, double dy, double dz, int positivity, double* t, double* vmax_out) {
  double vmax = 0.0;
  void* w = hyqo_step_begin(Nx, Ny, Nz, M, Kn, Ma, flag2D, CFL, dtmax, tmax, dx, dy, dz, positivity, &vmax);
  if (vmax_out) *vmax_out = vmax;
  return hyqo_step_end(w, M, vmax, t);
}

void hyqo_count_ops(int Nx, int Ny, int Nz, const double* M, double Kn, double Ma, int flag2D, int positivity, double dt,
                    double* out) {
  Params P{Nx, Ny, Nz, flag2D, positivity, Kn, Ma, 0, 0, 0, 0, 0, 0};
  const size_t N = size_t(Nx) * Ny * Nz;
  unsigned long long a = 0, e = 0;
  for (size_t c = 0; c < N; ++c) {
    Counted m[35], fx[35], fy[35], fz[35], mr[35], v[6], r[35], o[35];
    for (int n = 0; n < 35; ++n) m[n] = Counted(M[c + N * n]);
    Counted::ops = 0;
    phase_A<Counted>(m, P, fx, fy, fz, mr, v);
    a += Counted::ops;
    Counted::ops = 0;
    phase_E<Counted>(mr, P, r);
    collision35<Counted>(r, Counted(dt), Counted(Kn), positivity != 0, o);
    e += Counted::ops;
  }
  out[0] = double(a);
  out[1] = double(e);
  // HLL per face per moment: Wstar 7, flux 8, update 3; three sweeps + combine 4
  out[2] = (Nz > 1 ? 3.0 : 2.0) * 35.0 * 18.0 + 35.0 * 4.0;
}

// Per-kernel FP64 operation counts of the staged CUDA step, summed over cells:
// out[0..4] = A1 closure, A2 x eigenvalues, A3 y eigenvalues, A4 z eigenvalues,
// A5 closure with fluxes + 1-D closure speeds; out[5..8] = E1 closure,
// E2 x eigenvalues, E3 y eigenvalues, E4 closure + BGK.  Same per-cell chain as
// phase_A / phase_E + collision35.
void hyqo_count_ops_stages(int Nx, int Ny, int Nz, const double* M, double Kn, double Ma, int flag2D, int positivity, double dt,
                           double* out) {
  const size_t N = size_t(Nx) * Ny * Nz;
  unsigned long long c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const Counted ma(Ma);
  for (size_t q = 0; q < N; ++q) {
    Counted m[35], a[35], b[35], fx[35], fy[35], fz[35], mr[35], v0, v1;
    for (int n = 0; n < 35; ++n) m[n] = Counted(M[q + N * n]);
    Counted::ops = 0; flux_closure35(m, flag2D, ma, fx, fy, fz, a); c[0] += Counted::ops;
    Counted::ops = 0; eigenvalues6_hyperbolic_3D(a, 1, flag2D, ma, v0, v1, b); c[1] += Counted::ops;
    Counted::ops = 0; eigenvalues6_hyperbolic_3D(b, 2, flag2D, ma, v0, v1, a); c[2] += Counted::ops;
    Counted::ops = 0; eigenvalues6z_hyperbolic_3D(a, flag2D, ma, positivity != 0, v0, v1, b); c[3] += Counted::ops;
    Counted::ops = 0;
    flux_closure35(b, flag2D, ma, fx, fy, fz, mr);
    {
      Counted mx[5] = {mr[0], mr[1], mr[2], mr[3], mr[4]};
      Counted my[5] = {mr[0], mr[5], mr[9], mr[12], mr[14]};
      Counted mz[5] = {mr[0], mr[15], mr[19], mr[22], mr[24]};
      Counted Mp, lo, hi;
      closure_and_eigenvalues(mx, Mp, lo, hi);
      closure_and_eigenvalues(my, Mp, lo, hi);
      closure_and_eigenvalues(mz, Mp, lo, hi);
    }
    c[4] += Counted::ops;
    // phases E + F on the realized state (the HLL update is not replayed here)
    Counted::ops = 0; flux_closure35(mr, flag2D, ma, fx, fy, fz, a); c[5] += Counted::ops;
    Counted::ops = 0; eigenvalues6_hyperbolic_3D(a, 1, flag2D, ma, v0, v1, b); c[6] += Counted::ops;
    Counted::ops = 0; eigenvalues6_hyperbolic_3D(b, 2, flag2D, ma, v0, v1, a); c[7] += Counted::ops;
    Counted::ops = 0;
    flux_closure35(a, flag2D, ma, fx, fy, fz, b);
    collision35<Counted>(b, Counted(dt), Counted(Kn), positivity != 0, mr);
    c[8] += Counted::ops;
  }
  for (int k = 0; k < 9; ++k) out[k] = double(c[k]);
}

}  // extern "C"
