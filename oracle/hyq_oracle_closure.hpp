// ORACLE (test infrastructure): 3-D realizability, HyQMOM closure and the
// Flux_closure35_and_realizable_3D driver.  Restates the reference files cited
// per function; see hyq_oracle.hpp for the conventions.
#pragma once
#include "hyq_oracle.hpp"

namespace hyqo {

// ------------------------------------------------ edge / corner correction
// Averaging helpers (src/realizability/edge_corner_correction.jl:113-252).
template <class T> struct S19 { T s210, s201, s120, s111, s102, s021, s012, s310, s301, s220, s211, s202, s130, s121, s112, s103, s031, s022, s013; };

template <class T> S19<T> avg_edge_xy(T S110, T S030, T S040, T S300, T S400, T S021r, T S012r, T S013r, T S031r, T S022r,
                                      T S201r, T S102r, T S103r, T S301r, T S202r, T S003r, T S004r) {
  (void)S003r; (void)S004r;
  S19<T> o;
  T h = T(2);
  o.s210 = (S030 + S110 * S300) / h;
  o.s201 = (S021r + S201r) / h;
  o.s120 = (S110 * S030 + S300) / h;
  o.s111 = (S110 * S021r + S110 * S201r) / h;
  o.s102 = (S110 * S012r + S102r) / h;
  o.s021 = (S021r + S201r) / h;
  o.s012 = (S012r + S110 * S102r) / h;
  o.s310 = (S110 * S040 + S110 * S400) / h;
  o.s301 = (S110 * S031r + S301r) / h;
  o.s220 = (S040 + S400) / h;
  o.s211 = (S031r + S110 * S301r) / h;
  o.s202 = (S022r + S202r) / h;
  o.s130 = (S110 * S040 + S110 * S400) / h;
  o.s121 = (S110 * S031r + S301r) / h;
  o.s112 = (S110 * S022r + S110 * S202r) / h;
  o.s103 = (S110 * S013r + S103r) / h;
  o.s031 = (S031r + S110 * S301r) / h;
  o.s022 = (S022r + S202r) / h;
  o.s013 = (S013r + S110 * S103r) / h;
  return o;
}

template <class T> S19<T> avg_edge_xz(T S101, T S003, T S004, T S300, T S400, T S021r, T S012r, T S013r, T S031r, T S022r,
                                      T S030r, T S210r, T S120r, T S220r, T S130r, T S310r) {
  (void)S030r;
  S19<T> o;
  T h = T(2);
  o.s210 = (S013r + S210r) / h;
  o.s201 = (S003 + S101 * S300) / h;
  o.s120 = (S101 * S021r + S120r) / h;
  o.s111 = (S101 * S012r + S101 * S210r) / h;
  o.s102 = (S101 * S003 + S300) / h;
  o.s021 = (S021r + S101 * S120r) / h;
  o.s012 = (S012r + S210r) / h;
  o.s310 = (S101 * S013r + S310r) / h;
  o.s301 = (S101 * S004 + S101 * S400) / h;
  o.s220 = (S022r + S220r) / h;
  o.s211 = (S013r + S101 * S310r) / h;
  o.s202 = (S004 + S400) / h;
  o.s130 = (S101 * S031r + S130r) / h;
  o.s121 = (S101 * S022r + S101 * S220r) / h;
  o.s112 = (S101 * S013r + S310r) / h;
  o.s103 = (S101 * S004 + S101 * S400) / h;
  o.s031 = (S031r + S101 * S130r) / h;
  o.s022 = (S022r + S220r) / h;
  o.s013 = (S013r + S101 * S310r) / h;
  return o;
}

template <class T> S19<T> avg_edge_yz(T S011, T S003, T S004, T S030, T S040, T S201r, T S102r, T S103r, T S301r, T S202r,
                                      T S300r, T S210r, T S120r, T S220r, T S130r, T S310r) {
  (void)S300r;
  S19<T> o;
  T h = T(2);
  o.s210 = (S011 * S201r + S210r) / h;
  o.s201 = (S201r + S011 * S210r) / h;
  o.s120 = (S102r + S120r) / h;
  o.s111 = (S011 * S102r + S011 * S120r) / h;
  o.s102 = (S102r + S120r) / h;
  o.s021 = (S003 + S011 * S030) / h;
  o.s012 = (S011 * S003 + S030) / h;
  o.s310 = (S011 * S301r + S310r) / h;
  o.s301 = (S301r + S011 * S310r) / h;
  o.s220 = (S202r + S220r) / h;
  o.s211 = (S011 * S202r + S011 * S220r) / h;
  o.s202 = (S202r + S220r) / h;
  o.s130 = (S011 * S103r + S130r) / h;
  o.s121 = (S103r + S011 * S130r) / h;
  o.s112 = (S011 * S103r + S130r) / h;
  o.s103 = (S103r + S011 * S130r) / h;
  o.s031 = (S011 * S004 + S011 * S040) / h;
  o.s022 = (S004 + S040) / h;
  o.s013 = (S011 * S004 + S011 * S040) / h;
  return o;
}

template <class T> S19<T> avg_corner(T S110, T S101, T S011, T S030a, T S040a, T S030b, T S040b, T S300c, T S400c, T S003c, T S004c) {
  (void)S300c; (void)S400c;
  T th = T(3);
  S19<T> o;
  // variant a: SIJK = S110^J S101^K S(I+J+K)00 ; b: S110^I S011^K S0(I+J+K)0 ; c: S101^I S011^J S00(I+J+K)
  T a210 = S110 * S030a, a201 = S101 * S030a, a120 = S030a, a111 = S110 * S101 * S030a, a102 = S030a, a021 = S101 * S030a, a012 = S110 * S030a;
  T a310 = S110 * S040a, a301 = S101 * S040a, a220 = S040a, a211 = S110 * S101 * S040a, a202 = S040a, a130 = S110 * S040a, a121 = S101 * S040a,
    a112 = S110 * S040a, a103 = S101 * S040a, a031 = S110 * S101 * S040a, a022 = S040a, a013 = S110 * S101 * S040a;
  T b210 = S030b, b201 = S011 * S030b, b120 = S110 * S030b, b111 = S110 * S011 * S030b, b102 = S110 * S030b, b021 = S011 * S030b, b012 = S030b;
  T b310 = S110 * S040b, b301 = S110 * S011 * S040b, b220 = S040b, b211 = S011 * S040b, b202 = S040b, b130 = S110 * S040b, b121 = S110 * S011 * S040b,
    b112 = S110 * S040b, b103 = S110 * S011 * S040b, b031 = S011 * S040b, b022 = S040b, b013 = S011 * S040b;
  T c210 = S011 * S003c, c201 = S003c, c120 = S101 * S003c, c111 = S101 * S011 * S003c, c102 = S101 * S003c, c021 = S003c, c012 = S011 * S003c;
  T c310 = S101 * S011 * S004c, c301 = S101 * S004c, c220 = S004c, c211 = S011 * S004c, c202 = S004c, c130 = S101 * S011 * S004c,
    c121 = S101 * S004c, c112 = S101 * S011 * S004c, c103 = S101 * S004c, c031 = S011 * S004c, c022 = S004c, c013 = S011 * S004c;
  o.s210 = (a210 + b210 + c210) / th; o.s201 = (a201 + b201 + c201) / th; o.s120 = (a120 + b120 + c120) / th;
  o.s111 = (a111 + b111 + c111) / th; o.s102 = (a102 + b102 + c102) / th; o.s021 = (a021 + b021 + c021) / th;
  o.s012 = (a012 + b012 + c012) / th;
  o.s310 = (a310 + b310 + c310) / th; o.s301 = (a301 + b301 + c301) / th; o.s220 = (a220 + b220 + c220) / th;
  o.s211 = (a211 + b211 + c211) / th; o.s202 = (a202 + b202 + c202) / th; o.s130 = (a130 + b130 + c130) / th;
  o.s121 = (a121 + b121 + c121) / th; o.s112 = (a112 + b112 + c112) / th; o.s103 = (a103 + b103 + c103) / th;
  o.s031 = (a031 + b031 + c031) / th; o.s022 = (a022 + b022 + c022) / th; o.s013 = (a013 + b013 + c013) / th;
  return o;
}

// ------------------------------------------------------------ realizable_3D
// realizable_3D (src/realizability/realizable_3D.jl:39-624).  `s` holds the
// 28 moments in/out; returns flag220.
template <class T> S28<T> perm(const S28<T>& s, int which) {
  // delta2star3D_permutation (src/autogen/delta2star3D_permutation.jl:26-61)
  S28<T> r;
  switch (which) {
    case 1: r = s; break;
    case 2: r = {s.s300, s.s400, s.s101, s.s201, s.s301, s.s102, s.s202, s.s003, s.s103, s.s004,
                 s.s110, s.s210, s.s310, s.s120, s.s220, s.s030, s.s130, s.s040, s.s011, s.s111,
                 s.s211, s.s012, s.s112, s.s013, s.s021, s.s121, s.s031, s.s022}; break;
    case 3: r = {s.s030, s.s040, s.s110, s.s120, s.s130, s.s210, s.s220, s.s300, s.s310, s.s400,
                 s.s011, s.s021, s.s031, s.s012, s.s022, s.s003, s.s013, s.s004, s.s101, s.s111,
                 s.s121, s.s201, s.s211, s.s301, s.s102, s.s112, s.s103, s.s202}; break;
    case 4: r = {s.s003, s.s004, s.s101, s.s102, s.s103, s.s201, s.s202, s.s300, s.s301, s.s400,
                 s.s011, s.s012, s.s013, s.s021, s.s022, s.s030, s.s031, s.s040, s.s110, s.s111,
                 s.s112, s.s210, s.s211, s.s310, s.s120, s.s121, s.s130, s.s220}; break;
    case 5: r = {s.s030, s.s040, s.s011, s.s021, s.s031, s.s012, s.s022, s.s003, s.s013, s.s004,
                 s.s110, s.s120, s.s130, s.s210, s.s220, s.s300, s.s310, s.s400, s.s101, s.s111,
                 s.s121, s.s102, s.s112, s.s103, s.s201, s.s211, s.s301, s.s202}; break;
    default: r = {s.s003, s.s004, s.s011, s.s012, s.s013, s.s021, s.s022, s.s030, s.s031, s.s040,
                  s.s101, s.s102, s.s103, s.s201, s.s202, s.s300, s.s301, s.s400, s.s110, s.s111,
                  s.s112, s.s120, s.s121, s.s130, s.s210, s.s211, s.s310, s.s220}; break;
  }
  return r;
}

template <class T, int K> T lead_det(const T (&E)[6][6]) {
  T A[K][K];
  for (int i = 0; i < K; ++i) for (int j = 0; j < K; ++j) A[i][j] = E[i][j];
  return det_lu<T, K>(A);
}

template <class T> int realizable_3D(S28<T>& s) {
  using std::sqrt;
  int flag220 = 0;
  const T diagmin = T(1e-10), h2min = T(1e-10), S2min = T(1e-12);
  T H200 = jmax(T(EPS), s.s400 - s.s300 * s.s300 - T(1));
  T H020 = jmax(T(EPS), s.s040 - s.s030 * s.s030 - T(1));
  T H002 = jmax(T(EPS), s.s004 - s.s003 * s.s003 - T(1));
  T A220 = sqrt((H200 + s.s300 * s.s300) * (H020 + s.s030 * s.s030));
  T S220max = realizablity_S220(s.s110, s.s220, A220);
  T A202 = sqrt((H200 + s.s300 * s.s300) * (H002 + s.s003 * s.s003));
  T S202max = realizablity_S220(s.s101, s.s202, A202);
  T A022 = sqrt((H020 + s.s030 * s.s030) * (H002 + s.s003 * s.s003));
  T S022max = realizablity_S220(s.s011, s.s022, A022);
  s.s220 = jmin(s.s220, S220max);
  s.s202 = jmin(s.s202, S202max);
  s.s022 = jmin(s.s022, S022max);
  T S2;
  realizability_S2(s.s110, s.s101, s.s011, s.s110, s.s101, s.s011, S2);
  T R110 = sqrt(jmax(T(0), T(1) - s.s110 * s.s110));
  T R101 = sqrt(jmax(T(0), T(1) - s.s101 * s.s101));
  T R011 = sqrt(jmax(T(0), T(1) - s.s011 * s.s011));

  if (S2 <= S2min) {
    hit(BR_FACES);
    // faces (src/realizability/realizable_3D.jl:79-142)
    T Rmax = jmax(jmax(R110, R101), R011);
    if (R110 == Rmax) {
      T g1 = (s.s101 - s.s110 * s.s011) / (T(1) - s.s110 * s.s110);
      T g2 = (s.s011 - s.s110 * s.s101) / (T(1) - s.s110 * s.s110);
      s.s021 = g2 * s.s030 + g1 * s.s120;
      s.s201 = g2 * s.s210 + g1 * s.s300;
      s.s031 = g2 * s.s040 + g1 * s.s130;
      s.s301 = g2 * s.s310 + g1 * s.s400;
      s.s111 = g2 * s.s120 + g1 * s.s210;
      s.s211 = g2 * s.s220 + g1 * s.s310;
      s.s121 = g2 * s.s130 + g1 * s.s220;
      s.s012 = sq(g2) * s.s030 + T(2) * g1 * g2 * s.s120 + sq(g1) * s.s210;
      s.s102 = sq(g2) * s.s120 + T(2) * g1 * g2 * s.s210 + sq(g1) * s.s300;
      s.s022 = sq(g2) * s.s040 + T(2) * g1 * g2 * s.s130 + sq(g1) * s.s220;
      s.s202 = sq(g2) * s.s220 + T(2) * g1 * g2 * s.s310 + sq(g1) * s.s400;
      s.s112 = sq(g2) * s.s130 + T(2) * g1 * g2 * s.s220 + sq(g1) * s.s310;
      s.s003 = cube(g2) * s.s030 + T(3) * g1 * sq(g2) * s.s120 + T(3) * sq(g1) * g2 * s.s210 + cube(g1) * s.s300;
      s.s013 = cube(g2) * s.s040 + T(3) * g1 * sq(g2) * s.s130 + T(3) * sq(g1) * g2 * s.s220 + cube(g1) * s.s310;
      s.s103 = cube(g2) * s.s130 + T(3) * g1 * sq(g2) * s.s220 + T(3) * sq(g1) * g2 * s.s310 + cube(g1) * s.s400;
      s.s004 = pow4(g2) * s.s040 + T(4) * g1 * cube(g2) * s.s130 + T(6) * sq(g1) * sq(g2) * s.s220 + T(4) * cube(g1) * g2 * s.s310 + pow4(g1) * s.s400;
    } else if (R101 == Rmax) {
      T g3 = (s.s110 - s.s101 * s.s011) / (T(1) - s.s101 * s.s101);
      T g4 = (s.s011 - s.s110 * s.s101) / (T(1) - s.s101 * s.s101);
      s.s012 = g4 * s.s003 + g3 * s.s102;
      s.s210 = g4 * s.s201 + g3 * s.s300;
      s.s013 = g4 * s.s004 + g3 * s.s103;
      s.s310 = g4 * s.s301 + g3 * s.s400;
      s.s111 = g4 * s.s102 + g3 * s.s201;
      s.s211 = g4 * s.s202 + g3 * s.s301;
      s.s112 = g4 * s.s103 + g3 * s.s202;
      s.s021 = sq(g4) * s.s003 + T(2) * g3 * g4 * s.s102 + sq(g3) * s.s201;
      s.s120 = sq(g4) * s.s102 + T(2) * g3 * g4 * s.s201 + sq(g3) * s.s300;
      s.s022 = sq(g4) * s.s004 + T(2) * g3 * g4 * s.s103 + sq(g3) * s.s202;
      s.s220 = sq(g4) * s.s202 + T(2) * g3 * g4 * s.s301 + sq(g3) * s.s400;
      s.s121 = sq(g4) * s.s103 + T(2) * g3 * g4 * s.s202 + sq(g3) * s.s301;
      s.s030 = cube(g4) * s.s003 + T(3) * g3 * sq(g4) * s.s102 + T(3) * sq(g3) * g4 * s.s201 + cube(g3) * s.s300;
      s.s031 = cube(g4) * s.s004 + T(3) * g3 * sq(g4) * s.s103 + T(3) * sq(g3) * g4 * s.s202 + cube(g3) * s.s301;
      s.s130 = cube(g4) * s.s103 + T(3) * g3 * sq(g4) * s.s202 + T(3) * sq(g3) * g4 * s.s301 + cube(g3) * s.s400;
      s.s040 = pow4(g4) * s.s004 + T(4) * g3 * cube(g4) * s.s103 + T(6) * sq(g3) * sq(g4) * s.s202 + T(4) * cube(g3) * g4 * s.s301 + pow4(g3) * s.s400;
    } else {
      T g5 = (s.s101 - s.s110 * s.s011) / (T(1) - s.s011 * s.s011);
      T g6 = (s.s110 - s.s101 * s.s011) / (T(1) - s.s011 * s.s011);
      s.s102 = g6 * s.s003 + g5 * s.s012;
      s.s120 = g6 * s.s021 + g5 * s.s030;
      s.s103 = g6 * s.s004 + g5 * s.s013;
      s.s130 = g6 * s.s031 + g5 * s.s040;
      s.s111 = g6 * s.s012 + g5 * s.s021;
      s.s121 = g6 * s.s022 + g5 * s.s031;
      s.s112 = g6 * s.s013 + g5 * s.s022;
      s.s201 = sq(g6) * s.s003 + T(2) * g5 * g6 * s.s012 + sq(g5) * s.s021;
      s.s210 = sq(g6) * s.s012 + T(2) * g5 * g6 * s.s021 + sq(g5) * s.s030;
      s.s202 = sq(g6) * s.s004 + T(2) * g5 * g6 * s.s013 + sq(g5) * s.s022;
      s.s220 = sq(g6) * s.s022 + T(2) * g5 * g6 * s.s031 + sq(g5) * s.s040;
      s.s211 = sq(g6) * s.s013 + T(2) * g5 * g6 * s.s022 + sq(g5) * s.s031;
      s.s300 = cube(g6) * s.s003 + T(3) * g5 * sq(g6) * s.s012 + T(3) * sq(g5) * g6 * s.s021 + cube(g5) * s.s030;
      s.s301 = cube(g6) * s.s004 + T(3) * g5 * sq(g6) * s.s013 + T(3) * sq(g5) * g6 * s.s022 + cube(g5) * s.s031;
      s.s310 = cube(g6) * s.s013 + T(3) * g5 * sq(g6) * s.s022 + T(3) * sq(g5) * g6 * s.s031 + cube(g5) * s.s040;
      s.s400 = pow4(g6) * s.s004 + T(4) * g5 * cube(g6) * s.s013 + T(6) * sq(g5) * sq(g6) * s.s022 + T(4) * cube(g5) * g6 * s.s031 + pow4(g5) * s.s040;
    }
    return flag220;
  }

  // interior (src/realizability/realizable_3D.jl:144-619)
  const T beta = T(1);
  T E[6][6];
  delta2star3D(s, E);
  int fE11 = 0, fE22 = 0, fE33 = 0, fE44 = 0, fE55 = 0, fE66 = 0;
  if (E[0][0] < T(0)) { realizability_S210(s.s110, s.s101, s.s011, s.s300, s.s210, s.s201, H200, beta, s.s210, s.s201); fE11 = 1; }
  if (E[3][3] < T(0)) { realizability_S210(s.s110, s.s011, s.s101, s.s030, s.s120, s.s021, H020, beta, s.s120, s.s021); fE44 = 1; }
  if (E[5][5] < T(0)) { realizability_S210(s.s011, s.s101, s.s110, s.s003, s.s012, s.s102, H002, beta, s.s012, s.s102); fE66 = 1; }
  T S111r = realizability_S111(s.s110, s.s101, s.s011, s.s210, s.s201, s.s120, s.s021, s.s102, s.s012, s.s111);
  if (S111r != s.s111) s.s111 = S111r;
  T S220_310 = realizability_S310_220(s.s110, s.s101, s.s011, s.s210, s.s120, s.s111, s.s220);
  T S202_310 = realizability_S310_220(s.s101, s.s110, s.s011, s.s201, s.s102, s.s111, s.s202);
  T S022_310 = realizability_S310_220(s.s011, s.s110, s.s101, s.s021, s.s012, s.s111, s.s022);
  T S220_diag = s.s220, S202_diag = s.s202, S022_diag = s.s022;
  T S22min[3];
  lower_bound_S220(s, S22min);
  if (s.s220 < S22min[0]) { S220_diag = S22min[0]; fE22 = 1; flag220 = 1; }
  if (s.s202 < S22min[1]) { S202_diag = S22min[1]; fE33 = 1; flag220 = 1; }
  if (s.s022 < S22min[2]) { S022_diag = S22min[2]; fE55 = 1; flag220 = 1; }
  delta2star3D(s, E);
  if (E[0][0] < diagmin) fE11 = 1;
  if (E[1][1] < diagmin) fE22 = 1;
  if (E[2][2] < diagmin) fE33 = 1;
  if (E[3][3] < diagmin) fE44 = 1;
  if (E[4][4] < diagmin) fE55 = 1;
  if (E[5][5] < diagmin) fE66 = 1;
  if (fE11 || fE22 || fE33 || fE44 || fE55 || fE66) {
    T Mb[12];
    bound_minor1(s, Mb);
    T S310b = Mb[0], S301b = Mb[1], S130b = Mb[2], S103b = Mb[3], S031b = Mb[4], S013b = Mb[5];
    T S211b = Mb[9], S121b = Mb[10], S112b = Mb[11];
    if (fE11) { s.s310 = S310b; s.s301 = S301b; s.s211 = S211b; }
    if (fE22) { s.s310 = S310b; s.s130 = S130b; s.s211 = S211b; s.s121 = S121b; s.s112 = S112b; }
    if (fE33) { s.s301 = S301b; s.s103 = S103b; s.s211 = S211b; s.s121 = S121b; s.s112 = S112b; }
    if (fE44) { s.s130 = S130b; s.s031 = S031b; s.s121 = S121b; }
    if (fE55) { s.s031 = S031b; s.s013 = S013b; s.s211 = S211b; s.s121 = S121b; s.s112 = S112b; }
    if (fE66) { s.s103 = S103b; s.s013 = S013b; s.s112 = S112b; }
  }
  if (fE11 && fE22 && fE33 && fE44 && fE55 && fE66) return flag220;

  // 2x2 minors (src/realizability/realizable_3D.jl:284-378)
  T S220a = s.s220, S220b = s.s220, S202a = s.s202, S202b = s.s202, S022a = s.s022, S022b = s.s022;
  T P[6][6][6];
  for (int p = 0; p < 6; ++p) { S28<T> sp = perm(s, p + 1); delta2star3D(sp, P[p]); }
  int flag310 = 0;
  if (!fE11 && !fE44 && lead_det<T, 2>(P[0]) < h2min) {
    realizability_S310(s.s110, s.s101, s.s011, s.s300, s.s210, s.s120, s.s201, s.s111, s.s310, s.s220, H200, beta, s.s310, S220a);
    flag310 = 1;
  }
  if (!fE22 && !fE44 && lead_det<T, 2>(P[2]) < h2min) {
    realizability_S310(s.s110, s.s011, s.s101, s.s030, s.s120, s.s021, s.s210, s.s111, s.s130, s.s220, H020, beta, s.s130, S220b);
    flag310 = 1;
  }
  if (!fE11 && !fE33 && lead_det<T, 2>(P[1]) < h2min) {
    realizability_S310(s.s101, s.s110, s.s011, s.s300, s.s201, s.s210, s.s102, s.s111, s.s301, s.s202, H200, beta, s.s301, S202a);
    flag310 = 1;
  }
  if (!fE33 && !fE66 && lead_det<T, 2>(P[3]) < h2min) {
    realizability_S310(s.s101, s.s011, s.s110, s.s003, s.s102, s.s012, s.s201, s.s111, s.s103, s.s202, H002, beta, s.s103, S202b);
    flag310 = 1;
  }
  if (!fE44 && !fE55 && lead_det<T, 2>(P[4]) < h2min) {
    realizability_S310(s.s011, s.s110, s.s101, s.s030, s.s021, s.s120, s.s012, s.s111, s.s031, s.s022, H020, beta, s.s031, S022a);
    flag310 = 1;
  }
  if (!fE55 && !fE66 && lead_det<T, 2>(P[5]) < h2min) {
    realizability_S310(s.s011, s.s101, s.s110, s.s003, s.s012, s.s102, s.s021, s.s111, s.s013, s.s022, H002, beta, s.s013, S022b);
    flag310 = 1;
  }
  T S220r = jmax(S220a, S220b);
  T S220_310r = S220_310;
  if (s.s220 < S220r) { S220_310r = S220r; flag220 = 1; }
  T S022r = jmax(S022a, S022b);
  T S022_310r = S022_310;
  if (s.s022 < S022r) { S022_310r = S022r; flag220 = 1; }
  T S202r = jmax(S202a, S202b);
  T S202_310r = S202_310;
  if (s.s202 < S202r) { S202_310r = S202r; flag220 = 1; }
  if (flag310) {
    for (int p = 0; p < 6; ++p) { S28<T> sp = perm(s, p + 1); delta2star3D(sp, P[p]); }
    T dm = lead_det<T, 2>(P[0]);
    for (int p = 1; p < 6; ++p) dm = jmin(dm, lead_det<T, 2>(P[p]));
    if (dm < T(0)) flag220 = 1;
  }

  // 3x3 minors (src/realizability/realizable_3D.jl:380-453); P still holds
  // the permutation matrices of the current (possibly updated) moments.
  S220a = s.s220; S220b = s.s220; S202a = s.s202; T S202c = s.s202; S022b = s.s022; T S022c = s.s022;
  if (!fE11 && !fE22 && !fE33 && !fE55) {
    if (lead_det<T, 3>(P[0]) <= h2min || lead_det<T, 3>(P[1]) <= h2min) {
      T e11 = P[0][0][0], e12 = P[0][0][1], e13 = P[0][0][2], e22 = P[0][1][1], e23 = P[0][1][2], e33 = P[0][2][2];
      T d23 = s.s211 - e23, d22 = s.s220 - e22, d33 = s.s202 - e33;
      if (e11 > diagmin) { S220a = d22 + e13 * e13 / e11; S202a = d33 + e12 * e12 / e11; }
      s.s211 = realizability_S211(e11, e22, e33, e12, e13, d23, s.s211, beta);
      flag220 = 1;
    }
  }
  if (!fE22 && !fE33 && !fE44 && !fE55) {
    if (lead_det<T, 3>(P[2]) < h2min || lead_det<T, 3>(P[4]) < h2min) {
      T e11 = P[2][0][0], e12 = P[2][0][1], e13 = P[2][0][2], e22 = P[2][1][1], e23 = P[2][1][2], e33 = P[2][2][2];
      T d23 = s.s121 - e23, d22 = s.s220 - e22, d33 = s.s022 - e33;
      if (e11 > diagmin) { S220b = d22 + e13 * e13 / e11; S022b = d33 + e12 * e12 / e11; }
      s.s121 = realizability_S211(e11, e22, e33, e12, e13, d23, s.s121, beta);
      flag220 = 1;
    }
  }
  if (!fE22 && !fE33 && !fE55 && !fE66) {
    if (lead_det<T, 3>(P[3]) < h2min || lead_det<T, 3>(P[5]) < h2min) {
      T e11 = P[5][0][0], e12 = P[5][0][1], e13 = P[5][0][2], e22 = P[5][1][1], e23 = P[5][1][2], e33 = P[5][2][2];
      T d23 = s.s112 - e23, d22 = s.s022 - e22, d33 = s.s202 - e33;
      if (e11 > diagmin) { S202c = d22 + e13 * e13 / e11; S022c = d33 + e12 * e12 / e11; }
      s.s112 = realizability_S211(e11, e22, e33, e12, e13, d23, s.s112, beta);
      flag220 = 1;
    }
  }
  T S220_211 = jmax(S220a, S220b);
  T S202_211 = jmax(S202a, S202c);
  T S022_211 = jmax(S022b, S022c);

  // 4x4 minors with rootsR_X_Y (src/realizability/realizable_3D.jl:455-608)
  auto minor4 = [&](const S28<T>& sp, T S22cur, T& lo, T& hi) {
    T Em[6][6];
    delta2star3D(sp, Em);
    lo = S22cur; hi = S22cur;
    if (lead_det<T, 4>(Em) < T(0)) {
      flag220 = 1;
      T ex = -Em[1][1] + Em[0][3];
      T d22 = S22cur - Em[1][1];
      T re[3], im[3];
      rootsR_X_Y(Em[2][2], Em[0][0], Em[0][1], Em[0][2], Em[1][2], Em[1][3], Em[2][3], Em[3][3], ex, re, im);
      T Rr[3] = {re[0], re[1], re[2]};
      sort3_nan_last(Rr);
      if (imag_ratio(re, im) < T(1000 * EPS)) { lo = Rr[1] + d22; hi = Rr[2] + d22; }
    }
  };
  T s220mina, s220maxa, s220minb, s220maxb, s202mina, s202maxa, s202minb, s202maxb, s022mina, s022maxa, s022minb, s022maxb;
  minor4(perm(s, 1), s.s220, s220mina, s220maxa);
  minor4(perm(s, 3), s.s220, s220minb, s220maxb);
  minor4(perm(s, 2), s.s202, s202mina, s202maxa);
  minor4(perm(s, 4), s.s202, s202minb, s202maxb);
  minor4(perm(s, 5), s.s022, s022mina, s022maxa);
  minor4(perm(s, 6), s.s022, s022minb, s022maxb);
  T v;
  v = jmax(jmax(jmax(jmax(jmax(s220mina, s220minb), S220_diag), S220_310), S220_310r), S220_211);
  s.s220 = jmin(jmin(jmin(v, S220max), s220maxa), s220maxb);
  v = jmax(jmax(jmax(jmax(jmax(s202mina, s202minb), S202_diag), S202_310), S202_310r), S202_211);
  s.s202 = jmin(jmin(jmin(v, S202max), s202maxa), s202maxb);
  v = jmax(jmax(jmax(jmax(jmax(s022mina, s022minb), S022_diag), S022_310), S022_310r), S022_211);
  s.s022 = jmin(jmin(jmin(v, S022max), s022maxa), s022maxb);
  return flag220;
}

// ------------------------------------------------------------ hyqmom_3D
// hyqmom_3D (src/moments/hyqmom_3D.jl:147-190): 21 fifth-order closures.
template <class T> struct S5 { T s500, s410, s320, s230, s140, s401, s302, s203, s104, s311, s221, s131, s212, s113, s122, s050, s041, s032, s023, s014, s005; };

template <class T> S5<T> hyqmom_3D(const S28<T>& s) {
  S5<T> o;
  const T h = T(0.5);
  o.s500 = h * s.s300 * (T(5) * s.s400 - T(3) * sq(s.s300) - T(1));
  o.s050 = h * s.s030 * (T(5) * s.s040 - T(3) * sq(s.s030) - T(1));
  o.s005 = h * s.s003 * (T(5) * s.s004 - T(3) * sq(s.s003) - T(1));
  // mixed (a=3,b=2) closure for a coordinate pair (i,j) with the given moments
  auto c32 = [&](T Sj3, T Si3, T Si4, T Sij, T Sijj, T Siij, T Siijj, T Siiij) {
    return ((Sj3 * sq(Si3)) / T(2) - Sj3 + Sj3 * (sq(Si3) - Si4 + T(1))) * Sij + (Si4 - (T(3) * sq(Si3)) / T(2)) * Sijj +
           (-(T(3) * Sj3 * Si3) / T(2)) * Siij + ((T(3) * Si3) / T(2)) * Siijj + Sj3 * Siiij - Si3 / T(2);
  };
  o.s320 = c32(s.s030, s.s300, s.s400, s.s110, s.s120, s.s210, s.s220, s.s310);
  o.s230 = c32(s.s300, s.s030, s.s040, s.s110, s.s210, s.s120, s.s220, s.s130);
  o.s302 = c32(s.s003, s.s300, s.s400, s.s101, s.s102, s.s201, s.s202, s.s301);
  o.s203 = c32(s.s300, s.s003, s.s004, s.s101, s.s201, s.s102, s.s202, s.s103);
  o.s032 = c32(s.s003, s.s030, s.s040, s.s011, s.s012, s.s021, s.s022, s.s031);
  o.s023 = c32(s.s030, s.s003, s.s004, s.s011, s.s021, s.s012, s.s022, s.s013);
  auto c41 = [&](T Si3, T Si4, T Sij, T Siij, T Siiij) {
    return (Si3 - T(2) * Si3 * Si4 + (T(9) * cube(Si3)) / T(4)) * Sij + ((T(5) * Si4) / T(2) - (T(15) * sq(Si3)) / T(4) - T(1.5)) * Siij +
           (T(2) * Si3) * Siiij;
  };
  o.s410 = c41(s.s300, s.s400, s.s110, s.s210, s.s310);
  o.s140 = c41(s.s030, s.s040, s.s110, s.s120, s.s130);
  o.s401 = c41(s.s300, s.s400, s.s101, s.s201, s.s301);
  o.s104 = c41(s.s003, s.s004, s.s101, s.s102, s.s103);
  o.s041 = c41(s.s030, s.s040, s.s011, s.s021, s.s031);
  o.s014 = c41(s.s003, s.s004, s.s011, s.s012, s.s013);
  o.s311 = T(3) * (s.s300 * s.s211) / T(2) + (T(2) * s.s400 - T(3) * sq(s.s300)) * s.s111 / T(2) - (s.s300 * s.s011) / T(2);
  o.s131 = T(3) * (s.s030 * s.s121) / T(2) + (T(2) * s.s040 - T(3) * sq(s.s030)) * s.s111 / T(2) - (s.s030 * s.s101) / T(2);
  o.s113 = T(3) * (s.s003 * s.s112) / T(2) + (T(2) * s.s004 - T(3) * sq(s.s003)) * s.s111 / T(2) - (s.s003 * s.s110) / T(2);
  o.s221 = s.s300 * (s.s121 - s.s101) + s.s030 * (s.s211 - s.s011) + s.s201 + s.s021 - s.s300 * s.s030 * s.s111;
  o.s212 = s.s300 * (s.s112 - s.s110) + s.s003 * (s.s211 - s.s011) + s.s210 + s.s012 - s.s300 * s.s003 * s.s111;
  o.s122 = s.s003 * (s.s121 - s.s101) + s.s030 * (s.s112 - s.s110) + s.s102 + s.s120 - s.s003 * s.s030 * s.s111;
  return o;
}

// ------------------------------------------ Flux_closure35_and_realizable_3D
// (src/numerics/Flux_closure35_and_realizable_3D.jl:33-234)
template <class T> void flux_closure35(const T* M4, int flag2D, T Ma, T* Fx, T* Fy, T* Fz, T* M4r) {
  using std::fabs; using std::sqrt;
  const T s3max = T(4) + fabs(Ma) / T(2);
  const T h2min = T(1e-8);
  const int itrealmax = 6;
  T M000 = M4[0];
  T umean = M4[1] / M000, vmean = M4[5] / M000, wmean = M4[15] / M000;
  T C4[35], S4[35];
  m2cs4_35(M4, C4, S4);
  T C200 = jmax(T(EPS), C4[2]), C020 = jmax(T(EPS), C4[9]), C002 = jmax(T(EPS), C4[19]);
  S28<T> s;
  s.s300 = S4[3]; s.s400 = S4[4]; s.s110 = S4[6]; s.s210 = S4[7]; s.s310 = S4[8];
  s.s120 = S4[10]; s.s220 = S4[11]; s.s030 = S4[12]; s.s130 = S4[13]; s.s040 = S4[14];
  s.s101 = S4[16]; s.s201 = S4[17]; s.s301 = S4[18]; s.s102 = S4[20]; s.s202 = S4[21];
  s.s003 = S4[22]; s.s103 = S4[23]; s.s004 = S4[24]; s.s011 = S4[25]; s.s111 = S4[26];
  s.s211 = S4[27]; s.s021 = S4[28]; s.s121 = S4[29]; s.s031 = S4[30]; s.s012 = S4[31];
  s.s112 = S4[32]; s.s013 = S4[33]; s.s022 = S4[34];
  T H200, H020, H002;
  enforce_univariate(s.s300, s.s400, h2min, s3max, H200);
  enforce_univariate(s.s030, s.s040, h2min, s3max, H020);
  enforce_univariate(s.s003, s.s004, h2min, s3max, H002);
  T A220 = sqrt((H200 + sq(s.s300)) * (H020 + sq(s.s030)));
  s.s220 = realizablity_S220(s.s110, s.s220, A220);
  T A202 = sqrt((H200 + sq(s.s300)) * (H002 + sq(s.s003)));
  s.s202 = realizablity_S220(s.s101, s.s202, A202);
  T A022 = sqrt((H020 + sq(s.s030)) * (H002 + sq(s.s003)));
  s.s022 = realizablity_S220(s.s011, s.s022, A022);

  // check2D_all_planes (src/utils/diagnostics.jl:168-187)
  T p1[10] = {s.s300, s.s400, s.s110, s.s210, s.s310, s.s120, s.s220, s.s030, s.s130, s.s040};
  T p2[10] = {s.s300, s.s400, s.s101, s.s201, s.s301, s.s102, s.s202, s.s003, s.s103, s.s004};
  T p3[10] = {s.s030, s.s040, s.s011, s.s021, s.s031, s.s012, s.s022, s.s003, s.s013, s.s004};
  check2D(p1[0], p1[1], p1[2], p1[3], p1[4], p1[5], p1[6], p1[7], p1[8], p1[9]);
  check2D(p2[0], p2[1], p2[2], p2[3], p2[4], p2[5], p2[6], p2[7], p2[8], p2[9]);
  check2D(p3[0], p3[1], p3[2], p3[3], p3[4], p3[5], p3[6], p3[7], p3[8], p3[9]);
  T S300r1 = p1[0], S400r1 = p1[1], S110r = p1[2], S210r = p1[3], S310r = p1[4], S120r = p1[5], S220r = p1[6], S030r1 = p1[7], S130r = p1[8], S040r1 = p1[9];
  T S300r2 = p2[0], S400r2 = p2[1], S101r = p2[2], S201r = p2[3], S301r = p2[4], S102r = p2[5], S202r = p2[6], S003r2 = p2[7], S103r = p2[8], S004r2 = p2[9];
  T S030r3 = p3[0], S040r3 = p3[1], S011r = p3[2], S021r = p3[3], S031r = p3[4], S012r = p3[5], S022r = p3[6], S003r3 = p3[7], S013r = p3[8], S004r3 = p3[9];
  (void)S130r;
  T S111r = s.s111, S211r = s.s211, S121r = s.s121, S112r = s.s112;
  T S300r = s.s300, S030r = s.s030, S003r = s.s003, S400r = s.s400, S040r = s.s040, S004r = s.s004;
  (void)S211r; (void)S121r; (void)S112r; (void)S111r;

  T R110 = T(1) - sq(s.s110), R101 = T(1) - sq(s.s101), R011 = T(1) - sq(s.s011);
  if (R110 <= T(0) || R101 <= T(0) || R011 <= T(0)) {
    hit(BR_EDGE_CORNER);
    // edge_corner_correction (src/realizability/edge_corner_correction.jl:24-110)
    S19<T> a;
    T S110, S101, S011, S300, S030, S003, S400, S040, S004, dummy;
    if (R110 <= T(0) && R101 > T(0) && R011 > T(0)) {
      S110 = jsign(S110r);
      T Smean = (S011r + S101r) / T(2);
      S011 = jsign(S011r) * Smean; S101 = jsign(S101r) * Smean;
      realizability_S2(S110, S101, S011, S110, S101, S011, dummy);
      S300 = S300r1; S030 = S030r1; S400 = S400r1; S040 = S040r1; S003 = S003r; S004 = S004r;
      a = avg_edge_xy(S110, S030, S040, S300r, S400r, S021r, S012r, S013r, S031r, S022r, S201r, S102r, S103r, S301r, S202r, S003r, S004r);
    } else if (R101 <= T(0) && R110 > T(0) && R011 > T(0)) {
      S101 = jsign(S101r);
      T Smean = (S011r + S110r) / T(2);
      S011 = jsign(S011r) * Smean; S110 = jsign(S110r) * Smean;
      realizability_S2(S110, S101, S011, S110, S101, S011, dummy);
      S300 = S300r2; S003 = S003r2; S400 = S400r2; S004 = S004r2; S030 = S030r; S040 = S040r;
      a = avg_edge_xz(S101, S003, S004, S300r, S400r, S021r, S012r, S013r, S031r, S022r, S030r, S210r, S120r, S220r, S130r, S310r);
    } else if (R011 <= T(0) && R101 > T(0) && R110 > T(0)) {
      S011 = jsign(S011r);
      T Smean = (S101r + S110r) / T(2);
      S101 = jsign(S101r) * Smean; S110 = jsign(S110r) * Smean;
      realizability_S2(S110, S101, S011, S110, S101, S011, dummy);
      S030 = S030r3; S003 = S003r3; S040 = S040r3; S004 = S004r3; S300 = S300r; S400 = S400r;
      a = avg_edge_yz(S011, S003, S004, S030r, S040r, S201r, S102r, S103r, S301r, S202r, S300r, S210r, S120r, S220r, S130r, S310r);
    } else {
      S110 = jsign(S110r); S101 = jsign(S101r); S011 = jsign(S011r);
      realizability_S2(S110, S101, S011, S110, S101, S011, dummy);
      S300 = (S030r1 + S030r + S300r) / T(3);
      S030 = (S030r1 + S030r + S030r3) / T(3);
      S003 = (S003r + S003r2 + S003r3) / T(3);
      S400 = (S040r1 + S040r + S400r) / T(3);
      S040 = (S040r1 + S040r + S040r3) / T(3);
      S004 = (S004r + S004r2 + S004r3) / T(3);
      a = avg_corner(S110, S101, S011, S030r1, S040r1, S030r, S040r, S300r, S400r, S003r3, S004r3);
    }
    s.s110 = S110; s.s101 = S101; s.s011 = S011; s.s300 = S300; s.s030 = S030; s.s003 = S003;
    s.s400 = S400; s.s040 = S040; s.s004 = S004;
    s.s210 = a.s210; s.s201 = a.s201; s.s120 = a.s120; s.s111 = a.s111; s.s102 = a.s102; s.s021 = a.s021; s.s012 = a.s012;
    s.s310 = a.s310; s.s301 = a.s301; s.s220 = a.s220; s.s211 = a.s211; s.s202 = a.s202; s.s130 = a.s130; s.s121 = a.s121;
    s.s112 = a.s112; s.s103 = a.s103; s.s031 = a.s031; s.s022 = a.s022; s.s013 = a.s013;
    realizable_2D(s.s300, s.s400, s.s110, s.s210, s.s310, s.s120, s.s220, s.s030, s.s130, s.s040);
    realizable_2D(s.s300, s.s400, s.s101, s.s201, s.s301, s.s102, s.s202, s.s003, s.s103, s.s004);
    realizable_2D(s.s030, s.s040, s.s011, s.s021, s.s031, s.s012, s.s022, s.s003, s.s013, s.s004);
  } else {
    int flag220 = realizable_3D(s);
    int itreal = 0;
    while (flag220 == 1 && itreal < itrealmax) {
      ++itreal;
      hit(BR_FLAG220);
      realizable_3D(s);
    }
  }
  if (flag2D == 1) {
    s.s011 = T(0); s.s101 = T(0); s.s201 = T(0); s.s021 = T(0); s.s012 = T(0); s.s102 = T(0); s.s111 = T(0);
    s.s202 = T(1); s.s022 = T(1); s.s112 = s.s110; s.s121 = T(0); s.s211 = T(0); s.s103 = T(0); s.s013 = T(0);
    s.s301 = T(0); s.s031 = T(0);
  }
  S5<T> f = hyqmom_3D(s);
  T sC200 = sqrt(jmax(T(EPS), C200)), sC020 = sqrt(jmax(T(EPS), C020)), sC002 = sqrt(jmax(T(EPS), C002));
  // S_to_C_batch (src/utils/moment_array_utils.jl:137-204)
  T Cc[216];
  for (int i = 0; i < 216; ++i) Cc[i] = T(0);
  auto put = [&](int i, int j, int k, T sv) {
    T d = sv;
    T f1[3] = {sC200, sC020, sC002};
    int ex[3] = {i, j, k};
    for (int r = 0; r < 3; ++r) {
      if (ex[r] == 0) continue;
      T p = ex[r] == 4 ? pow4(f1[r]) : (ex[r] == 5 ? pow5(f1[r]) : ipow(f1[r], ex[r]));
      d = d * p;
    }
    Cc[t3(i, j, k)] = d;
  };
  put(1, 1, 0, s.s110); put(1, 0, 1, s.s101); put(0, 1, 1, s.s011);
  put(3, 0, 0, s.s300); put(2, 1, 0, s.s210); put(2, 0, 1, s.s201); put(1, 2, 0, s.s120); put(1, 1, 1, s.s111);
  put(1, 0, 2, s.s102); put(0, 3, 0, s.s030); put(0, 2, 1, s.s021); put(0, 1, 2, s.s012); put(0, 0, 3, s.s003);
  put(4, 0, 0, s.s400); put(3, 1, 0, s.s310); put(3, 0, 1, s.s301); put(2, 2, 0, s.s220); put(2, 1, 1, s.s211);
  put(2, 0, 2, s.s202); put(1, 3, 0, s.s130); put(1, 2, 1, s.s121); put(1, 1, 2, s.s112); put(1, 0, 3, s.s103);
  put(0, 4, 0, s.s040); put(0, 3, 1, s.s031); put(0, 2, 2, s.s022); put(0, 1, 3, s.s013); put(0, 0, 4, s.s004);
  put(5, 0, 0, f.s500); put(4, 1, 0, f.s410); put(4, 0, 1, f.s401); put(3, 2, 0, f.s320); put(3, 1, 1, f.s311);
  put(3, 0, 2, f.s302); put(2, 3, 0, f.s230); put(2, 2, 1, f.s221); put(2, 1, 2, f.s212); put(2, 0, 3, f.s203);
  put(1, 4, 0, f.s140); put(1, 3, 1, f.s131); put(1, 2, 2, f.s122); put(1, 1, 3, f.s113); put(1, 0, 4, f.s104);
  put(0, 5, 0, f.s050); put(0, 4, 1, f.s041); put(0, 3, 2, f.s032); put(0, 2, 3, f.s023); put(0, 1, 4, f.s014);
  put(0, 0, 5, f.s005);
  Cc[t3(2, 0, 0)] = C200; Cc[t3(0, 2, 0)] = C020; Cc[t3(0, 0, 2)] = C002;
  T M5[216];
  c_to_m(M000, umean, vmean, wmean, Cc, M5, 5);
  for (int n = 0; n < 35; ++n) {
    int i = E35[n][0], j = E35[n][1], k = E35[n][2];
    M4r[n] = M5[t3(i, j, k)];
    Fx[n] = M5[t3(i + 1, j, k)];
    Fy[n] = M5[t3(i, j + 1, k)];
    Fz[n] = M5[t3(i, j, k + 1)];
  }
}

}  // namespace hyqo
