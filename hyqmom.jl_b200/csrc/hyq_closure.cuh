// 3-D realizability, 5th-order HyQMOM closure and the flux closure driver
// (device code).  Restates src/realizability/realizable_3D.jl:39-624,
// src/realizability/edge_corner_correction.jl:24-252,
// src/moments/hyqmom_3D.jl:147-190 and
// src/numerics/Flux_closure35_and_realizable_3D.jl:33-234.
#pragma once
#include "hyq_cell.cuh"

namespace hyq {

// realizable_3D on the 28-set s[] (enum order); returns flag220.
HQN int realizable_3D(double* s) {
  int flag220 = 0;
  const double diagmin = 1e-10, h2min = 1e-10, S2min = 1e-12;
  const double H200 = jmax(EPS, s[s400] - s[s300] * s[s300] - 1.0);
  const double H020 = jmax(EPS, s[s040] - s[s030] * s[s030] - 1.0);
  const double H002 = jmax(EPS, s[s004] - s[s003] * s[s003] - 1.0);
  const double A220 = sqrt((H200 + s[s300] * s[s300]) * (H020 + s[s030] * s[s030]));
  const double S220max = realizablity_S220(s[s110], s[s220], A220);
  const double A202 = sqrt((H200 + s[s300] * s[s300]) * (H002 + s[s003] * s[s003]));
  const double S202max = realizablity_S220(s[s101], s[s202], A202);
  const double A022 = sqrt((H020 + s[s030] * s[s030]) * (H002 + s[s003] * s[s003]));
  const double S022max = realizablity_S220(s[s011], s[s022], A022);
  s[s220] = jmin(s[s220], S220max);
  s[s202] = jmin(s[s202], S202max);
  s[s022] = jmin(s[s022], S022max);
  double S2;
  realizability_S2(s[s110], s[s101], s[s011], S2);
  const double R110 = sqrt(jmax(0.0, 1.0 - s[s110] * s[s110]));
  const double R101 = sqrt(jmax(0.0, 1.0 - s[s101] * s[s101]));
  const double R011 = sqrt(jmax(0.0, 1.0 - s[s011] * s[s011]));

  if (S2 <= S2min) {  // faces
    const double Rmax = jmax(jmax(R110, R101), R011);
    if (R110 == Rmax) {
      const double g1 = (s[s101] - s[s110] * s[s011]) / (1.0 - s[s110] * s[s110]);
      const double g2 = (s[s011] - s[s110] * s[s101]) / (1.0 - s[s110] * s[s110]);
      s[s021] = g2 * s[s030] + g1 * s[s120];
      s[s201] = g2 * s[s210] + g1 * s[s300];
      s[s031] = g2 * s[s040] + g1 * s[s130];
      s[s301] = g2 * s[s310] + g1 * s[s400];
      s[s111] = g2 * s[s120] + g1 * s[s210];
      s[s211] = g2 * s[s220] + g1 * s[s310];
      s[s121] = g2 * s[s130] + g1 * s[s220];
      s[s012] = sq(g2) * s[s030] + 2.0 * g1 * g2 * s[s120] + sq(g1) * s[s210];
      s[s102] = sq(g2) * s[s120] + 2.0 * g1 * g2 * s[s210] + sq(g1) * s[s300];
      s[s022] = sq(g2) * s[s040] + 2.0 * g1 * g2 * s[s130] + sq(g1) * s[s220];
      s[s202] = sq(g2) * s[s220] + 2.0 * g1 * g2 * s[s310] + sq(g1) * s[s400];
      s[s112] = sq(g2) * s[s130] + 2.0 * g1 * g2 * s[s220] + sq(g1) * s[s310];
      s[s003] = cube(g2) * s[s030] + 3.0 * g1 * sq(g2) * s[s120] + 3.0 * sq(g1) * g2 * s[s210] + cube(g1) * s[s300];
      s[s013] = cube(g2) * s[s040] + 3.0 * g1 * sq(g2) * s[s130] + 3.0 * sq(g1) * g2 * s[s220] + cube(g1) * s[s310];
      s[s103] = cube(g2) * s[s130] + 3.0 * g1 * sq(g2) * s[s220] + 3.0 * sq(g1) * g2 * s[s310] + cube(g1) * s[s400];
      s[s004] = pow4(g2) * s[s040] + 4.0 * g1 * cube(g2) * s[s130] + 6.0 * sq(g1) * sq(g2) * s[s220] + 4.0 * cube(g1) * g2 * s[s310] + pow4(g1) * s[s400];
    } else if (R101 == Rmax) {
      const double g3 = (s[s110] - s[s101] * s[s011]) / (1.0 - s[s101] * s[s101]);
      const double g4 = (s[s011] - s[s110] * s[s101]) / (1.0 - s[s101] * s[s101]);
      s[s012] = g4 * s[s003] + g3 * s[s102];
      s[s210] = g4 * s[s201] + g3 * s[s300];
      s[s013] = g4 * s[s004] + g3 * s[s103];
      s[s310] = g4 * s[s301] + g3 * s[s400];
      s[s111] = g4 * s[s102] + g3 * s[s201];
      s[s211] = g4 * s[s202] + g3 * s[s301];
      s[s112] = g4 * s[s103] + g3 * s[s202];
      s[s021] = sq(g4) * s[s003] + 2.0 * g3 * g4 * s[s102] + sq(g3) * s[s201];
      s[s120] = sq(g4) * s[s102] + 2.0 * g3 * g4 * s[s201] + sq(g3) * s[s300];
      s[s022] = sq(g4) * s[s004] + 2.0 * g3 * g4 * s[s103] + sq(g3) * s[s202];
      s[s220] = sq(g4) * s[s202] + 2.0 * g3 * g4 * s[s301] + sq(g3) * s[s400];
      s[s121] = sq(g4) * s[s103] + 2.0 * g3 * g4 * s[s202] + sq(g3) * s[s301];
      s[s030] = cube(g4) * s[s003] + 3.0 * g3 * sq(g4) * s[s102] + 3.0 * sq(g3) * g4 * s[s201] + cube(g3) * s[s300];
      s[s031] = cube(g4) * s[s004] + 3.0 * g3 * sq(g4) * s[s103] + 3.0 * sq(g3) * g4 * s[s202] + cube(g3) * s[s301];
      s[s130] = cube(g4) * s[s103] + 3.0 * g3 * sq(g4) * s[s202] + 3.0 * sq(g3) * g4 * s[s301] + cube(g3) * s[s400];
      s[s040] = pow4(g4) * s[s004] + 4.0 * g3 * cube(g4) * s[s103] + 6.0 * sq(g3) * sq(g4) * s[s202] + 4.0 * cube(g3) * g4 * s[s301] + pow4(g3) * s[s400];
    } else {
      const double g5 = (s[s101] - s[s110] * s[s011]) / (1.0 - s[s011] * s[s011]);
      const double g6 = (s[s110] - s[s101] * s[s011]) / (1.0 - s[s011] * s[s011]);
      s[s102] = g6 * s[s003] + g5 * s[s012];
      s[s120] = g6 * s[s021] + g5 * s[s030];
      s[s103] = g6 * s[s004] + g5 * s[s013];
      s[s130] = g6 * s[s031] + g5 * s[s040];
      s[s111] = g6 * s[s012] + g5 * s[s021];
      s[s121] = g6 * s[s022] + g5 * s[s031];
      s[s112] = g6 * s[s013] + g5 * s[s022];
      s[s201] = sq(g6) * s[s003] + 2.0 * g5 * g6 * s[s012] + sq(g5) * s[s021];
      s[s210] = sq(g6) * s[s012] + 2.0 * g5 * g6 * s[s021] + sq(g5) * s[s030];
      s[s202] = sq(g6) * s[s004] + 2.0 * g5 * g6 * s[s013] + sq(g5) * s[s022];
      s[s220] = sq(g6) * s[s022] + 2.0 * g5 * g6 * s[s031] + sq(g5) * s[s040];
      s[s211] = sq(g6) * s[s013] + 2.0 * g5 * g6 * s[s022] + sq(g5) * s[s031];
      s[s300] = cube(g6) * s[s003] + 3.0 * g5 * sq(g6) * s[s012] + 3.0 * sq(g5) * g6 * s[s021] + cube(g5) * s[s030];
      s[s301] = cube(g6) * s[s004] + 3.0 * g5 * sq(g6) * s[s013] + 3.0 * sq(g5) * g6 * s[s022] + cube(g5) * s[s031];
      s[s310] = cube(g6) * s[s013] + 3.0 * g5 * sq(g6) * s[s022] + 3.0 * sq(g5) * g6 * s[s031] + cube(g5) * s[s040];
      s[s400] = pow4(g6) * s[s004] + 4.0 * g5 * cube(g6) * s[s013] + 6.0 * sq(g5) * sq(g6) * s[s022] + 4.0 * cube(g5) * g6 * s[s031] + pow4(g5) * s[s040];
    }
    return flag220;
  }

  const double beta = 1.0;
  // one projection store for the whole function: each projection below is
  // formed, read and dropped before the next (a smaller per-thread frame)
  Delta D;
  delta2star_p(s, 0, D);
  int fE11 = 0, fE22 = 0, fE33 = 0, fE44 = 0, fE55 = 0, fE66 = 0;
  if (E_(D, 0, 0) < 0.0) { realizability_S210(s[s110], s[s101], s[s011], s[s300], s[s210], s[s201], H200, beta); fE11 = 1; }
  if (E_(D, 3, 3) < 0.0) { realizability_S210(s[s110], s[s011], s[s101], s[s030], s[s120], s[s021], H020, beta); fE44 = 1; }
  if (E_(D, 5, 5) < 0.0) { realizability_S210(s[s011], s[s101], s[s110], s[s003], s[s012], s[s102], H002, beta); fE66 = 1; }
  // delta2star_p is a pure function of s, so a projection of an unchanged s
  // is reused below instead of recomputed (same values as the reference's
  // recomputation); `written` records writes to s since D was formed
  bool written = (fE11 | fE44 | fE66) != 0;
  const double S111r = realizability_S111(s[s110], s[s101], s[s011], s[s210], s[s201], s[s120], s[s021], s[s102], s[s012], s[s111]);
  if (S111r != s[s111]) { s[s111] = S111r; written = true; }
  const double S220_310 = realizability_S310_220(s[s110], s[s101], s[s011], s[s210], s[s120], s[s111], s[s220]);
  const double S202_310 = realizability_S310_220(s[s101], s[s110], s[s011], s[s201], s[s102], s[s111], s[s202]);
  const double S022_310 = realizability_S310_220(s[s011], s[s110], s[s101], s[s021], s[s012], s[s111], s[s022]);
  double S220_diag = s[s220], S202_diag = s[s202], S022_diag = s[s022];
  // lower_bound_S220: projection diagonal of the current moments
  if (written) delta2star_p(s, 0, D);
  const double lb0 = Q_(D, 1, 1), lb1 = Q_(D, 2, 2), lb2 = Q_(D, 4, 4);
  if (s[s220] < lb0) { S220_diag = lb0; fE22 = 1; flag220 = 1; }
  if (s[s202] < lb1) { S202_diag = lb1; fE33 = 1; flag220 = 1; }
  if (s[s022] < lb2) { S022_diag = lb2; fE55 = 1; flag220 = 1; }
  // recheck diagonal (same moments as the projection above)
  if (E_(D, 0, 0) < diagmin) fE11 = 1;
  if (E_(D, 1, 1) < diagmin) fE22 = 1;
  if (E_(D, 2, 2) < diagmin) fE33 = 1;
  if (E_(D, 3, 3) < diagmin) fE44 = 1;
  if (E_(D, 4, 4) < diagmin) fE55 = 1;
  if (E_(D, 5, 5) < diagmin) fE66 = 1;
  if (fE11 | fE22 | fE33 | fE44 | fE55 | fE66) {
    // bound_minor1 values from the projection
    const double S310b = Q_(D, 0, 1), S301b = Q_(D, 0, 2), S130b = Q_(D, 1, 3), S103b = Q_(D, 2, 5);
    const double S031b = Q_(D, 3, 4), S013b = Q_(D, 4, 5);
    const double S211b = Q_(D, 0, 4), S121b = Q_(D, 2, 3), S112b = Q_(D, 1, 5);
    if (fE11) { s[s310] = S310b; s[s301] = S301b; s[s211] = S211b; }
    if (fE22) { s[s310] = S310b; s[s130] = S130b; s[s211] = S211b; s[s121] = S121b; s[s112] = S112b; }
    if (fE33) { s[s301] = S301b; s[s103] = S103b; s[s211] = S211b; s[s121] = S121b; s[s112] = S112b; }
    if (fE44) { s[s130] = S130b; s[s031] = S031b; s[s121] = S121b; }
    if (fE55) { s[s031] = S031b; s[s013] = S013b; s[s211] = S211b; s[s121] = S121b; s[s112] = S112b; }
    if (fE66) { s[s103] = S103b; s[s013] = S013b; s[s112] = S112b; }
  }
  if (fE11 & fE22 & fE33 & fE44 & fE55 & fE66) return flag220;

  // 2x2 minors of the six permutations
  double S220a = s[s220], S220b = s[s220], S202a = s[s202], S202b = s[s202], S022a = s[s022], S022b = s[s022];
  // Of the six projections only their 2x2, 3x3 and 4x4 leading minors and
  // the leading 3x3 entries of permutations 0, 2, 5 are used below (the 4x4
  // minors while s is unchanged), so those are kept instead of the six Delta
  // structs (a smaller per-thread frame; the values are the same).
  double d2[6], d3[6], d4[6];
  double Ee[3][6];  // (0,0),(0,1),(0,2),(1,1),(1,2),(2,2) of projections 0, 2, 5
  auto keep = [&](int p, const Delta& Dp) {
    d3[p] = lead_det_k<3>(Dp);
    d4[p] = lead_det_k<4>(Dp);
    const int slot = (p == 0) ? 0 : (p == 2) ? 1 : (p == 5) ? 2 : -1;
    if (slot >= 0) {
      Ee[slot][0] = E_(Dp, 0, 0); Ee[slot][1] = E_(Dp, 0, 1); Ee[slot][2] = E_(Dp, 0, 2);
      Ee[slot][3] = E_(Dp, 1, 1); Ee[slot][4] = E_(Dp, 1, 2); Ee[slot][5] = E_(Dp, 2, 2);
    }
  };
  // D is still the projection 0 of s unless the bound_minor1 block wrote s
  const bool reuseD = (fE11 | fE22 | fE33 | fE44 | fE55 | fE66) == 0;
  for (int p = 0; p < 6; ++p) {
    if (p == 0 && reuseD) {
      d2[0] = lead_det_k<2>(D);
      keep(0, D);
      continue;
    }
    delta2star_p(s, p, D);  // D is not needed after projection 0
    d2[p] = lead_det_k<2>(D);
    keep(p, D);
  }
  bool fresh = true;  // d2..Ee are those of the current s
  int flag310 = 0;
  if (!fE11 && !fE44 && d2[0] < h2min) {
    s[s310] = realizability_S310(s[s110], s[s101], s[s011], s[s300], s[s210], s[s120], s[s201], s[s111], s[s310], s[s220], H200, beta);
    S220a = s[s220]; flag310 = 1;
  }
  if (!fE22 && !fE44 && d2[2] < h2min) {
    s[s130] = realizability_S310(s[s110], s[s011], s[s101], s[s030], s[s120], s[s021], s[s210], s[s111], s[s130], s[s220], H020, beta);
    S220b = s[s220]; flag310 = 1;
  }
  if (!fE11 && !fE33 && d2[1] < h2min) {
    s[s301] = realizability_S310(s[s101], s[s110], s[s011], s[s300], s[s201], s[s210], s[s102], s[s111], s[s301], s[s202], H200, beta);
    S202a = s[s202]; flag310 = 1;
  }
  if (!fE33 && !fE66 && d2[3] < h2min) {
    s[s103] = realizability_S310(s[s101], s[s011], s[s110], s[s003], s[s102], s[s012], s[s201], s[s111], s[s103], s[s202], H002, beta);
    S202b = s[s202]; flag310 = 1;
  }
  if (!fE44 && !fE55 && d2[4] < h2min) {
    s[s031] = realizability_S310(s[s011], s[s110], s[s101], s[s030], s[s021], s[s120], s[s012], s[s111], s[s031], s[s022], H020, beta);
    S022a = s[s022]; flag310 = 1;
  }
  if (!fE55 && !fE66 && d2[5] < h2min) {
    s[s013] = realizability_S310(s[s011], s[s101], s[s110], s[s003], s[s012], s[s102], s[s021], s[s111], s[s013], s[s022], H002, beta);
    S022b = s[s022]; flag310 = 1;
  }
  const double S220r = jmax(S220a, S220b);
  double S220_310r = S220_310;
  if (s[s220] < S220r) { S220_310r = S220r; flag220 = 1; }
  const double S022r = jmax(S022a, S022b);
  double S022_310r = S022_310;
  if (s[s022] < S022r) { S022_310r = S022r; flag220 = 1; }
  const double S202r = jmax(S202a, S202b);
  double S202_310r = S202_310;
  if (s[s202] < S202r) { S202_310r = S202r; flag220 = 1; }
  if (flag310) {
    double dm = 0.0;
    for (int p = 0; p < 6; ++p) {
      delta2star_p(s, p, D);
      const double d = lead_det_k<2>(D);
      dm = (p == 0) ? d : jmin(dm, d);
      keep(p, D);
    }
    if (dm < 0.0) flag220 = 1;
  }

  // 3x3 minors
  S220a = s[s220]; S220b = s[s220]; S202a = s[s202];
  double S202c = s[s202];
  S022b = s[s022];
  double S022c = s[s022];
  if (!fE11 && !fE22 && !fE33 && !fE55) {
    if (d3[0] <= h2min || d3[1] <= h2min) {
      const double e11 = Ee[0][0], e12 = Ee[0][1], e13 = Ee[0][2], e22 = Ee[0][3], e23 = Ee[0][4], e33 = Ee[0][5];
      const double d23 = s[s211] - e23, d22 = s[s220] - e22, d33 = s[s202] - e33;
      if (e11 > diagmin) { S220a = d22 + e13 * e13 / e11; S202a = d33 + e12 * e12 / e11; }
      s[s211] = realizability_S211(e11, e22, e33, e12, e13, d23, s[s211], beta);
      flag220 = 1;
      fresh = false;
    }
  }
  if (!fE22 && !fE33 && !fE44 && !fE55) {
    if (d3[2] < h2min || d3[4] < h2min) {
      const double e11 = Ee[1][0], e12 = Ee[1][1], e13 = Ee[1][2], e22 = Ee[1][3], e23 = Ee[1][4], e33 = Ee[1][5];
      const double d23 = s[s121] - e23, d22 = s[s220] - e22, d33 = s[s022] - e33;
      if (e11 > diagmin) { S220b = d22 + e13 * e13 / e11; S022b = d33 + e12 * e12 / e11; }
      s[s121] = realizability_S211(e11, e22, e33, e12, e13, d23, s[s121], beta);
      flag220 = 1;
      fresh = false;
    }
  }
  if (!fE22 && !fE33 && !fE55 && !fE66) {
    if (d3[3] < h2min || d3[5] < h2min) {
      const double e11 = Ee[2][0], e12 = Ee[2][1], e13 = Ee[2][2], e22 = Ee[2][3], e23 = Ee[2][4], e33 = Ee[2][5];
      const double d23 = s[s112] - e23, d22 = s[s022] - e22, d33 = s[s202] - e33;
      if (e11 > diagmin) { S202c = d22 + e13 * e13 / e11; S022c = d33 + e12 * e12 / e11; }
      s[s112] = realizability_S211(e11, e22, e33, e12, e13, d23, s[s112], beta);
      flag220 = 1;
      fresh = false;
    }
  }
  const double S220_211 = jmax(S220a, S220b), S202_211 = jmax(S202a, S202c), S022_211 = jmax(S022b, S022c);

  // 4x4 minors: cubic roots bound the S220-type moments
  double lo[6], hi[6];
  const double cur[6] = {s[s220], s[s220], s[s202], s[s202], s[s022], s[s022]};
  for (int q = 0; q < 6; ++q) {
    // order of the reference: E1, E3 (S220), E2, E4 (S202), E5, E6 (S022)
    const int p = (q == 0) ? 0 : (q == 1) ? 2 : (q == 2) ? 1 : (q == 3) ? 3 : (q == 4) ? 4 : 5;
    lo[q] = cur[q]; hi[q] = cur[q];
    if (fresh && !(d4[p] < 0.0)) continue;  // its projection is the kept one
    Delta& E = D;
    delta2star_p(s, p, E);
    if (lead_det_k<4>(E) < 0.0) {
      flag220 = 1;
      const double ex = -E_(E, 1, 1) + E_(E, 0, 3);
      const double d22 = cur[q] - E_(E, 1, 1);
      Roots3 R = roots_X_Y(E_(E, 2, 2), E_(E, 0, 0), E_(E, 0, 1), E_(E, 0, 2), E_(E, 1, 2), E_(E, 1, 3), E_(E, 2, 3), E_(E, 3, 3), ex);
      double Rr[3] = {R.re[0], R.re[1], R.re[2]};
      sort3(Rr);
      if (imag_ratio(R) < 1000.0 * EPS) { lo[q] = Rr[1] + d22; hi[q] = Rr[2] + d22; }
    }
  }
  double v;
  v = jmax(jmax(jmax(jmax(jmax(lo[0], lo[1]), S220_diag), S220_310), S220_310r), S220_211);
  s[s220] = jmin(jmin(jmin(v, S220max), hi[0]), hi[1]);
  v = jmax(jmax(jmax(jmax(jmax(lo[2], lo[3]), S202_diag), S202_310), S202_310r), S202_211);
  s[s202] = jmin(jmin(jmin(v, S202max), hi[2]), hi[3]);
  v = jmax(jmax(jmax(jmax(jmax(lo[4], lo[5]), S022_diag), S022_310), S022_310r), S022_211);
  s[s022] = jmin(jmin(jmin(v, S022max), hi[4]), hi[5]);
  return flag220;
}

// Edge/corner correction + 2-D re-check (src/realizability/edge_corner_correction.jl:24-252)
// on the 28-set; r* are the check2D outputs, o* the post-univariate values.
struct Planes { double p1[10], p2[10], p3[10]; };
HQN void edge_corner(double* s, const Planes& pl, double R110, double R101, double R011) {
  const double S300r1 = pl.p1[0], S400r1 = pl.p1[1], S110r = pl.p1[2], S210r = pl.p1[3], S310r = pl.p1[4], S120r = pl.p1[5], S220r = pl.p1[6],
               S030r1 = pl.p1[7], S130r = pl.p1[8], S040r1 = pl.p1[9];
  const double S300r2 = pl.p2[0], S400r2 = pl.p2[1], S101r = pl.p2[2], S201r = pl.p2[3], S301r = pl.p2[4], S102r = pl.p2[5], S202r = pl.p2[6],
               S003r2 = pl.p2[7], S103r = pl.p2[8], S004r2 = pl.p2[9];
  const double S030r3 = pl.p3[0], S040r3 = pl.p3[1], S011r = pl.p3[2], S021r = pl.p3[3], S031r = pl.p3[4], S012r = pl.p3[5], S022r = pl.p3[6],
               S003r3 = pl.p3[7], S013r = pl.p3[8], S004r3 = pl.p3[9];
  const double S300r = s[s300], S030r = s[s030], S003r = s[s003], S400r = s[s400], S040r = s[s040], S004r = s[s004];
  double S110, S101, S011, S300, S030, S003, S400, S040, S004, dummy;
  double o[19];  // s210 s201 s120 s111 s102 s021 s012 s310 s301 s220 s211 s202 s130 s121 s112 s103 s031 s022 s013
  if (R110 <= 0.0 && R101 > 0.0 && R011 > 0.0) {
    S110 = jsign(S110r);
    const double Sm = (S011r + S101r) / 2.0;
    S011 = jsign(S011r) * Sm; S101 = jsign(S101r) * Sm;
    realizability_S2(S110, S101, S011, dummy);
    S300 = S300r1; S030 = S030r1; S400 = S400r1; S040 = S040r1; S003 = S003r; S004 = S004r;
    const double a = S110;
    o[0] = (S030 + a * S300r) / 2.0; o[1] = (S021r + S201r) / 2.0; o[2] = (a * S030 + S300r) / 2.0;
    o[3] = (a * S021r + a * S201r) / 2.0; o[4] = (a * S012r + S102r) / 2.0; o[5] = (S021r + S201r) / 2.0;
    o[6] = (S012r + a * S102r) / 2.0; o[7] = (a * S040 + a * S400r) / 2.0; o[8] = (a * S031r + S301r) / 2.0;
    o[9] = (S040 + S400r) / 2.0; o[10] = (S031r + a * S301r) / 2.0; o[11] = (S022r + S202r) / 2.0;
    o[12] = (a * S040 + a * S400r) / 2.0; o[13] = (a * S031r + S301r) / 2.0; o[14] = (a * S022r + a * S202r) / 2.0;
    o[15] = (a * S013r + S103r) / 2.0; o[16] = (S031r + a * S301r) / 2.0; o[17] = (S022r + S202r) / 2.0;
    o[18] = (S013r + a * S103r) / 2.0;
  } else if (R101 <= 0.0 && R110 > 0.0 && R011 > 0.0) {
    S101 = jsign(S101r);
    const double Sm = (S011r + S110r) / 2.0;
    S011 = jsign(S011r) * Sm; S110 = jsign(S110r) * Sm;
    realizability_S2(S110, S101, S011, dummy);
    S300 = S300r2; S003 = S003r2; S400 = S400r2; S004 = S004r2; S030 = S030r; S040 = S040r;
    const double a = S101;
    o[0] = (S013r + S210r) / 2.0; o[1] = (S003 + a * S300r) / 2.0; o[2] = (a * S021r + S120r) / 2.0;
    o[3] = (a * S012r + a * S210r) / 2.0; o[4] = (a * S003 + S300r) / 2.0; o[5] = (S021r + a * S120r) / 2.0;
    o[6] = (S012r + S210r) / 2.0; o[7] = (a * S013r + S310r) / 2.0; o[8] = (a * S004 + a * S400r) / 2.0;
    o[9] = (S022r + S220r) / 2.0; o[10] = (S013r + a * S310r) / 2.0; o[11] = (S004 + S400r) / 2.0;
    o[12] = (a * S031r + S130r) / 2.0; o[13] = (a * S022r + a * S220r) / 2.0; o[14] = (a * S013r + S310r) / 2.0;
    o[15] = (a * S004 + a * S400r) / 2.0; o[16] = (S031r + a * S130r) / 2.0; o[17] = (S022r + S220r) / 2.0;
    o[18] = (S013r + a * S310r) / 2.0;
  } else if (R011 <= 0.0 && R101 > 0.0 && R110 > 0.0) {
    S011 = jsign(S011r);
    const double Sm = (S101r + S110r) / 2.0;
    S101 = jsign(S101r) * Sm; S110 = jsign(S110r) * Sm;
    realizability_S2(S110, S101, S011, dummy);
    S030 = S030r3; S003 = S003r3; S040 = S040r3; S004 = S004r3; S300 = S300r; S400 = S400r;
    const double a = S011;
    o[0] = (a * S201r + S210r) / 2.0; o[1] = (S201r + a * S210r) / 2.0; o[2] = (S102r + S120r) / 2.0;
    o[3] = (a * S102r + a * S120r) / 2.0; o[4] = (S102r + S120r) / 2.0; o[5] = (S003 + a * S030r) / 2.0;
    o[6] = (a * S003 + S030r) / 2.0; o[7] = (a * S301r + S310r) / 2.0; o[8] = (S301r + a * S310r) / 2.0;
    o[9] = (S202r + S220r) / 2.0; o[10] = (a * S202r + a * S220r) / 2.0; o[11] = (S202r + S220r) / 2.0;
    o[12] = (a * S103r + S130r) / 2.0; o[13] = (S103r + a * S130r) / 2.0; o[14] = (a * S103r + S130r) / 2.0;
    o[15] = (S103r + a * S130r) / 2.0; o[16] = (a * S004 + a * S040r) / 2.0; o[17] = (S004 + S040r) / 2.0;
    o[18] = (a * S004 + a * S040r) / 2.0;
  } else {
    S110 = jsign(S110r); S101 = jsign(S101r); S011 = jsign(S011r);
    realizability_S2(S110, S101, S011, dummy);
    S300 = (S030r1 + S030r + S300r) / 3.0;
    S030 = (S030r1 + S030r + S030r3) / 3.0;
    S003 = (S003r + S003r2 + S003r3) / 3.0;
    S400 = (S040r1 + S040r + S400r) / 3.0;
    S040 = (S040r1 + S040r + S040r3) / 3.0;
    S004 = (S004r + S004r2 + S004r3) / 3.0;
    const double A3 = S030r1, A4 = S040r1, B3 = S030r, B4 = S040r, C3 = S003r3, C4 = S004r3;
    const double x = S110, y = S101, z = S011;
    o[0] = (x * A3 + B3 + z * C3) / 3.0;          o[1] = (y * A3 + z * B3 + C3) / 3.0;
    o[2] = (A3 + x * B3 + y * C3) / 3.0;          o[3] = (x * y * A3 + x * z * B3 + y * z * C3) / 3.0;
    o[4] = (A3 + x * B3 + y * C3) / 3.0;          o[5] = (y * A3 + z * B3 + C3) / 3.0;
    o[6] = (x * A3 + B3 + z * C3) / 3.0;
    o[7] = (x * A4 + x * B4 + y * z * C4) / 3.0;  o[8] = (y * A4 + x * z * B4 + y * C4) / 3.0;
    o[9] = (A4 + B4 + C4) / 3.0;                  o[10] = (x * y * A4 + z * B4 + z * C4) / 3.0;
    o[11] = (A4 + B4 + C4) / 3.0;                 o[12] = (x * A4 + x * B4 + y * z * C4) / 3.0;
    o[13] = (y * A4 + x * z * B4 + y * C4) / 3.0; o[14] = (x * A4 + x * B4 + y * z * C4) / 3.0;
    o[15] = (y * A4 + x * z * B4 + y * C4) / 3.0; o[16] = (x * y * A4 + z * B4 + z * C4) / 3.0;
    o[17] = (A4 + B4 + C4) / 3.0;                 o[18] = (x * y * A4 + z * B4 + z * C4) / 3.0;
  }
  s[s110] = S110; s[s101] = S101; s[s011] = S011; s[s300] = S300; s[s030] = S030; s[s003] = S003;
  s[s400] = S400; s[s040] = S040; s[s004] = S004;
  s[s210] = o[0]; s[s201] = o[1]; s[s120] = o[2]; s[s111] = o[3]; s[s102] = o[4]; s[s021] = o[5]; s[s012] = o[6];
  s[s310] = o[7]; s[s301] = o[8]; s[s220] = o[9]; s[s211] = o[10]; s[s202] = o[11]; s[s130] = o[12]; s[s121] = o[13];
  s[s112] = o[14]; s[s103] = o[15]; s[s031] = o[16]; s[s022] = o[17]; s[s013] = o[18];
  realizable_2D(s[s300], s[s400], s[s110], s[s210], s[s310], s[s120], s[s220], s[s030], s[s130], s[s040]);
  realizable_2D(s[s300], s[s400], s[s101], s[s201], s[s301], s[s102], s[s202], s[s003], s[s103], s[s004]);
  realizable_2D(s[s030], s[s040], s[s011], s[s021], s[s031], s[s012], s[s022], s[s003], s[s013], s[s004]);
}

// 5th-order HyQMOM closures (src/moments/hyqmom_3D.jl:147-190); indices of
// the output array: 0 s500 1 s410 2 s320 3 s230 4 s140 5 s401 6 s302 7 s203
// 8 s104 9 s311 10 s221 11 s131 12 s212 13 s113 14 s122 15 s050 16 s041
// 17 s032 18 s023 19 s014 20 s005.
HQD double c32f(double Sj3, double Si3, double Si4, double Sij, double Sijj, double Siij, double Siijj, double Siiij) {
  return ((Sj3 * sq(Si3)) / 2.0 - Sj3 + Sj3 * (sq(Si3) - Si4 + 1.0)) * Sij + (Si4 - (3.0 * sq(Si3)) / 2.0) * Sijj +
         (-(3.0 * Sj3 * Si3) / 2.0) * Siij + ((3.0 * Si3) / 2.0) * Siijj + Sj3 * Siiij - Si3 / 2.0;
}
HQD double c41f(double Si3, double Si4, double Sij, double Siij, double Siiij) {
  return (Si3 - 2.0 * Si3 * Si4 + (9.0 * cube(Si3)) / 4.0) * Sij + ((5.0 * Si4) / 2.0 - (15.0 * sq(Si3)) / 4.0 - 1.5) * Siij + (2.0 * Si3) * Siiij;
}
HQD void hyqmom_3D(const double* s, double* f) {
  f[0] = 0.5 * s[s300] * (5.0 * s[s400] - 3.0 * sq(s[s300]) - 1.0);
  f[15] = 0.5 * s[s030] * (5.0 * s[s040] - 3.0 * sq(s[s030]) - 1.0);
  f[20] = 0.5 * s[s003] * (5.0 * s[s004] - 3.0 * sq(s[s003]) - 1.0);
  f[2] = c32f(s[s030], s[s300], s[s400], s[s110], s[s120], s[s210], s[s220], s[s310]);
  f[3] = c32f(s[s300], s[s030], s[s040], s[s110], s[s210], s[s120], s[s220], s[s130]);
  f[6] = c32f(s[s003], s[s300], s[s400], s[s101], s[s102], s[s201], s[s202], s[s301]);
  f[7] = c32f(s[s300], s[s003], s[s004], s[s101], s[s201], s[s102], s[s202], s[s103]);
  f[17] = c32f(s[s003], s[s030], s[s040], s[s011], s[s012], s[s021], s[s022], s[s031]);
  f[18] = c32f(s[s030], s[s003], s[s004], s[s011], s[s021], s[s012], s[s022], s[s013]);
  f[1] = c41f(s[s300], s[s400], s[s110], s[s210], s[s310]);
  f[4] = c41f(s[s030], s[s040], s[s110], s[s120], s[s130]);
  f[5] = c41f(s[s300], s[s400], s[s101], s[s201], s[s301]);
  f[8] = c41f(s[s003], s[s004], s[s101], s[s102], s[s103]);
  f[16] = c41f(s[s030], s[s040], s[s011], s[s021], s[s031]);
  f[19] = c41f(s[s003], s[s004], s[s011], s[s012], s[s013]);
  f[9] = 3.0 * (s[s300] * s[s211]) / 2.0 + (2.0 * s[s400] - 3.0 * sq(s[s300])) * s[s111] / 2.0 - (s[s300] * s[s011]) / 2.0;
  f[11] = 3.0 * (s[s030] * s[s121]) / 2.0 + (2.0 * s[s040] - 3.0 * sq(s[s030])) * s[s111] / 2.0 - (s[s030] * s[s101]) / 2.0;
  f[13] = 3.0 * (s[s003] * s[s112]) / 2.0 + (2.0 * s[s004] - 3.0 * sq(s[s003])) * s[s111] / 2.0 - (s[s003] * s[s110]) / 2.0;
  f[10] = s[s300] * (s[s121] - s[s101]) + s[s030] * (s[s211] - s[s011]) + s[s201] + s[s021] - s[s300] * s[s030] * s[s111];
  f[12] = s[s300] * (s[s112] - s[s110]) + s[s003] * (s[s211] - s[s011]) + s[s210] + s[s012] - s[s300] * s[s003] * s[s111];
  f[14] = s[s003] * (s[s121] - s[s101]) + s[s030] * (s[s112] - s[s110]) + s[s102] + s[s120] - s[s003] * s[s030] * s[s111];
}

// index of a 3rd/4th-order moment in the 28-set, and of a fifth-order
// closure in the order above (tables in hyq_cell.cuh); -1 if absent
HQD int s28_of(int i, int j, int k) { return T_S28[i * 36 + j * 6 + k]; }
HQD int f5_of(int i, int j, int k) { return T_F5[i * 36 + j * 6 + k]; }

// Flux_closure35_and_realizable_3D: fluxes F (x,y,z) of order-4 moments and the
// realizable moments Mr.  Any of Fx/Fy/Fz may be null (not needed).  Moment n
// is read from M4[n * ist] and written to Mr[n * mst], Fx[n * fst], ...: the
// step kernels pass the cell's entry of the moment-major fields (stride N)
// so that nothing is staged through per-thread arrays.
// FLUX = false (no flux wanted): the fifth-order closure and the raw
// fifth-order moments are skipped; the order <= 4 entries of the raw-moment
// transform only read order <= 4 entries, in the same order, so Mr has the
// same bits either way.
template <bool FLUX>
HQN void flux_closure35_t(const double* M4, int flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr, long long ist,
                          long long mst, long long fst) {
  const double s3max = 4.0 + fabs(Ma) / 2.0;
  const double h2min = 1e-8;
  const double M000 = M4[0];
  const double u = M4[1 * ist] / M000, v = M4[5 * ist] / M000, w = M4[15 * ist] / M000;
  double C[35], S[35];
  raw_to_central_r(M4, ist, C);
  central_to_std(C, S);
  const double C200 = jmax(EPS, C[2]), C020 = jmax(EPS, C[9]), C002 = jmax(EPS, C[19]);
  double s[NS];
#pragma unroll
  for (int n = 0; n < 35; ++n) {
    const int q = s28_of(ex_i(n), ex_j(n), ex_k(n));
    if (q >= 0) s[q] = S[n];
  }
  double H200, H020, H002;
  enforce_univariate(s[s300], s[s400], h2min, s3max, H200);
  enforce_univariate(s[s030], s[s040], h2min, s3max, H020);
  enforce_univariate(s[s003], s[s004], h2min, s3max, H002);
  s[s220] = realizablity_S220(s[s110], s[s220], sqrt((H200 + sq(s[s300])) * (H020 + sq(s[s030]))));
  s[s202] = realizablity_S220(s[s101], s[s202], sqrt((H200 + sq(s[s300])) * (H002 + sq(s[s003]))));
  s[s022] = realizablity_S220(s[s011], s[s022], sqrt((H020 + sq(s[s030])) * (H002 + sq(s[s003]))));
  const double R110 = 1.0 - sq(s[s110]), R101 = 1.0 - sq(s[s101]), R011 = 1.0 - sq(s[s011]);
  if (R110 <= 0.0 || R101 <= 0.0 || R011 <= 0.0) {
    Planes pl = {{s[s300], s[s400], s[s110], s[s210], s[s310], s[s120], s[s220], s[s030], s[s130], s[s040]},
                 {s[s300], s[s400], s[s101], s[s201], s[s301], s[s102], s[s202], s[s003], s[s103], s[s004]},
                 {s[s030], s[s040], s[s011], s[s021], s[s031], s[s012], s[s022], s[s003], s[s013], s[s004]}};
    check2D(pl.p1[0], pl.p1[1], pl.p1[2], pl.p1[3], pl.p1[4], pl.p1[5], pl.p1[6], pl.p1[7], pl.p1[8], pl.p1[9]);
    check2D(pl.p2[0], pl.p2[1], pl.p2[2], pl.p2[3], pl.p2[4], pl.p2[5], pl.p2[6], pl.p2[7], pl.p2[8], pl.p2[9]);
    check2D(pl.p3[0], pl.p3[1], pl.p3[2], pl.p3[3], pl.p3[4], pl.p3[5], pl.p3[6], pl.p3[7], pl.p3[8], pl.p3[9]);
    edge_corner(s, pl, R110, R101, R011);
  } else {
    // interior branch: check2D_all_planes outputs are not used here
    const int flag220 = realizable_3D(s);
    if (flag220 == 1)
      for (int it = 0; it < 6; ++it) realizable_3D(s);
  }
  if (flag2D == 1) {
    s[s011] = 0.0; s[s101] = 0.0; s[s201] = 0.0; s[s021] = 0.0; s[s012] = 0.0; s[s102] = 0.0; s[s111] = 0.0;
    s[s202] = 1.0; s[s022] = 1.0; s[s112] = s[s110]; s[s121] = 0.0; s[s211] = 0.0; s[s103] = 0.0; s[s013] = 0.0;
    s[s301] = 0.0; s[s031] = 0.0;
  }
  double f[FLUX ? 21 : 1];
  if constexpr (FLUX) hyqmom_3D(s, f);
  // S -> C (S_to_C_batch) on the 56-entry store, then C -> raw (C5toM5_3D)
  const double sx = sqrt(jmax(EPS, C200)), sy = sqrt(jmax(EPS, C020)), sz = sqrt(jmax(EPS, C002));
  double px[6], py[6], pz[6];
  px[0] = py[0] = pz[0] = 1.0;
  px[1] = sx; py[1] = sy; pz[1] = sz;
  px[2] = sx * sx; py[2] = sy * sy; pz[2] = sz * sz;
  px[3] = sx * sx * sx; py[3] = sy * sy * sy; pz[3] = sz * sz * sz;
  px[4] = pow4(sx); py[4] = pow4(sy); pz[4] = pow4(sz);
  px[5] = pow5(sx); py[5] = pow5(sy); pz[5] = pow5(sz);
  constexpr int NA = FLUX ? 56 : 35;
  double A[NA];
#pragma unroll
  for (int q = 0; q < NA; ++q) {
    const int i = T_EX56I[q], j = T_EX56J[q], k = T_EX56K[q];
    const int o = i + j + k;
    double val;
    if (o == 0) val = 1.0;
    else if (o == 1) val = 0.0;
    else if (o == 2 && i == 2) val = C200;
    else if (o == 2 && j == 2) val = C020;
    else if (o == 2 && k == 2) val = C002;
    else {
      double d = (q >= 35) ? f[FLUX ? q - 35 : 0] : s[T_S28OF56[q]];
      if (i) d = d * px[i];
      if (j) d = d * py[j];
      if (k) d = d * pz[k];
      val = d;
    }
    A[q] = val;
  }
  central_to_raw_r<NA>(M000, u, v, w, A);
#pragma unroll
  for (int n = 0; n < 35; ++n) {
    Mr[n * mst] = A[n];
    if constexpr (FLUX) {
      if (Fx) Fx[n * fst] = A[T_FX[n]];
      if (Fy) Fy[n * fst] = A[T_FY[n]];
      if (Fz) Fz[n * fst] = A[T_FZ[n]];
    }
  }
}
// Flux_closure35_and_realizable_3D; null Fx, Fy and Fz (the realized moments
// only) select the variant without the fifth-order work.
HQD void flux_closure35(const double* M4, int flag2D, double Ma, double* Fx, double* Fy, double* Fz, double* Mr, long long ist = 1,
                        long long mst = 1, long long fst = 1) {
  if (Fx || Fy || Fz) flux_closure35_t<true>(M4, flag2D, Ma, Fx, Fy, Fz, Mr, ist, mst, fst);
  else flux_closure35_t<false>(M4, flag2D, Ma, nullptr, nullptr, nullptr, Mr, ist, mst, fst);
}

}  // namespace hyq
