// oracle_cell.h -- per-cell mathematics of PANGU's stage path, restated on
// the CPU. TEST INFRASTRUCTURE ONLY: used by the tests, the smoke check and
// the CPU baseline of bench.py as the checker; never linked into the engine.
//
// Every function follows the reference's operation order line by line
// (file:line cited on each) and is compiled with -ffp-contract=off so that
// no multiply-add is fused behind the source's back. The coordinate maps use
// the C library's exp/sin/cos, as the reference's host build does; pow, exp
// and log of the physics use the double-double routines of pgmath.h, which
// the engine runs bit-identically (the C2P chain is chaotic with respect to
// one-ulp differences in floor-dominated cells). Those routines agree with
// the C library's to the last bit on the golden vectors.
// Parity anchor: the per-cell functions are checked against golden vectors
// produced by the reference's own headers (tests/golden/make_golden.py).
#ifndef PANGU_ORACLE_CELL_H
#define PANGU_ORACLE_CELL_H

#include <cmath>

// pow/exp/log of the physics: the double-double routines shared with the
// engine (bit-identical on host and device); see pgmath.h.
#include "pgmath.h"

namespace orc {

using Real = double;

// variable_mnemonics.h:7-14
enum Index { RHO, ENY, UX1, UX2, UX3, BX1, BX2, BX3, ENT, KEL, NPRIM };
enum MType { MINKOWSKI = 0, BL = 1, CKS = 2, MKS = 3 };  // christoffel.h:19-21

// Kokkos::min / Kokkos::max semantics ((b < a) ? b : a and (a < b) ? b : a).
inline Real kmin(Real a, Real b) { return (b < a) ? b : a; }
inline Real kmax(Real a, Real b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------
// tensor_algebra.h
// ---------------------------------------------------------------------------
inline Real dot4(const Real a[4], const Real b[4]) {  // tensor_algebra.h:11-16
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

inline Real square3(const Real v[3], const Real m[3][3]) {  // :18-37
  return v[0] * m[0][0] * v[0] + v[0] * m[0][1] * v[1] + v[0] * m[0][2] * v[2] +
         v[1] * m[1][0] * v[0] + v[1] * m[1][1] * v[1] + v[1] * m[1][2] * v[2] +
         v[2] * m[2][0] * v[0] + v[2] * m[2][1] * v[1] + v[2] * m[2][2] * v[2];
}

inline Real determinant(const Real m[4][4]) {  // tensor_algebra.h:39-69
  return m[0][0] * (m[1][1] * (m[2][2] * m[3][3] - m[2][3] * m[3][2]) -
                    m[1][2] * (m[2][1] * m[3][3] - m[2][3] * m[3][1]) +
                    m[1][3] * (m[2][1] * m[3][2] - m[2][2] * m[3][1])) -
         m[0][1] * (m[1][0] * (m[2][2] * m[3][3] - m[2][3] * m[3][2]) -
                    m[1][2] * (m[2][0] * m[3][3] - m[2][3] * m[3][0]) +
                    m[1][3] * (m[2][0] * m[3][2] - m[2][2] * m[3][0])) +
         m[0][2] * (m[1][0] * (m[2][1] * m[3][3] - m[2][3] * m[3][1]) -
                    m[1][1] * (m[2][0] * m[3][3] - m[2][3] * m[3][0]) +
                    m[1][3] * (m[2][0] * m[3][1] - m[2][1] * m[3][0])) -
         m[0][3] * (m[1][0] * (m[2][1] * m[3][2] - m[2][2] * m[3][1]) -
                    m[1][1] * (m[2][0] * m[3][2] - m[2][2] * m[3][0]) +
                    m[1][2] * (m[2][0] * m[3][1] - m[2][1] * m[3][0]));
}

// Gauss-Jordan with a row swap only on an exactly zero pivot
// (tensor_algebra.h:71-124). Returns 0 when singular.
inline int invert(const Real m[4][4], Real inv[4][4]) {
  Real aug[4][8];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      aug[i][j] = m[i][j];
      aug[i][j + 4] = (i == j) ? 1.0 : 0.0;
    }
  for (int i = 0; i < 4; ++i) {
    if (aug[i][i] == 0.0) {
      int sw = -1;
      for (int j = i + 1; j < 4; ++j)
        if (aug[j][i] != 0.0) { sw = j; break; }
      if (sw == -1) return 0;
      for (int j = 0; j < 8; ++j) {
        const Real t = aug[i][j];
        aug[i][j] = aug[sw][j];
        aug[sw][j] = t;
      }
    }
    const Real pivot = aug[i][i];
    for (int j = 0; j < 8; ++j) aug[i][j] /= pivot;
    for (int j = 0; j < 4; ++j) {
      if (j == i) continue;
      const Real f = aug[j][i];
      for (int k = 0; k < 8; ++k) aug[j][k] -= f * aug[i][k];
    }
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) inv[i][j] = aug[i][j + 4];
  return 1;
}

// ---------------------------------------------------------------------------
// Coordinate maps and physical metrics: minkowski.h, BL.h, CKS.h, MKS.h
// ---------------------------------------------------------------------------
// MKS.h:15-23 and BL.h:15-23 (identical maps).
inline void log_theta_map(const Real x[4], Real y[4], Real h) {
  y[0] = x[0];
  y[1] = std::exp(x[1]);
  y[2] = M_PI_2 * (x[2] + 1.0) + 0.5 * h * std::sin(M_PI * (x[2] + 1.0));
  y[3] = x[3];
}

inline void physical_coords(int mt, const Real x[4], Real y[4], Real h) {
  if (mt == MKS || mt == BL) {
    log_theta_map(x, y, h);
  } else {  // minkowski.h:12-19, CKS.h:12-19: identity
    y[0] = x[0]; y[1] = x[1]; y[2] = x[2]; y[3] = x[3];
  }
}

// MKS.h:25-58: Kerr-Schild metric in (t, r, theta, phi).
inline void mks_physical_metric(const Real x[4], Real g[4][4], Real h, Real a) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = 0.0;
  Real y[4];
  log_theta_map(x, y, h);
  const Real r = y[1];
  const Real theta = y[2];
  const Real cth = std::cos(theta);
  const Real sth = std::sin(theta);
  const Real Sigma = r * r + a * a * cth * cth;
  g[0][0] = -1.0 + 2.0 * r / Sigma;
  g[0][1] = 2.0 * r / Sigma;
  g[0][3] = -2.0 * a * r * sth * sth / Sigma;
  g[1][0] = g[0][1];
  g[1][1] = 1.0 + 2.0 * r / Sigma;
  g[1][3] = -a * (1.0 + 2.0 * r / Sigma) * sth * sth;
  g[2][2] = Sigma;
  g[3][0] = g[0][3];
  g[3][1] = g[1][3];
  g[3][3] = sth * sth * (Sigma + a * a * sth * sth * (1.0 + 2.0 * r / Sigma));
}

// BL.h:25-58: Boyer-Lindquist metric.
inline void bl_physical_metric(const Real x[4], Real g[4][4], Real h, Real a) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = 0.0;
  Real y[4];
  log_theta_map(x, y, h);
  const Real r = y[1];
  const Real theta = y[2];
  const Real cth = std::cos(theta);
  const Real sth = std::sin(theta);
  const Real sth2 = sth * sth;
  const Real r2 = r * r;
  const Real a2 = a * a;
  const Real mu = 1.0 + a2 * cth * cth / r2;
  const Real delta = 1.0 - 2.0 / r + a2 / r2;
  const Real inv_r_mu = 1.0 / (r * mu);
  g[0][0] = -1.0 + 2.0 * inv_r_mu;
  g[0][3] = -2.0 * a * sth2 * inv_r_mu;
  g[1][1] = mu / delta;
  g[2][2] = r2 / mu;
  g[3][0] = g[0][3];
  g[3][3] = r2 * sth2 * (1.0 + a2 / r2 + 2.0 * a2 * sth2 / (r * r2 * mu));
}

// CKS.h:24-71: Cartesian Kerr-Schild metric.
inline void cks_physical_metric(const Real x[4], Real g[4][4], Real a) {
  const Real xx = x[1], yy = x[2], zz = x[3];
  const Real r2_cart = xx * xx + yy * yy + zz * zz;
  const Real a2 = a * a;
  const Real tmp = r2_cart - a2;
  const Real sqrtarg = tmp * tmp + 4.0 * a2 * zz * zz;
  const Real r = std::sqrt(0.5 * (tmp + std::sqrt(sqrtarg)));
  const Real r_safe = (r > 1.0e-15) ? r : 1.0e-15;
  const Real r2 = r_safe * r_safe;
  const Real r3 = r2 * r_safe;
  const Real r4 = r2 * r2;
  const Real xi_denom = r4 + a2 * zz * zz;
  const Real xi = (xi_denom > 0.0) ? (2.0 * r3 / xi_denom) : 0.0;
  const Real denom_l = r2 + a2;
  const Real l[4] = {1.0, (r_safe * xx + a * yy) / denom_l,
                     (r_safe * yy - a * xx) / denom_l, zz / r_safe};
  for (int m = 0; m < 4; ++m)
    for (int n = 0; n < 4; ++n) g[m][n] = 0.0;
  g[0][0] = -1.0;
  g[1][1] = 1.0;
  g[2][2] = 1.0;
  g[3][3] = 1.0;
  for (int m = 0; m < 4; ++m)
    for (int n = 0; n < 4; ++n) g[m][n] += xi * l[m] * l[n];
}

// minkowski.h:24-32
inline void minkowski_physical_metric(Real g[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = (i == j) * (1 - 2 * (i == 0));
}

// Code metric = finite-difference Jacobian (delta = 1e-5) of the coordinate
// map applied to the physical metric: MKS.h:60-107, BL.h:60-107,
// CKS.h:73-108, minkowski.h:34-70 (the same recipe in all four files).
inline void code_metric(int mt, const Real x[4], Real a, Real h,
                        Real gc[4][4]) {
  constexpr Real delta = 1.0e-5;
  Real gp[4][4];
  switch (mt) {
    case BL: bl_physical_metric(x, gp, h, a); break;
    case CKS: cks_physical_metric(x, gp, a); break;
    case MKS: mks_physical_metric(x, gp, h, a); break;
    default: minkowski_physical_metric(gp); break;
  }
  Real jac[4][4];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) jac[r][c] = 0.0;
  for (int col = 0; col < 4; ++col) {
    Real xh[4], xl[4];
    for (int d = 0; d < 4; ++d) { xh[d] = x[d]; xl[d] = x[d]; }
    xh[col] += delta;
    xl[col] -= delta;
    Real yh[4], yl[4];
    physical_coords(mt, xh, yh, h);
    physical_coords(mt, xl, yl, h);
    for (int row = 0; row < 4; ++row)
      jac[row][col] = (yh[row] - yl[row]) / (xh[col] - xl[col]);
  }
  for (int row = 0; row < 4; ++row)
    for (int col = 0; col < 4; ++col) {
      gc[row][col] = 0.0;
      for (int p = 0; p < 4; ++p)
        for (int q = 0; q < 4; ++q)
          gc[row][col] += gp[p][q] * jac[row][p] * jac[q][col];
    }
}

// christoffel.h:33-62 (ComputeMetricAtLocation).
inline void metric_at(int mt, const Real x[4], Real a, Real h, Real gcov[4][4],
                      Real gcon[4][4], Real &gdet) {
  code_metric(mt, x, a, h, gcov);
  invert(gcov, gcon);
  gdet = determinant(gcov);
}

// christoffel.h:64-148 (ComputeChristoffelConnection): conn[m][a][b].
inline void christoffel(int mt, const Real x[4], Real a, Real h,
                        Real conn[4][4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) conn[i][j][k] = 0.0;
  if (mt == MINKOWSKI) return;
  Real gcov[4][4], gcon[4][4], gdet;
  metric_at(mt, x, a, h, gcov, gcon, gdet);
  constexpr Real delta = 1.0e-5;
  Real dg[4][4][4];
  for (int d = 0; d < 4; ++d) {
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) dg[d][r][c] = 0.0;
    if (d > 0) {
      Real xp[4] = {x[0], x[1], x[2], x[3]};
      Real xm[4] = {x[0], x[1], x[2], x[3]};
      xp[d] += delta;
      xm[d] -= delta;
      Real gp[4][4], gm[4][4];
      code_metric(mt, xp, a, h, gp);
      code_metric(mt, xm, a, h, gm);
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
          dg[d][r][c] = (gp[r][c] - gm[r][c]) / (2.0 * delta);
    }
  }
  Real cc[4][4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k)
        cc[i][j][k] = 0.5 * (dg[j][i][k] + dg[k][i][j] - dg[i][j][k]);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        Real v = 0.0;
        for (int l = 0; l < 4; ++l) v += gcon[i][l] * cc[l][j][k];
        conn[i][j][k] = v;
      }
}

// ---------------------------------------------------------------------------
// physics/
// ---------------------------------------------------------------------------
struct State {  // state_calculation.h:11-17
  Real ucon[4], ucov[4], bcon[4], bcov[4], bsq;
};

// state_calculation.h:19-69
inline void calc_state(const Real P[NPRIM], const Real gcov[4][4],
                       const Real gcon[4][4], State &s) {
  const Real alpha = 1.0 / std::sqrt(-gcon[0][0]);
  Real gij[3][3];
  for (int r = 1; r < 4; ++r)
    for (int c = 1; c < 4; ++c) gij[r - 1][c - 1] = gcov[r][c];
  const Real ut[3] = {P[UX1], P[UX2], P[UX3]};
  const Real lsq = 1.0 + square3(ut, gij);
  const Real lor = std::sqrt(lsq);
  s.ucon[0] = lor / alpha;
  s.ucon[1] = P[UX1] - s.ucon[0] * gcon[0][1] * alpha * alpha;
  s.ucon[2] = P[UX2] - s.ucon[0] * gcon[0][2] * alpha * alpha;
  s.ucon[3] = P[UX3] - s.ucon[0] * gcon[0][3] * alpha * alpha;
  for (int r = 0; r < 4; ++r) {
    s.ucov[r] = 0.0;
    for (int c = 0; c < 4; ++c) s.ucov[r] += gcov[r][c] * s.ucon[c];
  }
  s.bcon[0] = P[BX1] * s.ucov[1] + P[BX2] * s.ucov[2] + P[BX3] * s.ucov[3];
  s.bcon[1] = (P[BX1] + s.bcon[0] * s.ucon[1]) / s.ucon[0];
  s.bcon[2] = (P[BX2] + s.bcon[0] * s.ucon[2]) / s.ucon[0];
  s.bcon[3] = (P[BX3] + s.bcon[0] * s.ucon[3]) / s.ucon[0];
  for (int r = 0; r < 4; ++r) {
    s.bcov[r] = 0.0;
    for (int c = 0; c < 4; ++c) s.bcov[r] += gcov[r][c] * s.bcon[c];
  }
  s.bsq = s.bcon[0] * s.bcov[0] + s.bcon[1] * s.bcov[1] +
          s.bcon[2] * s.bcov[2] + s.bcon[3] * s.bcov[3];
}

// energy_momentum_tensor.h:11-29: T^{dir}_m.
inline void emt(Real gam, const Real P[NPRIM], const Real gcov[4][4],
                const Real gcon[4][4], int dir, Real t[4]) {
  State s;
  calc_state(P, gcov, gcon, s);
  const Real p_gas = (gam - 1.) * P[ENY];
  const Real hh = P[RHO] + gam * P[ENY];
  const Real e_tot = hh + s.bsq;
  const Real p_tot = p_gas + 0.5 * s.bsq;
  for (int m = 0; m < 4; ++m)
    t[m] = e_tot * s.ucon[dir] * s.ucov[m] + p_tot * (dir == m) -
           s.bcon[dir] * s.bcov[m];
}

// contravariant_flux.h:12-39
inline void contravariant_flux(Real gam, const Real P[NPRIM],
                               const Real gcov[4][4], const Real gcon[4][4],
                               Real gdet, int dir, Real f[NPRIM]) {
  State s;
  calc_state(P, gcov, gcon, s);
  Real t[4];
  emt(gam, P, gcov, gcon, dir, t);
  f[RHO] = P[RHO] * s.ucon[dir];
  f[ENY] = t[0] + f[RHO];
  f[UX1] = t[1];
  f[UX2] = t[2];
  f[UX3] = t[3];
  f[BX1] = s.bcon[1] * s.ucon[dir] - s.bcon[dir] * s.ucon[1];
  f[BX2] = s.bcon[2] * s.ucon[dir] - s.bcon[dir] * s.ucon[2];
  f[BX3] = s.bcon[3] * s.ucon[dir] - s.bcon[dir] * s.ucon[3];
  f[ENT] = P[ENT] * f[RHO];
  f[KEL] = P[KEL] * f[RHO];
  const Real sg = std::sqrt(std::fabs(gdet));
  for (int n = 0; n < NPRIM; ++n) f[n] *= sg;
}

// fast_magnetosonic_speed.h:11-81
inline void fast_speed(Real gam, const Real P[NPRIM], const Real gcov[4][4],
                       const Real gcon[4][4], int dir, Real &vmax,
                       Real &vmin) {
  Real ncon[4] = {0., 0., 0., 0.}, ncov[4] = {0., 0., 0., 0.};
  Real tcon[4] = {0., 0., 0., 0.}, tcov[4] = {0., 0., 0., 0.};
  ncov[dir] = 1.0;
  tcov[0] = 1.0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      ncon[r] += gcon[r][c] * ncov[c];
      tcon[r] += gcon[r][c] * tcov[c];
    }
  State s;
  calc_state(P, gcov, gcon, s);
  const Real hh = P[RHO] + gam * P[ENY];
  const Real h_tot = s.bsq + hh;
  const Real va_sq = s.bsq / h_tot;
  const Real cs_sq = gam * (gam - 1.) * P[ENY] / hh;
  Real cf_sq = cs_sq + va_sq - cs_sq * va_sq;
  if (cf_sq < 0.) cf_sq = 1e-10;
  if (cf_sq > 1.) cf_sq = 1.;
  const Real n_sq = dot4(ncon, ncov);
  const Real t_sq = dot4(tcon, tcov);
  const Real n_dot_u = dot4(ncov, s.ucon);
  const Real t_dot_u = dot4(tcov, s.ucon);
  const Real n_dot_t = dot4(ncon, tcov);
  const Real nu2 = n_dot_u * n_dot_u;
  const Real tu2 = t_dot_u * t_dot_u;
  const Real nutu = n_dot_u * t_dot_u;
  const Real A = tu2 - (t_sq + tu2) * cf_sq;
  const Real B = 2. * (nutu - (n_dot_t + nutu) * cf_sq);
  const Real C = nu2 - (n_sq + nu2) * cf_sq;
  Real disc = B * B - 4. * A * C;
  if ((disc < 0.0) && (disc > -1.e-10)) disc = 0.0;
  else if (disc < -1.e-10) disc = 0.;
  disc = std::sqrt(disc);
  const Real vp = -(-B + disc) / (2. * A);
  const Real vm = -(-B - disc) / (2. * A);
  if (vp > vm) { vmax = vp; vmin = vm; }
  else { vmax = vm; vmin = vp; }
}

// ---------------------------------------------------------------------------
// interpolation/
// ---------------------------------------------------------------------------
inline Real minmod3(Real a, Real b, Real c) {  // interpolater_mc.h:16-23
  if (a > 0.0 && b > 0.0 && c > 0.0) return std::fmin(std::fmin(a, b), c);
  if (a < 0.0 && b < 0.0 && c < 0.0) return std::fmax(std::fmax(a, b), c);
  return 0.0;
}

// interpolater_mc.h:38-48
inline void mc(Real qm2, Real qm1, Real q, Real qp1, Real qp2, Real &ql_ip1,
               Real &qr_i) {
  (void)qm2; (void)qp2;
  const Real slope =
      minmod3(2.0 * (q - qm1), 0.5 * (qp1 - qm1), 2.0 * (qp1 - q));
  ql_ip1 = q + 0.5 * slope;
  qr_i = q - 0.5 * slope;
}

// interpolater_ppm4.h:29-67
inline void ppm4(Real qm2, Real qm1, Real q, Real qp1, Real qp2, Real &ql_ip1,
                 Real &qr_i) {
  Real qlv = (7.0 * (q + qm1) - (qm2 + qp1)) / 12.0;
  Real qrv = (7.0 * (q + qp1) - (qm1 + qp2)) / 12.0;
  qlv = std::fmax(qlv, std::fmin(q, qm1));
  qlv = std::fmin(qlv, std::fmax(q, qm1));
  qrv = std::fmax(qrv, std::fmin(q, qp1));
  qrv = std::fmin(qrv, std::fmax(q, qp1));
  const Real qc = qrv - q;
  const Real qd = qlv - q;
  if ((qc * qd) >= 0.0) {
    qlv = q;
    qrv = q;
  } else {
    if (std::fabs(qc) >= 2.0 * std::fabs(qd)) qrv = q - 2.0 * qd;
    if (std::fabs(qd) >= 2.0 * std::fabs(qc)) qlv = q - 2.0 * qc;
  }
  ql_ip1 = qrv;
  qr_i = qlv;
}

// ---------------------------------------------------------------------------
// recovery/ (constants.h:14-23)
// ---------------------------------------------------------------------------
constexpr int MAX_NEWT_ITER = 30;
constexpr Real NEWT_TOL = 1e-10;
constexpr Real MIN_NEWT_TOL = 1e-10;
constexpr int EXTRA_NEWT_ITER = 2;
constexpr Real NEWT_TOL2 = 1.0e-15;
constexpr Real W_TOO_BIG = 1.e20;
constexpr Real UTSQ_TOO_BIG = 1.e20;
constexpr Real FAIL_VAL = 1.e30;

inline void raise_g(const Real v[4], const Real gcon[4][4], Real o[4]) {
  for (int i = 0; i < 4; i++) {
    o[i] = 0;
    for (int j = 0; j < 4; j++) o[i] += gcon[i][j] * v[j];
  }
}
inline void lower_g(const Real v[4], const Real gcov[4][4], Real o[4]) {
  for (int i = 0; i < 4; i++) {
    o[i] = 0;
    for (int j = 0; j < 4; j++) o[i] += gcov[i][j] * v[j];
  }
}
inline void ncov_calc(const Real gcon[4][4], Real ncov[4]) {
  const Real lapse = std::sqrt(-1.0 / gcon[0][0]);
  for (int i = 0; i < 4; i++) ncov[i] = -lapse * (i == 0);
}

// The projections shared by the three HARM schemes
// (scheme_2d.h:271-306, scheme_1d_vsq.h:234-269, scheme_1d.h:423-458).
struct HarmSetup {
  Real Bcon[4], Bcov[4], Qcov[4], Qcon[4], ncov[4], ncon[4];
  Real Bsq, QdotB, QdotBsq, Qdotn, Qsq, Qtsq, D;
};

inline void harm_setup(const Real U[9], const Real gcov[4][4],
                       const Real gcon[4][4], HarmSetup &s) {
  s.Bcon[0] = 0.;
  s.Bcon[1] = U[BX1];
  s.Bcon[2] = U[BX2];
  s.Bcon[3] = U[BX3];
  lower_g(s.Bcon, gcov, s.Bcov);
  s.Qcov[0] = U[ENY];
  s.Qcov[1] = U[UX1];
  s.Qcov[2] = U[UX2];
  s.Qcov[3] = U[UX3];
  raise_g(s.Qcov, gcon, s.Qcon);
  s.Bsq = 0.;
  for (int i = 1; i < 4; i++) s.Bsq += s.Bcon[i] * s.Bcov[i];
  s.QdotB = 0.;
  for (int i = 0; i < 4; i++) s.QdotB += s.Qcov[i] * s.Bcon[i];
  s.QdotBsq = s.QdotB * s.QdotB;
  ncov_calc(gcon, s.ncov);
  raise_g(s.ncov, gcon, s.ncon);
  s.Qdotn = s.Qcon[0] * s.ncov[0];
  s.Qsq = 0.;
  for (int i = 0; i < 4; i++) s.Qsq += s.Qcov[i] * s.Qcon[i];
  s.Qtsq = s.Qsq + s.Qdotn * s.Qdotn;
  s.D = U[RHO];
}

// utsq from the stale primitive guess (scheme_2d.h:310-323 and twins).
// Returns false when the guess is rejected (retval 2).
inline bool harm_utsq(const Real prim[9], const Real gcov[4][4], Real &utsq) {
  utsq = 0.;
  for (int i = 1; i < 4; i++)
    for (int j = 1; j < 4; j++)
      utsq += gcov[i][j] * prim[UX1 + i - 1] * prim[UX1 + j - 1];
  if ((utsq < 0.) && (std::fabs(utsq) < 1.0e-13)) utsq = std::fabs(utsq);
  if (utsq < 0. || utsq > UTSQ_TOO_BIG) return false;
  return true;
}

// Velocity write-back shared by the schemes (scheme_2d.h:395-398).
inline void harm_velocity(const HarmSetup &s, Real Gamma, Real W, Real prim[9]) {
  Real Qtcon[4];
  for (int i = 1; i < 4; i++) Qtcon[i] = s.Qcon[i] + s.ncon[i] * s.Qdotn;
  for (int i = 1; i < 4; i++)
    prim[UX1 + i - 1] =
        Gamma / (W + s.Bsq) * (Qtcon[i] + s.QdotB * s.Bcon[i] / W);
}

// ---- Scheme2D (scheme_2d.h) -------------------------------------------------
namespace s2d {
inline Real pressure_W_vsq(Real D, Real W, Real vsq, Real g) {  // :60-64
  Real gtmp = 1. - vsq;
  return ((g - 1.) * (W * gtmp - D * std::sqrt(gtmp)) / g);
}
inline Real vsq_calc(Real Bsq, Real QdotBsq, Real Qtsq, Real W) {  // :66-74
  Real Wsq = W * W;
  Real Xsq = (Bsq + W) * (Bsq + W);
  return ((Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * Xsq));
}
inline Real x1_of_x0(Real Bsq, Real QdotBsq, Real Qtsq, Real x0) {  // :76-83
  Real dv = 1.e-15;
  Real vsq = std::fabs(vsq_calc(Bsq, QdotBsq, Qtsq, x0));
  return ((vsq > 1.) ? (1.0 - dv) : vsq);
}
inline void validate_x(Real x[2], const Real x0[2]) {  // :85-97
  Real dv = 1.e-15;
  x[0] = std::fabs(x[0]);
  x[0] = (x[0] > W_TOO_BIG) ? x0[0] : x[0];
  x[1] = (x[1] < 0.) ? 0. : x[1];
  x[1] = (x[1] > 1.) ? (1. - dv) : x[1];
}
// :99-156
inline void func_vsq(Real Bsq, Real QdotBsq, Real Qtsq, Real Qdotn, Real D,
                     const Real x[2], Real dx[2], Real *f, Real *df, Real g) {
  const Real W = x[0];
  const Real vsq = x[1];
  const Real Wsq = W * W;
  const Real p_tmp = pressure_W_vsq(D, W, vsq, g);
  const Real dPdW = ((g - 1.) * (1. - vsq) / g);
  const Real dPdvsq = ((g - 1.) * (0.5 * D / std::sqrt(1. - vsq) - W) / g);
  const Real t2 = -0.5 * Bsq + dPdvsq;
  const Real t3 = Bsq + W;
  const Real t4 = t3 * t3;
  const Real t9 = 1.0 / Wsq;
  const Real t11 = Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.0 * W) * t9;
  const Real t16 = QdotBsq * t9;
  const Real t18 = -Qdotn - 0.5 * Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
  const Real t21 = 1.0 / t3;
  const Real t23 = 1.0 / W;
  const Real t24 = t16 * t23;
  const Real t25 = -1.0 + dPdW - t24;
  const Real t35 =
      t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
  const Real t36 = 1.0 / t35;
  dx[0] = -(t2 * t11 + t4 * t18) * t21 * t36;
  const Real t40 = (vsq + t24) * t3;
  dx[1] = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
  const Real r0 = t11, r1 = t18;
  *df = -r0 * r0 - r1 * r1;
  *f = -0.5 * (*df);
}
// :158-255
inline int newton(Real Bsq, Real QdotBsq, Real Qtsq, Real Qdotn, Real D,
                  Real x[2], Real g, int *iters) {
  Real f = 1., df = 1., dx[2], x_old[2];
  Real errx = 1.;
  int i_extra = 0, doing_extra = 0, n_iter = 0;
  int keep = 1;
  while (keep) {
    func_vsq(Bsq, QdotBsq, Qtsq, Qdotn, D, x, dx, &f, &df, g);
    errx = 0.;
    x_old[0] = x[0];
    x_old[1] = x[1];
    x[0] += dx[0];
    x[1] += dx[1];
    errx = (x[0] == 0.) ? std::fabs(dx[0]) : std::fabs(dx[0] / x[0]);
    errx += (x[1] == 0.) ? std::fabs(dx[1]) : std::fabs(dx[1] / x[1]);
    validate_x(x, x_old);
    if ((std::fabs(errx) <= NEWT_TOL) && (doing_extra == 0) &&
        (EXTRA_NEWT_ITER > 0))
      doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((std::fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) ||
        (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (iters) *iters = n_iter;
  if ((std::isfinite(f) == 0) || (std::isfinite(df) == 0)) return 2;
  if (std::fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}
// :257-404
inline int invert(const Real U[9], Real prim[9], Real g,
                  const Real gcov[4][4], const Real gcon[4][4]) {
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  HarmSetup s;
  harm_setup(U, gcov, gcon, s);
  Real utsq;
  if (!harm_utsq(prim, gcov, utsq)) return 2;
  const Real gammasq = 1. + utsq;
  Real Gamma = std::sqrt(gammasq);
  Real rho0 = s.D / Gamma;
  Real uu = prim[ENY];
  Real p = (g - 1.) * uu;
  Real w = rho0 + uu + p;
  Real W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) -
           s.QdotBsq * (2. * W_last + s.Bsq)) <=
          W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  Real x[2];
  x[0] = std::fabs(W_last);
  x[1] = x1_of_x0(s.Bsq, s.QdotBsq, s.Qtsq, W_last);
  int retval = newton(s.Bsq, s.QdotBsq, s.Qtsq, s.Qdotn, s.D, x, g, nullptr);
  const Real W = x[0];
  const Real vsq = x[1];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  if (vsq >= 1.) return 4;
  const Real gtmp = std::sqrt(1. - vsq);
  Gamma = 1. / gtmp;
  rho0 = s.D * gtmp;
  w = W * (1. - vsq);
  p = ((g - 1.) * (w - rho0) / g);
  uu = w - (rho0 + p);
  if ((rho0 <= 0.) || (uu <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[ENY] = uu;
  prim[ENT] = (g - 1.) * uu * pgm::pow(rho0, -g);
  harm_velocity(s, Gamma, W, prim);
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  return 0;
}
}  // namespace s2d

// ---- Scheme1Dvsq (scheme_1d_vsq.h) ---------------------------------------
namespace s1dvsq {
inline void validate_x(Real x[1], const Real x0[1]) {  // :52-61
  Real small = 1.e-10;
  x[0] = (x[0] >= 1.0) ? (0.5 * (x0[0] + 1.)) : x[0];
  x[0] = (x[0] < -small) ? (0.5 * x0[0]) : x[0];
  x[0] = std::fabs(x[0]);
}
// :71-82
inline Real W_of_vsq(Real D, Real K, Real vsq, Real *p, Real *rho, Real *uu,
                     Real g) {
  Real gtmp = (1. - vsq);
  *rho = D * std::sqrt(gtmp);
  *p = (K * pgm::pow(*rho, g));
  *uu = (*p / (g - 1.));
  return ((*rho + *uu + *p) / gtmp);
}
// :84-88
inline Real dWdvsq_calc(Real vsq, Real rho, Real p, Real g) {
  return ((g * (2. - g) * p + (g - 1.) * rho) /
          (2. * (g - 1.) * (1. - vsq) * (1. - vsq)));
}
// :90-117
inline void func_1d_gnr(Real Bsq, Real QdotBsq, Real Qtsq, Real D, Real K,
                        const Real x[1], Real dx[1], Real *f, Real *df,
                        Real g) {
  Real rho, p, uu;
  const Real vsq = x[0];
  const Real W = W_of_vsq(D, K, vsq, &p, &rho, &uu, g);
  const Real Wsq = W * W;
  const Real W3 = W * Wsq;
  const Real dWdvsq = dWdvsq_calc(vsq, rho, p, g);
  const Real ft = (Bsq + W);
  const Real resid = Qtsq - vsq * ft * ft + QdotBsq * (Bsq + 2. * W) / Wsq;
  const Real jac = -ft * (ft + 2. * dWdvsq * (vsq + QdotBsq / W3));
  dx[0] = -resid / jac;
  *f = 0.5 * resid * resid;
  *df = -2. * (*f);
}
// :119-220
inline int newton(Real Bsq, Real QdotBsq, Real Qtsq, Real D, Real K, Real x[1],
                  Real g) {
  Real f = 1., df = 1., dx[1], x_old[1];
  Real errx = 1.;
  int i_extra = 0, doing_extra = 0, n_iter = 0, keep = 1;
  Real W = 0., W_old = 0., rho, p, uu;
  while (keep) {
    func_1d_gnr(Bsq, QdotBsq, Qtsq, D, K, x, dx, &f, &df, g);
    errx = 0.;
    x_old[0] = x[0];
    x[0] += dx[0];
    validate_x(x, x_old);
    W_old = W;
    W = W_of_vsq(D, K, x[0], &p, &rho, &uu, g);
    errx = (W == 0.) ? std::fabs(W - W_old) : std::fabs((W - W_old) / W);
    errx += (x[0] == 0.) ? std::fabs(x[0] - x_old[0])
                         : std::fabs((x[0] - x_old[0]) / x[0]);
    if ((std::fabs(errx) <= NEWT_TOL) && (doing_extra == 0) &&
        (EXTRA_NEWT_ITER > 0))
      doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((std::fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) ||
        (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if ((std::isfinite(f) == 0) || (std::isfinite(df) == 0)) return 2;
  if (std::fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}
// :222-351
inline int invert(const Real U[9], Real prim[9], Real g,
                  const Real gcov[4][4], const Real gcon[4][4]) {
  Real K = prim[ENT];
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  HarmSetup s;
  harm_setup(U, gcov, gcon, s);
  Real utsq;
  if (!harm_utsq(prim, gcov, utsq)) return 2;
  const Real gammasq = 1. + utsq;
  Real x[1];
  x[0] = 1. - 1. / gammasq;
  int retval = newton(s.Bsq, s.QdotBsq, s.Qtsq, s.D, K, x, g);
  if (retval != 0) return retval * 100 + 1;
  const Real vsq = x[0];
  if ((vsq >= 1.) || (vsq < 0.)) return 4;
  Real p, rho0, uu;
  const Real W = W_of_vsq(s.D, K, vsq, &p, &rho0, &uu, g);
  const Real gtmp = std::sqrt(1. - vsq);
  const Real Gamma = 1. / gtmp;
  if ((rho0 <= 0.) || (uu <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[ENY] = uu;
  prim[ENT] = (g - 1.) * uu * pgm::pow(rho0, -g);
  harm_velocity(s, Gamma, W, prim);
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  return 0;
}
}  // namespace s1dvsq

// ---- Scheme1D (scheme_1d.h; USE_ISENTROPIC undefined -> func_1d_orig2) ----
namespace s1d {
// :376-409
inline void func_1d_orig2(Real QdotBsq, Real K, Real D, Real Bsq, Real Qtsq,
                          const Real x[1], Real dx[1], Real *f, Real *df,
                          Real g) {
  const Real W = x[0];
  const Real t1 = D * D;
  const Real t2 = QdotBsq * t1;
  const Real t3 = t2 * Bsq;
  const Real t5 = Bsq * Bsq;
  const Real t8 = t1 * Bsq;
  const Real t10 = t1 * W;
  const Real t21 = W * W;
  const Real rho = t1 * (1. + g * K / (g - 1.)) / W;
  const Real t23 = rho * rho;
  const Real t26 = 1 / t1;
  const Real resid =
      (t3 + (2.0 * t2 + ((Qtsq - t5) * t1 + (-2.0 * t8 - t10) * W) * W) * W +
       (t5 + (2.0 * Bsq + W) * W) * t21 * t23) *
      t26 / t21;
  const Real jac = -2.0 *
                   (t3 + (t2 + (t8 + t10) * t21) * W +
                    (t5 + Bsq * W) * t21 * t23) *
                   t26 / t21 / W;
  dx[0] = -resid / jac;
  *f = 0.5 * resid * resid;
  *df = -2. * (*f);
}
// :196-304
inline int newton(Real QdotBsq, Real K, Real D, Real Bsq, Real Qtsq, Real x[1],
                  Real g) {
  Real f = 1., df = 1., dx[1];
  Real errx = 1.;
  int i_extra = 0, doing_extra = 0, n_iter = 0, keep = 1;
  while (keep) {
    func_1d_orig2(QdotBsq, K, D, Bsq, Qtsq, x, dx, &f, &df, g);
    errx = 0.;
    x[0] += dx[0];
    int i_increase = 0;
    while (((x[0] * x[0] * x[0] * (x[0] + 2. * Bsq) -
             QdotBsq * (2. * x[0] + Bsq)) <= x[0] * x[0] * (Qtsq - Bsq * Bsq)) &&
           (i_increase < 10)) {
      x[0] -= (1. * i_increase) * dx[0] / 10.;
      i_increase++;
    }
    errx = (x[0] == 0.) ? std::fabs(dx[0]) : std::fabs(dx[0] / x[0]);
    x[0] = std::fabs(x[0]);
    if ((std::fabs(errx) <= NEWT_TOL) && (doing_extra == 0) &&
        (EXTRA_NEWT_ITER > 0))
      doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((std::fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) ||
        (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if ((std::isfinite(f) == 0) || (std::isfinite(df) == 0) ||
      (std::isfinite(x[0]) == 0))
    return 2;
  if (std::fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}
// :411-568
inline int invert(const Real U[9], Real prim[9], Real g,
                  const Real gcov[4][4], const Real gcon[4][4]) {
  Real K = prim[ENT];
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  HarmSetup s;
  harm_setup(U, gcov, gcon, s);
  Real utsq;
  if (!harm_utsq(prim, gcov, utsq)) return 2;
  const Real uvsq = 1. + utsq;
  Real Gamma = std::sqrt(uvsq);
  Real rho0 = s.D / Gamma;
  Real p = (K * pgm::pow(rho0, g));
  Real uu = (p / (g - 1.));
  Real w = rho0 + uu + p;
  Real W_last = w * uvsq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) -
           s.QdotBsq * (2. * W_last + s.Bsq)) <=
          W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  Real x[1] = {W_last};
  int retval = newton(s.QdotBsq, K, s.D, s.Bsq, s.Qtsq, x, g);
  const Real W = x[0];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  const Real vsq = s2d::vsq_calc(s.Bsq, s.QdotBsq, s.Qtsq, W);  // :531
  if (vsq >= 1.) return 4;
  const Real gtmp = std::sqrt(1. - vsq);
  Gamma = 1. / gtmp;
  rho0 = s.D * gtmp;
  w = W * (1. - vsq);
  p = (K * pgm::pow(rho0, g));
  uu = (p / (g - 1.));
  if ((rho0 <= 0.) || (uu <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[ENY] = uu;
  prim[ENT] = (g - 1.) * uu * pgm::pow(rho0, -g);
  harm_velocity(s, Gamma, W, prim);
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  return 0;
}
}  // namespace s1d

// ---- SchemeKastaun (scheme_kastaun.h) ------------------------------------
namespace kastaun {
inline Real sq(Real x) { return x * x; }
// :83-108
inline Real root_function(Real mu, Real D, Real q, Real bsq, Real rsq,
                          Real rbsq, Real g) {
  const Real x = 1.0 / (1.0 + mu * bsq);
  const Real xsq = x * x;
  const Real rbarsq = x * (rsq * x + mu * (x + 1.0) * rbsq);
  const Real musq = mu * mu;
  Real vsq = musq * rbarsq;
  vsq = kmin(kmax(vsq, 0.0), 1.0 - 1.0e-14);
  const Real inv_lorentz = std::sqrt(1.0 - vsq);
  const Real qbar = q - 0.5 * bsq - 0.5 * musq * xsq * (bsq * rsq - rbsq);
  const Real eoverD = qbar - mu * rbarsq + 1.0;
  const Real rho = D * inv_lorentz;
  Real eps = D * eoverD - rho;
  eps = kmax(eps, 1.0e-300);
  const Real pressure = (g - 1.0) * eps;
  const Real hh = 1.0 + (eps + pressure) / rho;
  const Real nu_a = hh * inv_lorentz;
  const Real nu_b = eoverD + pressure / D;
  const Real nu = kmax(nu_a, nu_b);
  const Real mu_hat = 1.0 / (nu + mu * rbarsq);
  return mu - mu_hat;
}
// :110-165
inline int false_position(Real &mu, Real D, Real q, Real bsq, Real rsq,
                          Real rbsq, Real g) {
  Real lower = 0.0, upper = 1.0;
  Real f_lower = root_function(lower, D, q, bsq, rsq, rbsq, g);
  Real f_upper = root_function(upper, D, q, bsq, rsq, rbsq, g);
  if (!std::isfinite(f_lower) || !std::isfinite(f_upper)) return 1;
  if (std::fabs(f_lower) <= NEWT_TOL) { mu = lower; return 0; }
  if (std::fabs(f_upper) <= NEWT_TOL) { mu = upper; return 0; }
  if (f_lower * f_upper > 0.0) return 2;
  int side = 0;
  mu = lower;
  for (int iter = 0; iter < MAX_NEWT_ITER; ++iter) {
    const Real old_mu = mu;
    mu = (f_upper * lower - f_lower * upper) / (f_upper - f_lower);
    const Real f_mu = root_function(mu, D, q, bsq, rsq, rbsq, g);
    if (!std::isfinite(mu) || !std::isfinite(f_mu)) return 3;
    if (std::fabs((mu - old_mu) / (mu + 1.0e-300)) <= NEWT_TOL) return 0;
    if (f_mu * f_lower >= 0.0) {
      if (side == 1) {
        const Real weight = 1.0 - f_mu / f_lower;
        f_upper = (weight > 0.0) ? f_upper * weight : 0.5 * f_upper;
      }
      lower = mu;
      f_lower = f_mu;
      side = 1;
    } else {
      if (side == -1) {
        const Real weight = 1.0 - f_mu / f_upper;
        f_lower = (weight > 0.0) ? f_lower * weight : 0.5 * f_lower;
      }
      upper = mu;
      f_upper = f_mu;
      side = -1;
    }
  }
  return 4;
}
// :167-259
inline int invert(const Real U[9], Real prim[9], Real g,
                  const Real gcov[4][4], const Real gcon[4][4]) {
  const Real gm[6] = {gcov[1][1], gcov[1][2], gcov[1][3],
                      gcov[2][2], gcov[2][3], gcov[3][3]};
  const Real det = gm[0] * gm[3] * gm[5] + 2.0 * gm[1] * gm[2] * gm[4] -
                   gm[0] * gm[4] * gm[4] - gm[1] * gm[1] * gm[5] -
                   gm[2] * gm[2] * gm[3];
  if (!(det > 0.0) || !std::isfinite(det)) return 1;
  const Real idet = 1.0 / det;
  Real gi[6];
  gi[0] = (gm[3] * gm[5] - gm[4] * gm[4]) * idet;
  gi[1] = (gm[2] * gm[4] - gm[1] * gm[5]) * idet;
  gi[2] = (gm[1] * gm[4] - gm[2] * gm[3]) * idet;
  gi[3] = (gm[0] * gm[5] - gm[2] * gm[2]) * idet;
  gi[4] = (gm[1] * gm[2] - gm[0] * gm[4]) * idet;
  gi[5] = (gm[0] * gm[3] - gm[1] * gm[1]) * idet;
  const Real D = U[RHO];
  if (!(D > 0.0) || !std::isfinite(D)) return 2;
  Real ncov[4], Qcov[4], Qcon[4];
  ncov_calc(gcon, ncov);
  Qcov[0] = U[ENY];
  Qcov[1] = U[UX1];
  Qcov[2] = U[UX2];
  Qcov[3] = U[UX3];
  raise_g(Qcov, gcon, Qcon);
  const Real Qdotn = Qcon[0] * ncov[0];
  const Real tau = -Qdotn - D;
  if (!std::isfinite(tau)) return 3;
  const Real S_d[3] = {U[UX1], U[UX2], U[UX3]};
  Real S_u[3];
  S_u[0] = gi[0] * S_d[0] + gi[1] * S_d[1] + gi[2] * S_d[2];
  S_u[1] = gi[1] * S_d[0] + gi[3] * S_d[1] + gi[4] * S_d[2];
  S_u[2] = gi[2] * S_d[0] + gi[4] * S_d[1] + gi[5] * S_d[2];
  const Real B_u[3] = {U[BX1], U[BX2], U[BX3]};
  Real B_d[3];
  B_d[0] = gm[0] * B_u[0] + gm[1] * B_u[1] + gm[2] * B_u[2];
  B_d[1] = gm[1] * B_u[0] + gm[3] * B_u[1] + gm[4] * B_u[2];
  B_d[2] = gm[2] * B_u[0] + gm[4] * B_u[1] + gm[5] * B_u[2];
  const Real Bsq = B_u[0] * B_d[0] + B_u[1] * B_d[1] + B_u[2] * B_d[2];
  const Real Ssq = S_u[0] * S_d[0] + S_u[1] * S_d[1] + S_u[2] * S_d[2];
  const Real SdotB = B_u[0] * S_d[0] + B_u[1] * S_d[1] + B_u[2] * S_d[2];
  if (!std::isfinite(Bsq) || !std::isfinite(Ssq) || !std::isfinite(SdotB))
    return 4;
  const Real inv_D = 1.0 / D;
  const Real sqrt_D = std::sqrt(D);
  const Real bsq = Bsq * inv_D;
  const Real rsq = Ssq * inv_D * inv_D;
  const Real rbsq = sq(SdotB / (D * sqrt_D));
  const Real q = tau * inv_D;
  Real mu;
  const int rs = false_position(mu, D, q, bsq, rsq, rbsq, g);
  if (rs != 0) return 100 + rs;
  const Real x = 1.0 / (1.0 + mu * bsq);
  const Real rb = SdotB / (D * sqrt_D);
  const Real rbarsq = x * (rsq * x + mu * (x + 1.0) * rbsq);
  const Real vsq = mu * mu * rbarsq;
  if (!(vsq >= 0.0) || vsq >= 1.0 || !std::isfinite(vsq)) return 5;
  const Real lorentz = 1.0 / std::sqrt(1.0 - vsq);
  const Real rho = D / lorentz;
  const Real qbar = q - 0.5 * bsq - 0.5 * mu * mu * x * x * (bsq * rsq - rbsq);
  const Real eoverD = qbar - mu * rbarsq + 1.0;
  const Real eps = D * eoverD - rho;
  if (!(rho > 0.0) || !(eps > 0.0) || !std::isfinite(eps)) return 6;
  const Real r_u[3] = {S_u[0] * inv_D, S_u[1] * inv_D, S_u[2] * inv_D};
  const Real b_u[3] = {B_u[0] / sqrt_D, B_u[1] / sqrt_D, B_u[2] / sqrt_D};
  const Real Wmu_x = lorentz * mu * x;
  prim[RHO] = rho;
  prim[ENY] = eps;
  prim[ENT] = (g - 1.) * eps * pgm::pow(rho, -g);
  for (int d = 0; d < 3; ++d) prim[UX1 + d] = Wmu_x * (r_u[d] + rb * mu * b_u[d]);
  prim[BX1] = U[BX1];
  prim[BX2] = U[BX2];
  prim[BX3] = U[BX3];
  return 0;
}
}  // namespace kastaun

// ---------------------------------------------------------------------------
// physics/heating_model.h
// ---------------------------------------------------------------------------
struct HeatParams {  // heating_model.h:27-37
  int model;
  Real gamma, gamma_p, gamma_e, fel_constant, ratio_min, ratio_max;
  bool limit_kel, suppress_highb_heat, enforce_positive_dissipation;
};
struct HeatCell {  // heating_model.h:39-46
  Real rho, energy, bsq, adv_total, rec_total, adv_electron;
};

inline Real clip(Real v, Real lo, Real hi) { return kmax(lo, kmin(v, hi)); }

// heating_model.h:53-109
inline Real heating_fraction(const HeatParams &p, const HeatCell &c) {
  constexpr Real kElectronMass = 9.1093826e-28;
  constexpr Real kProtonMass = 1.67262171e-24;
  const Real tpr = (p.gamma_p - 1.0) * c.energy / c.rho;
  const Real tel = c.adv_electron * pgm::pow(c.rho, p.gamma_e - 1.0);
  switch (p.model) {
    case 0:
      return p.fel_constant;
    case 1: {
      const Real trat = tpr / tel;
      const Real pres = c.rho * tpr;
      const Real beta = kmin(2.0 * pres / c.bsq, 1.0e20);
      const Real log_trat = pgm::log(trat) / pgm::log(10.0);
      const Real mbeta = 2.0 - 0.2 * log_trat;
      const Real c2 = (trat <= 1.0) ? 1.6 / trat : 1.2 / trat;
      const Real c3 = (trat <= 1.0) ? 18.0 + 5.0 * log_trat : 18.0;
      const Real beta_pow = pgm::pow(beta, mbeta);
      const Real qrat = 0.92 * (c2 * c2 + beta_pow) / (c3 * c3 + beta_pow) *
                        pgm::exp(-1.0 / beta) *
                        std::sqrt(kProtonMass / kElectronMass * trat);
      return 1.0 / (1.0 + qrat);
    }
    case 2: {
      const Real trat = tpr / tel;
      const Real pres = c.rho * tpr;
      const Real beta = kmin(2.0 * pres / c.bsq, 1.0e20);
      const Real qi_qe =
          35.0 / (1.0 + pgm::pow(beta / 15.0, -1.4) * pgm::exp(-0.1 / trat));
      return 1.0 / (1.0 + qi_qe);
    }
    case 3: {
      const Real sigma = c.bsq / c.rho;
      return 0.25 * (1.0 + std::sqrt((sigma / 5.0) / (2.0 + sigma / 5.0)));
    }
    case 4: {
      const Real pres = (p.gamma_p - 1.0) * c.energy;
      const Real pg = (p.gamma - 1.0) * c.energy;
      const Real beta = 2.0 * pres / c.bsq;
      const Real sigma = c.bsq / (c.rho + c.energy + pg);
      const Real betamax = 0.25 / sigma;
      return 0.5 * pgm::exp(-pgm::pow(1.0 - beta / betamax, 3.3) /
                            (1.0 + 1.2 * pgm::pow(sigma, 0.7)));
    }
    case 5: {
      const Real trat_inv = tel / tpr;
      const Real qe_qi = 0.33 * std::sqrt(trat_inv);
      return 1.0 / (1.0 + 1.0 / qe_qi);
    }
  }
  return p.fel_constant;
}

// heating_model.h:141-170
inline Real heating_apply(const HeatParams &p, const HeatCell &c) {
  const Real fel = heating_fraction(p, c);
  Real diss = (p.gamma_e - 1.0) / (p.gamma - 1.0) *
              pgm::pow(c.rho, p.gamma - p.gamma_e) * (c.rec_total - c.adv_total);
  if (p.suppress_highb_heat && (c.bsq / c.rho > 1.0)) diss = 0.0;
  if (p.enforce_positive_dissipation) diss = kmax(diss, 0.0);
  Real kel = c.adv_electron + fel * diss;
  if (!p.limit_kel && p.model == 0) return kel;
  const Real kel_max =
      c.adv_total * pgm::pow(c.rho, p.gamma - p.gamma_e) /
      (p.ratio_min * (p.gamma - 1.0) / (p.gamma_p - 1.0) +
       (p.gamma - 1.0) / (p.gamma_e - 1.0));
  const Real kel_min =
      c.adv_total * pgm::pow(c.rho, p.gamma - p.gamma_e) /
      (p.ratio_max * (p.gamma - 1.0) / (p.gamma_p - 1.0) +
       (p.gamma - 1.0) / (p.gamma_e - 1.0));
  return clip(kel, kel_min, kel_max);
}

// heating_model.h:172-179
inline Real clamp_by_ratio(Real rmin, Real rmax, Real total, Real electron) {
  const Real lo = total / (1.0 + rmax);
  const Real hi = total / (1.0 + rmin);
  const Real b = kmax(0.0, kmin(electron, total));
  return kmax(lo, kmin(b, hi));
}

}  // namespace orc
#endif  // PANGU_ORACLE_CELL_H
