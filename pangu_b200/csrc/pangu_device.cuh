// pangu_device.cuh -- per-cell device mathematics of the stage engine (FP64).
//
// The FP64 engine is built with --fmad=false and calls the double-double
// pow/exp/log of pgmath.h, so every operation rounds as in a plain C++ build
// of the reference: the conservative-to-primitive chain is chaotic in
// floor-dominated cells (whether a Newton solve converges flips on one-ulp
// input differences), so parity needs bit-identical arithmetic. The metric
// algebra additionally spells its operations with explicit round-to-nearest
// intrinsics, which keeps it exact even in a build that allows contraction.
#ifndef PANGU_DEVICE_CUH
#define PANGU_DEVICE_CUH

#include <cstdint>

#include "pgmath.h"

// Powers, exponentials and logarithms: correctly rounded (pgmath.h) in the
// exact build; an includer may substitute the CUDA math library.
#ifndef PGD_POW
#define PGD_POW pgm::pow
#define PGD_EXP pgm::exp
#define PGD_LOG pgm::log
#endif

namespace pgd {

// variable_mnemonics.h:7-14
enum { RHO, ENY, UX1, UX2, UX3, BX1, BX2, BX3, ENT, KEL, NPRIM };
enum { MINKOWSKI = 0, BL = 1, CKS = 2, MKS = 3 };

#define PGD __device__ __forceinline__

PGD double MUL(double a, double b) { return __dmul_rn(a, b); }
PGD double ADD(double a, double b) { return __dadd_rn(a, b); }
PGD double SUB(double a, double b) { return __dsub_rn(a, b); }
PGD double DIV(double a, double b) { return __ddiv_rn(a, b); }

// Kokkos::min / Kokkos::max semantics.
PGD double kmin(double a, double b) { return (b < a) ? b : a; }
PGD double kmax(double a, double b) { return (a < b) ? b : a; }

struct Geo {
  double gcov[4][4];
  double gcon[4][4];
  double gdet;
  double sg;     // sqrt(|gdet|), as every reference task computes it
  double alpha;  // 1 / sqrt(-gcon[0][0]), as state_calculation.h:24 computes it
};

// Coordinate values along x1 and x2 that fully determine the MKS / BL
// metric: r = exp(x1), J1 = d exp / dx1 (finite difference), and sin, cos of
// theta(x2) with J2 = d theta / dx2. Built on the host (engine.cu).
struct MapPt {
  double r, J1, sth, cth, J2;
};

// ---------------------------------------------------------------------------
// Physical metrics with the code Jacobian applied (MKS.h:25-107, BL.h:25-107,
// CKS.h:24-108, minkowski.h:24-70). The Jacobian of every map is diagonal,
// so the quadruple sum reduces to (g[r][c] J[r]) J[c] (+0.0, which turns a
// negative zero into the positive zero of the reference's accumulation).
// ---------------------------------------------------------------------------
PGD void ks_code_gcov(const MapPt &m, double a, double g[4][4]) {
  const double r = m.r, sth = m.sth, cth = m.cth;
  const double Sigma = ADD(MUL(r, r), MUL(MUL(MUL(a, a), cth), cth));
  const double trS = DIV(MUL(2.0, r), Sigma);
  const double J[4] = {1.0, m.J1, m.J2, 1.0};
  double p[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) p[i][j] = 0.0;
  p[0][0] = ADD(-1.0, trS);
  p[0][1] = trS;
  p[0][3] = DIV(MUL(MUL(MUL(MUL(-2.0, a), r), sth), sth), Sigma);
  p[1][0] = p[0][1];
  p[1][1] = ADD(1.0, trS);
  p[1][3] = MUL(MUL(MUL(-a, ADD(1.0, trS)), sth), sth);
  p[2][2] = Sigma;
  p[3][0] = p[0][3];
  p[3][1] = p[1][3];
  p[3][3] = MUL(MUL(sth, sth), ADD(Sigma, MUL(MUL(MUL(MUL(a, a), sth), sth), ADD(1.0, trS))));
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = ADD(MUL(MUL(p[i][j], J[i]), J[j]), 0.0);
}

PGD void bl_code_gcov(const MapPt &m, double a, double g[4][4]) {
  const double r = m.r, sth = m.sth, cth = m.cth;
  const double sth2 = MUL(sth, sth);
  const double r2 = MUL(r, r);
  const double a2 = MUL(a, a);
  const double mu = ADD(1.0, DIV(MUL(MUL(a2, cth), cth), r2));
  const double delta = ADD(SUB(1.0, DIV(2.0, r)), DIV(a2, r2));
  const double inv_r_mu = DIV(1.0, MUL(r, mu));
  const double J[4] = {1.0, m.J1, m.J2, 1.0};
  double p[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) p[i][j] = 0.0;
  p[0][0] = ADD(-1.0, MUL(2.0, inv_r_mu));
  p[0][3] = MUL(MUL(MUL(-2.0, a), sth2), inv_r_mu);
  p[1][1] = DIV(mu, delta);
  p[2][2] = DIV(r2, mu);
  p[3][0] = p[0][3];
  p[3][3] = MUL(MUL(r2, sth2),
                ADD(ADD(1.0, DIV(a2, r2)), DIV(MUL(MUL(2.0, a2), sth2), MUL(MUL(r, r2), mu))));
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = ADD(MUL(MUL(p[i][j], J[i]), J[j]), 0.0);
}

PGD void cks_code_gcov(double xx, double yy, double zz, double a, double g[4][4]) {
  const double r2c = ADD(ADD(MUL(xx, xx), MUL(yy, yy)), MUL(zz, zz));
  const double a2 = MUL(a, a);
  const double tmp = SUB(r2c, a2);
  const double sqrtarg = ADD(MUL(tmp, tmp), MUL(MUL(MUL(4.0, a2), zz), zz));
  const double r = __dsqrt_rn(MUL(0.5, ADD(tmp, __dsqrt_rn(sqrtarg))));
  const double rs = (r > 1.0e-15) ? r : 1.0e-15;
  const double r2 = MUL(rs, rs);
  const double r3 = MUL(r2, rs);
  const double r4 = MUL(r2, r2);
  const double xd = ADD(r4, MUL(MUL(a2, zz), zz));
  const double xi = (xd > 0.0) ? DIV(MUL(2.0, r3), xd) : 0.0;
  const double dl = ADD(r2, a2);
  const double l[4] = {1.0, DIV(ADD(MUL(rs, xx), MUL(a, yy)), dl),
                       DIV(SUB(MUL(rs, yy), MUL(a, xx)), dl), DIV(zz, rs)};
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      const double eta = (m == n) ? ((m == 0) ? -1.0 : 1.0) : 0.0;
      g[m][n] = ADD(ADD(eta, MUL(MUL(xi, l[m]), l[n])), 0.0);
    }
}

PGD void minkowski_gcov(double g[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = (i == j) ? ((i == 0) ? -1.0 : 1.0) : 0.0;
}

// tensor_algebra.h:71-124, rounding step by step. Returns 0 if singular
// (gcon then untouched).
PGD int gj_invert(const double m[4][4], double inv[4][4]) {
  double aug[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      aug[i][j] = m[i][j];
      aug[i][j + 4] = (i == j) ? 1.0 : 0.0;
    }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (aug[i][i] == 0.0) {
      int sw = -1;
#pragma unroll
      for (int j = i + 1; j < 4; ++j)
        if (sw < 0 && aug[j][i] != 0.0) sw = j;
      if (sw == -1) return 0;
#pragma unroll
      for (int j = i + 1; j < 4; ++j)
        if (j == sw)
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const double t = aug[i][c];
            aug[i][c] = aug[j][c];
            aug[j][c] = t;
          }
    }
    const double piv = aug[i][i];
#pragma unroll
    for (int c = 0; c < 8; ++c) aug[i][c] = DIV(aug[i][c], piv);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j == i) continue;
      const double f = aug[j][i];
#pragma unroll
      for (int c = 0; c < 8; ++c) aug[j][c] = SUB(aug[j][c], MUL(f, aug[i][c]));
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) inv[i][j] = aug[i][j + 4];
  return 1;
}

// tensor_algebra.h:39-69, rounding step by step.
PGD double determinant(const double m[4][4]) {
#define D2(a, b, c, d) SUB(MUL(a, b), MUL(c, d))
  const double t0 = MUL(m[0][0], ADD(SUB(MUL(m[1][1], D2(m[2][2], m[3][3], m[2][3], m[3][2])),
                                         MUL(m[1][2], D2(m[2][1], m[3][3], m[2][3], m[3][1]))),
                                     MUL(m[1][3], D2(m[2][1], m[3][2], m[2][2], m[3][1]))));
  const double t1 = MUL(m[0][1], ADD(SUB(MUL(m[1][0], D2(m[2][2], m[3][3], m[2][3], m[3][2])),
                                         MUL(m[1][2], D2(m[2][0], m[3][3], m[2][3], m[3][0]))),
                                     MUL(m[1][3], D2(m[2][0], m[3][2], m[2][2], m[3][0]))));
  const double t2 = MUL(m[0][2], ADD(SUB(MUL(m[1][0], D2(m[2][1], m[3][3], m[2][3], m[3][1])),
                                         MUL(m[1][1], D2(m[2][0], m[3][3], m[2][3], m[3][0]))),
                                     MUL(m[1][3], D2(m[2][0], m[3][1], m[2][1], m[3][0]))));
  const double t3 = MUL(m[0][3], ADD(SUB(MUL(m[1][0], D2(m[2][1], m[3][2], m[2][2], m[3][1])),
                                         MUL(m[1][1], D2(m[2][0], m[3][2], m[2][2], m[3][0]))),
                                     MUL(m[1][2], D2(m[2][0], m[3][1], m[2][1], m[3][0]))));
#undef D2
  return SUB(ADD(SUB(t0, t1), t2), t3);
}

// ---------------------------------------------------------------------------
// Structural zeros of the code metrics. The MKS and BL metrics couple only
// (t, r, phi) with theta apart, and the Minkowski metric is diagonal; their
// zero entries are exact zeros by construction (ks_code_gcov, bl_code_gcov).
// Operations on a structural zero change at most the sign of a zero result,
// so skipping them leaves every non-zero value bit-identical to the dense
// computation of the reference.
// ---------------------------------------------------------------------------
struct Pattern {
  bool nz[4][4];
};
__host__ __device__ constexpr Pattern metric_pattern(int mt) {
  Pattern p{};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      if (mt == MKS) {
        const bool tr = (r != 2), tc = (c != 2);
        p.nz[r][c] = (tr && tc) || (r == 2 && c == 2);
      } else if (mt == BL) {
        p.nz[r][c] = (r == c) || (r == 0 && c == 3) || (r == 3 && c == 0);
      } else if (mt == MINKOWSKI) {
        p.nz[r][c] = (r == c);
      } else {
        p.nz[r][c] = true;
      }
    }
  return p;
}

// Fill pattern of the Gauss-Jordan elimination of tensor_algebra.h:71-124:
// a[i][r][c] is true when entry (r, c) of the augmented matrix may be
// non-zero before pivot step i. After step i, column i of every other row is
// exactly zero (x - x * 1).
struct GJPlan {
  bool a[4][4][8];
};
__host__ __device__ constexpr GJPlan gj_plan(int mt) {
  GJPlan P{};
  bool cur[4][8] = {};
  const Pattern pt = metric_pattern(mt);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      cur[r][c] = pt.nz[r][c];
      cur[r][c + 4] = (r == c);
    }
  for (int i = 0; i < 4; ++i) {
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 8; ++c) P.a[i][r][c] = cur[r][c];
    bool prow[8] = {};
    for (int c = 0; c < 8; ++c) prow[c] = cur[i][c];
    for (int j = 0; j < 4; ++j) {
      if (j == i || !cur[j][i]) continue;
      for (int c = 0; c < 8; ++c) cur[j][c] = cur[j][c] || prow[c];
      cur[j][i] = false;
    }
  }
  return P;
}

// Gauss-Jordan inverse restricted to the fill pattern of metric type MT.
// A pivot that is exactly zero needs the reference's row swap: the dense
// routine then redoes the inversion from scratch.
template <int MT>
PGD int gj_invert_s(const double m[4][4], double inv[4][4]) {
  constexpr GJPlan P = gj_plan(MT);
  double aug[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      aug[i][j] = m[i][j];
      aug[i][j + 4] = (i == j) ? 1.0 : 0.0;
    }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double piv = aug[i][i];
    if (piv == 0.0) return gj_invert(m, inv);
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (P.a[i][i][c]) aug[i][c] = DIV(aug[i][c], piv);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j == i || !P.a[i][j][i]) continue;
      const double f = aug[j][i];
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (P.a[i][i][c]) aug[j][c] = SUB(aug[j][c], MUL(f, aug[i][c]));
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) inv[i][j] = aug[i][j + 4];
  return 1;
}

// The cofactor determinant of tensor_algebra.h:39-69 with the structural
// zeros of MT folded away at compile time: Zr stands for a value known to be
// a (signed) zero, and the operator overloads return what the dense
// arithmetic returns for it (x - 0 = x, 0 - x = -x, 0 * x = 0).
struct Zr {};
PGD double op_mul(double a, double b) { return MUL(a, b); }
PGD Zr op_mul(Zr, double) { return {}; }
PGD Zr op_mul(double, Zr) { return {}; }
PGD Zr op_mul(Zr, Zr) { return {}; }
PGD double op_sub(double a, double b) { return SUB(a, b); }
PGD double op_sub(double a, Zr) { return a; }
PGD double op_sub(Zr, double b) { return -b; }
PGD Zr op_sub(Zr, Zr) { return {}; }
PGD double op_add(double a, double b) { return ADD(a, b); }
PGD double op_add(double a, Zr) { return a; }
PGD double op_add(Zr, double b) { return b; }
PGD Zr op_add(Zr, Zr) { return {}; }
PGD double to_double(double a) { return a; }
PGD double to_double(Zr) { return 0.0; }

template <int MT, int r, int c>
PGD auto el(const double (&m)[4][4]) {
  if constexpr (metric_pattern(MT).nz[r][c]) {
    return m[r][c];
  } else {
    return Zr{};
  }
}

template <int MT>
PGD double determinant_s(const double (&m)[4][4]) {
#define E(r, c) el<MT, r, c>(m)
#define D2(a, b, c, d) op_sub(op_mul(a, b), op_mul(c, d))
  const auto t0 = op_mul(E(0, 0), op_add(op_sub(op_mul(E(1, 1), D2(E(2, 2), E(3, 3), E(2, 3), E(3, 2))),
                                                op_mul(E(1, 2), D2(E(2, 1), E(3, 3), E(2, 3), E(3, 1)))),
                                         op_mul(E(1, 3), D2(E(2, 1), E(3, 2), E(2, 2), E(3, 1)))));
  const auto t1 = op_mul(E(0, 1), op_add(op_sub(op_mul(E(1, 0), D2(E(2, 2), E(3, 3), E(2, 3), E(3, 2))),
                                                op_mul(E(1, 2), D2(E(2, 0), E(3, 3), E(2, 3), E(3, 0)))),
                                         op_mul(E(1, 3), D2(E(2, 0), E(3, 2), E(2, 2), E(3, 0)))));
  const auto t2 = op_mul(E(0, 2), op_add(op_sub(op_mul(E(1, 0), D2(E(2, 1), E(3, 3), E(2, 3), E(3, 1))),
                                                op_mul(E(1, 1), D2(E(2, 0), E(3, 3), E(2, 3), E(3, 0)))),
                                         op_mul(E(1, 3), D2(E(2, 0), E(3, 1), E(2, 1), E(3, 0)))));
  const auto t3 = op_mul(E(0, 3), op_add(op_sub(op_mul(E(1, 0), D2(E(2, 1), E(3, 2), E(2, 2), E(3, 1))),
                                                op_mul(E(1, 1), D2(E(2, 0), E(3, 2), E(2, 2), E(3, 0)))),
                                         op_mul(E(1, 2), D2(E(2, 0), E(3, 1), E(2, 1), E(3, 0)))));
#undef D2
#undef E
  return to_double(op_sub(op_add(op_sub(t0, t1), t2), t3));
}

// ---------------------------------------------------------------------------
// physics/ (state_calculation.h, energy_momentum_tensor.h,
// contravariant_flux.h, fast_magnetosonic_speed.h)
// ---------------------------------------------------------------------------
struct State {
  double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
};

template <int MT>
PGD void calc_state(const double P[NPRIM], const Geo &g, State &s) {
  constexpr Pattern PT = metric_pattern(MT);
  const double alpha = g.alpha;
  const double u[3] = {P[UX1], P[UX2], P[UX3]};
  // 1 + gamma_ij u^i u^j, summed left to right over (i, j) as square3 does
  // (tensor_algebra.h:18-37); structurally zero terms are skipped.
  double sq = 0.0;
#pragma unroll
  for (int i = 1; i < 4; ++i)
#pragma unroll
    for (int j = 1; j < 4; ++j)
      if (PT.nz[i][j]) sq = sq + u[i - 1] * g.gcov[i][j] * u[j - 1];
  const double lor = sqrt(1.0 + sq);
  s.ucon[0] = lor / alpha;
#pragma unroll
  for (int i = 1; i < 4; ++i)
    s.ucon[i] = PT.nz[0][i] ? u[i - 1] - s.ucon[0] * g.gcon[0][i] * alpha * alpha : u[i - 1];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (PT.nz[r][c]) v += g.gcov[r][c] * s.ucon[c];
    s.ucov[r] = v;
  }
  s.bcon[0] = P[BX1] * s.ucov[1] + P[BX2] * s.ucov[2] + P[BX3] * s.ucov[3];
  s.bcon[1] = (P[BX1] + s.bcon[0] * s.ucon[1]) / s.ucon[0];
  s.bcon[2] = (P[BX2] + s.bcon[0] * s.ucon[2]) / s.ucon[0];
  s.bcon[3] = (P[BX3] + s.bcon[0] * s.ucon[3]) / s.ucon[0];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (PT.nz[r][c]) v += g.gcov[r][c] * s.bcon[c];
    s.bcov[r] = v;
  }
  s.bsq = s.bcon[0] * s.bcov[0] + s.bcon[1] * s.bcov[1] + s.bcon[2] * s.bcov[2] +
          s.bcon[3] * s.bcov[3];
}

// T^{dir}_m for a given state (energy_momentum_tensor.h:11-29).
PGD void emt_from_state(double gam, const double P[NPRIM], const State &s, int dir, double t[4]) {
  const double p_gas = (gam - 1.) * P[ENY];
  const double hh = P[RHO] + gam * P[ENY];
  const double e_tot = hh + s.bsq;
  const double p_tot = p_gas + 0.5 * s.bsq;
#pragma unroll
  for (int m = 0; m < 4; ++m)
    t[m] = e_tot * s.ucon[dir] * s.ucov[m] + p_tot * (dir == m) - s.bcon[dir] * s.bcov[m];
}

// contravariant_flux.h:12-39 for a given state; sg = sqrt(|gdet|).
PGD void flux_from_state(double gam, const double P[NPRIM], const State &s, double sg, int dir,
                         double f[NPRIM]) {
  double t[4];
  emt_from_state(gam, P, s, dir, t);
  f[RHO] = P[RHO] * s.ucon[dir];
  f[ENY] = t[0] + f[RHO];
  f[UX1] = t[1];
  f[UX2] = t[2];
  f[UX3] = t[3];
  // Induction fluxes: rounded step by step, so the component along dir
  // cancels to exactly zero as in the reference (a fused multiply-add would
  // leave the rounding error of one product).
  f[BX1] = SUB(MUL(s.bcon[1], s.ucon[dir]), MUL(s.bcon[dir], s.ucon[1]));
  f[BX2] = SUB(MUL(s.bcon[2], s.ucon[dir]), MUL(s.bcon[dir], s.ucon[2]));
  f[BX3] = SUB(MUL(s.bcon[3], s.ucon[dir]), MUL(s.bcon[dir], s.ucon[3]));
  f[ENT] = P[ENT] * f[RHO];
  f[KEL] = P[KEL] * f[RHO];
#pragma unroll
  for (int n = 0; n < NPRIM; ++n) f[n] *= sg;
}

// fast_magnetosonic_speed.h:11-81 for a given state.
PGD void fast_speed_from_state(double gam, const double P[NPRIM], const Geo &g, const State &s,
                               int dir, double &vmax, double &vmin) {
  // ncov = e_dir, tcov = e_0: ncon = gcon[.][dir], tcon = gcon[.][0]
  const double hh = P[RHO] + gam * P[ENY];
  const double h_tot = s.bsq + hh;
  const double va_sq = s.bsq / h_tot;
  const double cs_sq = gam * (gam - 1.) * P[ENY] / hh;
  double cf_sq = cs_sq + va_sq - cs_sq * va_sq;
  if (cf_sq < 0.) cf_sq = 1e-10;
  if (cf_sq > 1.) cf_sq = 1.;
  const double n_sq = g.gcon[dir][dir];
  const double t_sq = g.gcon[0][0];
  const double n_dot_u = s.ucon[dir];
  const double t_dot_u = s.ucon[0];
  const double n_dot_t = g.gcon[0][dir];
  const double nu2 = n_dot_u * n_dot_u;
  const double tu2 = t_dot_u * t_dot_u;
  const double nutu = n_dot_u * t_dot_u;
  const double A = tu2 - (t_sq + tu2) * cf_sq;
  const double B = 2. * (nutu - (n_dot_t + nutu) * cf_sq);
  const double C = nu2 - (n_sq + nu2) * cf_sq;
  double disc = B * B - 4. * A * C;
  if ((disc < 0.0) && (disc > -1.e-10))
    disc = 0.0;
  else if (disc < -1.e-10)
    disc = 0.;
  disc = sqrt(disc);
  const double vp = -(-B + disc) / (2. * A);
  const double vm = -(-B - disc) / (2. * A);
  if (vp > vm) {
    vmax = vp;
    vmin = vm;
  } else {
    vmax = vm;
    vmin = vp;
  }
}

// ---------------------------------------------------------------------------
// interpolation/ (interpolater_mc.h:16-48, interpolater_ppm4.h:29-67)
// ---------------------------------------------------------------------------
PGD double minmod3(double a, double b, double c) {
  if (a > 0.0 && b > 0.0 && c > 0.0) return fmin(fmin(a, b), c);
  if (a < 0.0 && b < 0.0 && c < 0.0) return fmax(fmax(a, b), c);
  return 0.0;
}
// Right value at the upper face (ql_ip1) and left value at the lower face
// (qr_i) of the centre cell of a 3-point MC stencil.
PGD void mc(double qm1, double q, double qp1, double &ql_ip1, double &qr_i) {
  const double slope = minmod3(2.0 * (q - qm1), 0.5 * (qp1 - qm1), 2.0 * (qp1 - q));
  ql_ip1 = q + 0.5 * slope;
  qr_i = q - 0.5 * slope;
}
PGD void ppm4(double qm2, double qm1, double q, double qp1, double qp2, double &ql_ip1,
              double &qr_i) {
  double qlv = (7.0 * (q + qm1) - (qm2 + qp1)) / 12.0;
  double qrv = (7.0 * (q + qp1) - (qm1 + qp2)) / 12.0;
  qlv = fmax(qlv, fmin(q, qm1));
  qlv = fmin(qlv, fmax(q, qm1));
  qrv = fmax(qrv, fmin(q, qp1));
  qrv = fmin(qrv, fmax(q, qp1));
  const double qc = qrv - q;
  const double qd = qlv - q;
  if ((qc * qd) >= 0.0) {
    qlv = q;
    qrv = q;
  } else {
    if (fabs(qc) >= 2.0 * fabs(qd)) qrv = q - 2.0 * qd;
    if (fabs(qd) >= 2.0 * fabs(qc)) qlv = q - 2.0 * qc;
  }
  ql_ip1 = qrv;
  qr_i = qlv;
}

// ---------------------------------------------------------------------------
// recovery/ (constants.h:14-23; scheme_2d.h, scheme_1d_vsq.h, scheme_1d.h,
// scheme_kastaun.h)
// ---------------------------------------------------------------------------
constexpr int MAX_NEWT_ITER = 30;
constexpr double NEWT_TOL = 1e-10;
constexpr double MIN_NEWT_TOL = 1e-10;
constexpr int EXTRA_NEWT_ITER = 2;
constexpr double W_TOO_BIG = 1.e20;
constexpr double UTSQ_TOO_BIG = 1.e20;
constexpr double FAIL_VAL = 1.e30;

struct Harm {
  double Bcon[4], Qcon[4], ncon[4];
  double Bsq, QdotB, QdotBsq, Qdotn, Qsq, Qtsq, D;
};

// Bcon[0] = 0 and the structural zeros of the metric contribute signed
// zeros only; they are skipped.
template <int MT>
PGD void harm_setup(const double U[9], const Geo &g, Harm &s) {
  constexpr Pattern PT = metric_pattern(MT);
  s.Bcon[0] = 0.;
  s.Bcon[1] = U[BX1];
  s.Bcon[2] = U[BX2];
  s.Bcon[3] = U[BX3];
  double Bcov[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double v = 0.0;
#pragma unroll
    for (int j = 1; j < 4; j++)
      if (PT.nz[i][j]) v += g.gcov[i][j] * s.Bcon[j];
    Bcov[i] = v;
  }
  const double Qcov[4] = {U[ENY], U[UX1], U[UX2], U[UX3]};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double v = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (PT.nz[i][j]) v += g.gcon[i][j] * Qcov[j];
    s.Qcon[i] = v;
  }
  s.Bsq = s.Bcon[1] * Bcov[1] + s.Bcon[2] * Bcov[2] + s.Bcon[3] * Bcov[3];
  s.QdotB = Qcov[1] * s.Bcon[1] + Qcov[2] * s.Bcon[2] + Qcov[3] * s.Bcon[3];
  s.QdotBsq = s.QdotB * s.QdotB;
  const double lapse = sqrt(-1.0 / g.gcon[0][0]);
  const double n0 = -lapse;
#pragma unroll
  for (int i = 0; i < 4; i++) s.ncon[i] = PT.nz[i][0] ? g.gcon[i][0] * n0 : 0.0;
  s.Qdotn = s.Qcon[0] * n0;
  s.Qsq = Qcov[0] * s.Qcon[0] + Qcov[1] * s.Qcon[1] + Qcov[2] * s.Qcon[2] + Qcov[3] * s.Qcon[3];
  s.Qtsq = s.Qsq + s.Qdotn * s.Qdotn;
  s.D = U[RHO];
}

template <int MT>
PGD bool harm_utsq(const double prim[9], const Geo &g, double &utsq) {
  constexpr Pattern PT = metric_pattern(MT);
  const double u[3] = {prim[UX1], prim[UX2], prim[UX3]};
  double v = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++)
      if (PT.nz[i][j]) v += g.gcov[i][j] * u[i - 1] * u[j - 1];
  if ((v < 0.) && (fabs(v) < 1.0e-13)) v = fabs(v);
  utsq = v;
  return !(v < 0. || v > UTSQ_TOO_BIG);
}

template <int MT>
PGD void harm_velocity(const Harm &s, double Gamma, double W, double prim[9]) {
  constexpr Pattern PT = metric_pattern(MT);
#pragma unroll
  for (int i = 1; i < 4; i++) {
    const double qt = PT.nz[i][0] ? s.Qcon[i] + s.ncon[i] * s.Qdotn : s.Qcon[i];
    prim[UX1 + i - 1] = Gamma / (W + s.Bsq) * (qt + s.QdotB * s.Bcon[i] / W);
  }
}

PGD double vsq_calc(double Bsq, double QdotBsq, double Qtsq, double W) {
  const double Wsq = W * W;
  const double Xsq = (Bsq + W) * (Bsq + W);
  return ((Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * Xsq));
}

PGD bool w_too_small(double W, double Bsq, double QdotBsq, double Qtsq) {
  return (W * W * W * (W + 2. * Bsq) - QdotBsq * (2. * W + Bsq)) <= W * W * (Qtsq - Bsq * Bsq);
}

// Scheme2D::invert (scheme_2d.h:257-404) with general_newton_raphson
// (:158-255) and func_vsq (:99-156).
template <int MT>
PGD int invert_2d(const double U[9], double prim[9], double g, const Geo &geo,
                  const Harm &s) {
  double utsq;
  if (!harm_utsq<MT>(prim, geo, utsq)) return 2;
  const double gammasq = 1. + utsq;
  double Gamma = sqrt(gammasq);
  double rho0 = s.D / Gamma;
  double uu = prim[ENY];
  double p = (g - 1.) * uu;
  double w = rho0 + uu + p;
  double W_last = w * gammasq;
  for (int i = 0; i < 10 && w_too_small(W_last, s.Bsq, s.QdotBsq, s.Qtsq); ++i) W_last *= 10.;
  double x0 = fabs(W_last);
  double x1;
  {
    const double vsq = fabs(vsq_calc(s.Bsq, s.QdotBsq, s.Qtsq, W_last));
    x1 = (vsq > 1.) ? (1.0 - 1.e-15) : vsq;
  }
  const double Bsq = s.Bsq, QdotBsq = s.QdotBsq, Qtsq = s.Qtsq, Qdotn = s.Qdotn, D = s.D;
  const double gm1g = (g - 1.) / g;
  double f = 1., df = 1., errx = 1.;
  int i_extra = 0, doing_extra = 0;
  for (int n_iter = 0;; ++n_iter) {
    const double W = x0, vsq = x1;
    const double Wsq = W * W;
    const double gtmp = 1. - vsq;
    const double sgt = sqrt(gtmp);
    const double p_tmp = ((g - 1.) * (W * gtmp - D * sgt) / g);
    const double dPdW = ((g - 1.) * (1. - vsq) / g);
    const double dPdvsq = ((g - 1.) * (0.5 * D / sgt - W) / g);
    (void)gm1g;
    const double t2 = -0.5 * Bsq + dPdvsq;
    const double t3 = Bsq + W;
    const double t4 = t3 * t3;
    const double t9 = 1.0 / Wsq;
    const double t11 = Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.0 * W) * t9;
    const double t16 = QdotBsq * t9;
    const double t18 = -Qdotn - 0.5 * Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
    const double t21 = 1.0 / t3;
    const double t23 = 1.0 / W;
    const double t24 = t16 * t23;
    const double t25 = -1.0 + dPdW - t24;
    const double t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
    const double t36 = 1.0 / t35;
    const double dx0 = -(t2 * t11 + t4 * t18) * t21 * t36;
    const double t40 = (vsq + t24) * t3;
    const double dx1 = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
    df = -t11 * t11 - t18 * t18;
    f = -0.5 * df;
    const double xo0 = x0;
    x0 += dx0;
    x1 += dx1;
    errx = (x0 == 0.) ? fabs(dx0) : fabs(dx0 / x0);
    errx += (x1 == 0.) ? fabs(dx1) : fabs(dx1 / x1);
    x0 = fabs(x0);
    x0 = (x0 > W_TOO_BIG) ? xo0 : x0;
    x1 = (x1 < 0.) ? 0. : x1;
    x1 = (x1 > 1.) ? (1. - 1.e-15) : x1;
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      break;
  }
  int retval = 0;
  if (!isfinite(f) || !isfinite(df)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  const double W = x0, vsq = x1;
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  if (vsq >= 1.) return 4;
  const double gtmp = sqrt(1. - vsq);
  Gamma = 1. / gtmp;
  rho0 = D * gtmp;
  w = W * (1. - vsq);
  p = ((g - 1.) * (w - rho0) / g);
  uu = w - (rho0 + p);
  if ((rho0 <= 0.) || (uu <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[ENY] = uu;
  prim[ENT] = (g - 1.) * uu * PGD_POW(rho0, -g);
  harm_velocity<MT>(s, Gamma, W, prim);
  return 0;
}

// Scheme1Dvsq::invert (scheme_1d_vsq.h:222-351), K = stale prim[ENT].
PGD double w_of_vsq(double D, double K, double vsq, double g, double &p, double &rho,
                    double &uu) {
  const double gtmp = (1. - vsq);
  rho = D * sqrt(gtmp);
  p = (K * PGD_POW(rho, g));
  uu = (p / (g - 1.));
  return ((rho + uu + p) / gtmp);
}

template <int MT>
PGD int invert_1dvsq(const double U[9], double prim[9], double g, const Geo &geo,
                     const Harm &s) {
  (void)U;
  const double K = prim[ENT];
  double utsq;
  if (!harm_utsq<MT>(prim, geo, utsq)) return 2;
  const double gammasq = 1. + utsq;
  double x = 1. - 1. / gammasq;
  const double Bsq = s.Bsq, QdotBsq = s.QdotBsq, Qtsq = s.Qtsq, D = s.D;
  double f = 1., df = 1., errx = 1., W = 0., W_old;
  int i_extra = 0, doing_extra = 0;
  // W_of_vsq at the current x: func_1d_gnr evaluates it at the start of each
  // iteration (scheme_1d_vsq.h:100) at the point where the previous
  // iteration's convergence test evaluated it (:174); the value is reused.
  double pA, rhoA, uuA;
  double WA = w_of_vsq(D, K, x, g, pA, rhoA, uuA);
  for (int n_iter = 0;; ++n_iter) {
    {
      const double vsq = x;
      const double Wv = WA;
      const double Wsq = Wv * Wv;
      const double W3 = Wv * Wsq;
      const double dWdvsq = ((g * (2. - g) * pA + (g - 1.) * rhoA) /
                             (2. * (g - 1.) * (1. - vsq) * (1. - vsq)));
      const double ft = (Bsq + Wv);
      const double resid = Qtsq - vsq * ft * ft + QdotBsq * (Bsq + 2. * Wv) / Wsq;
      const double jac = -ft * (ft + 2. * dWdvsq * (vsq + QdotBsq / W3));
      const double dx = -resid / jac;
      f = 0.5 * resid * resid;
      df = -2. * f;
      const double xo = x;
      x += dx;
      x = (x >= 1.0) ? (0.5 * (xo + 1.)) : x;
      x = (x < -1.e-10) ? (0.5 * xo) : x;
      x = fabs(x);
      W_old = W;
      W = w_of_vsq(D, K, x, g, pA, rhoA, uuA);
      WA = W;
      errx = (W == 0.) ? fabs(W - W_old) : fabs((W - W_old) / W);
      errx += (x == 0.) ? fabs(x - xo) : fabs((x - xo) / x);
    }
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      break;
  }
  int retval = 0;
  if (!isfinite(f) || !isfinite(df)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  if (retval != 0) return retval * 100 + 1;
  const double vsq = x;
  if ((vsq >= 1.) || (vsq < 0.)) return 4;
  const double Wf = WA, rho0 = rhoA, uu = uuA;  // W_of_vsq(D, K, vsq) of :321
  const double Gamma = 1. / sqrt(1. - vsq);
  if ((rho0 <= 0.) || (uu <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[ENY] = uu;
  prim[ENT] = (g - 1.) * uu * PGD_POW(rho0, -g);
  harm_velocity<MT>(s, Gamma, Wf, prim);
  return 0;
}

// Scheme1D::invert (scheme_1d.h:411-568) with func_1d_orig2 (:376-409).
template <int MT>
PGD int invert_1d(const double U[9], double prim[9], double g, const Geo &geo, const Harm &s) {
  (void)U;
  const double K = prim[ENT];
  double utsq;
  if (!harm_utsq<MT>(prim, geo, utsq)) return 2;
  const double uvsq = 1. + utsq;
  double Gamma = sqrt(uvsq);
  const double Bsq = s.Bsq, QdotBsq = s.QdotBsq, Qtsq = s.Qtsq, D = s.D;
  double rho0 = D / Gamma;
  double p = (K * PGD_POW(rho0, g));
  double uu = (p / (g - 1.));
  double w = rho0 + uu + p;
  double W_last = w * uvsq;
  for (int i = 0; i < 10 && w_too_small(W_last, Bsq, QdotBsq, Qtsq); ++i) W_last *= 10.;
  double x = W_last;
  double f = 1., df = 1., errx = 1.;
  int i_extra = 0, doing_extra = 0;
  const double t1 = D * D;
  const double t2 = QdotBsq * t1;
  const double t3 = t2 * Bsq;
  const double t5 = Bsq * Bsq;
  const double t8 = t1 * Bsq;
  const double t26 = 1 / t1;
  const double rho_num = t1 * (1. + g * K / (g - 1.));
  for (int n_iter = 0;; ++n_iter) {
    const double W = x;
    const double t10 = t1 * W;
    const double t21 = W * W;
    const double rho = rho_num / W;
    const double t23 = rho * rho;
    const double resid =
        (t3 + (2.0 * t2 + ((Qtsq - t5) * t1 + (-2.0 * t8 - t10) * W) * W) * W +
         (t5 + (2.0 * Bsq + W) * W) * t21 * t23) *
        t26 / t21;
    const double jac =
        -2.0 * (t3 + (t2 + (t8 + t10) * t21) * W + (t5 + Bsq * W) * t21 * t23) * t26 / t21 / W;
    const double dx = -resid / jac;
    f = 0.5 * resid * resid;
    df = -2. * f;
    x += dx;
    for (int i = 0; i < 10 && w_too_small(x, Bsq, QdotBsq, Qtsq); ++i) x -= (1. * i) * dx / 10.;
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      break;
  }
  int retval = 0;
  if (!isfinite(f) || !isfinite(df) || !isfinite(x)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  const double W = x;
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  const double vsq = vsq_calc(Bsq, QdotBsq, Qtsq, W);
  if (vsq >= 1.) return 4;
  const double gtmp = sqrt(1. - vsq);
  Gamma = 1. / gtmp;
  rho0 = D * gtmp;
  p = (K * PGD_POW(rho0, g));
  uu = (p / (g - 1.));
  if ((rho0 <= 0.) || (uu <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[ENY] = uu;
  prim[ENT] = (g - 1.) * uu * PGD_POW(rho0, -g);
  harm_velocity<MT>(s, Gamma, W, prim);
  return 0;
}

// SchemeKastaun (scheme_kastaun.h:83-259).
PGD double kastaun_root(double mu, double D, double q, double bsq, double rsq, double rbsq,
                        double g) {
  const double x = 1.0 / (1.0 + mu * bsq);
  const double xsq = x * x;
  const double rbarsq = x * (rsq * x + mu * (x + 1.0) * rbsq);
  const double musq = mu * mu;
  double vsq = musq * rbarsq;
  vsq = kmin(kmax(vsq, 0.0), 1.0 - 1.0e-14);
  const double inv_lorentz = sqrt(1.0 - vsq);
  const double qbar = q - 0.5 * bsq - 0.5 * musq * xsq * (bsq * rsq - rbsq);
  const double eoverD = qbar - mu * rbarsq + 1.0;
  const double rho = D * inv_lorentz;
  double eps = D * eoverD - rho;
  eps = kmax(eps, 1.0e-300);
  const double pressure = (g - 1.0) * eps;
  const double hh = 1.0 + (eps + pressure) / rho;
  const double nu = kmax(hh * inv_lorentz, eoverD + pressure / D);
  return mu - 1.0 / (nu + mu * rbarsq);
}

PGD int invert_kastaun(const double U[9], double prim[9], double g, const Geo &geo) {
  const double gm[6] = {geo.gcov[1][1], geo.gcov[1][2], geo.gcov[1][3],
                        geo.gcov[2][2], geo.gcov[2][3], geo.gcov[3][3]};
  const double det = gm[0] * gm[3] * gm[5] + 2.0 * gm[1] * gm[2] * gm[4] -
                     gm[0] * gm[4] * gm[4] - gm[1] * gm[1] * gm[5] - gm[2] * gm[2] * gm[3];
  if (!(det > 0.0) || !isfinite(det)) return 1;
  const double idet = 1.0 / det;
  const double gi[6] = {(gm[3] * gm[5] - gm[4] * gm[4]) * idet,
                        (gm[2] * gm[4] - gm[1] * gm[5]) * idet,
                        (gm[1] * gm[4] - gm[2] * gm[3]) * idet,
                        (gm[0] * gm[5] - gm[2] * gm[2]) * idet,
                        (gm[1] * gm[2] - gm[0] * gm[4]) * idet,
                        (gm[0] * gm[3] - gm[1] * gm[1]) * idet};
  const double D = U[RHO];
  if (!(D > 0.0) || !isfinite(D)) return 2;
  const double lapse = sqrt(-1.0 / geo.gcon[0][0]);
  const double Qcov[4] = {U[ENY], U[UX1], U[UX2], U[UX3]};
  double Qcon0 = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) Qcon0 += geo.gcon[0][c] * Qcov[c];
  const double Qdotn = Qcon0 * (-lapse);
  const double tau = -Qdotn - D;
  if (!isfinite(tau)) return 3;
  const double Sd[3] = {U[UX1], U[UX2], U[UX3]};
  const double Su[3] = {gi[0] * Sd[0] + gi[1] * Sd[1] + gi[2] * Sd[2],
                        gi[1] * Sd[0] + gi[3] * Sd[1] + gi[4] * Sd[2],
                        gi[2] * Sd[0] + gi[4] * Sd[1] + gi[5] * Sd[2]};
  const double Bu[3] = {U[BX1], U[BX2], U[BX3]};
  const double Bd[3] = {gm[0] * Bu[0] + gm[1] * Bu[1] + gm[2] * Bu[2],
                        gm[1] * Bu[0] + gm[3] * Bu[1] + gm[4] * Bu[2],
                        gm[2] * Bu[0] + gm[4] * Bu[1] + gm[5] * Bu[2]};
  const double Bsq = Bu[0] * Bd[0] + Bu[1] * Bd[1] + Bu[2] * Bd[2];
  const double Ssq = Su[0] * Sd[0] + Su[1] * Sd[1] + Su[2] * Sd[2];
  const double SdotB = Bu[0] * Sd[0] + Bu[1] * Sd[1] + Bu[2] * Sd[2];
  if (!isfinite(Bsq) || !isfinite(Ssq) || !isfinite(SdotB)) return 4;
  const double inv_D = 1.0 / D;
  const double sqrt_D = sqrt(D);
  const double bsq = Bsq * inv_D;
  const double rsq = Ssq * inv_D * inv_D;
  const double rbv = SdotB / (D * sqrt_D);
  const double rbsq = rbv * rbv;
  const double q = tau * inv_D;
  // false_position (:110-165)
  double lower = 0.0, upper = 1.0, mu;
  double f_lower = kastaun_root(lower, D, q, bsq, rsq, rbsq, g);
  double f_upper = kastaun_root(upper, D, q, bsq, rsq, rbsq, g);
  int rs = -1;
  if (!isfinite(f_lower) || !isfinite(f_upper)) rs = 1;
  else if (fabs(f_lower) <= NEWT_TOL) { mu = lower; rs = 0; }
  else if (fabs(f_upper) <= NEWT_TOL) { mu = upper; rs = 0; }
  else if (f_lower * f_upper > 0.0) rs = 2;
  if (rs < 0) {
    int side = 0;
    mu = lower;
    rs = 4;
    for (int iter = 0; iter < MAX_NEWT_ITER; ++iter) {
      const double old_mu = mu;
      mu = (f_upper * lower - f_lower * upper) / (f_upper - f_lower);
      const double f_mu = kastaun_root(mu, D, q, bsq, rsq, rbsq, g);
      if (!isfinite(mu) || !isfinite(f_mu)) { rs = 3; break; }
      if (fabs((mu - old_mu) / (mu + 1.0e-300)) <= NEWT_TOL) { rs = 0; break; }
      if (f_mu * f_lower >= 0.0) {
        if (side == 1) {
          const double w = 1.0 - f_mu / f_lower;
          f_upper = (w > 0.0) ? f_upper * w : 0.5 * f_upper;
        }
        lower = mu;
        f_lower = f_mu;
        side = 1;
      } else {
        if (side == -1) {
          const double w = 1.0 - f_mu / f_upper;
          f_lower = (w > 0.0) ? f_lower * w : 0.5 * f_lower;
        }
        upper = mu;
        f_upper = f_mu;
        side = -1;
      }
    }
  }
  if (rs != 0) return 100 + rs;
  const double x = 1.0 / (1.0 + mu * bsq);
  const double rbarsq = x * (rsq * x + mu * (x + 1.0) * rbsq);
  const double vsq = mu * mu * rbarsq;
  if (!(vsq >= 0.0) || vsq >= 1.0 || !isfinite(vsq)) return 5;
  const double lorentz = 1.0 / sqrt(1.0 - vsq);
  const double rho = D / lorentz;
  const double qbar = q - 0.5 * bsq - 0.5 * mu * mu * x * x * (bsq * rsq - rbsq);
  const double eoverD = qbar - mu * rbarsq + 1.0;
  const double eps = D * eoverD - rho;
  if (!(rho > 0.0) || !(eps > 0.0) || !isfinite(eps)) return 6;
  const double Wmu_x = lorentz * mu * x;
  prim[RHO] = rho;
  prim[ENY] = eps;
  prim[ENT] = (g - 1.) * eps * PGD_POW(rho, -g);
#pragma unroll
  for (int d = 0; d < 3; ++d) prim[UX1 + d] = Wmu_x * (Su[d] * inv_D + rbv * mu * (Bu[d] / sqrt_D));
  return 0;
}

// ---------------------------------------------------------------------------
// physics/heating_model.h:53-179
// ---------------------------------------------------------------------------
struct HeatParams {
  int model;
  double gamma, gamma_p, gamma_e, fel_constant, ratio_min, ratio_max;
  int limit_kel, suppress_highb_heat, enforce_positive_dissipation;
};

// The proton and electron temperatures (tpr, tel) are formed only by the
// models that read them: the same values, without the electron power in the
// constant, Werner and Rowan models.
PGD double heating_fraction(const HeatParams &p, double rho, double energy, double bsq,
                            double adv_electron) {
  const auto tpr = [&] { return (p.gamma_p - 1.0) * energy / rho; };
  const auto tel = [&] { return adv_electron * PGD_POW(rho, p.gamma_e - 1.0); };
  switch (p.model) {
    case 0:
      return p.fel_constant;
    case 1: {
      const double trat = tpr() / tel();
      const double pres = rho * tpr();
      const double beta = kmin(2.0 * pres / bsq, 1.0e20);
      const double log_trat = PGD_LOG(trat) / PGD_LOG(10.0);
      const double mbeta = 2.0 - 0.2 * log_trat;
      const double c2 = (trat <= 1.0) ? 1.6 / trat : 1.2 / trat;
      const double c3 = (trat <= 1.0) ? 18.0 + 5.0 * log_trat : 18.0;
      const double bp = PGD_POW(beta, mbeta);
      const double qrat = 0.92 * (c2 * c2 + bp) / (c3 * c3 + bp) * PGD_EXP(-1.0 / beta) *
                          sqrt(1.67262171e-24 / 9.1093826e-28 * trat);
      return 1.0 / (1.0 + qrat);
    }
    case 2: {
      const double trat = tpr() / tel();
      const double pres = rho * tpr();
      const double beta = kmin(2.0 * pres / bsq, 1.0e20);
      const double qi_qe = 35.0 / (1.0 + PGD_POW(beta / 15.0, -1.4) * PGD_EXP(-0.1 / trat));
      return 1.0 / (1.0 + qi_qe);
    }
    case 3: {
      const double sigma = bsq / rho;
      return 0.25 * (1.0 + sqrt((sigma / 5.0) / (2.0 + sigma / 5.0)));
    }
    case 4: {
      const double pres = (p.gamma_p - 1.0) * energy;
      const double pg = (p.gamma - 1.0) * energy;
      const double beta = 2.0 * pres / bsq;
      const double sigma = bsq / (rho + energy + pg);
      const double betamax = 0.25 / sigma;
      return 0.5 * PGD_EXP(-PGD_POW(1.0 - beta / betamax, 3.3) / (1.0 + 1.2 * PGD_POW(sigma, 0.7)));
    }
    case 5: {
      const double trat_inv = tel() / tpr();
      const double qe_qi = 0.33 * sqrt(trat_inv);
      return 1.0 / (1.0 + 1.0 / qe_qi);
    }
  }
  return p.fel_constant;
}

PGD double heating_apply(const HeatParams &p, double rho, double energy, double bsq,
                         double adv_total, double rec_total, double adv_electron) {
  const double fel = heating_fraction(p, rho, energy, bsq, adv_electron);
  const double rpow = PGD_POW(rho, p.gamma - p.gamma_e);
  double diss = (p.gamma_e - 1.0) / (p.gamma - 1.0) * rpow * (rec_total - adv_total);
  if (p.suppress_highb_heat && (bsq / rho > 1.0)) diss = 0.0;
  if (p.enforce_positive_dissipation) diss = kmax(diss, 0.0);
  const double kel = adv_electron + fel * diss;
  if (!p.limit_kel && p.model == 0) return kel;
  const double kel_max = adv_total * rpow /
                         (p.ratio_min * (p.gamma - 1.0) / (p.gamma_p - 1.0) +
                          (p.gamma - 1.0) / (p.gamma_e - 1.0));
  const double kel_min = adv_total * rpow /
                         (p.ratio_max * (p.gamma - 1.0) / (p.gamma_p - 1.0) +
                          (p.gamma - 1.0) / (p.gamma_e - 1.0));
  return kmax(kel_min, kmin(kel, kel_max));
}

PGD double clamp_by_ratio(double rmin, double rmax, double total, double electron) {
  const double lo = total / (1.0 + rmax);
  const double hi = total / (1.0 + rmin);
  const double b = kmax(0.0, kmin(electron, total));
  return kmax(lo, kmin(b, hi));
}

// ---------------------------------------------------------------------------
// Generic-precision forms of the face and heating physics, in the operation
// order of the FP64 forms above. The mixed-precision engine instantiates them
// with float for reconstruction, Riemann fluxes and electron heating.
// ---------------------------------------------------------------------------
PGD float tmin(float a, float b) { return fminf(a, b); }
PGD float tmax(float a, float b) { return fmaxf(a, b); }
PGD double tmin(double a, double b) { return fmin(a, b); }
PGD double tmax(double a, double b) { return fmax(a, b); }
PGD float tpow(float a, float b) { return powf(a, b); }
PGD double tpow(double a, double b) { return pow(a, b); }
PGD float texp(float a) { return expf(a); }
PGD double texp(double a) { return exp(a); }
PGD float tlog(float a) { return logf(a); }
PGD double tlog(double a) { return log(a); }

template <typename T>
struct GeoT {
  T gcov[4][4];
  T gcon[4][4];
  T gdet, sg, alpha;
};

template <typename T>
struct StateT {
  T ucon[4], ucov[4], bcon[4], bcov[4], bsq;
};

// Rounds an FP64 metric to T, keeping its structural zeros exact.
template <int MT, typename T>
PGD void geo_cast(const Geo &g, GeoT<T> &o) {
  constexpr Pattern PT = metric_pattern(MT);
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      o.gcov[r][c] = PT.nz[r][c] ? (T)g.gcov[r][c] : T(0);
      o.gcon[r][c] = PT.nz[r][c] ? (T)g.gcon[r][c] : T(0);
    }
  o.gdet = (T)g.gdet;
  o.sg = (T)g.sg;
  o.alpha = (T)g.alpha;
}

// state_calculation.h:19-69
template <int MT, typename T>
PGD void calc_state_t(const T P[NPRIM], const GeoT<T> &g, StateT<T> &s) {
  constexpr Pattern PT = metric_pattern(MT);
  const T alpha = g.alpha;
  const T u[3] = {P[UX1], P[UX2], P[UX3]};
  T sq = T(0);
#pragma unroll
  for (int i = 1; i < 4; ++i)
#pragma unroll
    for (int j = 1; j < 4; ++j)
      if (PT.nz[i][j]) sq = sq + u[i - 1] * g.gcov[i][j] * u[j - 1];
  const T lor = sqrt(T(1) + sq);
  s.ucon[0] = lor / alpha;
#pragma unroll
  for (int i = 1; i < 4; ++i)
    s.ucon[i] = PT.nz[0][i] ? u[i - 1] - s.ucon[0] * g.gcon[0][i] * alpha * alpha : u[i - 1];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    T v = T(0);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (PT.nz[r][c]) v += g.gcov[r][c] * s.ucon[c];
    s.ucov[r] = v;
  }
  s.bcon[0] = P[BX1] * s.ucov[1] + P[BX2] * s.ucov[2] + P[BX3] * s.ucov[3];
  const T iu0 = T(1) / s.ucon[0];
  s.bcon[1] = (P[BX1] + s.bcon[0] * s.ucon[1]) * iu0;
  s.bcon[2] = (P[BX2] + s.bcon[0] * s.ucon[2]) * iu0;
  s.bcon[3] = (P[BX3] + s.bcon[0] * s.ucon[3]) * iu0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    T v = T(0);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (PT.nz[r][c]) v += g.gcov[r][c] * s.bcon[c];
    s.bcov[r] = v;
  }
  s.bsq = s.bcon[0] * s.bcov[0] + s.bcon[1] * s.bcov[1] + s.bcon[2] * s.bcov[2] +
          s.bcon[3] * s.bcov[3];
}

// fast_magnetosonic_speed.h:11-81
template <typename T>
PGD void fast_speed_t(T gam, const T P[NPRIM], const GeoT<T> &g, const StateT<T> &s, int dir,
                      T &vmax, T &vmin) {
  const T hh = P[RHO] + gam * P[ENY];
  const T h_tot = s.bsq + hh;
  const T va_sq = s.bsq / h_tot;
  const T cs_sq = gam * (gam - T(1)) * P[ENY] / hh;
  T cf_sq = cs_sq + va_sq - cs_sq * va_sq;
  if (cf_sq < T(0)) cf_sq = T(1e-10);
  if (cf_sq > T(1)) cf_sq = T(1);
  const T n_sq = g.gcon[dir][dir];
  const T t_sq = g.gcon[0][0];
  const T n_dot_u = s.ucon[dir];
  const T t_dot_u = s.ucon[0];
  const T n_dot_t = g.gcon[0][dir];
  const T nu2 = n_dot_u * n_dot_u;
  const T tu2 = t_dot_u * t_dot_u;
  const T nutu = n_dot_u * t_dot_u;
  const T A = tu2 - (t_sq + tu2) * cf_sq;
  const T B = T(2) * (nutu - (n_dot_t + nutu) * cf_sq);
  const T C = nu2 - (n_sq + nu2) * cf_sq;
  T disc = B * B - T(4) * A * C;
  if (disc < T(0)) disc = T(0);
  disc = sqrt(disc);
  const T i2a = T(1) / (T(2) * A);
  const T vp = -(-B + disc) * i2a;
  const T vm = -(-B - disc) * i2a;
  vmax = vp > vm ? vp : vm;
  vmin = vp > vm ? vm : vp;
}

// interpolater_mc.h:16-48
template <typename T>
PGD void mc_t(T qm1, T q, T qp1, T &ql_ip1, T &qr_i) {
  const T a = T(2) * (q - qm1), b = T(0.5) * (qp1 - qm1), c = T(2) * (qp1 - q);
  T slope = T(0);
  if (a > T(0) && b > T(0) && c > T(0)) slope = tmin(tmin(a, b), c);
  if (a < T(0) && b < T(0) && c < T(0)) slope = tmax(tmax(a, b), c);
  ql_ip1 = q + T(0.5) * slope;
  qr_i = q - T(0.5) * slope;
}

// interpolater_ppm4.h:29-67
template <typename T>
PGD void ppm4_t(T qm2, T qm1, T q, T qp1, T qp2, T &ql_ip1, T &qr_i) {
  const T c12 = T(1) / T(12);
  T qlv = (T(7) * (q + qm1) - (qm2 + qp1)) * c12;
  T qrv = (T(7) * (q + qp1) - (qm1 + qp2)) * c12;
  qlv = tmax(qlv, tmin(q, qm1));
  qlv = tmin(qlv, tmax(q, qm1));
  qrv = tmax(qrv, tmin(q, qp1));
  qrv = tmin(qrv, tmax(q, qp1));
  const T qc = qrv - q;
  const T qd = qlv - q;
  if ((qc * qd) >= T(0)) {
    qlv = q;
    qrv = q;
  } else {
    if (fabs(qc) >= T(2) * fabs(qd)) qrv = q - T(2) * qd;
    if (fabs(qd) >= T(2) * fabs(qc)) qlv = q - T(2) * qc;
  }
  ql_ip1 = qrv;
  qr_i = qlv;
}

// heating_model.h:53-179
template <typename T>
PGD T heating_fraction_t(const HeatParams &p, T rho, T energy, T bsq, T adv_electron) {
  const auto tpr = [&] { return (T(p.gamma_p) - T(1)) * energy / rho; };
  const auto tel = [&] { return adv_electron * tpow(rho, T(p.gamma_e) - T(1)); };
  switch (p.model) {
    case 0:
      return T(p.fel_constant);
    case 1: {
      const T trat = tpr() / tel();
      const T beta = tmin(T(2) * rho * tpr() / bsq, T(1.0e20));
      const T log_trat = tlog(trat) / tlog(T(10));
      const T mbeta = T(2) - T(0.2) * log_trat;
      const T c2 = (trat <= T(1)) ? T(1.6) / trat : T(1.2) / trat;
      const T c3 = (trat <= T(1)) ? T(18) + T(5) * log_trat : T(18);
      const T bp = tpow(beta, mbeta);
      const T qrat = T(0.92) * (c2 * c2 + bp) / (c3 * c3 + bp) * texp(T(-1) / beta) *
                     sqrt(T(1.67262171e-24 / 9.1093826e-28) * trat);
      return T(1) / (T(1) + qrat);
    }
    case 2: {
      const T trat = tpr() / tel();
      const T beta = tmin(T(2) * rho * tpr() / bsq, T(1.0e20));
      const T qi_qe = T(35) / (T(1) + tpow(beta / T(15), T(-1.4)) * texp(T(-0.1) / trat));
      return T(1) / (T(1) + qi_qe);
    }
    case 3: {
      const T sigma = bsq / rho;
      return T(0.25) * (T(1) + sqrt((sigma / T(5)) / (T(2) + sigma / T(5))));
    }
    case 4: {
      const T pres = (T(p.gamma_p) - T(1)) * energy;
      const T pg = (T(p.gamma) - T(1)) * energy;
      const T beta = T(2) * pres / bsq;
      const T sigma = bsq / (rho + energy + pg);
      const T betamax = T(0.25) / sigma;
      return T(0.5) * texp(-tpow(T(1) - beta / betamax, T(3.3)) /
                           (T(1) + T(1.2) * tpow(sigma, T(0.7))));
    }
    case 5: {
      const T qe_qi = T(0.33) * sqrt(tel() / tpr());
      return T(1) / (T(1) + T(1) / qe_qi);
    }
  }
  return T(p.fel_constant);
}

template <typename T>
PGD T heating_apply_t(const HeatParams &p, T rho, T energy, T bsq, T adv_total, T rec_total,
                      T adv_electron) {
  const T fel = heating_fraction_t<T>(p, rho, energy, bsq, adv_electron);
  const T gam = T(p.gamma), ge = T(p.gamma_e), gp = T(p.gamma_p);
  const T rpow = tpow(rho, gam - ge);
  T diss = (ge - T(1)) / (gam - T(1)) * rpow * (rec_total - adv_total);
  if (p.suppress_highb_heat && (bsq / rho > T(1))) diss = T(0);
  if (p.enforce_positive_dissipation) diss = diss < T(0) ? T(0) : diss;
  const T kel = adv_electron + fel * diss;
  if (!p.limit_kel && p.model == 0) return kel;
  const T kel_max = adv_total * rpow /
                    (T(p.ratio_min) * (gam - T(1)) / (gp - T(1)) + (gam - T(1)) / (ge - T(1)));
  const T kel_min = adv_total * rpow /
                    (T(p.ratio_max) * (gam - T(1)) / (gp - T(1)) + (gam - T(1)) / (ge - T(1)));
  const T lo = kel < kel_max ? kel : kel_max;
  return kel_min < lo ? lo : kel_min;
}

}  // namespace pgd
#endif  // PANGU_DEVICE_CUH
