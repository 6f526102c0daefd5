// oracle.cc -- CPU restatement of PANGU's per-RK-stage task path.
//
// TEST INFRASTRUCTURE ONLY. The tests, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py call it as the checker; the engine never links
// or calls it.
//
// Each task restates the loop ranges and arithmetic of the reference task
// (file:line cited per function); the per-cell mathematics is in
// oracle_cell.h. The behaviour that the reference leaves to Parthenon (which
// is not vendored) is fixed here as explicit choices, shared with the
// engine:
//   * rk2: beta = {1.0, 0.5} indexed by stage % 2; stage names
//     {"base", "1", "base"}; mc_init = "base" (ideal_grmhd.cc:29-31,56).
//   * FluxDivergence in the area/volume form of a uniform Cartesian
//     coordinate object; UpdateIndependentData out = in + (beta dt) dudt on
//     the interior.
//   * Ghost exchange at send time: right after the update, periodic and
//     block-to-block ghosts of prim and flag receive the neighbour's interior
//     values as they are then (post-update, pre-recovery).
//   * Physical BCs (outflow / reflecting) after FixRecovery, in face order
//     ix1, ox1, ix2, ox2, ix3, ox3, each over the full transverse range;
//     reflecting negates the normal component of weighted_velocity and
//     magnetic_field (Metadata::Vector, package_registration.cc:113-128).
//   * FixRecovery reads a snapshot of prim and flag taken before it writes
//     (deterministic; the reference reads and writes in place, which is
//     order dependent for adjacent failed cells).
//   * Coordinates: Xc(i) = (xmin_block - ng dx) + (i + 0.5) dx,
//     Xf(i) = (xmin_block - ng dx) + i dx.
// Built -O2 -ffp-contract=off (oracle/build.py), OpenMP over cells.
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle_cell.h"
#include "pangu_b200.h"

using namespace orc;

namespace {

struct Geom {
  int N1, N2, N3;          // entire extents
  int is, ie, js, je, ks, ke;
  int o1, o2, o3;          // 1 if the direction is active
  int ndim;
  int NF, NB;
  int ng;
  double dx[3];
  std::vector<double> origin;  // [NB][3]: xmin_block - ng*dx (or xmin for inactive)
  // pack index of each logical slot (-1 if absent)
  int pidx[NPRIM];
};

Geom make_geom(const pangu_params &p, const pangu_mesh &m) {
  Geom g;
  g.ng = m.ng;
  g.o1 = m.nx1 > 1;
  g.o2 = m.nx2 > 1;
  g.o3 = m.nx3 > 1;
  g.ndim = 1 + g.o2 + g.o3;
  g.N1 = m.nx1 + 2 * m.ng * g.o1;
  g.N2 = m.nx2 + 2 * m.ng * g.o2;
  g.N3 = m.nx3 + 2 * m.ng * g.o3;
  g.is = m.ng * g.o1; g.ie = g.is + m.nx1 - 1;
  g.js = m.ng * g.o2; g.je = g.js + m.nx2 - 1;
  g.ks = m.ng * g.o3; g.ke = g.ks + m.nx3 - 1;
  g.NB = m.nbx1 * m.nbx2 * m.nbx3;
  g.dx[0] = (m.x1max - m.x1min) / (double)(m.nbx1 * m.nx1);
  g.dx[1] = (m.x2max - m.x2min) / (double)(m.nbx2 * m.nx2);
  g.dx[2] = (m.x3max - m.x3min) / (double)(m.nbx3 * m.nx3);
  g.origin.resize(3 * g.NB);
  const double mins[3] = {m.x1min, m.x2min, m.x3min};
  const int nx[3] = {m.nx1, m.nx2, m.nx3};
  const int act[3] = {g.o1, g.o2, g.o3};
  for (int b = 0; b < g.NB; ++b) {
    const int bl[3] = {b % m.nbx1, (b / m.nbx1) % m.nbx2, b / (m.nbx1 * m.nbx2)};
    for (int d = 0; d < 3; ++d) {
      const double bxmin = mins[d] + (double)(bl[d] * nx[d]) * g.dx[d];
      g.origin[3 * b + d] = bxmin - (double)(m.ng * act[d]) * g.dx[d];
    }
  }
  int n = 0;
  for (int s = 0; s < NPRIM; ++s) g.pidx[s] = -1;
  g.pidx[RHO] = n++; g.pidx[ENY] = n++;
  g.pidx[UX1] = n++; g.pidx[UX2] = n++; g.pidx[UX3] = n++;
  if (p.enable_B) { g.pidx[BX1] = n++; g.pidx[BX2] = n++; g.pidx[BX3] = n++; }
  g.pidx[ENT] = n++;
  if (p.enable_heating) g.pidx[KEL] = n++;
  g.NF = n;
  return g;
}

inline size_t at(const Geom &g, int b, int v, int k, int j, int i, int nv) {
  return ((((size_t)b * nv + v) * g.N3 + k) * g.N2 + j) * g.N1 + i;
}
inline size_t cell(const Geom &g, int b, int k, int j, int i) {
  return (((size_t)b * g.N3 + k) * g.N2 + j) * g.N1 + i;
}
inline double Xc(const Geom &g, int b, int d, int idx) {
  return g.origin[3 * b + d] + ((double)idx + 0.5) * g.dx[d];
}
inline double Xf(const Geom &g, int b, int d, int idx) {
  return g.origin[3 * b + d] + (double)idx * g.dx[d];
}

// Loads the prims of one cell into a zero-filled NPRIM array (pcarr = {0}).
inline void load_prim(const Geom &g, const double *P, int b, int k, int j,
                      int i, Real out[NPRIM]) {
  for (int s = 0; s < NPRIM; ++s)
    out[s] = (g.pidx[s] >= 0) ? P[at(g, b, g.pidx[s], k, j, i, g.NF)] : 0.0;
}

struct Ctx {
  pangu_params p;
  pangu_mesh m;
  Geom g;
  uint64_t cnt[PANGU_NCOUNTERS];
};

// ----------------------------------------------------------------------------
// FixPrimitive (primitive_fixer.cc:15-169), entire domain.
// ----------------------------------------------------------------------------
void fix_primitive(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
  const double gam = p.adiabatic_index;
  const double a2 = p.a * p.a;
  const double e_excise = p.pexcise / (gam - 1.0);
  const double umax2 = p.lorentz_max * p.lorentz_max - 1.0;
  double *P = md.prim;
  uint64_t n_rho = 0, n_eng = 0, n_lor = 0;
#pragma omp parallel for collapse(3) reduction(+ : n_rho, n_eng, n_lor)
  for (int b = 0; b < g.NB; ++b)
    for (int k = 0; k < g.N3; ++k)
      for (int j = 0; j < g.N2; ++j)
        for (int i = 0; i < g.N1; ++i) {
          constexpr Real small = 1.0e-20;
          const Real sigma_max_safe = kmax(p.sigma_max, small);
          const Real rho_before = kmax(P[at(g, b, g.pidx[RHO], k, j, i, g.NF)], small);
          const Real x = Xc(g, b, 0, i), y = Xc(g, b, 1, j), z = Xc(g, b, 2, k);
          const Real xc[4] = {0.0, x, y, z};
          Real r = 1.0;
          if (p.metric_type == MKS) {
            r = std::exp(x);
          } else if (p.metric_type == CKS) {
            const Real rad2 = x * x + y * y + z * z;
            const Real sa = (rad2 - a2) * (rad2 - a2) + 4.0 * a2 * z * z;
            r = std::sqrt(0.5 * (rad2 - a2 + std::sqrt(sa)));
          }
          Real rho_floor = p.density_floor * pgm::pow(std::fmax(r, 1.0), p.density_floor_pow);
          const Real eng_floor = p.energy_floor * pgm::pow(std::fmax(r, 1.0), p.energy_floor_pow);
          Real gcov[4][4], gcon[4][4], gdet;
          metric_at(p.metric_type, xc, p.a, p.h, gcov, gcon, gdet);
          Real pc[NPRIM];
          load_prim(g, P, b, k, j, i, pc);
          const Real rho = pc[RHO];
          const Real ug = pc[ENY];
          State st;
          calc_state(pc, gcov, gcon, st);
          if (rho_floor < ug / sigma_max_safe) rho_floor = ug / sigma_max_safe;
          const Real sigma = st.bsq / rho;
          if (sigma > p.sigma_max) rho_floor = st.bsq / sigma_max_safe;
          double &pr = P[at(g, b, g.pidx[RHO], k, j, i, g.NF)];
          double &pu = P[at(g, b, g.pidx[ENY], k, j, i, g.NF)];
          if (pr < rho_floor) { pr = rho_floor; ++n_rho; }
          if (pu < eng_floor) { pu = eng_floor; ++n_eng; }
          double &u1 = P[at(g, b, g.pidx[UX1], k, j, i, g.NF)];
          double &u2 = P[at(g, b, g.pidx[UX2], k, j, i, g.NF)];
          double &u3 = P[at(g, b, g.pidx[UX3], k, j, i, g.NF)];
          const Real uvsq = gcov[1][1] * u1 * u1 + gcov[2][2] * u2 * u2 +
                            gcov[3][3] * u3 * u3 +
                            2.0 * (gcov[1][2] * u1 * u2 + gcov[1][3] * u1 * u3 +
                                   gcov[2][3] * u2 * u3);
          if (umax2 > 0.0 && uvsq > umax2) {
            const Real f = std::sqrt(umax2 / kmax(uvsq, small));
            u1 *= f; u2 *= f; u3 *= f;
            ++n_lor;
          }
          const Real rho_after = kmax(pr, small);
          double *pk = p.enable_heating ? &P[at(g, b, g.pidx[KEL], k, j, i, g.NF)] : nullptr;
          if (p.enable_heating && rho_after != rho_before)
            *pk *= pgm::pow(rho_after / rho_before, -gam);
          double &pe = P[at(g, b, g.pidx[ENT], k, j, i, g.NF)];
          pe = (gam - 1.0) * pu * pgm::pow(pr, -gam);
          if (p.enable_heating) *pk = clamp_by_ratio(p.ratio_min, p.ratio_max, pe, *pk);
          if (p.metric_type == CKS && r < p.r_excise) {
            pr = p.dexcise;
            pu = e_excise;
            u1 = 0.0; u2 = 0.0; u3 = 0.0;
            pe = (gam - 1.0) * e_excise * pgm::pow(p.dexcise, -gam);
            if (p.enable_heating) *pk = e_excise;
          }
        }
  c.cnt[PANGU_CNT_RHO_FLOOR] += n_rho;
  c.cnt[PANGU_CNT_ENG_FLOOR] += n_eng;
  c.cnt[PANGU_CNT_LORENTZ_CAP] += n_lor;
}

// ----------------------------------------------------------------------------
// CalculateConservative (conservative.cc:15-110), interior.
// ----------------------------------------------------------------------------
void calc_conservative(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          const Real xc[4] = {0.0, Xc(g, b, 0, i), Xc(g, b, 1, j), Xc(g, b, 2, k)};
          Real gcov[4][4], gcon[4][4], gdet;
          metric_at(p.metric_type, xc, p.a, p.h, gcov, gcon, gdet);
          Real pc[NPRIM];
          load_prim(g, md.prim, b, k, j, i, pc);
          Real cc[NPRIM];
          contravariant_flux(p.adiabatic_index, pc, gcov, gcon, gdet, 0, cc);
          for (int s = 0; s < NPRIM; ++s)
            if (g.pidx[s] >= 0) md.cons[at(g, b, g.pidx[s], k, j, i, g.NF)] = cc[s];
        }
}

// ----------------------------------------------------------------------------
// CalculateLAXF / CalculateHLL (laxf.cc:19-396, hll.cc:19-401).
// ----------------------------------------------------------------------------
void flux_dir(Ctx &c, pangu_pack &md, int dir) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
  const bool use_mc = p.limiter == PANGU_LIMITER_MC;
  const bool hll = p.riemann_solver == PANGU_RIEMANN_HLL;
  double *F = dir == 1 ? md.flux1 : (dir == 2 ? md.flux2 : md.flux3);
  // loop ranges (laxf.cc:79-82, 185-188, 291-294; hll.cc:293-296)
  int k0 = g.ks - g.o3, k1 = g.ke + g.o3;
  int j0 = g.js - g.o2, j1 = g.je + g.o2;
  int i0 = g.is - g.o1, i1 = g.ie + g.o1;
  if (dir == 1) { i0 = g.is; i1 = g.ie + 1; }
  if (dir == 2) { j0 = g.js; j1 = g.je + 1; }
  if (dir == 3) {
    k0 = g.ks; k1 = g.ke + 1;
    if (hll) { j0 = g.js; j1 = g.je; i0 = g.is; i1 = g.ie; }
  }
  const int di = dir == 1, dj = dir == 2, dk = dir == 3;
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = k0; k <= k1; ++k)
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
          Real PL[NPRIM] = {0}, PR[NPRIM] = {0};
          for (int s = 0; s < NPRIM; ++s) {
            if (g.pidx[s] < 0) continue;
            const int v = g.pidx[s];
            Real q[6];  // q[n] = value at offset n-3 along dir
            for (int n = 0; n < 6; ++n) {
              const int o = n - 3;
              const int kk = k + o * dk, jj = j + o * dj, ii = i + o * di;
              // MC never reads the outermost two values (interpolater_mc.h:39-47)
              if (use_mc && (n == 0 || n == 5)) { q[n] = 0.0; continue; }
              q[n] = md.prim[at(g, b, v, kk, jj, ii, g.NF)];
            }
            Real ql_i, qr_im1, ql_ip1, qr_i;
            if (use_mc) {
              mc(q[0], q[1], q[2], q[3], q[4], ql_i, qr_im1);
              mc(q[1], q[2], q[3], q[4], q[5], ql_ip1, qr_i);
            } else {
              ppm4(q[0], q[1], q[2], q[3], q[4], ql_i, qr_im1);
              ppm4(q[1], q[2], q[3], q[4], q[5], ql_ip1, qr_i);
            }
            PL[s] = ql_i;
            PR[s] = qr_i;
          }
          Real xf[4] = {0.0, Xc(g, b, 0, i), Xc(g, b, 1, j), Xc(g, b, 2, k)};
          xf[dir] = Xf(g, b, dir - 1, dir == 1 ? i : (dir == 2 ? j : k));
          Real gcov[4][4], gcon[4][4], gdet;
          code_metric(p.metric_type, xf, p.a, p.h, gcov);
          if (!invert(gcov, gcon)) {
            // Singular code metric (theta = 0 exactly on a polar face): the
            // reference reads an unwritten inverse here (tensor_algebra.h:91-93
            // returns before filling it). Defined as zero flux, zero speed.
            md.alfven[at(g, b, dir - 1, k, j, i, 3)] = 0.0;
            for (int s = 0; s < NPRIM; ++s)
              if (g.pidx[s] >= 0) F[at(g, b, g.pidx[s], k, j, i, g.NF)] = 0.0;
            continue;
          }
          gdet = determinant(gcov);
          Real vmaxL, vminL, vmaxR, vminR;
          const Real gam = p.adiabatic_index;
          fast_speed(gam, PL, gcov, gcon, dir, vmaxL, vminL);
          fast_speed(gam, PR, gcov, gcon, dir, vmaxR, vminR);
          const Real cmax = std::fabs(kmax(kmax(0., vmaxL), vmaxR));
          const Real cmin = std::fabs(kmax(kmax(0., -vminL), -vminR));
          const Real cms = kmax(cmax, cmin);
          md.alfven[at(g, b, dir - 1, k, j, i, 3)] = cms;
          Real UL[NPRIM], UR[NPRIM], FL[NPRIM], FR[NPRIM];
          contravariant_flux(gam, PL, gcov, gcon, gdet, 0, UL);
          contravariant_flux(gam, PR, gcov, gcon, gdet, 0, UR);
          contravariant_flux(gam, PL, gcov, gcon, gdet, dir, FL);
          contravariant_flux(gam, PR, gcov, gcon, gdet, dir, FR);
          for (int s = 0; s < NPRIM; ++s) {
            if (g.pidx[s] < 0) continue;
            Real fx;
            if (hll)
              fx = (cmax * FL[s] + cmin * FR[s] - cmax * cmin * (UR[s] - UL[s])) /
                   (cmax + cmin + 1e-20);
            else
              fx = 0.5 * (FL[s] + FR[s] - cms * (UR[s] - UL[s]));
            F[at(g, b, g.pidx[s], k, j, i, g.NF)] = fx;
          }
        }
}

void calc_fluxes(Ctx &c, pangu_pack &md) {
  flux_dir(c, md, 1);
  if (c.g.ndim >= 2) flux_dir(c, md, 2);
  if (c.g.ndim == 3) flux_dir(c, md, 3);
}

// ----------------------------------------------------------------------------
// ConstraintedTransport (constrained_transport.cc:13-130).
// Flux component indices BX1..BX3 = 5..7 (enable_B layout).
// ----------------------------------------------------------------------------
void constrained_transport(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const int o1 = g.N1 > 1, o2 = g.N2 > 1, o3 = g.N3 > 1;
  const int E1 = o2 && o3, E2 = o3 && o1, E3 = o1 && o2;
  double *F1 = md.flux1, *F2 = md.flux2, *F3 = md.flux3, *E = md.efield;
  auto f = [&](double *Fa, int v, int b, int k, int j, int i) -> double & {
    return Fa[at(g, b, v, k, j, i, g.NF)];
  };
  auto e = [&](int d, int b, int k, int j, int i) -> double & {
    return E[at(g, b, d, k, j, i, 3)];
  };
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke + o3; ++k)
      for (int j = g.js; j <= g.je + o2; ++j)
        for (int i = g.is; i <= g.ie + o1; ++i) {
          e(0, b, k, j, i) = 0.0;
          e(1, b, k, j, i) = 0.0;
          e(2, b, k, j, i) = 0.0;
          if (E1)
            e(0, b, k, j, i) = 0.25 * ((f(F2, BX3, b, k, j, i) + f(F2, BX3, b, k - 1, j, i)) -
                                       (f(F3, BX2, b, k, j, i) + f(F3, BX2, b, k, j - 1, i)));
          if (E2)
            e(1, b, k, j, i) = 0.25 * ((f(F3, BX1, b, k, j, i) + f(F3, BX1, b, k, j, i - 1)) -
                                       (f(F1, BX3, b, k, j, i) + f(F1, BX3, b, k - 1, j, i)));
          if (E3)
            e(2, b, k, j, i) = 0.25 * ((f(F1, BX2, b, k, j, i) + f(F1, BX2, b, k, j - 1, i)) -
                                       (f(F2, BX1, b, k, j, i) + f(F2, BX1, b, k, j, i - 1)));
        }
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie + o1; ++i) {
          if (o1) f(F1, BX1, b, k, j, i) = 0;
          if (E2) f(F1, BX3, b, k, j, i) = -0.5 * (e(1, b, k, j, i) + e(1, b, k + 1, j, i));
          if (E3) f(F1, BX2, b, k, j, i) = 0.5 * (e(2, b, k, j, i) + e(2, b, k, j + 1, i));
        }
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je + o2; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          if (E1) f(F2, BX3, b, k, j, i) = 0.5 * (e(0, b, k, j, i) + e(0, b, k + 1, j, i));
          if (o2) f(F2, BX2, b, k, j, i) = 0.;
          if (E3) f(F2, BX1, b, k, j, i) = -0.5 * (e(2, b, k, j, i) + e(2, b, k, j, i + 1));
        }
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke + o3; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          if (E1) f(F3, BX2, b, k, j, i) = -0.5 * (e(0, b, k, j, i) + e(0, b, k, j + 1, i));
          if (E2) f(F3, BX1, b, k, j, i) = 0.5 * (e(1, b, k, j, i) + e(1, b, k, j, i + 1));
          if (o3) f(F3, BX3, b, k, j, i) = 0;
        }
}

// ----------------------------------------------------------------------------
// FluxDivergence + UpdateIndependentData (Parthenon, ideal_grmhd.cc:73-76).
// ----------------------------------------------------------------------------
void flux_div_update(Ctx &c, const pangu_pack &mc_init, const pangu_pack &mc0,
                     pangu_pack &mc1, double bdt) {
  const Geom &g = c.g;
  const double A1 = g.dx[1] * g.dx[2], A2 = g.dx[0] * g.dx[2],
               A3 = g.dx[0] * g.dx[1];
  const double V = g.dx[0] * g.dx[1] * g.dx[2];
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int v = 0; v < g.NF; ++v)
      for (int k = g.ks; k <= g.ke; ++k)
        for (int j = g.js; j <= g.je; ++j)
          for (int i = g.is; i <= g.ie; ++i) {
            double du = A1 * mc0.flux1[at(g, b, v, k, j, i + 1, g.NF)] -
                        A1 * mc0.flux1[at(g, b, v, k, j, i, g.NF)];
            if (g.ndim >= 2)
              du += A2 * mc0.flux2[at(g, b, v, k, j + 1, i, g.NF)] -
                    A2 * mc0.flux2[at(g, b, v, k, j, i, g.NF)];
            if (g.ndim == 3)
              du += A3 * mc0.flux3[at(g, b, v, k + 1, j, i, g.NF)] -
                    A3 * mc0.flux3[at(g, b, v, k, j, i, g.NF)];
            const double dudt = -du / V;
            const size_t q = at(g, b, v, k, j, i, g.NF);
            mc1.cons[q] = mc_init.cons[q] + bdt * dudt;
          }
}

// ----------------------------------------------------------------------------
// AddGeometricSource (source_term.cc:15-121), interior, prims of mc1.
// ----------------------------------------------------------------------------
void add_geometric_source(Ctx &c, pangu_pack &md, double bdt) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          const Real xc[4] = {0.0, Xc(g, b, 0, i), Xc(g, b, 1, j), Xc(g, b, 2, k)};
          Real gcov[4][4], gcon[4][4], gdet;
          metric_at(p.metric_type, xc, p.a, p.h, gcov, gcon, gdet);
          const Real sg = std::sqrt(std::fabs(gdet));
          Real conn[4][4][4];
          christoffel(p.metric_type, xc, p.a, p.h, conn);
          Real pc[NPRIM];
          load_prim(g, md.prim, b, k, j, i, pc);
          Real T[4][4];
          for (int r = 0; r < 4; ++r) emt(p.adiabatic_index, pc, gcov, gcon, r, T[r]);
          for (int d = 0; d < 4; ++d) {
            Real con = 0.0;
            for (int r = 0; r < 4; ++r)
              for (int cc = 0; cc < 4; ++cc) con += T[r][cc] * conn[cc][d][r];
            const int v = (d == 0) ? g.pidx[ENY] : g.pidx[UX1] + (d - 1);
            md.cons[at(g, b, v, k, j, i, g.NF)] += con * sg * bdt;
          }
        }
}

// ----------------------------------------------------------------------------
// Recovery (invertor.cc:18-210).
// ----------------------------------------------------------------------------
void recovery(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
  const bool robuster = p.recovery == PANGU_RECOVERY_ROBUSTER;
  const bool is_cks = p.metric_type == CKS;
  const double a2 = p.a * p.a;
  uint64_t n2d = 0, nvsq = 0, n1d = 0, nfail = 0, nkf = 0, nexc = 0;
#pragma omp parallel for collapse(3) reduction(+ : n2d, nvsq, n1d, nfail, nkf, nexc)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          const Real x = Xc(g, b, 0, i), y = Xc(g, b, 1, j), z = Xc(g, b, 2, k);
          const Real xc[4] = {0.0, x, y, z};
          double *flag = robuster ? nullptr : &md.flag[cell(g, b, k, j, i)];
          if (is_cks) {
            const Real rad2 = x * x + y * y + z * z;
            const Real sa = (rad2 - a2) * (rad2 - a2) + 4.0 * a2 * z * z;
            const Real r_bl = std::sqrt(0.5 * (rad2 - a2 + std::sqrt(sa)));
            if (r_bl < p.r_excise) {
              if (!robuster) *flag = 0;
              ++nexc;
              continue;
            }
          }
          Real gcov[4][4], gcon[4][4], gdet;
          metric_at(p.metric_type, xc, p.a, p.h, gcov, gcon, gdet);
          if (!robuster) *flag = 0;
          const Real sg = std::sqrt(std::fabs(gdet));
          const Real alpha = 1.0 / std::sqrt(-gcon[0][0]);
          Real C[9] = {0}, Pp[9] = {0};
          auto ld = [&](const double *A, int s) {
            return A[at(g, b, g.pidx[s], k, j, i, g.NF)];
          };
          C[RHO] = ld(md.cons, RHO); C[ENY] = ld(md.cons, ENY);
          C[UX1] = ld(md.cons, UX1); C[UX2] = ld(md.cons, UX2); C[UX3] = ld(md.cons, UX3);
          if (p.enable_B) { C[BX1] = ld(md.cons, BX1); C[BX2] = ld(md.cons, BX2); C[BX3] = ld(md.cons, BX3); }
          C[ENT] = ld(md.cons, ENT);
          Pp[RHO] = ld(md.prim, RHO); Pp[ENY] = ld(md.prim, ENY);
          Pp[UX1] = ld(md.prim, UX1); Pp[UX2] = ld(md.prim, UX2); Pp[UX3] = ld(md.prim, UX3);
          if (p.enable_B) { Pp[BX1] = ld(md.prim, BX1); Pp[BX2] = ld(md.prim, BX2); Pp[BX3] = ld(md.prim, BX3); }
          Pp[ENT] = ld(md.prim, ENT);
          const Real isg = 1.0 / sg;
          const Real aisg = alpha * isg;
          if (p.enable_B) {
            md.prim[at(g, b, g.pidx[BX1], k, j, i, g.NF)] = C[BX1] * isg;
            md.prim[at(g, b, g.pidx[BX2], k, j, i, g.NF)] = C[BX2] * isg;
            md.prim[at(g, b, g.pidx[BX3], k, j, i, g.NF)] = C[BX3] * isg;
          }
          Real UH[9], PH[9];
          UH[RHO] = aisg * C[RHO];
          UH[ENY] = aisg * (C[ENY] - C[RHO]);
          UH[UX1] = aisg * C[UX1]; UH[UX2] = aisg * C[UX2]; UH[UX3] = aisg * C[UX3];
          UH[BX1] = aisg * C[BX1]; UH[BX2] = aisg * C[BX2]; UH[BX3] = aisg * C[BX3];
          UH[ENT] = aisg * C[ENT];
          PH[RHO] = Pp[RHO]; PH[ENY] = Pp[ENY];
          PH[UX1] = Pp[UX1]; PH[UX2] = Pp[UX2]; PH[UX3] = Pp[UX3];
          PH[BX1] = PH[BX2] = PH[BX3] = 0.0;
          if (p.enable_B) {
            PH[BX1] = alpha * C[BX1] * isg;
            PH[BX2] = alpha * C[BX2] * isg;
            PH[BX3] = alpha * C[BX3] * isg;
          }
          PH[ENT] = Pp[ENT];
          const Real gam = p.adiabatic_index;
          if (robuster) {
            if (kastaun::invert(UH, PH, gam, gcov, gcon) != 0) { ++nkf; continue; }
          } else {
            int ok = s2d::invert(UH, PH, gam, gcov, gcon) == 0;
            if (ok) ++n2d;
            if (!ok) {
              ok = s1dvsq::invert(UH, PH, gam, gcov, gcon) == 0;
              if (ok) ++nvsq;
              if (!ok) {
                ok = s1d::invert(UH, PH, gam, gcov, gcon) == 0;
                if (ok) ++n1d; else ++nfail;
              }
            }
            *flag = ok;
          }
          md.prim[at(g, b, g.pidx[RHO], k, j, i, g.NF)] = PH[RHO];
          md.prim[at(g, b, g.pidx[ENY], k, j, i, g.NF)] = PH[ENY];
          md.prim[at(g, b, g.pidx[UX1], k, j, i, g.NF)] = PH[UX1];
          md.prim[at(g, b, g.pidx[UX2], k, j, i, g.NF)] = PH[UX2];
          md.prim[at(g, b, g.pidx[UX3], k, j, i, g.NF)] = PH[UX3];
        }
  c.cnt[PANGU_CNT_C2P_2D] += n2d;
  c.cnt[PANGU_CNT_C2P_1DVSQ] += nvsq;
  c.cnt[PANGU_CNT_C2P_1D] += n1d;
  c.cnt[PANGU_CNT_C2P_FAIL] += nfail;
  c.cnt[PANGU_CNT_KASTAUN_FAIL] += nkf;
  c.cnt[PANGU_CNT_EXCISED] += nexc;
}

// ----------------------------------------------------------------------------
// ApplyElectronHeating (electron_heating.cc:14-112), interior.
// ----------------------------------------------------------------------------
void apply_heating(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
  if (!p.enable_heating) return;
  const HeatParams hp = {p.model, p.adiabatic_index, p.gamma_p, p.gamma_e,
                         p.fel_constant, p.ratio_min, p.ratio_max,
                         (bool)p.limit_kel, (bool)p.suppress_highb_heat,
                         (bool)p.enforce_positive_dissipation};
#pragma omp parallel for collapse(3)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          const Real xc[4] = {0.0, Xc(g, b, 0, i), Xc(g, b, 1, j), Xc(g, b, 2, k)};
          Real gcov[4][4], gcon[4][4], gdet;
          metric_at(p.metric_type, xc, p.a, p.h, gcov, gcon, gdet);
          Real pc[NPRIM];
          load_prim(g, md.prim, b, k, j, i, pc);
          State st;
          calc_state(pc, gcov, gcon, st);
          const Real cr = md.cons[at(g, b, g.pidx[RHO], k, j, i, g.NF)];
          const HeatCell hc = {pc[RHO], pc[ENY], st.bsq,
                               md.cons[at(g, b, g.pidx[ENT], k, j, i, g.NF)] / cr,
                               pc[ENT],
                               md.cons[at(g, b, g.pidx[KEL], k, j, i, g.NF)] / cr};
          md.prim[at(g, b, g.pidx[KEL], k, j, i, g.NF)] = heating_apply(hp, hc);
        }
}

// ----------------------------------------------------------------------------
// FixRecovery (recovery_fixer.cc:12-119), two-phase deterministic form.
// ----------------------------------------------------------------------------
void fix_recovery(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_params &p = c.p;
  const bool is_cks = p.metric_type == CKS;
  const double a2 = p.a * p.a;
  const size_t ncell = (size_t)g.NB * g.N3 * g.N2 * g.N1;
  std::vector<double> P0(md.prim, md.prim + ncell * g.NF);
  std::vector<double> F0(md.flag, md.flag + ncell);
  const int off2 = (g.js != g.je) ? 1 : 0;  // recovery_fixer.cc:46
  uint64_t nfix = 0;
#pragma omp parallel for collapse(3) reduction(+ : nfix)
  for (int b = 0; b < g.NB; ++b)
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          if (F0[cell(g, b, k, j, i)] != 0) continue;
          if (is_cks) {
            const Real xr = Xc(g, b, 0, i), yr = Xc(g, b, 1, j), zr = Xc(g, b, 2, k);
            const Real rad2 = xr * xr + yr * yr + zr * zr;
            const Real sa = (rad2 - a2) * (rad2 - a2) + 4.0 * a2 * zr * zr;
            if (std::sqrt(0.5 * (rad2 - a2 + std::sqrt(sa))) < p.r_excise) continue;
          }
          auto fl = [&](int jj, int ii) { return (int)F0[cell(g, b, k, jj, ii)]; };
          const int pf1 = fl(j + off2, i - 1), pf2 = fl(j + off2, i);
          const int pf3 = fl(j + off2, i + 1), pf4 = fl(j, i + 1);
          const int pf5 = fl(j - off2, i + 1), pf6 = fl(j - off2, i);
          const int pf7 = fl(j - off2, i - 1), pf8 = fl(j, i - 1);
          auto q = [&](int v, int jj, int ii) { return P0[at(g, b, v, k, jj, ii, g.NF)]; };
          for (int v = 0; v < g.NF; ++v) {
            double val;
            if (pf2 && pf4 && pf6 && pf8)
              val = 0.25 * (q(v, j + off2, i) + q(v, j - off2, i) + q(v, j, i - 1) +
                            q(v, j, i + 1));
            else if (pf1 && pf3 && pf5 && pf7)
              val = 0.25 * (q(v, j + off2, i + 1) + q(v, j + off2, i - 1) +
                            q(v, j - off2, i + 1) + q(v, j - off2, i - 1));
            else
              val = 0.125 * (q(v, j + off2, i - 1) + q(v, j + off2, i) +
                             q(v, j + off2, i + 1) + q(v, j, i + 1) +
                             q(v, j - off2, i + 1) + q(v, j - off2, i) +
                             q(v, j - off2, i - 1) + q(v, j, i - 1));
            md.prim[at(g, b, v, k, j, i, g.NF)] = val;
          }
          md.prim[at(g, b, g.pidx[UX1], k, j, i, g.NF)] = 0.;
          md.prim[at(g, b, g.pidx[UX2], k, j, i, g.NF)] = 0.;
          md.prim[at(g, b, g.pidx[UX3], k, j, i, g.NF)] = 0.;
          md.flag[cell(g, b, k, j, i)] = 1;
          ++nfix;
        }
  c.cnt[PANGU_CNT_FIXRECOVERY] += nfix;
}

// ----------------------------------------------------------------------------
// Ghost exchange (periodic / block-to-block), prim and flag.
// ----------------------------------------------------------------------------
void exchange_ghosts(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_mesh &m = c.m;
  const int nb[3] = {m.nbx1, m.nbx2, m.nbx3};
  const int nx[3] = {m.nx1, m.nx2, m.nx3};
  const int st[3] = {g.is, g.js, g.ks};
  const int act[3] = {g.o1, g.o2, g.o3};
  const int Nn[3] = {g.N1, g.N2, g.N3};
  const bool periodic[3] = {m.bc[0] == PANGU_BC_PERIODIC, m.bc[2] == PANGU_BC_PERIODIC,
                            m.bc[4] == PANGU_BC_PERIODIC};
  // Values are read from a snapshot so that the copy order does not matter.
  const size_t ncell = (size_t)g.NB * g.N3 * g.N2 * g.N1;
  std::vector<double> P0(md.prim, md.prim + ncell * g.NF);
  std::vector<double> F0;
  if (md.flag) F0.assign(md.flag, md.flag + ncell);
  for (int b = 0; b < g.NB; ++b) {
    const int bl[3] = {b % m.nbx1, (b / m.nbx1) % m.nbx2, b / (m.nbx1 * m.nbx2)};
    for (int k = 0; k < g.N3; ++k)
      for (int j = 0; j < g.N2; ++j)
        for (int i = 0; i < g.N1; ++i) {
          const int idx[3] = {i, j, k};
          int src_bl[3], src_idx[3];
          bool ghost = false, ok = true;
          for (int d = 0; d < 3; ++d) {
            src_bl[d] = bl[d];
            src_idx[d] = idx[d];
            if (!act[d]) continue;
            int side = 0;
            if (idx[d] < st[d]) side = -1;
            else if (idx[d] >= st[d] + nx[d]) side = 1;
            if (side == 0) continue;
            ghost = true;
            int nbl = bl[d] + side;
            if (nbl < 0 || nbl >= nb[d]) {
              if (!periodic[d]) { ok = false; break; }
              nbl = (nbl + nb[d]) % nb[d];
            }
            src_bl[d] = nbl;
            src_idx[d] = idx[d] - side * nx[d];
          }
          (void)Nn;
          if (!ghost || !ok) continue;
          const int sb = (src_bl[2] * m.nbx2 + src_bl[1]) * m.nbx1 + src_bl[0];
          for (int v = 0; v < g.NF; ++v)
            md.prim[at(g, b, v, k, j, i, g.NF)] =
                P0[at(g, sb, v, src_idx[2], src_idx[1], src_idx[0], g.NF)];
          if (md.flag)
            md.flag[cell(g, b, k, j, i)] = F0[cell(g, sb, src_idx[2], src_idx[1], src_idx[0])];
        }
  }
}

// ----------------------------------------------------------------------------
// Physical boundary conditions (outflow / reflecting), prim and flag.
// ----------------------------------------------------------------------------
void physical_bcs(Ctx &c, pangu_pack &md) {
  const Geom &g = c.g;
  const pangu_mesh &m = c.m;
  const pangu_params &p = c.p;
  const int nb[3] = {m.nbx1, m.nbx2, m.nbx3};
  const int act[3] = {g.o1, g.o2, g.o3};
  const int s[3] = {g.is, g.js, g.ks};
  const int e[3] = {g.ie, g.je, g.ke};
  for (int face = 0; face < 6; ++face) {
    const int d = face / 2;
    const int outer = face % 2;
    const int kind = m.bc[face];
    if (!act[d] || kind == PANGU_BC_PERIODIC) continue;
    for (int b = 0; b < g.NB; ++b) {
      const int bl[3] = {b % m.nbx1, (b / m.nbx1) % m.nbx2, b / (m.nbx1 * m.nbx2)};
      if (outer ? (bl[d] != nb[d] - 1) : (bl[d] != 0)) continue;
      for (int k = 0; k < g.N3; ++k)
        for (int j = 0; j < g.N2; ++j)
          for (int i = 0; i < g.N1; ++i) {
            int idx[3] = {i, j, k};
            const int x = idx[d];
            if (outer ? (x <= e[d]) : (x >= s[d])) continue;
            int src = idx[d];
            if (kind == PANGU_BC_OUTFLOW) src = outer ? e[d] : s[d];
            else src = outer ? (2 * e[d] + 1 - x) : (2 * s[d] - 1 - x);
            int sidx[3] = {i, j, k};
            sidx[d] = src;
            for (int v = 0; v < g.NF; ++v) {
              double val = md.prim[at(g, b, v, sidx[2], sidx[1], sidx[0], g.NF)];
              if (kind == PANGU_BC_REFLECTING) {
                const bool vel = v == g.pidx[UX1] + d;
                const bool mag = p.enable_B && v == g.pidx[BX1] + d;
                if (vel || mag) val = -val;
              }
              md.prim[at(g, b, v, k, j, i, g.NF)] = val;
            }
            if (md.flag)
              md.flag[cell(g, b, k, j, i)] = md.flag[cell(g, b, sidx[2], sidx[1], sidx[0])];
          }
    }
  }
}

// ----------------------------------------------------------------------------
// EstimateTimestepMesh (timestep_estimation.cc:13-102).
// ----------------------------------------------------------------------------
double estimate_dt(Ctx &c, const pangu_pack &md) {
  const Geom &g = c.g;
  const double big = std::numeric_limits<double>::max();
  double gmin = big;
  const int off[3] = {g.N1 > 1, g.N2 > 1, g.N3 > 1};
  for (int b = 0; b < g.NB; ++b) {
    double mins[3] = {big, big, big};
    for (int d = 0; d < 3; ++d) {
      if (!off[d]) continue;
      double mn = big;
      const double cdx = c.p.cfl_number * g.dx[d];
#pragma omp parallel for collapse(3) reduction(min : mn)
      for (int k = g.ks; k <= g.ke; ++k)
        for (int j = g.js; j <= g.je; ++j)
          for (int i = g.is; i <= g.ie; ++i) {
            const double cs = md.alfven[at(g, b, d, k, j, i, 3)];
            const double dt = cdx / cs;
            if (mn > dt) mn = dt;
          }
      mins[d] = mn;
    }
    const double bdt = 1.0 / (1.0 / mins[0] + 1.0 / mins[1] + 1.0 / mins[2]);
    if (bdt < gmin) gmin = bdt;
  }
  return gmin;
}

void stage(Ctx &c, int st, pangu_pack &base, pangu_pack &one, double beta,
           double dt, double *dt_est) {
  pangu_pack &mc0 = (st == 1) ? base : one;
  pangu_pack &mc1 = (st == 1) ? one : base;
  pangu_pack &mc_init = base;
  fix_primitive(c, mc0);
  calc_conservative(c, mc0);
  calc_fluxes(c, mc0);
  if (c.p.enable_B) constrained_transport(c, mc0);
  flux_div_update(c, mc_init, mc0, mc1, beta * dt);
  exchange_ghosts(c, mc1);
  add_geometric_source(c, mc1, beta * dt);
  recovery(c, mc1);
  if (c.p.enable_heating) apply_heating(c, mc1);
  if (c.p.recovery == PANGU_RECOVERY_CHAINER) fix_recovery(c, mc1);
  physical_bcs(c, mc1);
  if (st == 2 && dt_est) *dt_est = estimate_dt(c, mc1);
}

}  // namespace

// ============================================================================
// C API (ctypes from the tests and bench.py)
// ============================================================================
extern "C" {

struct or_ctx;

or_ctx *or_create(const pangu_params *p, const pangu_mesh *m) {
  Ctx *c = new Ctx;
  c->p = *p;
  c->m = *m;
  c->g = make_geom(*p, *m);
  std::memset(c->cnt, 0, sizeof(c->cnt));
  return reinterpret_cast<or_ctx *>(c);
}
void or_destroy(or_ctx *h) { delete reinterpret_cast<Ctx *>(h); }
int or_num_fields(or_ctx *h) { return reinterpret_cast<Ctx *>(h)->g.NF; }
void or_counters(or_ctx *h, uint64_t *out) {
  std::memcpy(out, reinterpret_cast<Ctx *>(h)->cnt, sizeof(uint64_t) * PANGU_NCOUNTERS);
}
void or_reset_counters(or_ctx *h) {
  std::memset(reinterpret_cast<Ctx *>(h)->cnt, 0, sizeof(uint64_t) * PANGU_NCOUNTERS);
}
void or_set_threads(int n) { omp_set_num_threads(n); }

#define CTX reinterpret_cast<Ctx *>(h)
void or_fix_primitive(or_ctx *h, pangu_pack *md) { fix_primitive(*CTX, *md); }
void or_calculate_conservative(or_ctx *h, pangu_pack *md) { calc_conservative(*CTX, *md); }
void or_calculate_fluxes(or_ctx *h, pangu_pack *md) { calc_fluxes(*CTX, *md); }
void or_constrained_transport(or_ctx *h, pangu_pack *md) { constrained_transport(*CTX, *md); }
void or_flux_divergence_update(or_ctx *h, const pangu_pack *mi, const pangu_pack *m0,
                               pangu_pack *m1, double bdt) {
  flux_div_update(*CTX, *mi, *m0, *m1, bdt);
}
void or_exchange_ghosts(or_ctx *h, pangu_pack *md) { exchange_ghosts(*CTX, *md); }
void or_add_geometric_source(or_ctx *h, pangu_pack *md, double bdt) {
  add_geometric_source(*CTX, *md, bdt);
}
void or_recovery(or_ctx *h, pangu_pack *md) { recovery(*CTX, *md); }
void or_apply_electron_heating(or_ctx *h, pangu_pack *md) { apply_heating(*CTX, *md); }
void or_fix_recovery(or_ctx *h, pangu_pack *md) { fix_recovery(*CTX, *md); }
void or_apply_boundary_conditions(or_ctx *h, pangu_pack *md) { physical_bcs(*CTX, *md); }
double or_estimate_dt(or_ctx *h, const pangu_pack *md) { return estimate_dt(*CTX, *md); }
void or_stage(or_ctx *h, int st, pangu_pack *base, pangu_pack *one, double beta,
              double dt, double *dt_est) {
  stage(*CTX, st, *base, *one, beta, dt, dt_est);
}
#undef CTX

// Per-cell entry points for the golden-vector checks.
void or_cell_metric(int mt, const double x[4], double a, double h, double gcov[16],
                    double gcon[16], double *gdet) {
  metric_at(mt, x, a, h, reinterpret_cast<Real(*)[4]>(gcov),
            reinterpret_cast<Real(*)[4]>(gcon), *gdet);
}
void or_cell_christoffel(int mt, const double x[4], double a, double h, double conn[64]) {
  christoffel(mt, x, a, h, reinterpret_cast<Real(*)[4][4]>(conn));
}
void or_cell_flux(double gam, const double P[10], const double gcov[16],
                  const double gcon[16], double gdet, int dir, double f[10]) {
  contravariant_flux(gam, P, reinterpret_cast<const Real(*)[4]>(gcov),
                     reinterpret_cast<const Real(*)[4]>(gcon), gdet, dir, f);
}
void or_cell_fast_speed(double gam, const double P[10], const double gcov[16],
                        const double gcon[16], int dir, double out[2]) {
  fast_speed(gam, P, reinterpret_cast<const Real(*)[4]>(gcov),
             reinterpret_cast<const Real(*)[4]>(gcon), dir, out[0], out[1]);
}
void or_cell_recon(int use_mc, const double q[5], double out[2]) {
  if (use_mc) mc(q[0], q[1], q[2], q[3], q[4], out[0], out[1]);
  else ppm4(q[0], q[1], q[2], q[3], q[4], out[0], out[1]);
}
// scheme: 0 = 2D, 1 = 1Dvsq, 2 = 1D, 3 = Kastaun. Returns the scheme status.
int or_cell_invert(int scheme, const double U[9], double prim[9], double gam,
                   const double gcov[16], const double gcon[16]) {
  auto gc = reinterpret_cast<const Real(*)[4]>(gcov);
  auto gn = reinterpret_cast<const Real(*)[4]>(gcon);
  switch (scheme) {
    case 0: return s2d::invert(U, prim, gam, gc, gn);
    case 1: return s1dvsq::invert(U, prim, gam, gc, gn);
    case 2: return s1d::invert(U, prim, gam, gc, gn);
    default: return kastaun::invert(U, prim, gam, gc, gn);
  }
}
double or_cell_heating(const double hp[6], const int flags[4], const double cell[6]) {
  HeatParams p = {flags[0], hp[0], hp[1], hp[2], hp[3], hp[4], hp[5],
                  (bool)flags[1], (bool)flags[2], (bool)flags[3]};
  HeatCell c = {cell[0], cell[1], cell[2], cell[3], cell[4], cell[5]};
  return heating_apply(p, c);
}
double or_cell_clamp(double rmin, double rmax, double total, double electron) {
  return clamp_by_ratio(rmin, rmax, total, electron);
}

// The shared double-double routines, for their accuracy test.
void or_pgm_pow(int n, const double *x, const double *y, double *out) {
  for (int i = 0; i < n; ++i) out[i] = pgm::pow(x[i], y[i]);
}
// The slow double-double path of pgm::pow alone (finite x > 0), for tests of
// the table-driven fast path.
void or_pgm_pow_slow(int n, const double *x, const double *y, double *out) {
  for (int i = 0; i < n; ++i) out[i] = pgm::exp_round(pgm::mul_d(pgm::log_dd(x[i]), y[i]));
}
// The fast path alone (finite x > 0): ok[i] = 1 where its error bound decided
// the rounding, with out[i] its result; 0 where the slow path would decide.
void or_pgm_pow_fast(int n, const double *x, const double *y, double *out, int *ok) {
  for (int i = 0; i < n; ++i) {
    double r = 0.0;
    ok[i] = pgm::pow_fast(x[i], y[i], r) ? 1 : 0;
    out[i] = r;
  }
}
// The fast path's log and exp parts (hi + lo, and exp's power of two), for
// the test of their error bounds.
void or_pgm_log_fast(int n, const double *x, double *hi, double *lo) {
  for (int i = 0; i < n; ++i) {
    const pgm::dd l = pgm::log_fast(x[i]);
    hi[i] = l.hi;
    lo[i] = l.lo;
  }
}
void or_pgm_exp_fast(int n, const double *th, const double *tl, double *hi, double *lo,
                     int *scale) {
  for (int i = 0; i < n; ++i) {
    const pgm::dd v = pgm::exp_fast(th[i], tl[i], scale[i]);
    hi[i] = v.hi;
    lo[i] = v.lo;
  }
}
void or_pgm_exp(int n, const double *x, double *out) {
  for (int i = 0; i < n; ++i) out[i] = pgm::exp(x[i]);
}
void or_pgm_log(int n, const double *x, double *out) {
  for (int i = 0; i < n; ++i) out[i] = pgm::log(x[i]);
}

}  // extern "C"
