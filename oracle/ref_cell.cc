// ref_cell.cc -- extern "C" wrappers around the REFERENCE's own per-cell
// functions, compiled from its headers where they lie (pangu/src/...) with
// the stand-in headers of oracle/refshim. Built by oracle/build.py into
// oracle/_ref/ only when the reference sources are present. Test
// infrastructure: it produces the golden vectors that pin oracle_cell.h
// (tests/golden/make_golden.py); nothing else links it.
#include <cstdint>

#include "interpolation/interpolater_mc.h"
#include "interpolation/interpolater_ppm4.h"
#include "metric/christoffel.h"
#include "physics/contravariant_flux.h"
#include "physics/fast_magnetosonic_speed.h"
#include "physics/heating_model.h"
#include "recovery/scheme_1d.h"
#include "recovery/scheme_1d_vsq.h"
#include "recovery/scheme_2d.h"
#include "recovery/scheme_kastaun.h"

using parthenon::Real;

namespace {
void to44(const double *a, Real m[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) m[i][j] = a[4 * i + j];
}
void from44(Real m[4][4], double *a) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) a[4 * i + j] = m[i][j];
}
}  // namespace

extern "C" {

void ref_cell_metric(int mt, const double x[4], double a, double h,
                     double gcov[16], double gcon[16], double *gdet) {
  Real gc[4][4], gn[4][4];
  ComputeMetricAtLocation(mt, x, a, h, gc, gn, *gdet);
  from44(gc, gcov);
  from44(gn, gcon);
}

void ref_cell_christoffel(int mt, const double x[4], double a, double h,
                          double conn[64]) {
  Real c[4][4][4];
  ComputeChristoffelConnection(mt, x, a, h, c);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) conn[16 * i + 4 * j + k] = c[i][j][k];
}

void ref_cell_flux(double gam, const double P[10], const double gcov[16],
                   const double gcon[16], double gdet, int dir, double f[10]) {
  Real gc[4][4], gn[4][4], pp[NPRIM];
  to44(gcov, gc);
  to44(gcon, gn);
  for (int n = 0; n < NPRIM; ++n) pp[n] = P[n];
  CalculateContravariantFlux(gam, pp, gc, gn, gdet, dir, f);
}

void ref_cell_fast_speed(double gam, const double P[10], const double gcov[16],
                         const double gcon[16], int dir, double out[2]) {
  Real gc[4][4], gn[4][4], pp[NPRIM];
  to44(gcov, gc);
  to44(gcon, gn);
  for (int n = 0; n < NPRIM; ++n) pp[n] = P[n];
  CalculateFastMagnetosonicSpeed(gam, pp, gc, gn, dir, out[0], out[1]);
}

void ref_cell_recon(int use_mc, const double q[5], double out[2]) {
  if (use_mc)
    MC(q[0], q[1], q[2], q[3], q[4], out[0], out[1]);
  else
    PPM4(q[0], q[1], q[2], q[3], q[4], out[0], out[1]);
}

int ref_cell_invert(int scheme, const double U[9], double prim[9], double gam,
                    const double gcov[16], const double gcon[16]) {
  Real gc[4][4], gn[4][4], uu[9], pp[9];
  to44(gcov, gc);
  to44(gcon, gn);
  for (int n = 0; n < 9; ++n) { uu[n] = U[n]; pp[n] = prim[n]; }
  const Real gdet = 0.0;  // unused by every scheme
  int st;
  switch (scheme) {
    case 0: st = Scheme2D::invert(uu, pp, gam, gc, gn, gdet); break;
    case 1: st = Scheme1Dvsq::invert(uu, pp, gam, gc, gn, gdet); break;
    case 2: st = Scheme1D::invert(uu, pp, gam, gc, gn, gdet); break;
    default: st = SchemeKastaun::invert(uu, pp, gam, gc, gn, gdet); break;
  }
  for (int n = 0; n < 9; ++n) prim[n] = pp[n];
  return st;
}

double ref_cell_heating(const double hp[6], const int flags[4],
                        const double cell[6]) {
  const Parameters p = {static_cast<Model>(flags[0]), hp[0], hp[1], hp[2],
                        hp[3], {hp[4], hp[5]}, (bool)flags[1],
                        (bool)flags[2], (bool)flags[3]};
  const CellState c = {cell[0], cell[1], cell[2], cell[3], cell[4], cell[5]};
  return apply(p, c);
}

double ref_cell_clamp(double rmin, double rmax, double total, double electron) {
  return clampByRatio({rmin, rmax}, total, electron);
}

}  // extern "C"
