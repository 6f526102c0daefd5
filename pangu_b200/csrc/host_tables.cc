// host_tables.cc -- coordinate tables and ghost-exchange map of the engine,
// built on the host once per engine.
//
// The MKS and BL code metrics (MKS.h:60-107, BL.h:60-107) take a centred
// finite difference of the coordinate map with delta = 1e-5, which amplifies
// a one-ulp difference of exp/sin by 1e5. The values of the map that the
// metric needs -- r = exp(x1), its difference quotient J1, sin and cos of
// theta(x2) and its difference quotient J2, at cell centres, faces and the
// +-delta points of the Christoffel differences (christoffel.h:74-148) -- are
// therefore evaluated here, with the C library's exp/sin/cos, in the
// reference's operation order, and compiled with -ffp-contract=off. The
// device only does the algebra on top (pangu_device.cuh).
#include <cmath>
#include <cstdint>
#include <vector>

#include "pangu_b200.h"
#include "pgmath.h"

namespace pgh {

constexpr double kDelta = 1.0e-5;

// MKS.h:15-23 / BL.h:15-23
static double theta_of(double x2, double h) {
  return M_PI_2 * (x2 + 1.0) + 0.5 * h * std::sin(M_PI * (x2 + 1.0));
}

// Jacobian entry (yh - yl) / (xh - xl) of MKS.h:76-94.
static double jac_exp(double x) {
  const double xh = x + kDelta, xl = x - kDelta;
  return (std::exp(xh) - std::exp(xl)) / (xh - xl);
}
static double jac_theta(double x, double h) {
  const double xh = x + kDelta, xl = x - kDelta;
  return (theta_of(xh, h) - theta_of(xl, h)) / (xh - xl);
}

struct Layout {
  int N[3], st[3], nx[3], act[3], nb[3], NB, ng, NF;
  double dx[3];
  std::vector<double> origin;  // [NB][3]
};

Layout make_layout(const pangu_params &p, const pangu_mesh &m) {
  Layout L;
  L.nx[0] = m.nx1; L.nx[1] = m.nx2; L.nx[2] = m.nx3;
  L.nb[0] = m.nbx1; L.nb[1] = m.nbx2; L.nb[2] = m.nbx3;
  L.ng = m.ng;
  L.NB = m.nbx1 * m.nbx2 * m.nbx3;
  L.NF = 6 + (p.enable_B ? 3 : 0) + (p.enable_heating ? 1 : 0);
  const double mins[3] = {m.x1min, m.x2min, m.x3min};
  const double maxs[3] = {m.x1max, m.x2max, m.x3max};
  for (int d = 0; d < 3; ++d) {
    L.act[d] = L.nx[d] > 1;
    L.N[d] = L.nx[d] + 2 * m.ng * L.act[d];
    L.st[d] = m.ng * L.act[d];
    L.dx[d] = (maxs[d] - mins[d]) / (double)(L.nb[d] * L.nx[d]);
  }
  L.origin.resize(3 * L.NB);
  for (int b = 0; b < L.NB; ++b) {
    const int bl[3] = {b % m.nbx1, (b / m.nbx1) % m.nbx2, b / (m.nbx1 * m.nbx2)};
    for (int d = 0; d < 3; ++d) {
      const double bxmin = mins[d] + (double)(bl[d] * L.nx[d]) * L.dx[d];
      L.origin[3 * b + d] = bxmin - (double)(m.ng * L.act[d]) * L.dx[d];
    }
  }
  return L;
}

// Table of the x1 map per block: 10 rows of N1 + 1 entries
//   0 r(xc)  1 J1(xc)  2 r(xc+d)  3 J1(xc+d)  4 r(xc-d)  5 J1(xc-d)
//   6 r(xf)  7 J1(xf)
//   8, 9: the density and energy floors of FixPrimitive at r(xc)
//         (primitive_fixer.cc:79-89, MKS radius)
// and of the x2 map: 12 rows of N2 + 1 entries
//   0 sin th(xc) 1 cos th(xc) 2 J2(xc)  3..5 at xc+d  6..8 at xc-d
//   9..11 at xf.
void build_tables(const pangu_params &p, const Layout &L, std::vector<double> &t1,
                  std::vector<double> &t2) {
  const int W1 = L.N[0] + 1, W2 = L.N[1] + 1;
  t1.assign((size_t)L.NB * 10 * W1, 0.0);
  t2.assign((size_t)L.NB * 12 * W2, 0.0);
  for (int b = 0; b < L.NB; ++b) {
    const double o1 = L.origin[3 * b + 0], o2 = L.origin[3 * b + 1];
    double *T1 = &t1[(size_t)b * 10 * W1];
    double *T2 = &t2[(size_t)b * 12 * W2];
    for (int i = 0; i < W1; ++i) {
      const double xc = o1 + ((double)i + 0.5) * L.dx[0];
      const double xf = o1 + (double)i * L.dx[0];
      double xp = xc, xm = xc;
      xp += kDelta;
      xm -= kDelta;
      T1[0 * W1 + i] = std::exp(xc);
      T1[1 * W1 + i] = jac_exp(xc);
      T1[2 * W1 + i] = std::exp(xp);
      T1[3 * W1 + i] = jac_exp(xp);
      T1[4 * W1 + i] = std::exp(xm);
      T1[5 * W1 + i] = jac_exp(xm);
      T1[6 * W1 + i] = std::exp(xf);
      T1[7 * W1 + i] = jac_exp(xf);
      const double r = std::exp(xc);
      T1[8 * W1 + i] = p.density_floor * pgm::pow(std::fmax(r, 1.0), p.density_floor_pow);
      T1[9 * W1 + i] = p.energy_floor * pgm::pow(std::fmax(r, 1.0), p.energy_floor_pow);
    }
    for (int j = 0; j < W2; ++j) {
      const double xc = o2 + ((double)j + 0.5) * L.dx[1];
      const double xf = o2 + (double)j * L.dx[1];
      double xp = xc, xm = xc;
      xp += kDelta;
      xm -= kDelta;
      const double pts[4] = {xc, xp, xm, xf};
      for (int q = 0; q < 4; ++q) {
        const double th = theta_of(pts[q], p.h);
        T2[(3 * q + 0) * W2 + j] = std::sin(th);
        T2[(3 * q + 1) * W2 + j] = std::cos(th);
        T2[(3 * q + 2) * W2 + j] = jac_theta(pts[q], p.h);
      }
    }
  }
}

// Ghost exchange map: for every ghost cell whose every ghost direction has a
// neighbour block (periodic wrap included), the interior cell it copies.
// Entries are cell offsets b * ncell + c.
void build_exchange(const pangu_mesh &m, const Layout &L, std::vector<int64_t> &dst,
                    std::vector<int64_t> &src) {
  const bool periodic[3] = {m.bc[0] == PANGU_BC_PERIODIC, m.bc[2] == PANGU_BC_PERIODIC,
                            m.bc[4] == PANGU_BC_PERIODIC};
  const int64_t ncell = (int64_t)L.N[0] * L.N[1] * L.N[2];
  dst.clear();
  src.clear();
  for (int b = 0; b < L.NB; ++b) {
    const int bl[3] = {b % L.nb[0], (b / L.nb[0]) % L.nb[1], b / (L.nb[0] * L.nb[1])};
    for (int k = 0; k < L.N[2]; ++k)
      for (int j = 0; j < L.N[1]; ++j)
        for (int i = 0; i < L.N[0]; ++i) {
          const int idx[3] = {i, j, k};
          int sbl[3], sidx[3];
          bool ghost = false, ok = true;
          for (int d = 0; d < 3 && ok; ++d) {
            sbl[d] = bl[d];
            sidx[d] = idx[d];
            if (!L.act[d]) continue;
            int side = 0;
            if (idx[d] < L.st[d]) side = -1;
            else if (idx[d] >= L.st[d] + L.nx[d]) side = 1;
            if (!side) continue;
            ghost = true;
            int nbl = bl[d] + side;
            if (nbl < 0 || nbl >= L.nb[d]) {
              if (!periodic[d]) { ok = false; break; }
              nbl = (nbl + L.nb[d]) % L.nb[d];
            }
            sbl[d] = nbl;
            sidx[d] = idx[d] - side * L.nx[d];
          }
          if (!ghost || !ok) continue;
          const int sb = (sbl[2] * L.nb[1] + sbl[1]) * L.nb[0] + sbl[0];
          dst.push_back((int64_t)b * ncell + ((int64_t)k * L.N[1] + j) * L.N[0] + i);
          src.push_back((int64_t)sb * ncell + ((int64_t)sidx[2] * L.N[1] + sidx[1]) * L.N[0] +
                        sidx[0]);
        }
  }
}

// Block sharding of one mesh over several ranks: splits the exchange map for
// `rank`. Entries with both blocks on `rank` stay local (ldst, lsrc). An entry
// whose source block is on `rank` and whose destination block is on peer q is
// sent to q (its source cell appended to send[q]); one whose destination is on
// `rank` and whose source is on q is received from q (its destination cell
// appended to recv[q]). Both sides walk the same map in the same order, so the
// k-th cell that `rank` sends to q is the k-th cell q receives from `rank`.
void shard_exchange(const std::vector<int64_t> &dst, const std::vector<int64_t> &src,
                    int64_t ncell, const int32_t *block_rank, int nranks, int rank,
                    std::vector<int64_t> &ldst, std::vector<int64_t> &lsrc,
                    std::vector<std::vector<int64_t>> &send,
                    std::vector<std::vector<int64_t>> &recv) {
  ldst.clear();
  lsrc.clear();
  send.assign(nranks, {});
  recv.assign(nranks, {});
  for (size_t q = 0; q < dst.size(); ++q) {
    const int rd = block_rank[dst[q] / ncell], rs = block_rank[src[q] / ncell];
    if (rd == rank && rs == rank) {
      ldst.push_back(dst[q]);
      lsrc.push_back(src[q]);
    } else if (rs == rank) {
      send[rd].push_back(src[q]);
    } else if (rd == rank) {
      recv[rs].push_back(dst[q]);
    }
  }
}

}  // namespace pgh
