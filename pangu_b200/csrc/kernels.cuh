// kernels.cuh -- the engine's kernels and launch helpers, compiled four
// times: engine.cu instantiates them in namespace pgk64 (FP64 throughout,
// built with --fmad=false for bit-exact parity) and engine_mixed.cu in
// namespace pgkmx (mixed precision), both for packs in the contiguous layout;
// engine_tables.cu (pgk64t) and engine_mixed_tables.cu (pgkmxt) are the same
// kernels for packs that give arrays through per-(block, component) pointer
// tables. The includer defines PGK_NS, PGK_MIXED and (for the table forms)
// PGK_TABLES; the table test then costs the contiguous kernels nothing.
#ifndef PGK_NS
#error "define PGK_NS before including kernels.cuh"
#endif
#ifndef PGK_TABLES
#define PGK_TABLES 0
#endif

#include <cuda.h>  // CUtensorMap (types only; the encoder comes from the runtime)
#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>

namespace PGK_NS {
using namespace pgd;

// An NVTX range per task of the stage, named as the reference's tasks (the
// counterpart of PARTHENON_INSTRUMENT, e.g. laxf.cc:21); free when no
// profiler is attached.
struct TaskRange {
  explicit TaskRange(const char *name) { nvtxRangePushA(name); }
  ~TaskRange() { nvtxRangePop(); }
};

// Storage type of the primitives and arithmetic type of reconstruction and
// Riemann flux: FP64 in the exact build, FP32 in the mixed one.
#if PGK_MIXED
using PT = float;
using FT = float;
#define PGK_POW ::pow
#else
using PT = double;
using FT = double;
#define PGK_POW pgm::pow
#endif

// The FP64 flux kernels of curved metrics evaluate the two sides of a face
// one after the other through shared memory (face_flux_split); the others
// hold both states in registers (face_flux).
#define PGK_SPLIT_FACES (!PGK_MIXED)

template <class Pack>
__host__ __forceinline__ PT *prim_of(const Pack *md) {
  return reinterpret_cast<PT *>(md->prim);
}

// CTA size of the per-cell kernels. FixPrimitive, the geometric source and
// electron heating are bounded to 4 resident CTAs per SM (64 registers): the
// extra occupancy outweighs their few spills (measured 2 % per RK2 cycle on
// the 2D and 3D tori), and 148 x 1024 threads hold a 512 x 256 grid in one
// wave. The first C2P pass runs in CTAs of 128 threads bounded to 7 per SM
// (72 registers, a few spills): 148 x 896 threads hold the 512 x 256 grid in
// one wave (1.2 % per cycle; at 64 registers its Newton loop spills too much).
constexpr int kThreads = 256;
constexpr int kRecoveryThreads = 128;

// Programmatic dependent launch: the stage's kernels are launched with
// programmatic stream serialisation (launch_pdl), so the launch of a kernel
// overlaps the end of the previous one. Every kernel therefore first waits
// until the previous grid has completed and its writes are visible
// (griddepcontrol.wait; a no-op in a normal launch). No kernel triggers its
// dependents early: measured, an early trigger (dependents' CTAs resident
// and waiting during the last wave) cost 4 % per cycle on the 2D torus, while
// the launch overlap alone gains 2.6 % on the 256^2 Orszag-Tang problem and
// is neutral on the tori.
__device__ __forceinline__ void pdl_grid_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
constexpr int kT1Rows = 10;  // rows of the x1 table (host_tables.cc)

__device__ __forceinline__ int slot_of(const Dims &d, int bb) {
  return d.slot ? __ldg(d.slot + bb) : bb;
}
__device__ __forceinline__ int job_of(const Dims &d, int b) {
  return d.slot_job ? __ldg(d.slot_job + b) : 0;
}
__device__ __forceinline__ double dx_of(const Dims &d, int b, int dir) {
  return d.bdx ? __ldg(d.bdx + 3 * b + dir) : d.dx[dir];
}

__device__ __forceinline__ long long cidx(const Dims &d, int b, int k, int j, int i) {
  return ((long long)b * d.N3 + k) * (long long)d.N2 * d.N1 + (long long)j * d.N1 + i;
}

// Offset of cell (k, j, i) inside one component's [N3][N2][N1] array.
__device__ __forceinline__ long long coff(const Dims &d, int k, int j, int i) {
  return ((long long)k * d.N2 + j) * d.N1 + i;
}
// Base of component v of slot b of an array with nc components per slot: in
// the table forms the pack's table entry when it gives one, else (and always
// in the contiguous forms) the contiguous layout.
template <class T, class Tab>
__device__ __forceinline__ T *comp(const Dims &d, T *base, Tab *const *tab, int nc, int b, int v) {
#if PGK_TABLES
  if (tab) {
    const unsigned long long a =
        __ldg(reinterpret_cast<const unsigned long long *>(tab) + (long long)b * nc + v);
    return reinterpret_cast<T *>(a);
  }
#else
  (void)tab;
#endif
  return base + ((long long)b * nc + v) * d.ncell;
}
// The roles of Dims' tables: primitives, the task's conserved variables,
// the RK starting state's, the launch's flux array, the three flux arrays,
// alfven, efield and flag.
template <class T> __device__ __forceinline__ T *a_prim(const Dims &d, T *P, int b, int v) {
  return comp(d, P, d.tP, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_cons(const Dims &d, T *U, int b, int v) {
  return comp(d, U, d.tU, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_cons0(const Dims &d, T *U, int b, int v) {
  return comp(d, U, d.tUi, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_flux(const Dims &d, T *F, int b, int v) {
  return comp(d, F, d.tF, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_flux1(const Dims &d, T *F, int b, int v) {
  return comp(d, F, d.tF1, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_flux2(const Dims &d, T *F, int b, int v) {
  return comp(d, F, d.tF2, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_flux3(const Dims &d, T *F, int b, int v) {
  return comp(d, F, d.tF3, d.NF, b, v);
}
template <class T> __device__ __forceinline__ T *a_alfven(const Dims &d, T *A, int b, int c) {
  return comp(d, A, d.tA, 3, b, c);
}
template <class T> __device__ __forceinline__ T *a_efield(const Dims &d, T *E, int b, int c) {
  return comp(d, E, d.tE, 3, b, c);
}
template <class T> __device__ __forceinline__ T *a_flag(const Dims &d, T *G, int b) {
  return comp(d, G, d.tG, 1, b, 0);
}

__device__ __forceinline__ void load_prim(const Dims &d, const PT *P, int b, int k, int j,
                                          int i, double out[NPRIM]) {
  const long long o = coff(d, k, j, i);
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) out[s] = d.pidx[s] >= 0 ? a_prim(d, P, b, d.pidx[s])[o] : 0.0;
}

// Cell-centre coordinate (origin + (idx + 1/2) dx, rounded step by step).
__device__ __forceinline__ double xc(const Dims &d, int b, int dir, int idx) {
  return ADD(d.origin[3 * b + dir], MUL((double)idx + 0.5, dx_of(d, b, dir)));
}
__device__ __forceinline__ double xf(const Dims &d, int b, int dir, int idx) {
  return ADD(d.origin[3 * b + dir], MUL((double)idx, dx_of(d, b, dir)));
}

// Map point of the x1/x2 tables: q1/q2 select centre (0), +delta (1),
// -delta (2) or face (3).
__device__ __forceinline__ MapPt map_pt(const Dims &d, int b, int i, int q1, int j, int q2) {
  const int W1 = d.N1 + 1, W2 = d.N2 + 1;
  const double *T1 = d.t1 + (long long)b * kT1Rows * W1;
  const double *T2 = d.t2 + (long long)b * 12 * W2;
  MapPt m;
  m.r = T1[(2 * q1) * W1 + i];
  m.J1 = T1[(2 * q1 + 1) * W1 + i];
  m.sth = T2[(3 * q2) * W2 + j];
  m.cth = T2[(3 * q2 + 1) * W2 + j];
  m.J2 = T2[(3 * q2 + 2) * W2 + j];
  return m;
}

// Covariant code metric at a point given by table selectors (MKS/BL) or
// coordinates (CKS).
template <int MT>
__device__ __forceinline__ void gcov_at(const Dims &d, const pangu_params &p, int b, int i, int q1,
                                        int j, int q2, const double x[4], double g[4][4]) {
  if (MT == MKS) {
    ks_code_gcov(map_pt(d, b, i, q1, j, q2), p.a, g);
  } else if (MT == BL) {
    bl_code_gcov(map_pt(d, b, i, q1, j, q2), p.a, g);
  } else if (MT == CKS) {
    cks_code_gcov(x[1], x[2], x[3], p.a, g);
  } else {
    minkowski_gcov(g);
  }
}

// ---------------------------------------------------------------------------
// Static metric tables. The MKS and BL metrics depend on (x1, x2) only and not
// on time, so ComputeMetricAtLocation (christoffel.h:53-62) and
// ComputeChristoffelConnection (christoffel.h:74-148) are evaluated once per
// (j, i) point by the dense reference arithmetic (k_build_tables) and stored:
// the structurally non-zero entries of gcov (upper triangle: the code metric
// is symmetric bit for bit) and of gcon (every entry: the Gauss-Jordan inverse
// leaves g^rc and g^cr unequal in the last bits in most cells, and the C2P
// schemes read both), gdet, sqrt|gdet|, the lapse 1/sqrt(-gcon00), a validity
// flag (0 where the inversion is singular) and, at cell centres, the
// structurally non-zero Christoffel symbols (symmetric in their lower
// indices). Loads reproduce the dense values bit for bit.
// ---------------------------------------------------------------------------
struct TabLayout {
  int nsym, ncon, nmet, nconn, ncen;
  int sym[4][4];      // slot of g_rc (r, c symmetric), -1 if structurally zero
  int con[4][4];      // slot of g^rc (not symmetric), -1 if structurally zero
  int conn[4][4][4];  // slot of Gamma^a_bc (b, c symmetric), -1 if zero
};

__host__ __device__ constexpr TabLayout tab_layout(int mt) {
  TabLayout L{};
  const Pattern pt = metric_pattern(mt);
  int n = 0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) L.sym[r][c] = -1;
  for (int r = 0; r < 4; ++r)
    for (int c = r; c < 4; ++c)
      if (pt.nz[r][c]) {
        L.sym[r][c] = n;
        L.sym[c][r] = n;
        ++n;
      }
  L.nsym = n;
  int nc = 0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) L.con[r][c] = pt.nz[r][c] ? nc++ : -1;
  L.ncon = nc;
  L.nmet = L.nsym + L.ncon + 4;
  // derivative directions with non-zero metric derivatives
  bool ddir[4] = {false, true, true, mt == CKS};
  if (mt == MINKOWSKI) ddir[1] = ddir[2] = ddir[3] = false;
  bool dg[4][4][4] = {};
  for (int dd = 0; dd < 4; ++dd)
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) dg[dd][r][c] = ddir[dd] && pt.nz[r][c];
  int m = 0;
  for (int a = 0; a < 4; ++a)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) L.conn[a][j][k] = -1;
  for (int a = 0; a < 4; ++a)
    for (int j = 0; j < 4; ++j)
      for (int k = j; k < 4; ++k) {
        bool nz = false;
        for (int l = 0; l < 4; ++l)
          nz = nz || (pt.nz[a][l] && (dg[j][l][k] || dg[k][l][j] || dg[l][j][k]));
        if (nz) {
          L.conn[a][j][k] = m;
          L.conn[a][k][j] = m;
          ++m;
        }
      }
  L.nconn = m;
  L.ncen = L.nmet + m;
  return L;
}

template <int MT>
__device__ __forceinline__ int load_geo(const double *__restrict__ tab, long long plane,
                                        long long off, Geo &g) {
  constexpr TabLayout L = tab_layout(MT);
  double cov[L.nsym], con[L.ncon];
#pragma unroll
  for (int q = 0; q < L.nsym; ++q) cov[q] = __ldg(tab + off + q * plane);
#pragma unroll
  for (int q = 0; q < L.ncon; ++q) con[q] = __ldg(tab + off + (L.nsym + q) * plane);
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      g.gcov[r][c] = L.sym[r][c] >= 0 ? cov[L.sym[r][c]] : 0.0;
      g.gcon[r][c] = L.con[r][c] >= 0 ? con[L.con[r][c]] : 0.0;
    }
  const long long s0 = L.nsym + L.ncon;
  g.gdet = __ldg(tab + off + s0 * plane);
  g.sg = __ldg(tab + off + (s0 + 1) * plane);
  g.alpha = __ldg(tab + off + (s0 + 2) * plane);
  return __ldg(tab + off + (s0 + 3) * plane) != 0.0;
}

#if PGK_MIXED
// load_geo from an FP32 copy of a table: the values geo_cast would give.
template <int MT>
__device__ __forceinline__ int load_geo_f32(const float *__restrict__ tab, long long plane,
                                            long long off, GeoT<float> &g) {
  constexpr TabLayout L = tab_layout(MT);
  float cov[L.nsym], con[L.ncon];
#pragma unroll
  for (int q = 0; q < L.nsym; ++q) cov[q] = __ldg(tab + off + q * plane);
#pragma unroll
  for (int q = 0; q < L.ncon; ++q) con[q] = __ldg(tab + off + (L.nsym + q) * plane);
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      g.gcov[r][c] = L.sym[r][c] >= 0 ? cov[L.sym[r][c]] : 0.0f;
      g.gcon[r][c] = L.con[r][c] >= 0 ? con[L.con[r][c]] : 0.0f;
    }
  const long long s0 = L.nsym + L.ncon;
  g.gdet = __ldg(tab + off + s0 * plane);
  g.sg = __ldg(tab + off + (s0 + 1) * plane);
  g.alpha = __ldg(tab + off + (s0 + 2) * plane);
  return __ldg(tab + off + (s0 + 3) * plane) != 0.0f;
}
#endif

__device__ __forceinline__ void minkowski_geo(Geo &g) {
  minkowski_gcov(g.gcov);
  minkowski_gcov(g.gcon);
  g.gdet = -1.0;
  g.sg = 1.0;
  g.alpha = 1.0;
}

// Dense reference arithmetic at an analytic point (CKS; table building).
template <int MT>
__device__ __forceinline__ int analytic_geo(const Dims &d, const pangu_params &p, int b, int i,
                                            int q1, int j, int q2, const double x[4], Geo &g) {
  gcov_at<MT>(d, p, b, i, q1, j, q2, x, g.gcov);
  const int ok = gj_invert(g.gcov, g.gcon);
  g.gdet = determinant(g.gcov);
  g.sg = sqrt(fabs(g.gdet));
  g.alpha = 1.0 / sqrt(-g.gcon[0][0]);
  return ok;
}

// ComputeMetricAtLocation (christoffel.h:53-62) at cell centre (b, k, j, i).
// Returns 0 if the metric is singular.
template <int MT>
__device__ __forceinline__ int cell_metric(const Dims &d, const pangu_params &p, int b, int k,
                                           int j, int i, Geo &g) {
  if (MT == MKS || MT == BL) {
    constexpr TabLayout L = tab_layout(MT);
    const long long plane = (long long)d.N2 * d.N1;
    return load_geo<MT>(d.ctab, plane, (long long)b * L.ncen * plane + (long long)j * d.N1 + i, g);
  } else if (MT == CKS) {
    const double x[4] = {0.0, xc(d, b, 0, i), xc(d, b, 1, j), xc(d, b, 2, k)};
    return analytic_geo<MT>(d, p, b, i, 0, j, 0, x, g);
  } else {
    minkowski_geo(g);
    return 1;
  }
}

// Metric at the lower face of (b, k, j, i) along dir (1..3).
template <int MT>
__device__ __forceinline__ int face_metric(const Dims &d, const pangu_params &p, int dir, int b,
                                           int k, int j, int i, Geo &g) {
  if (MT == MKS || MT == BL) {
    constexpr TabLayout L = tab_layout(MT);
    if (dir == 1) {
      const long long plane = (long long)d.N2 * (d.N1 + 1);
      return load_geo<MT>(d.f1tab, plane,
                          (long long)b * L.nmet * plane + (long long)j * (d.N1 + 1) + i, g);
    } else if (dir == 2) {
      const long long plane = (long long)(d.N2 + 1) * d.N1;
      return load_geo<MT>(d.f2tab, plane, (long long)b * L.nmet * plane + (long long)j * d.N1 + i,
                          g);
    }
    return cell_metric<MT>(d, p, b, k, j, i, g);  // independent of x3
  } else if (MT == CKS) {
    const double x[4] = {0.0, dir == 1 ? xf(d, b, 0, i) : xc(d, b, 0, i),
                         dir == 2 ? xf(d, b, 1, j) : xc(d, b, 1, j),
                         dir == 3 ? xf(d, b, 2, k) : xc(d, b, 2, k)};
    return analytic_geo<MT>(d, p, b, i, 0, j, 0, x, g);
  } else {
    minkowski_geo(g);
    return 1;
  }
}

// Warp-aggregated increment of a hit counter of `job` (counters are
// [job][PANGU_NCOUNTERS]); a warp may straddle blocks of several jobs.
__device__ __forceinline__ void count(unsigned long long *cnt, int job, int which, bool pred) {
  const unsigned mask = __activemask();
  const unsigned hits = __ballot_sync(mask, pred);
  if (!hits) return;
  const unsigned peers = __match_any_sync(mask, job);
  const unsigned mine = hits & peers;
  if (mine && (threadIdx.x & 31) == (__ffs(peers) - 1))
    atomicAdd(&cnt[job * PANGU_NCOUNTERS + which], (unsigned long long)__popc(mine));
}

// Decomposes a flat index over the box [k0,k1] x [j0,j1] x [i0,i1] of every
// block. Returns false past the end.
__device__ __forceinline__ bool box_index(long long t, int NB, int k0, int k1, int j0, int j1,
                                          int i0, int i1, int &b, int &k, int &j, int &i) {
  const long long ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return false;
  const long long per = ni * nj * nk;
  if (t >= per * NB) return false;
  if (per * NB <= 0x7fffffffLL) {
    // 32-bit unsigned division (a 64-bit one is a long software routine)
    const unsigned ut = (unsigned)t, up = (unsigned)per, uij = (unsigned)(ni * nj),
                   ui = (unsigned)ni;
    const unsigned ub = ut / up;
    unsigned r = ut - ub * up;
    const unsigned uk = r / uij;
    r -= uk * uij;
    const unsigned uj = r / ui;
    b = (int)ub;
    k = k0 + (int)uk;
    j = j0 + (int)uj;
    i = i0 + (int)(r - uj * ui);
    return true;
  }
  b = (int)(t / per);
  long long r = t - (long long)b * per;
  k = k0 + (int)(r / (ni * nj));
  r -= (long long)(k - k0) * ni * nj;
  j = j0 + (int)(r / ni);
  i = i0 + (int)(r - (long long)(j - j0) * ni);
  return true;
}

// q = a / b and r = a % b for a >= 0, b > 0, in 32-bit arithmetic when both
// fit (a 64-bit division is a long software routine).
__device__ __forceinline__ long long div_fast(long long a, long long b, long long &r) {
  if (((a | b) >> 31) == 0) {
    const unsigned q = (unsigned)a / (unsigned)b;
    r = (unsigned)a - q * (unsigned)b;
    return q;
  }
  const long long q = a / b;
  r = a - q * b;
  return q;
}

// Block and in-block offset of a cell offset c = b * ncell + o.
__device__ __forceinline__ void split_cell(long long c, long long ncell, long long &b,
                                           long long &o) {
  if (c <= 0x7fffffffLL && ncell <= 0x7fffffffLL) {
    const unsigned uc = (unsigned)c, un = (unsigned)ncell;
    const unsigned ub = uc / un;
    b = ub;
    o = uc - ub * un;
  } else {
    b = c / ncell;
    o = c - b * ncell;
  }
}

inline unsigned grid_for(long long n) {
  const long long g = (n + kThreads - 1) / kThreads;
  return (unsigned)std::max<long long>(1, std::min<long long>(g, 0x7fffffffLL));
}

// ---------------------------------------------------------------------------
// FixPrimitive (primitive_fixer.cc:15-169), entire domain.
// ---------------------------------------------------------------------------
template <int MT>
// With with_cons set the kernel also computes the conserved variables of the
// interior cells from the primitives it has just stored, which is what
// CalculateConservative (the next task of the stage) would read back
// (with_b = 0: conserved B left as is, see k_calc_cons).
// zero0, zero1 (may be null) are list counters of later tasks of the stage,
// set to 0 here so that the stage needs no memset.
__global__ void __launch_bounds__(kThreads, 4) k_fix_primitive(Dims d, pangu_params p, PT *P,
                                                            unsigned long long *cnt, double *U,
                                                            int with_cons, int with_b, int *zero0,
                                                            int *zero1) {
  pdl_grid_wait();
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0 && zero0) {
    *zero0 = 0;
    *zero1 = 0;
  }
  if (!box_index(t, d.NB, 0, d.N3 - 1, 0, d.N2 - 1, 0, d.N1 - 1, b, k, j, i)) return;
  b = slot_of(d, b);
  const double gam = p.adiabatic_index;
  constexpr double small = 1.0e-20;
  const double sigma_max_safe = kmax(p.sigma_max, small);
  const long long o = coff(d, k, j, i);
  const double rho_before = kmax(a_prim(d, P, b, 0)[o], small);
  double r = 1.0;
  double rho_floor, eng_floor;
  if (MT == MKS) {
    // r = exp(Xc1) and the radial floor profiles, from the host tables
    const double *T1 = d.t1 + (long long)b * kT1Rows * (d.N1 + 1);
    r = T1[i];
    rho_floor = T1[8 * (d.N1 + 1) + i];
    eng_floor = T1[9 * (d.N1 + 1) + i];
  } else if (MT == CKS) {
    const double x = xc(d, b, 0, i), y = xc(d, b, 1, j), z = xc(d, b, 2, k);
    const double a2 = p.a * p.a;
    const double rad2 = x * x + y * y + z * z;
    const double sa = (rad2 - a2) * (rad2 - a2) + 4.0 * a2 * z * z;
    r = sqrt(0.5 * (rad2 - a2 + sqrt(sa)));
    rho_floor = p.density_floor * PGK_POW(fmax(r, 1.0), p.density_floor_pow);
    eng_floor = p.energy_floor * PGK_POW(fmax(r, 1.0), p.energy_floor_pow);
  } else {
    rho_floor = p.density_floor;  // pow(max(1, 1), q) == 1
    eng_floor = p.energy_floor;
  }
  Geo g;
  cell_metric<MT>(d, p, b, k, j, i, g);
  double pc[NPRIM];
  load_prim(d, P, b, k, j, i, pc);
#if PGK_MIXED
  // The mixed form stores these primitives in FP32, and applies the floors,
  // the Lorentz cap and the entropies in FT: the same steps as below, with
  // the metric rounded once (geo_cast) and the CUDA math library's float pow.
  // Measured 5-6 % per RK2 cycle on the 2D and 3D tori and the 48-torus batch
  // against the same steps in FP64.
  double pr, pu, u1, u2, u3, ent, kel;
  bool hit_r, hit_u, cap;
  {
    GeoT<FT> gf;
    geo_cast<MT>(g, gf);
    FT q[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; ++v) q[v] = (FT)pc[v];
    StateT<FT> sf;
    calc_state_t<MT>(q, gf, sf);
    const FT gamf = (FT)gam, smallf = (FT)small, smax = (FT)sigma_max_safe;
    FT rfl = (FT)rho_floor;
    const FT efl = (FT)eng_floor;
    if (rfl < q[ENY] / smax) rfl = q[ENY] / smax;
    if (sf.bsq / q[RHO] > (FT)p.sigma_max) rfl = sf.bsq / smax;
    FT rr = q[RHO], uu = q[ENY];
    hit_r = rr < rfl;
    if (hit_r) rr = rfl;
    hit_u = uu < efl;
    if (hit_u) uu = efl;
    FT v1 = q[UX1], v2 = q[UX2], v3 = q[UX3];
    const FT umax2 = (FT)(p.lorentz_max * p.lorentz_max - 1.0);
    constexpr Pattern PAT = metric_pattern(MT);
    FT uvsq = gf.gcov[1][1] * v1 * v1 + gf.gcov[2][2] * v2 * v2 + gf.gcov[3][3] * v3 * v3;
    if (PAT.nz[1][2] || PAT.nz[1][3] || PAT.nz[2][3]) {
      FT cross = FT(0);
      if (PAT.nz[1][2]) cross = cross + gf.gcov[1][2] * v1 * v2;
      if (PAT.nz[1][3]) cross = cross + gf.gcov[1][3] * v1 * v3;
      if (PAT.nz[2][3]) cross = cross + gf.gcov[2][3] * v2 * v3;
      uvsq = uvsq + FT(2) * cross;
    }
    cap = umax2 > FT(0) && uvsq > umax2;
    if (cap) {
      const FT f = sqrt(umax2 / tmax(uvsq, smallf));
      v1 *= f;
      v2 *= f;
      v3 *= f;
    }
    const FT rho_after = tmax(rr, smallf);
    FT kf = q[KEL];
    if (p.enable_heating && rho_after != (FT)rho_before)
      kf *= tpow(rho_after / (FT)rho_before, -gamf);
    FT ef = (gamf - FT(1)) * uu * tpow(rr, -gamf);
    kel = kf;
    if (p.enable_heating) kel = clamp_by_ratio(p.ratio_min, p.ratio_max, (double)ef, kel);
    pr = rr;
    pu = uu;
    u1 = v1;
    u2 = v2;
    u3 = v3;
    ent = ef;
  }
  if (MT == CKS && r < p.r_excise) {
    const double e_excise = p.pexcise / (gam - 1.0);
    pr = p.dexcise;
    pu = e_excise;
    u1 = u2 = u3 = 0.0;
    ent = (FT)(gam - 1.0) * (FT)e_excise * tpow((FT)p.dexcise, -(FT)gam);
    if (p.enable_heating) kel = e_excise;
  }
#else
  const double rho = pc[RHO], ug = pc[ENY];
  State st;
  calc_state<MT>(pc, g, st);
  if (rho_floor < ug / sigma_max_safe) rho_floor = ug / sigma_max_safe;
  const double sigma = st.bsq / rho;
  if (sigma > p.sigma_max) rho_floor = st.bsq / sigma_max_safe;
  double pr = pc[RHO], pu = pc[ENY];
  const bool hit_r = pr < rho_floor;
  if (hit_r) pr = rho_floor;
  const bool hit_u = pu < eng_floor;
  if (hit_u) pu = eng_floor;
  double u1 = pc[UX1], u2 = pc[UX2], u3 = pc[UX3];
  const double umax2 = p.lorentz_max * p.lorentz_max - 1.0;
  // primitive_fixer.cc:131-134; structurally zero cross terms skipped
  constexpr Pattern PAT = metric_pattern(MT);
  double uvsq = g.gcov[1][1] * u1 * u1 + g.gcov[2][2] * u2 * u2 + g.gcov[3][3] * u3 * u3;
  if (PAT.nz[1][2] || PAT.nz[1][3] || PAT.nz[2][3]) {
    double cross = 0.0;
    if (PAT.nz[1][2]) cross = cross + g.gcov[1][2] * u1 * u2;
    if (PAT.nz[1][3]) cross = cross + g.gcov[1][3] * u1 * u3;
    if (PAT.nz[2][3]) cross = cross + g.gcov[2][3] * u2 * u3;
    uvsq = uvsq + 2.0 * cross;
  }
  const bool cap = umax2 > 0.0 && uvsq > umax2;
  if (cap) {
    const double f = sqrt(umax2 / kmax(uvsq, small));
    u1 *= f;
    u2 *= f;
    u3 *= f;
  }
  const double rho_after = kmax(pr, small);
  double kel = pc[KEL];
  if (p.enable_heating && rho_after != rho_before) kel *= PGK_POW(rho_after / rho_before, -gam);
  double ent = (gam - 1.0) * pu * PGK_POW(pr, -gam);
  if (p.enable_heating) kel = clamp_by_ratio(p.ratio_min, p.ratio_max, ent, kel);
  if (MT == CKS && r < p.r_excise) {
    const double e_excise = p.pexcise / (gam - 1.0);
    pr = p.dexcise;
    pu = e_excise;
    u1 = u2 = u3 = 0.0;
    ent = (gam - 1.0) * e_excise * PGK_POW(p.dexcise, -gam);
    if (p.enable_heating) kel = e_excise;
  }
#endif
  a_prim(d, P, b, 0)[o] = pr;
  a_prim(d, P, b, 1)[o] = pu;
  a_prim(d, P, b, 2)[o] = u1;
  a_prim(d, P, b, 3)[o] = u2;
  a_prim(d, P, b, 4)[o] = u3;
  a_prim(d, P, b, d.pidx[ENT])[o] = ent;
  if (p.enable_heating) a_prim(d, P, b, d.pidx[KEL])[o] = kel;
  count(cnt, job_of(d, b), PANGU_CNT_RHO_FLOOR, hit_r);
  count(cnt, job_of(d, b), PANGU_CNT_ENG_FLOOR, hit_u);
  count(cnt, job_of(d, b), PANGU_CNT_LORENTZ_CAP, cap);
  if (with_cons && k >= d.ks && k <= d.ke && j >= d.js && j <= d.je && i >= d.is && i <= d.ie) {
    // the stored values, as a reload would see them
    double pf[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; ++v) pf[v] = pc[v];
    pf[RHO] = (PT)pr;
    pf[ENY] = (PT)pu;
    pf[UX1] = (PT)u1;
    pf[UX2] = (PT)u2;
    pf[UX3] = (PT)u3;
    pf[ENT] = (PT)ent;
    if (p.enable_heating) pf[KEL] = (PT)kel;
    State sf;
    calc_state<MT>(pf, g, sf);
    double f[NPRIM];
    flux_from_state(gam, pf, sf, g.sg, 0, f);
#pragma unroll
    for (int v = 0; v < NPRIM; ++v)
      if (d.pidx[v] >= 0 && (with_b || v < BX1 || v > BX3)) a_cons(d, U, b, d.pidx[v])[o] = f[v];
  }
}

// ---------------------------------------------------------------------------
// CalculateConservative (conservative.cc:15-110), interior.
// ---------------------------------------------------------------------------
template <int MT>
// with_b = 0 leaves the conserved magnetic field as it is: the mixed form
// evolves B only through the FP64 flux-CT update, because rebuilding it from
// FP32-stored primitives every stage would add FP32 rounding to div B.
__global__ void __launch_bounds__(kThreads) k_calc_cons(Dims d, pangu_params p, const PT *P,
                                                        double *U, int with_b) {
  pdl_grid_wait();
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, b, k, j, i)) return;
  b = slot_of(d, b);
  Geo g;
  cell_metric<MT>(d, p, b, k, j, i, g);
  double pc[NPRIM];
  load_prim(d, P, b, k, j, i, pc);
  State s;
  calc_state<MT>(pc, g, s);
  double f[NPRIM];
  flux_from_state(p.adiabatic_index, pc, s, g.sg, 0, f);
#pragma unroll
  for (int v = 0; v < NPRIM; ++v)
    if (d.pidx[v] >= 0 && (with_b || v < BX1 || v > BX3))
      a_cons(d, U, b, d.pidx[v])[coff(d, k, j, i)] = f[v];
}

// ---------------------------------------------------------------------------
// CalculateLAXF / CalculateHLL (laxf.cc:78-393, hll.cc:78-399).
//
// Each cell's reconstruction is computed once and shared by its two faces
// (the reference calls MC/PPM4 twice per variable and face,
// laxf.cc:86-105): x1 faces by warp shuffles, x2/x3 faces by marching along
// the column. The Riemann flux is then assembled component by component
// from the two states, in the reference's operation order.
// ---------------------------------------------------------------------------

// Riemann solver and limiter of an FP64 flux kernel instance, fixed at
// compile time so that the other option's arithmetic is not in the kernel
// (measured 3.4 % per RK2 cycle on the 3D torus against runtime flags): bit 0
// HLL (else LAXF), bit 1 MC (else PPM4). The mixed form keeps runtime flags
// (one instance, OPT 0): compiled in, the options change ptxas's contraction
// choices there, and its errors against FP64 came out larger (entropies
// 2.0e-2 against 6.9e-3 on the MC/HLL torus after 10 cycles).
constexpr int kFluxHLL = 1, kFluxMC = 2;
#if PGK_MIXED
#define PGK_FLUX_HLL(p) ((p).riemann_solver == PANGU_RIEMANN_HLL)
#define PGK_FLUX_MC(p) ((p).limiter == PANGU_LIMITER_MC)
#else
#define PGK_FLUX_HLL(p) ((OPT & kFluxHLL) != 0)
#define PGK_FLUX_MC(p) ((OPT & kFluxMC) != 0)
#endif

// Reconstruction of one variable in cell q (stride s along the direction):
// ql_ip1 = value at the upper face, qr_i = value at the lower face
// (interpolater_mc.h:38-48, interpolater_ppm4.h:29-67).
__device__ __forceinline__ void recon_cell(bool use_mc, const PT *q, long long s, FT &ql_ip1,
                                           FT &qr_i) {
#if PGK_MIXED
  if (use_mc) {
    mc_t<FT>(q[-s], q[0], q[s], ql_ip1, qr_i);
  } else {
    ppm4_t<FT>(q[-2 * s], q[-s], q[0], q[s], q[2 * s], ql_ip1, qr_i);
  }
#else
  if (use_mc) {
    mc(q[-s], q[0], q[s], ql_ip1, qr_i);
  } else {
    ppm4(q[-2 * s], q[-s], q[0], q[s], q[2 * s], ql_ip1, qr_i);
  }
#endif
}

// One flux component from a state (contravariant_flux.h:12-39).
template <int c>
__device__ __forceinline__ double flux_component(double gam, const double P[NPRIM],
                                                 const State &s, double sg, int dir) {
  const double f_rho = P[RHO] * s.ucon[dir];
  if (c == RHO) return f_rho * sg;
  if (c == ENT) return (P[ENT] * f_rho) * sg;
  if (c == KEL) return (P[KEL] * f_rho) * sg;
  if (c >= BX1 && c <= BX3) {
    const int m = c - BX1 + 1;
    return SUB(MUL(s.bcon[m], s.ucon[dir]), MUL(s.bcon[dir], s.ucon[m])) * sg;
  }
  const double hh = P[RHO] + gam * P[ENY];
  const double e_tot = hh + s.bsq;
  const double p_tot = (gam - 1.) * P[ENY] + 0.5 * s.bsq;
  const int m = (c == ENY) ? 0 : c - UX1 + 1;
  const double t = e_tot * s.ucon[dir] * s.ucov[m] + p_tot * (dir == m) - s.bcon[dir] * s.bcov[m];
  if (c == ENY) return (t + f_rho) * sg;
  return t * sg;
}

#if PGK_MIXED
// One flux component from a state in FT arithmetic (contravariant_flux.h:12-39).
template <int c>
__device__ __forceinline__ FT flux_component_t(FT gam, const FT P[NPRIM], const StateT<FT> &s,
                                               FT sg, int dir) {
  const FT f_rho = P[RHO] * s.ucon[dir];
  if (c == RHO) return f_rho * sg;
  if (c == ENT) return (P[ENT] * f_rho) * sg;
  if (c == KEL) return (P[KEL] * f_rho) * sg;
  if (c >= BX1 && c <= BX3) {
    const int m = c - BX1 + 1;
    return (s.bcon[m] * s.ucon[dir] - s.bcon[dir] * s.ucon[m]) * sg;
  }
  const FT hh = P[RHO] + gam * P[ENY];
  const FT e_tot = hh + s.bsq;
  const FT p_tot = (gam - FT(1)) * P[ENY] + FT(0.5) * s.bsq;
  const int m = (c == ENY) ? 0 : c - UX1 + 1;
  const FT t = e_tot * s.ucon[dir] * s.ucov[m] + p_tot * FT(dir == m) - s.bcon[dir] * s.bcov[m];
  if (c == ENY) return (t + f_rho) * sg;
  return t * sg;
}

// Riemann flux and fast speed at the lower face of (b, k, j, i) along DIR in
// FT arithmetic; the metric is evaluated in FP64 and rounded once.
template <int MT, int DIR, int OPT>
__device__ __forceinline__ void face_flux(const Dims &d, const pangu_params &p, int b, int k, int j,
                                          int i, const FT PL[NPRIM], const FT PR[NPRIM],
                                          double *F, double *alfven) {
  const long long fo = coff(d, k, j, i);
  GeoT<FT> g;
  int ok;
  if ((MT == MKS || MT == BL) && DIR != 3) {
    // the FP32 face tables (pool_init builds them for every mixed engine)
    constexpr TabLayout L = tab_layout(MT);
    if (DIR == 1) {
      const long long plane = (long long)d.N2 * (d.N1 + 1);
      ok = load_geo_f32<MT>(d.f1tab32, plane,
                            (long long)b * L.nmet * plane + (long long)j * (d.N1 + 1) + i, g);
    } else {
      const long long plane = (long long)(d.N2 + 1) * d.N1;
      ok = load_geo_f32<MT>(d.f2tab32, plane, (long long)b * L.nmet * plane + (long long)j * d.N1 + i,
                            g);
    }
  } else {
    Geo g64;
    ok = face_metric<MT>(d, p, DIR, b, k, j, i, g64);
    if (ok) geo_cast<MT>(g64, g);
  }
  if (!ok) {
    a_alfven(d, alfven, b, DIR - 1)[fo] = 0.0;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s)
      if (d.pidx[s] >= 0) a_flux(d, F, b, d.pidx[s])[fo] = 0.0;
    return;
  }
  const FT gam = (FT)p.adiabatic_index;
  const FT sg = g.sg;
  StateT<FT> sL, sR;
  calc_state_t<MT>(PL, g, sL);
  calc_state_t<MT>(PR, g, sR);
  FT vmaxL, vminL, vmaxR, vminR;
  fast_speed_t<FT>(gam, PL, g, sL, DIR, vmaxL, vminL);
  fast_speed_t<FT>(gam, PR, g, sR, DIR, vmaxR, vminR);
  const FT cmax = fabs(tmax(tmax(FT(0), vmaxL), vmaxR));
  const FT cmin = fabs(tmax(tmax(FT(0), -vminL), -vminR));
  const FT cms = tmax(cmax, cmin);
  a_alfven(d, alfven, b, DIR - 1)[fo] = cms;
  const bool hll = PGK_FLUX_HLL(p);
  const FT ihll = FT(1) / (cmax + cmin + FT(1e-20));
#define PGD_FACE_COMPONENT(C)                                                         \
  if (d.pidx[C] >= 0) {                                                               \
    const FT fl = flux_component_t<C>(gam, PL, sL, sg, DIR);                          \
    const FT fr = flux_component_t<C>(gam, PR, sR, sg, DIR);                          \
    const FT ul = flux_component_t<C>(gam, PL, sL, sg, 0);                            \
    const FT ur = flux_component_t<C>(gam, PR, sR, sg, 0);                            \
    a_flux(d, F, b, d.pidx[C])[fo] =                                                     \
        hll ? (cmax * fl + cmin * fr - cmax * cmin * (ur - ul)) * ihll                 \
            : FT(0.5) * (fl + fr - cms * (ur - ul));                                   \
  }
  PGD_FACE_COMPONENT(RHO)
  PGD_FACE_COMPONENT(ENY)
  PGD_FACE_COMPONENT(UX1)
  PGD_FACE_COMPONENT(UX2)
  PGD_FACE_COMPONENT(UX3)
  PGD_FACE_COMPONENT(BX1)
  PGD_FACE_COMPONENT(BX2)
  PGD_FACE_COMPONENT(BX3)
  PGD_FACE_COMPONENT(ENT)
  PGD_FACE_COMPONENT(KEL)
#undef PGD_FACE_COMPONENT
}
#else
// Riemann flux and fast speed at the lower face of (b, k, j, i) along DIR
// from the left and right states.
template <int MT, int DIR, int OPT>
__device__ __forceinline__ void face_flux(const Dims &d, const pangu_params &p, int b, int k, int j,
                                          int i, const double PL[NPRIM], const double PR[NPRIM],
                                          double *F, double *alfven) {
  Geo g;
  const long long fo = coff(d, k, j, i);
  if (!face_metric<MT>(d, p, DIR, b, k, j, i, g)) {
    // Singular code metric (theta = 0 exactly on a polar face): zero flux,
    // zero speed (the reference reads an unwritten inverse here).
    a_alfven(d, alfven, b, DIR - 1)[fo] = 0.0;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s)
      if (d.pidx[s] >= 0) a_flux(d, F, b, d.pidx[s])[fo] = 0.0;
    return;
  }
  const double gam = p.adiabatic_index;
  const double sg = g.sg;
  State sL, sR;
  calc_state<MT>(PL, g, sL);
  calc_state<MT>(PR, g, sR);
  double vmaxL, vminL, vmaxR, vminR;
  fast_speed_from_state(gam, PL, g, sL, DIR, vmaxL, vminL);
  fast_speed_from_state(gam, PR, g, sR, DIR, vmaxR, vminR);
  const double cmax = fabs(kmax(kmax(0., vmaxL), vmaxR));
  const double cmin = fabs(kmax(kmax(0., -vminL), -vminR));
  const double cms = kmax(cmax, cmin);
  a_alfven(d, alfven, b, DIR - 1)[fo] = cms;
  const bool hll = PGK_FLUX_HLL(p);
#define PGD_FACE_COMPONENT(C)                                                         \
  if (d.pidx[C] >= 0) {                                                               \
    const double fl = flux_component<C>(gam, PL, sL, sg, DIR);                        \
    const double fr = flux_component<C>(gam, PR, sR, sg, DIR);                        \
    const double ul = flux_component<C>(gam, PL, sL, sg, 0);                          \
    const double ur = flux_component<C>(gam, PR, sR, sg, 0);                          \
    a_flux(d, F, b, d.pidx[C])[fo] =                                                     \
        hll ? (cmax * fl + cmin * fr - cmax * cmin * (ur - ul)) / (cmax + cmin + 1e-20) \
            : 0.5 * (fl + fr - cms * (ur - ul));                                      \
  }
  PGD_FACE_COMPONENT(RHO)
  PGD_FACE_COMPONENT(ENY)
  PGD_FACE_COMPONENT(UX1)
  PGD_FACE_COMPONENT(UX2)
  PGD_FACE_COMPONENT(UX3)
  PGD_FACE_COMPONENT(BX1)
  PGD_FACE_COMPONENT(BX2)
  PGD_FACE_COMPONENT(BX3)
  PGD_FACE_COMPONENT(ENT)
  PGD_FACE_COMPONENT(KEL)
#undef PGD_FACE_COMPONENT
}

// face_flux with the two sides evaluated one after the other through shared
// memory, so that only one side's state is held in registers at a time.
// On entry sl[s * ss] holds the left state and sr[s * ss] the right one; the
// left side's fluxes go to sl (over its state) and its conserved values to
// su, and the right side combines them with its own. Every value is the one
// face_flux computes, from the same operations on the same operands.
template <int MT, int DIR, int OPT>
__device__ __forceinline__ void face_flux_split(const Dims &d, const pangu_params &p, int b, int k,
                                                int j, int i, double *sl, const double *sr,
                                                double *su, int ss, double *F, double *alfven) {
  Geo g;
  const long long fo = coff(d, k, j, i);
  if (!face_metric<MT>(d, p, DIR, b, k, j, i, g)) {
    a_alfven(d, alfven, b, DIR - 1)[fo] = 0.0;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s)
      if (d.pidx[s] >= 0) a_flux(d, F, b, d.pidx[s])[fo] = 0.0;
    return;
  }
  const double gam = p.adiabatic_index;
  const double sg = g.sg;
  double vmaxL, vminL;
  {
    double P[NPRIM];
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) P[s] = sl[s * ss];
    State st;
    calc_state<MT>(P, g, st);
    fast_speed_from_state(gam, P, g, st, DIR, vmaxL, vminL);
#define PGD_LEFT_COMPONENT(C)                                 \
  if (d.pidx[C] >= 0) {                                       \
    sl[C * ss] = flux_component<C>(gam, P, st, sg, DIR);      \
    su[C * ss] = flux_component<C>(gam, P, st, sg, 0);        \
  }
    PGD_LEFT_COMPONENT(RHO)
    PGD_LEFT_COMPONENT(ENY)
    PGD_LEFT_COMPONENT(UX1)
    PGD_LEFT_COMPONENT(UX2)
    PGD_LEFT_COMPONENT(UX3)
    PGD_LEFT_COMPONENT(BX1)
    PGD_LEFT_COMPONENT(BX2)
    PGD_LEFT_COMPONENT(BX3)
    PGD_LEFT_COMPONENT(ENT)
    PGD_LEFT_COMPONENT(KEL)
#undef PGD_LEFT_COMPONENT
  }
  // the right side reads the left side's results back from shared memory
  asm volatile("" ::: "memory");
  double P[NPRIM];
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) P[s] = sr[s * ss];
  State st;
  calc_state<MT>(P, g, st);
  double vmaxR, vminR;
  fast_speed_from_state(gam, P, g, st, DIR, vmaxR, vminR);
  const double cmax = fabs(kmax(kmax(0., vmaxL), vmaxR));
  const double cmin = fabs(kmax(kmax(0., -vminL), -vminR));
  const double cms = kmax(cmax, cmin);
  a_alfven(d, alfven, b, DIR - 1)[fo] = cms;
  const bool hll = PGK_FLUX_HLL(p);
#define PGD_RIGHT_COMPONENT(C)                                                        \
  if (d.pidx[C] >= 0) {                                                               \
    const double fl = sl[C * ss];                                                     \
    const double fr = flux_component<C>(gam, P, st, sg, DIR);                         \
    const double ul = su[C * ss];                                                     \
    const double ur = flux_component<C>(gam, P, st, sg, 0);                           \
    a_flux(d, F, b, d.pidx[C])[fo] =                                                     \
        hll ? (cmax * fl + cmin * fr - cmax * cmin * (ur - ul)) / (cmax + cmin + 1e-20) \
            : 0.5 * (fl + fr - cms * (ur - ul));                                      \
  }
  PGD_RIGHT_COMPONENT(RHO)
  PGD_RIGHT_COMPONENT(ENY)
  PGD_RIGHT_COMPONENT(UX1)
  PGD_RIGHT_COMPONENT(UX2)
  PGD_RIGHT_COMPONENT(UX3)
  PGD_RIGHT_COMPONENT(BX1)
  PGD_RIGHT_COMPONENT(BX2)
  PGD_RIGHT_COMPONENT(BX3)
  PGD_RIGHT_COMPONENT(ENT)
  PGD_RIGHT_COMPONENT(KEL)
#undef PGD_RIGHT_COMPONENT
}
#endif

// x1 faces: a warp covers 31 consecutive faces of one row. Lane l
// reconstructs cell c = f0 - 1 + l; face c takes its left state from lane
// l - 1 (upper-face value of cell c - 1) and its right state from lane l.
constexpr int kFacesPerWarp = 31;
// Flux kernels holding both states of a face in registers: at most 128
// registers (4 CTAs of 4 warps per SM, a few spills). For them, bounds of 3
// CTAs (168 registers) and of 5 or 6 (96 or 80) were measured slower on the
// 2D torus (the latter two faster on the 3D one).
constexpr int kFluxThreads = 128;
// With one side's state in registers at a time (FP64, curved metrics) the
// flux kernels run at 5 CTAs per SM (96 registers): measured 1.1 % faster per
// cycle on the 2D and the 3D torus than both states at 4 CTAs (at 4 CTAs the
// split alone gained nothing); on Minkowski (Orszag-Tang) it cost 1.6 %, so
// it is not used there.
constexpr bool split_faces(int mt) { return PGK_SPLIT_FACES && mt != MINKOWSKI; }
constexpr int flux_blocks(int mt) { return split_faces(mt) ? 5 : 4; }

template <int MT, int OPT>
__global__ void __launch_bounds__(kFluxThreads, flux_blocks(MT)) k_flux_x1(Dims d, pangu_params p, int k0, int k1,
                                                      int j0, int j1, int i0, int i1,
                                                      const PT *P, double *F,
                                                      double *alfven) {
  pdl_grid_wait();
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nf = i1 - i0 + 1;
  const int nseg = (nf + kFacesPerWarp - 1) / kFacesPerWarp;
  const long long nrow = (long long)(k1 - k0 + 1) * (j1 - j0 + 1);
  if (warp >= nrow * d.NB * nseg) return;  // whole warps exit together
  long long seg_l, rr, jr;
  const long long row = div_fast(warp, nseg, seg_l);
  const int seg = (int)seg_l;
  const int bb = (int)div_fast(row, nrow, rr);
  const int b = slot_of(d, bb);
  const int k = k0 + (int)div_fast(rr, j1 - j0 + 1, jr);
  const int j = j0 + (int)jr;
  const int c = i0 - 1 + seg * kFacesPerWarp + lane;
  const bool active = c <= i1;  // cell c is needed by face c (and c + 1)
  const bool use_mc = PGK_FLUX_MC(p);
#if PGK_SPLIT_FACES
  if (split_faces(MT)) {
    // [3][NPRIM][blockDim.x]: upper-face values, lower-face values, and the
    // left side's conserved values of face c. Face c reads the upper-face
    // values of lane - 1, which no other lane reads, and writes its left
    // fluxes over them.
    extern __shared__ double fsm[];
    const int ss = blockDim.x, t = threadIdx.x;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) {
      FT up = 0, lo = 0;
      if (d.pidx[s] >= 0 && active)
        recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, k, j, c), 1, up, lo);
      fsm[s * ss + t] = up;
      fsm[(NPRIM + s) * ss + t] = lo;
    }
    __syncwarp();
    if (lane == 0 || !active) return;
    face_flux_split<MT, 1, OPT>(d, p, b, k, j, c, fsm + t - 1, fsm + NPRIM * ss + t,
                           fsm + 2 * NPRIM * ss + t, ss, F, alfven);
    return;
  }
#endif
  FT PL[NPRIM], PR[NPRIM];
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) {
    FT up = 0, lo = 0;
    if (d.pidx[s] >= 0 && active)
      recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, k, j, c), 1, up, lo);
    PL[s] = __shfl_up_sync(0xffffffffu, up, 1);
    PR[s] = lo;
  }
  if (lane == 0 || !active) return;
  face_flux<MT, 1, OPT>(d, p, b, k, j, c, PL, PR, F, alfven);
}

// x2 / x3 faces: a thread marches over MARCH consecutive faces of one
// column, carrying the upper-face value of the previous cell. A deeper march
// reconstructs fewer cells twice but gives fewer threads; the autotuner picks
// the depth (and the CTA size) for the engine's grid.
template <int MT, int DIR, int MARCH, int OPT>
__device__ __forceinline__ void flux_march_body(const Dims &d, const pangu_params &p, int k0,
                                                int k1, int j0, int j1, int i0, int i1,
                                                const PT *P, double *F, double *alfven) {
  // the marching index is j (DIR 2) or k (DIR 3); the other two form the column
  const int m0 = DIR == 2 ? j0 : k0, m1 = DIR == 2 ? j1 : k1;
  const int a0 = DIR == 2 ? k0 : j0, a1 = DIR == 2 ? k1 : j1;  // outer transverse index
  const int ni = i1 - i0 + 1, na = a1 - a0 + 1;
  const int nruns = (m1 - m0 + 1 + MARCH - 1) / MARCH;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.NB * na * nruns * ni) return;
  long long ir, runr, ar;
  long long r = div_fast(t, ni, ir);
  const int i = i0 + (int)ir;
  r = div_fast(r, nruns, runr);
  const int run = (int)runr;
  const int b = slot_of(d, (int)div_fast(r, na, ar));
  const int a = a0 + (int)ar;
  const long long stride = DIR == 2 ? (long long)d.N1 : (long long)d.N1 * d.N2;
  const bool use_mc = PGK_FLUX_MC(p);
  const int f0 = m0 + run * MARCH;
  const int f1 = min(f0 + MARCH - 1, m1);
#if PGK_SPLIT_FACES
  if (split_faces(MT)) {
    // [4][NPRIM][blockDim.x], each thread's own: the upper-face values of the
    // previous cell (then the left fluxes), the lower-face values of this
    // cell, the left conserved values, and the upper-face values of this cell.
    extern __shared__ double fsm[];
    const int ss = blockDim.x;
    double *carry = fsm + threadIdx.x, *next = fsm + 3 * NPRIM * ss + threadIdx.x;
    double *lower = fsm + NPRIM * ss + threadIdx.x;
    double *left_u = fsm + 2 * NPRIM * ss + threadIdx.x;
    {
      const int c = f0 - 1;
      const int kk = DIR == 2 ? a : c, jj = DIR == 2 ? c : a;
#pragma unroll
      for (int s = 0; s < NPRIM; ++s) {
        FT up = 0, lo;
        if (d.pidx[s] >= 0)
          recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, kk, jj, i), stride, up, lo);
        carry[s * ss] = up;
      }
    }
    for (int f = f0; f <= f1; ++f) {
      const int kk = DIR == 2 ? a : f, jj = DIR == 2 ? f : a;
#pragma unroll
      for (int s = 0; s < NPRIM; ++s) {
        FT up = 0, lo = 0;
        if (d.pidx[s] >= 0)
          recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, kk, jj, i), stride, up, lo);
        next[s * ss] = up;
        lower[s * ss] = lo;
      }
      face_flux_split<MT, DIR, OPT>(d, p, b, kk, jj, i, carry, lower, left_u, ss, F, alfven);
      double *tmp = carry;
      carry = next;
      next = tmp;
    }
    return;
  }
#endif
  FT carry[NPRIM];
  {
    const int c = f0 - 1;
    const int kk = DIR == 2 ? a : c, jj = DIR == 2 ? c : a;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) {
      FT up = 0, lo;
      if (d.pidx[s] >= 0) recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, kk, jj, i), stride, up, lo);
      carry[s] = up;
    }
  }
  for (int f = f0; f <= f1; ++f) {
    const int kk = DIR == 2 ? a : f, jj = DIR == 2 ? f : a;
    FT PR[NPRIM], up[NPRIM];
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) {
      up[s] = 0.0;
      PR[s] = 0.0;
      if (d.pidx[s] >= 0)
        recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, kk, jj, i), stride, up[s], PR[s]);
    }
    face_flux<MT, DIR, OPT>(d, p, b, kk, jj, i, carry, PR, F, alfven);
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) carry[s] = up[s];
  }
}

// x2 / x3 faces by tiles: a CTA of 32 x TF threads reconstructs each cell of
// a tile of 32 consecutive i by TF + 1 cells along the face direction once,
// into shared memory, then computes the TF x 32 faces from the stored upper
// and lower values (a march reconstructs (MARCH + 1) / MARCH cells per face,
// a tile (TF + 1) / TF). The face arithmetic is face_flux's, so the results
// are those of the march kernels.
template <int MT, int DIR, int TF, int OPT>
__device__ __forceinline__ void flux_tile_body(const Dims &d, const pangu_params &p, int k0, int k1,
                                               int j0, int j1, int i0, int i1, const PT *P,
                                               double *F, double *alfven) {
  __shared__ FT sup[TF + 1][NPRIM][32], slo[TF + 1][NPRIM][32];
  const int m0 = DIR == 2 ? j0 : k0, m1 = DIR == 2 ? j1 : k1;
  const int a0 = DIR == 2 ? k0 : j0, a1 = DIR == 2 ? k1 : j1;
  const int ni = i1 - i0 + 1, na = a1 - a0 + 1, nm = m1 - m0 + 1;
  const int nti = (ni + 31) / 32, ntm = (nm + TF - 1) / TF;
  long long ti, tm, al;
  long long r = div_fast(blockIdx.x, nti, ti);
  r = div_fast(r, ntm, tm);
  const long long bb = div_fast(r, na, al);
  if (bb >= d.NB) return;  // whole CTAs exit together
  const int b = slot_of(d, (int)bb);
  const int a = a0 + (int)al;
  const int mt0 = m0 + (int)tm * TF;
  const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
  const int i = i0 + (int)ti * 32 + lane;
  const long long stride = DIR == 2 ? (long long)d.N1 : (long long)d.N1 * d.N2;
  const bool use_mc = PGK_FLUX_MC(p);
  // cells mt0 - 1 .. mt0 + TF - 1: the lower neighbour of every face of the tile
  for (int cr = row; cr <= TF; cr += TF) {
    const int c = mt0 - 1 + cr;
    if (i <= i1 && c <= m1) {
      const int kk = DIR == 2 ? a : c, jj = DIR == 2 ? c : a;
#pragma unroll
      for (int s = 0; s < NPRIM; ++s) {
        FT up = 0, lo = 0;
        if (d.pidx[s] >= 0) recon_cell(use_mc, a_prim(d, P, b, d.pidx[s]) + coff(d, kk, jj, i), stride, up, lo);
        sup[cr][s][lane] = up;
        slo[cr][s][lane] = lo;
      }
    }
  }
  __syncthreads();
  const int f = mt0 + row;
  if (i > i1 || f > m1) return;
  const int kk = DIR == 2 ? a : f, jj = DIR == 2 ? f : a;
#if PGK_SPLIT_FACES
  // sup[row][.][lane] and slo[row + 1][.][lane] are read by this thread only.
  // Tiles of 8 rows keep both states in registers (their static shared
  // memory would pass 48 KB).
  constexpr bool split = split_faces(MT) && TF <= 4;
  __shared__ double sul[split ? TF : 1][NPRIM][32];
  if (split) {
    face_flux_split<MT, DIR, OPT>(d, p, b, kk, jj, i, &sup[row][0][lane], &slo[row + 1][0][lane],
                             &sul[split ? row : 0][0][lane], 32, F, alfven);
    return;
  }
#endif
  FT PL[NPRIM], PR[NPRIM];
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) {
    PL[s] = sup[row][s][lane];
    PR[s] = slo[row + 1][s][lane];
  }
  face_flux<MT, DIR, OPT>(d, p, b, kk, jj, i, PL, PR, F, alfven);
}

template <int MT, int DIR, int TF, int OPT>
__global__ void __launch_bounds__(32 * TF, TF == 4 ? flux_blocks(MT) : 2) k_flux_tile(Dims d, pangu_params p, int k0,
                                                                     int k1, int j0, int j1, int i0,
                                                                     int i1, const PT *P, double *F,
                                                                     double *alfven) {
  pdl_grid_wait();
  flux_tile_body<MT, DIR, TF, OPT>(d, p, k0, k1, j0, j1, i0, i1, P, F, alfven);
}

// ---------------------------------------------------------------------------
// Flux kernels whose primitives are staged into shared memory by TMA: one
// cp.async.bulk.tensor load per CTA brings every component of the cells the
// CTA's stencils reach from this GPU's memory, completing on an mbarrier; the
// threads then reconstruct from shared memory (recon_cell reads the stencil
// there) and evaluate their faces with face_flux / face_flux_split, so the
// results are those of the other flux kernels bit for bit. No multicast: each
// load reads this GPU's own memory and serves one CTA.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int c0, int c1,
                                            int c2, int c3, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_u32(bar))
      : "memory");
}

// Elements per 16 bytes: a copy's first column is rounded down to a multiple.
constexpr int kTmaAlign = 16 / (int)sizeof(PT);
// Bound on the mbarrier wait (polls of try_wait, each of which suspends for
// a while itself): far beyond any copy's completion; past it the kernel
// records an error and returns instead of waiting on.
constexpr long long kTmaWaitPolls = 1ll << 26;

// Waits for the CTA's copy; false (after recording the error) if the bound
// ran out.
__device__ __forceinline__ bool tma_wait(unsigned long long *bar, int *err) {
  long long polls = 0;
  while (!mbar_try_wait(bar, 0))
    if (++polls == kTmaWaitPolls) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      return false;
    }
  return true;
}

// x2 / x3 faces: tiles of 32 x TF faces. The copy holds the tile's 32 columns
// (plus the few that align its start) and the TF + 5 cells along the face
// direction that the TF faces' stencils reach; each thread reconstructs the
// two cells of its face.
constexpr int kTmaCols = 32 + kTmaAlign;

template <int TF>
inline size_t tma_tile_smem(int nf) {
  // the staged primitives, whose space then holds the split faces' states
  const size_t staged = (size_t)nf * (TF + 5) * kTmaCols * sizeof(PT);
  const size_t split = split_faces(MKS) ? 3 * (size_t)TF * NPRIM * 32 * sizeof(double) : 0;
  return std::max(staged, split);
}

template <int MT, int DIR, int TF, int OPT>
__global__ void __launch_bounds__(32 * TF, flux_blocks(MT))
    k_flux_tile_tma(const __grid_constant__ CUtensorMap tm, Dims d, pangu_params p, int k0,
                    int k1, int j0, int j1, int i0, int i1, double *F, double *alfven,
                    int *err) {
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) unsigned long long bar;
  pdl_grid_wait();
  const int m0 = DIR == 2 ? j0 : k0, m1 = DIR == 2 ? j1 : k1;
  const int a0 = DIR == 2 ? k0 : j0, a1 = DIR == 2 ? k1 : j1;
  const int ni = i1 - i0 + 1, na = a1 - a0 + 1, nm = m1 - m0 + 1;
  const int nti = (ni + 31) / 32, ntm = (nm + TF - 1) / TF;
  long long ti, tmi, al;
  long long r = div_fast(blockIdx.x, nti, ti);
  r = div_fast(r, ntm, tmi);
  const long long bb = div_fast(r, na, al);
  if (bb >= d.NB) return;  // whole CTAs exit together
  const int b = slot_of(d, (int)bb);
  const int a = a0 + (int)al;
  const int mt0 = m0 + (int)tmi * TF;
  const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
  const int x0 = i0 + (int)ti * 32;
  const int xs = x0 & ~(kTmaAlign - 1);  // 16-byte aligned first column
  const int off = x0 - xs;
  constexpr int R = TF + 5;  // cells mt0 - 3 .. mt0 + TF + 1
  PT *raw = reinterpret_cast<PT *>(dsm);
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, (unsigned)(d.NF * R * kTmaCols * sizeof(PT)));
    if (DIR == 2)
      tma_load_4d(raw, &tm, xs, mt0 - 3, a, b * d.NF, &bar);
    else
      tma_load_4d(raw, &tm, xs, a, mt0 - 3, b * d.NF, &bar);
  }
  if (!tma_wait(&bar, err)) return;
  const int i = x0 + lane, f = mt0 + row;
  const bool active = i <= i1 && f <= m1;
  const bool use_mc = PGK_FLUX_MC(p);
  FT PL[NPRIM], PR[NPRIM];
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) {
    PL[s] = 0;
    PR[s] = 0;
    if (active && d.pidx[s] >= 0) {
      // cell f - 1 sits at tile row row + 2, cell f at row + 3
      const PT *q = raw + ((size_t)d.pidx[s] * R + row + 2) * kTmaCols + lane + off;
      FT lo, up;
      recon_cell(use_mc, q, kTmaCols, PL[s], lo);
      recon_cell(use_mc, q + kTmaCols, kTmaCols, up, PR[s]);
    }
  }
  __syncthreads();  // the staged tile is read; its space is reused below
  if (!active) return;
  const int kk = DIR == 2 ? a : f, jj = DIR == 2 ? f : a;
#if PGK_SPLIT_FACES
  if (split_faces(MT)) {
    double *sl = reinterpret_cast<double *>(dsm);
    double *pl = sl + ((size_t)0 * TF + row) * NPRIM * 32 + lane;
    double *pr = sl + ((size_t)1 * TF + row) * NPRIM * 32 + lane;
    double *ul = sl + ((size_t)2 * TF + row) * NPRIM * 32 + lane;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) {
      pl[s * 32] = PL[s];
      pr[s * 32] = PR[s];
    }
    face_flux_split<MT, DIR, OPT>(d, p, b, kk, jj, i, pl, pr, ul, 32, F, alfven);
    return;
  }
#endif
  face_flux<MT, DIR, OPT>(d, p, b, kk, jj, i, PL, PR, F, alfven);
}

// x1 faces: a CTA of 4 warps takes 4 consecutive rows (j) of one k and one
// segment of 31 faces; the copy holds the segment's 32 cells and 2 more on
// each side (from a 16-byte aligned first column) of every component and row.
// Lane l reconstructs cell i0 - 1 + 31 seg + l and hands its upper-face value
// to lane l + 1, as k_flux_x1 does from global memory.
constexpr int kTmaRowsX1 = 4;
constexpr int kTmaColsX1 = (kFacesPerWarp + 5 + kTmaAlign - 1 + kTmaAlign - 1) / kTmaAlign *
                           kTmaAlign;

inline size_t tma_x1_smem(int nf) {
  const size_t staged = (size_t)nf * kTmaRowsX1 * kTmaColsX1 * sizeof(PT);
  const size_t split = split_faces(MKS) ? 3 * (size_t)NPRIM * 32 * kTmaRowsX1 * sizeof(double)
                                        : 0;
  return std::max(staged, split);
}

template <int MT, int OPT>
__global__ void __launch_bounds__(32 * kTmaRowsX1, flux_blocks(MT))
    k_flux_x1_tma(const __grid_constant__ CUtensorMap tm, Dims d, pangu_params p, int k0, int k1,
                  int j0, int j1, int i0, int i1, double *F, double *alfven, int *err) {
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) unsigned long long bar;
  pdl_grid_wait();
  const int nf = i1 - i0 + 1;
  const int nseg = (nf + kFacesPerWarp - 1) / kFacesPerWarp;
  const int nj = j1 - j0 + 1, njc = (nj + kTmaRowsX1 - 1) / kTmaRowsX1;
  long long segl, jcl, kl;
  long long r = div_fast(blockIdx.x, nseg, segl);
  r = div_fast(r, njc, jcl);
  const long long bb = div_fast(r, k1 - k0 + 1, kl);
  if (bb >= d.NB) return;  // whole CTAs exit together
  const int b = slot_of(d, (int)bb);
  const int k = k0 + (int)kl, seg = (int)segl;
  const int jr0 = j0 + (int)jcl * kTmaRowsX1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c0 = i0 - 1 + seg * kFacesPerWarp;  // the segment's first cell
  const int xs = (c0 - 2) & ~(kTmaAlign - 1);
  const int off = c0 - xs;  // column of cell c0 in the staged rows
  PT *raw = reinterpret_cast<PT *>(dsm);
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, (unsigned)(d.NF * kTmaRowsX1 * kTmaColsX1 * sizeof(PT)));
    tma_load_4d(raw, &tm, xs, jr0, k, b * d.NF, &bar);
  }
  if (!tma_wait(&bar, err)) return;
  const int j = jr0 + w, c = c0 + lane;
  const bool active = c <= i1 && j <= j1;  // cell c is needed by face c (and c + 1)
  const bool use_mc = PGK_FLUX_MC(p);
  FT up[NPRIM], lo[NPRIM];
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) {
    up[s] = 0;
    lo[s] = 0;
    if (d.pidx[s] >= 0 && active)
      recon_cell(use_mc, raw + ((size_t)d.pidx[s] * kTmaRowsX1 + w) * kTmaColsX1 + off + lane, 1,
                 up[s], lo[s]);
  }
#if PGK_SPLIT_FACES
  if (split_faces(MT)) {
    __syncthreads();  // the staged rows are read; their space is reused below
    // [3][NPRIM][blockDim.x] as in k_flux_x1
    double *fsm = reinterpret_cast<double *>(dsm);
    const int ss = blockDim.x, t = threadIdx.x;
#pragma unroll
    for (int s = 0; s < NPRIM; ++s) {
      fsm[s * ss + t] = up[s];
      fsm[(NPRIM + s) * ss + t] = lo[s];
    }
    __syncwarp();
    if (lane == 0 || !active) return;
    face_flux_split<MT, 1, OPT>(d, p, b, k, j, c, fsm + t - 1, fsm + NPRIM * ss + t,
                                fsm + 2 * NPRIM * ss + t, ss, F, alfven);
    return;
  }
#endif
  FT PL[NPRIM];
#pragma unroll
  for (int s = 0; s < NPRIM; ++s) PL[s] = __shfl_up_sync(0xffffffffu, up[s], 1);
  if (lane == 0 || !active) return;
  face_flux<MT, 1, OPT>(d, p, b, k, j, c, PL, lo, F, alfven);
}

template <int MT, int MARCH, int OPT>
__global__ void __launch_bounds__(kFluxThreads, flux_blocks(MT)) k_flux_march2(Dims d, pangu_params p, int k0, int k1,
                                                          int j0, int j1, int i0, int i1,
                                                          const PT *P, double *F,
                                                          double *alfven) {
  pdl_grid_wait();
  flux_march_body<MT, 2, MARCH, OPT>(d, p, k0, k1, j0, j1, i0, i1, P, F, alfven);
}
template <int MT, int MARCH, int OPT>
__global__ void __launch_bounds__(kFluxThreads, flux_blocks(MT)) k_flux_march3(Dims d, pangu_params p, int k0, int k1,
                                                          int j0, int j1, int i0, int i1,
                                                          const PT *P, double *F,
                                                          double *alfven) {
  pdl_grid_wait();
  flux_march_body<MT, 3, MARCH, OPT>(d, p, k0, k1, j0, j1, i0, i1, P, F, alfven);
}

// ---------------------------------------------------------------------------
// ConstraintedTransport (constrained_transport.cc:13-130).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_ct_emf(Dims d, const double *F1, const double *F2,
                                                     const double *F3, double *E) {
  pdl_grid_wait();
  int b, k, j, i;
  const int o1 = d.N1 > 1, o2 = d.N2 > 1, o3 = d.N3 > 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke + o3, d.js, d.je + o2, d.is, d.ie + o1, b, k, j, i)) return;
  b = slot_of(d, b);
  const long long sj = d.N1, sk = (long long)d.N1 * d.N2, o = coff(d, k, j, i);
  double e1 = 0.0, e2 = 0.0, e3 = 0.0;
  if (o2 && o3) {
    const double *a = a_flux2(d, F2, b, BX3) + o, *c = a_flux3(d, F3, b, BX2) + o;
    e1 = 0.25 * ((a[0] + a[-sk]) - (c[0] + c[-sj]));
  }
  if (o3 && o1) {
    const double *a = a_flux3(d, F3, b, BX1) + o, *c = a_flux1(d, F1, b, BX3) + o;
    e2 = 0.25 * ((a[0] + a[-1]) - (c[0] + c[-sk]));
  }
  if (o1 && o2) {
    const double *a = a_flux1(d, F1, b, BX2) + o, *c = a_flux2(d, F2, b, BX1) + o;
    e3 = 0.25 * ((a[0] + a[-sj]) - (c[0] + c[-1]));
  }
  a_efield(d, E, b, 0)[o] = e1;
  a_efield(d, E, b, 1)[o] = e2;
  a_efield(d, E, b, 2)[o] = e3;
}

// Face-B overwrite (constrained_transport.cc:78-127) of every direction in
// one launch: a thread at (k, j, i) of the union of the face ranges writes the
// x1 face (i - 1/2) when j and k are interior, the x2 face when i and k are,
// and the x3 face when i and j are.
__global__ void __launch_bounds__(kThreads) k_ct_faces(Dims d, double *F1, double *F2,
                                                       double *F3, const double *E) {
  pdl_grid_wait();
  int b, k, j, i;
  const int o1 = d.N1 > 1, o2 = d.N2 > 1, o3 = d.N3 > 1;
  const int E1 = o2 && o3, E2 = o3 && o1, E3 = o1 && o2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke + o3, d.js, d.je + o2, d.is, d.ie + o1, b, k, j, i)) return;
  b = slot_of(d, b);
  const long long sj = d.N1, sk = (long long)d.N1 * d.N2, o = coff(d, k, j, i);
  const double *Ea = a_efield(d, E, b, 0) + o, *Eb = a_efield(d, E, b, 1) + o, *Ec = a_efield(d, E, b, 2) + o;
  const bool in_i = i <= d.ie, in_j = j <= d.je, in_k = k <= d.ke;
  if (in_j && in_k) {
    if (o1) a_flux1(d, F1, b, BX1)[o] = 0;
    if (E2) a_flux1(d, F1, b, BX3)[o] = -0.5 * (Eb[0] + Eb[sk]);
    if (E3) a_flux1(d, F1, b, BX2)[o] = 0.5 * (Ec[0] + Ec[sj]);
  }
  if (d.ndim >= 2 && in_i && in_k) {
    if (E1) a_flux2(d, F2, b, BX3)[o] = 0.5 * (Ea[0] + Ea[sk]);
    if (o2) a_flux2(d, F2, b, BX2)[o] = 0.;
    if (E3) a_flux2(d, F2, b, BX1)[o] = -0.5 * (Ec[0] + Ec[1]);
  }
  if (d.ndim == 3 && in_i && in_j) {
    if (E1) a_flux3(d, F3, b, BX2)[o] = -0.5 * (Ea[0] + Ea[sj]);
    if (E2) a_flux3(d, F3, b, BX1)[o] = 0.5 * (Eb[0] + Eb[1]);
    if (o3) a_flux3(d, F3, b, BX3)[o] = 0;
  }
}

// ---------------------------------------------------------------------------
// FluxDivergence + UpdateIndependentData, interior (ideal_grmhd.cc:73-76).
// ---------------------------------------------------------------------------
// One thread per interior cell for all NF variables: the index decode, the
// block's widths, areas, volume and beta dt are formed once per cell, not once
// per (cell, variable) (4x fewer instructions; every variable's value is
// computed as before).
__global__ void __launch_bounds__(kThreads, 4) k_flux_div_update(Dims d, const double *F1,
                                                                 const double *F2,
                                                                 const double *F3,
                                                                 const double *Uinit,
                                                                 double *Uout, double beta,
                                                                 const double *dt) {
  pdl_grid_wait();
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, b, k, j, i)) return;
  b = slot_of(d, b);
  const long long q = coff(d, k, j, i);
  const double dx0 = dx_of(d, b, 0), dx1 = dx_of(d, b, 1), dx2 = dx_of(d, b, 2);
  const double A1 = MUL(dx1, dx2), A2 = MUL(dx0, dx2), A3 = MUL(dx0, dx1);
  const double V = MUL(MUL(dx0, dx1), dx2);
  const double bdt = MUL(beta, dt[job_of(d, b)]);
  const long long sj = d.N1, sk = (long long)d.N1 * d.N2;
  // Components in groups of kUpdGroup: every load of a group is issued before
  // its first store (Uout may be Uinit, so the compiler would not move a
  // later component's loads above an earlier store). Two per group: measured
  // 2-4 % faster per RK2 cycle than one at a time on the 2D and 3D tori and
  // Orszag-Tang; groups of three or more spill at the 64-register bound.
  constexpr int kUpdGroup = 2;
#pragma unroll
  for (int v0 = 0; v0 < NPRIM; v0 += kUpdGroup) {
    double f1l[kUpdGroup], f1r[kUpdGroup], f2l[kUpdGroup], f2r[kUpdGroup], f3l[kUpdGroup],
        f3r[kUpdGroup], u0[kUpdGroup];
#pragma unroll
    for (int c = 0; c < kUpdGroup; ++c) {
      const int v = v0 + c;
      if (v >= d.NF) break;
      const double *f1 = a_flux1(d, F1, b, v) + q;
      f1l[c] = f1[0];
      f1r[c] = f1[1];
      if (d.ndim >= 2) {
        const double *f2 = a_flux2(d, F2, b, v) + q;
        f2l[c] = f2[0];
        f2r[c] = f2[sj];
      }
      if (d.ndim == 3) {
        const double *f3 = a_flux3(d, F3, b, v) + q;
        f3l[c] = f3[0];
        f3r[c] = f3[sk];
      }
      u0[c] = a_cons0(d, Uinit, b, v)[q];
    }
#pragma unroll
    for (int c = 0; c < kUpdGroup; ++c) {
      const int v = v0 + c;
      if (v >= d.NF) break;
      double du = SUB(MUL(A1, f1r[c]), MUL(A1, f1l[c]));
      if (d.ndim >= 2) du = ADD(du, SUB(MUL(A2, f2r[c]), MUL(A2, f2l[c])));
      if (d.ndim == 3) du = ADD(du, SUB(MUL(A3, f3r[c]), MUL(A3, f3l[c])));
      const double dudt = DIV(-du, V);
      a_cons(d, Uout, b, v)[q] = ADD(u0[c], MUL(bdt, dudt));
    }
  }
}

// ---------------------------------------------------------------------------
// Ghost exchange: ghost <- neighbour interior, prim and flag.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_exchange(Dims d, long long n, const long long *dst,
                                                       const long long *src, PT *P,
                                                       double *flag) {
  pdl_grid_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long dc = dst[t], sc = src[t];
  long long db, dof, sb, sof;
  split_cell(dc, d.ncell, db, dof);
  split_cell(sc, d.ncell, sb, sof);
  // every load before the first store (a source is an interior cell, which
  // the exchange never writes): one memory latency instead of NF in a row
  PT val[NPRIM];
#pragma unroll
  for (int v = 0; v < NPRIM; ++v)
    if (v < d.NF) val[v] = a_prim(d, P, (int)sb, v)[sof];
  const bool has_flag = flag || d.tG;
  const double fl = has_flag ? a_flag(d, flag, (int)sb)[sof] : 0.0;
#pragma unroll
  for (int v = 0; v < NPRIM; ++v)
    if (v < d.NF) a_prim(d, P, (int)db, v)[dof] = val[v];
  if (has_flag) a_flag(d, flag, (int)db)[dof] = fl;
}

// Halo messages of a sharded mesh: the cells of the exchange whose other end
// is on another GPU, as [entry][Nf primitives, flag] in FP64 (an FP32
// primitive converts to FP64 and back exactly), so a message is a plain
// contiguous buffer for NCCL or a peer copy.
__global__ void __launch_bounds__(kThreads) k_halo_pack(Dims d, long long n, const long long *cells,
                                                        const PT *P, const double *flag,
                                                        double *buf) {
  pdl_grid_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long c = cells[t];
  long long b, off;
  split_cell(c, d.ncell, b, off);
  double *o = buf + t * (d.NF + 1);
  for (int v = 0; v < d.NF; ++v) o[v] = (double)a_prim(d, P, (int)b, v)[off];
  o[d.NF] = (flag || d.tG) ? a_flag(d, flag, (int)b)[off] : 0.0;
}

__global__ void __launch_bounds__(kThreads) k_halo_unpack(Dims d, long long n,
                                                          const long long *cells, PT *P,
                                                          double *flag, const double *buf) {
  pdl_grid_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long c = cells[t];
  long long b, off;
  split_cell(c, d.ncell, b, off);
  const double *o = buf + t * (d.NF + 1);
  for (int v = 0; v < d.NF; ++v) a_prim(d, P, (int)b, v)[off] = (PT)o[v];
  if (flag || d.tG) a_flag(d, flag, (int)b)[off] = o[d.NF];
}

// ---------------------------------------------------------------------------
// AddGeometricSource (source_term.cc:15-121): Christoffel symbols by central
// differences of the code metric (christoffel.h:74-148), rounded step by
// step like the metric itself.
// ---------------------------------------------------------------------------
template <int MT>
__device__ __forceinline__ void metric_derivs(const Dims &d, const pangu_params &p, int b, int k,
                                              int j, int i, double dg[4][4][4]) {
  constexpr double twod = 2.0 * 1.0e-5;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) dg[a][r][c] = 0.0;
  double x[4] = {0.0, 0.0, 0.0, 0.0};
  if (MT == CKS) {
    x[1] = xc(d, b, 0, i);
    x[2] = xc(d, b, 1, j);
    x[3] = xc(d, b, 2, k);
  }
#pragma unroll
  for (int dir = 1; dir < 4; ++dir) {
    if ((MT == MKS || MT == BL) && dir == 3) continue;  // metric independent of x3: exactly 0
    double gp[4][4], gm[4][4];
    double xp[4] = {x[0], x[1], x[2], x[3]}, xm[4] = {x[0], x[1], x[2], x[3]};
    xp[dir] = ADD(xp[dir], 1.0e-5);
    xm[dir] = SUB(xm[dir], 1.0e-5);
    gcov_at<MT>(d, p, b, i, dir == 1 ? 1 : 0, j, dir == 2 ? 1 : 0, xp, gp);
    gcov_at<MT>(d, p, b, i, dir == 1 ? 2 : 0, j, dir == 2 ? 2 : 0, xm, gm);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) dg[dir][r][c] = DIV(SUB(gp[r][c], gm[r][c]), twod);
  }
}

// Gamma^a_jk = g^al (d_j g_lk + d_k g_lj - d_l g_jk) / 2 in the order of
// christoffel.h:120-146, with every term.
__device__ __forceinline__ void connection(const double dg[4][4][4], const Geo &g,
                                           double conn[4][4][4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const double cc = MUL(0.5, SUB(ADD(dg[jj][l][kk], dg[kk][l][jj]), dg[l][jj][kk]));
          v = ADD(v, MUL(g.gcon[a][l], cc));
        }
        conn[a][jj][kk] = v;
      }
}

template <int MT>
__device__ __forceinline__ void christoffel(const Dims &d, const pangu_params &p, int b, int k,
                                            int j, int i, const Geo &g, double conn[4][4][4]) {
  double dg[4][4][4];
  metric_derivs<MT>(d, p, b, k, j, i, dg);
  connection(dg, g, conn);
}

// Geometric source of one interior cell: U += (T^r_c Gamma^c_{dir r})
// sqrt|g| beta dt for the energy and momentum components, from the cell's
// (stale) primitives as they stand in memory.
template <int MT>
__device__ __forceinline__ void source_cell(const Dims &d, const pangu_params &p, const PT *P,
                                            double *U, int b, int k, int j, int i, const Geo &g,
                                            double bdt) {
  if (MT == MINKOWSKI) return;  // connection identically zero (christoffel.h:90)
  const double sg = g.sg;
#if PGK_MIXED
  if (MT == MKS || MT == BL) {
    // Mixed form: T^r_c Gamma^c_{dir r} evaluated in FT from the FP32
    // primitives and the tabulated FP64 metric rounded once; the increment is
    // accumulated into the FP64 conserved variables.
    constexpr TabLayout L = tab_layout(MT);
    const long long q0 = coff(d, k, j, i);
    FT pf[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; ++v) pf[v] = d.pidx[v] >= 0 ? a_prim(d, P, b, d.pidx[v])[q0] : FT(0);
    GeoT<FT> gf;
    geo_cast<MT>(g, gf);
    StateT<FT> sf;
    calc_state_t<MT>(pf, gf, sf);
    const FT gam = (FT)p.adiabatic_index;
    const FT hh = pf[RHO] + gam * pf[ENY];
    const FT e_tot = hh + sf.bsq;
    const FT p_tot = (gam - FT(1)) * pf[ENY] + FT(0.5) * sf.bsq;
    const long long plane = (long long)d.N2 * d.N1;
    // the FP32 Christoffel planes (pool_init builds them for every mixed engine)
    const float *cn = d.ctab32 + (long long)b * L.nconn * plane + (long long)j * d.N1 + i;
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
      FT con = FT(0);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (L.conn[c][dir][r] >= 0) {
            const FT T = e_tot * sf.ucon[r] * sf.ucov[c] + p_tot * FT(r == c) -
                         sf.bcon[r] * sf.bcov[c];
            con += T * (FT)__ldg(cn + L.conn[c][dir][r] * plane);
          }
      const int v = dir == 0 ? d.pidx[ENY] : d.pidx[UX1] + dir - 1;
      a_cons(d, U, b, v)[q0] += (double)con * sg * bdt;
    }
    return;
  }
#endif
  double pc[NPRIM];
  load_prim(d, P, b, k, j, i, pc);
  State s;
  calc_state<MT>(pc, g, s);
  double T[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r) emt_from_state(p.adiabatic_index, pc, s, r, T[r]);
  if (MT == MKS || MT == BL) {
    // Christoffel symbols from the centre table; structural zeros skipped
    constexpr TabLayout L = tab_layout(MT);
    const long long plane = (long long)d.N2 * d.N1;
    const double *cn = d.ctab + (long long)b * L.ncen * plane + (long long)j * d.N1 + i +
                       (long long)L.nmet * plane;
    // the four contractions first, then the four updates: no Christoffel load
    // waits behind a store to U
    double con[4];
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
      con[dir] = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (L.conn[c][dir][r] >= 0)
            con[dir] += T[r][c] * __ldg(cn + L.conn[c][dir][r] * plane);
    }
    const long long q = coff(d, k, j, i);
    double u[4];
#pragma unroll
    for (int dir = 0; dir < 4; ++dir)
      u[dir] = a_cons(d, U, b, dir == 0 ? d.pidx[ENY] : d.pidx[UX1] + dir - 1)[q];
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
      const int v = dir == 0 ? d.pidx[ENY] : d.pidx[UX1] + dir - 1;
      a_cons(d, U, b, v)[q] = u[dir] + con[dir] * sg * bdt;
    }
  } else {
    double conn[4][4][4];
    christoffel<MT>(d, p, b, k, j, i, g, conn);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
      double con = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) con += T[r][c] * conn[c][dir][r];
      const int v = dir == 0 ? d.pidx[ENY] : d.pidx[UX1] + dir - 1;
      a_cons(d, U, b, v)[coff(d, k, j, i)] += con * sg * bdt;
    }
  }
}

template <int MT>
__global__ void __launch_bounds__(kThreads, 4) k_source(Dims d, pangu_params p, const PT *P,
                                                     double *U, double beta, const double *dt) {
  pdl_grid_wait();
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, b, k, j, i)) return;
  b = slot_of(d, b);
  if (MT == MINKOWSKI) return;
  Geo g;
  cell_metric<MT>(d, p, b, k, j, i, g);
  source_cell<MT>(d, p, P, U, b, k, j, i, g, beta * dt[job_of(d, b)]);
}

// Builds the static metric tables of an MKS or BL engine with the dense
// reference arithmetic (one thread per table point).
template <int MT>
__global__ void __launch_bounds__(kThreads) k_build_tables(Dims d, pangu_params p, double *ctab,
                                                           double *f1tab, double *f2tab) {
  pdl_grid_wait();
  constexpr TabLayout L = tab_layout(MT);
  const long long pc = (long long)d.N2 * d.N1, p1 = (long long)d.N2 * (d.N1 + 1),
                  p2 = (long long)(d.N2 + 1) * d.N1;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = pc + p1 + p2;
  if (t >= per * d.NB) return;
  const int bb = (int)(t / per);
  t -= (long long)bb * per;
  const int b = slot_of(d, bb);
  int which, W;
  long long plane;
  double *tab;
  int nc;
  if (t < pc) {
    which = 0, W = d.N1, plane = pc, tab = ctab, nc = L.ncen;
  } else if (t < pc + p1) {
    t -= pc;
    which = 1, W = d.N1 + 1, plane = p1, tab = f1tab, nc = L.nmet;
  } else {
    t -= pc + p1;
    which = 2, W = d.N1, plane = p2, tab = f2tab, nc = L.nmet;
  }
  const int j = (int)(t / W), i = (int)(t % W);
  const double x[4] = {0.0, 0.0, 0.0, 0.0};
  Geo g;
  const int ok = analytic_geo<MT>(d, p, b, i, which == 1 ? 3 : 0, j, which == 2 ? 3 : 0, x, g);
  double *o = tab + (long long)b * nc * plane + t;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= r && L.sym[r][c] >= 0) o[L.sym[r][c] * plane] = g.gcov[r][c];
      if (L.con[r][c] >= 0) o[(L.nsym + L.con[r][c]) * plane] = g.gcon[r][c];
    }
  const long long s0 = L.nsym + L.ncon;
  o[s0 * plane] = g.gdet;
  o[(s0 + 1) * plane] = g.sg;
  o[(s0 + 2) * plane] = g.alpha;
  o[(s0 + 3) * plane] = ok ? 1.0 : 0.0;
  if (which == 0) {
    double conn[4][4][4];
    christoffel<MT>(d, p, b, 0, j, i, g, conn);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int kk = jj; kk < 4; ++kk)
          if (L.conn[a][jj][kk] >= 0) o[(L.nmet + L.conn[a][jj][kk]) * plane] = conn[a][jj][kk];
  }
}

// Mixed form: ncomp planes of a slot-major table, for the job's slots,
// rounded once to FP32.
__global__ void __launch_bounds__(kThreads) k_planes_to_f32(Dims d, const double *src, float *dst,
                                                            int ncomp, long long plane) {
  pdl_grid_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.NB * ncomp * plane) return;
  long long off, q;
  const long long bq = div_fast(t, plane, off);
  const int bb = (int)div_fast(bq, ncomp, q);
  const long long at = ((long long)slot_of(d, bb) * ncomp + q) * plane + off;
  dst[at] = (float)src[at];
}

// Mixed form: the centre table's Christoffel planes of the job's slots
// rounded once to FP32 (what the FP32 source term converts each value to
// anyway), so that the source term reads half the bytes.
template <int MT>
__global__ void __launch_bounds__(kThreads) k_conn_to_f32(Dims d, float *out) {
  pdl_grid_wait();
  constexpr TabLayout L = tab_layout(MT);
  const long long plane = (long long)d.N2 * d.N1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.NB * L.nconn * plane) return;
  long long off, q;
  const long long bq = div_fast(t, plane, off);
  const int bb = (int)div_fast(bq, L.nconn, q);
  const long long sl = slot_of(d, bb);
  out[(sl * L.nconn + q) * plane + off] =
      (float)d.ctab[(sl * L.ncen + L.nmet + q) * plane + off];
}

// ---------------------------------------------------------------------------
// ApplyElectronHeating (electron_heating.cc:14-112).
// ---------------------------------------------------------------------------
// Electron heating of one interior cell from its primitives and conserved
// variables as they stand in memory: writes the electron entropy. The mixed
// form computes the state and the heating in FT (FP32).
template <int MT>
__device__ __forceinline__ void heat_cell(const Dims &d, const pangu_params &p, PT *P,
                                          const double *U, int b, int k, int j, int i,
                                          const Geo &g) {
  const long long q = coff(d, k, j, i);
  const double cr = a_cons(d, U, b, 0)[q];
  const HeatParams hp = {p.model, p.adiabatic_index, p.gamma_p, p.gamma_e, p.fel_constant,
                         p.ratio_min, p.ratio_max, p.limit_kel, p.suppress_highb_heat,
                         p.enforce_positive_dissipation};
#if PGK_MIXED
  FT pc[NPRIM];
#pragma unroll
  for (int v = 0; v < NPRIM; ++v) pc[v] = d.pidx[v] >= 0 ? a_prim(d, P, b, d.pidx[v])[q] : FT(0);
  GeoT<FT> gf;
  geo_cast<MT>(g, gf);
  StateT<FT> s;
  calc_state_t<MT>(pc, gf, s);
  a_prim(d, P, b, d.pidx[KEL])[q] =
      heating_apply_t<FT>(hp, pc[RHO], pc[ENY], s.bsq, (FT)(a_cons(d, U, b, d.pidx[ENT])[q] / cr),
                          pc[ENT], (FT)(a_cons(d, U, b, d.pidx[KEL])[q] / cr));
#else
  double pc[NPRIM];
  load_prim(d, P, b, k, j, i, pc);
  State s;
  calc_state<MT>(pc, g, s);
  a_prim(d, P, b, d.pidx[KEL])[q] =
      heating_apply(hp, pc[RHO], pc[ENY], s.bsq, a_cons(d, U, b, d.pidx[ENT])[q] / cr, pc[ENT],
                    a_cons(d, U, b, d.pidx[KEL])[q] / cr);
#endif
}

template <int MT>
__global__ void __launch_bounds__(kThreads, 4) k_heating(Dims d, pangu_params p, PT *P,
                                                      const double *U) {
  pdl_grid_wait();
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, b, k, j, i)) return;
  b = slot_of(d, b);
  Geo g;
  cell_metric<MT>(d, p, b, k, j, i, g);
  heat_cell<MT>(d, p, P, U, b, k, j, i, g);
}

// ---------------------------------------------------------------------------
// Recovery (invertor.cc:18-210).
// ---------------------------------------------------------------------------
// Warp-aggregated append of `value` to list[*count] for the lanes with pred.
__device__ __forceinline__ void append(int *count, long long *list, bool pred, long long value) {
  const unsigned mask = __activemask();
  const unsigned hits = __ballot_sync(mask, pred);
  if (!hits) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(hits));
  base = __shfl_sync(mask, base, leader);
  if (pred) list[base + __popc(hits & ((1u << lane) - 1u))] = value;
}

// The HARM-normalised conserved state and the stale primitive guess of one
// cell (invertor.cc:100-174); writes the magnetic primitives
// (invertor.cc:137-147).
template <int MT>
__device__ __forceinline__ void c2p_inputs(const Dims &d, const pangu_params &p, PT *P,
                                           const double *U, int b, int k, int j, int i,
                                           const Geo &g, double UH[9], double PH[9],
                                           bool write_b) {
  const long long q = coff(d, k, j, i);
  double C[9];
#pragma unroll
  for (int s = 0; s < 9; ++s) {
    C[s] = d.pidx[s] >= 0 ? a_cons(d, U, b, d.pidx[s])[q] : 0.0;
    PH[s] = d.pidx[s] >= 0 ? a_prim(d, P, b, d.pidx[s])[q] : 0.0;
  }
  const double isg = 1.0 / g.sg;
  const double aisg = g.alpha * isg;
  if (p.enable_B && write_b) {
    a_prim(d, P, b, d.pidx[BX1])[q] = C[BX1] * isg;
    a_prim(d, P, b, d.pidx[BX2])[q] = C[BX2] * isg;
    a_prim(d, P, b, d.pidx[BX3])[q] = C[BX3] * isg;
  }
  UH[RHO] = aisg * C[RHO];
  UH[ENY] = aisg * (C[ENY] - C[RHO]);
  UH[UX1] = aisg * C[UX1];
  UH[UX2] = aisg * C[UX2];
  UH[UX3] = aisg * C[UX3];
  UH[BX1] = aisg * C[BX1];
  UH[BX2] = aisg * C[BX2];
  UH[BX3] = aisg * C[BX3];
  UH[ENT] = aisg * C[ENT];
}

__device__ __forceinline__ void c2p_write(const Dims &d, PT *P, int b, int k, int j, int i,
                                          const double PH[9]) {
  const long long q = coff(d, k, j, i);
  a_prim(d, P, b, 0)[q] = PH[RHO];
  a_prim(d, P, b, 1)[q] = PH[ENY];
  a_prim(d, P, b, 2)[q] = PH[UX1];
  a_prim(d, P, b, 3)[q] = PH[UX2];
  a_prim(d, P, b, 4)[q] = PH[UX3];
}

// Recovery, first pass: Kastaun (robuster), or the chain from Scheme2D.
// CHAIN = false: cells where Scheme2D fails are appended to `list` (their
// primitives left untouched) and finished by k_recovery_retry, so the long
// 1Dvsq/1D Newton loops of a few cells do not hold whole warps of converged
// cells. CHAIN = true: the failing lanes run Scheme1Dvsq and Scheme1D at
// once (the retry pass's arithmetic, from the same inputs), and `list` (may
// be null) receives the cells the whole chain fails, FixRecovery's list.
// The chained form is used when the pass fits in one wave of CTAs: then the
// few long chains overlap the rest of the wave instead of running as a
// separate latency-bound launch (2D 512 x 256 torus at steady state: 0.387
// against 0.403 ms per cycle), while on larger grids the registers the
// chain adds (spills) cost more than the retry launch (3D torus 11.17
// against 10.98 ms, 48-torus batch 7.15 against 7.05 ms).
// (Folding the geometric source and electron heating into this kernel was
// measured slower: their registers cut the occupancy of the Newton loops.)
template <int MT, bool CHAIN>
__device__ __forceinline__ void recovery_cell(const Dims &d, const pangu_params &p, PT *P,
                                              const double *U, double *flag,
                                              unsigned long long *cnt, int *nlist,
                                              long long *list) {
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, b, k, j, i)) return;
  b = slot_of(d, b);
  const bool robuster = p.recovery == PANGU_RECOVERY_ROBUSTER;
  const long long fc = cidx(d, b, k, j, i);
  if (MT == CKS) {
    const double x = xc(d, b, 0, i), y = xc(d, b, 1, j), z = xc(d, b, 2, k);
    const double a2 = p.a * p.a;
    const double rad2 = x * x + y * y + z * z;
    const double sa = (rad2 - a2) * (rad2 - a2) + 4.0 * a2 * z * z;
    const bool exc = sqrt(0.5 * (rad2 - a2 + sqrt(sa))) < p.r_excise;
    count(cnt, job_of(d, b), PANGU_CNT_EXCISED, exc);
    if (exc) {
      if (!robuster) a_flag(d, flag, b)[fc - (long long)b * d.ncell] = 0;
      return;
    }
  }
  Geo g;
  cell_metric<MT>(d, p, b, k, j, i, g);
  double UH[9], PH[9];
  c2p_inputs<MT>(d, p, P, U, b, k, j, i, g, UH, PH, true);
  const double gam = p.adiabatic_index;
  if (robuster) {
    const int st = invert_kastaun(UH, PH, gam, g);
    count(cnt, job_of(d, b), PANGU_CNT_KASTAUN_FAIL, st != 0);
    if (st != 0) return;
  } else {
    Harm hs;
    harm_setup<MT>(UH, g, hs);
    bool ok = invert_2d<MT>(UH, PH, gam, g, hs) == 0;
    count(cnt, job_of(d, b), PANGU_CNT_C2P_2D, ok);
    if (!CHAIN) {
      append(nlist, list, !ok, fc);
      a_flag(d, flag, b)[fc - (long long)b * d.ncell] = ok ? 1.0 : 0.0;
      if (!ok) return;
    } else {
      if (!ok) {
        // Scheme1Dvsq, then Scheme1D (invertor.cc:185-197), from the stale
        // guess as it stands in memory
        c2p_inputs<MT>(d, p, P, U, b, k, j, i, g, UH, PH, false);
        harm_setup<MT>(UH, g, hs);
        ok = invert_1dvsq<MT>(UH, PH, gam, g, hs) == 0;
        count(cnt, job_of(d, b), PANGU_CNT_C2P_1DVSQ, ok);
        if (!ok) {
          ok = invert_1d<MT>(UH, PH, gam, g, hs) == 0;
          count(cnt, job_of(d, b), PANGU_CNT_C2P_1D, ok);
          count(cnt, job_of(d, b), PANGU_CNT_C2P_FAIL, !ok);
        }
        if (list) append(nlist, list, !ok, fc);
      }
      a_flag(d, flag, b)[fc - (long long)b * d.ncell] = ok ? 1.0 : 0.0;
    }
  }
  c2p_write(d, P, b, k, j, i, PH);
}

template <int MT>
__global__ void __launch_bounds__(kRecoveryThreads, 7) k_recovery(Dims d, pangu_params p, PT *P,
                                                       const double *U, double *flag,
                                                       unsigned long long *cnt, int *nretry,
                                                       long long *retry) {
  pdl_grid_wait();
  recovery_cell<MT, false>(d, p, P, U, flag, cnt, nretry, retry);
}

template <int MT>
__global__ void __launch_bounds__(kRecoveryThreads, 7)
    k_recovery_chain(Dims d, pangu_params p, PT *P, const double *U, double *flag,
                     unsigned long long *cnt, int *nfix, long long *fix) {
  pdl_grid_wait();
  recovery_cell<MT, true>(d, p, P, U, flag, cnt, nfix, fix);
}

// Recovery, second pass over the cells Scheme2D failed: Scheme1Dvsq, then
// Scheme1D (invertor.cc:185-197).
template <int MT>
// With fix non-null the cells the whole chain failed are appended to the
// FixRecovery list (nfix, fix): exactly the cells whose flag ends at 0.
__global__ void __launch_bounds__(kThreads) k_recovery_retry(Dims d, pangu_params p, PT *P,
                                                             const double *U, double *flag,
                                                             unsigned long long *cnt,
                                                             const int *nretry,
                                                             const long long *retry,
                                                             int *nfix, long long *fix) {
  pdl_grid_wait();
  const int n = *nretry;
  // A few cells per stage run the isentropic schemes here, one thread each:
  // their chains of pow calls would wait on L2 for every table load.
  if ((long long)blockIdx.x * blockDim.x < n) pgm::prefetch_tables_l1();
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fc = retry[t];
    const int b = (int)(fc / d.ncell);
    long long c = fc - (long long)b * d.ncell;
    const int k = (int)(c / ((long long)d.N2 * d.N1));
    c -= (long long)k * d.N2 * d.N1;
    const int j = (int)(c / d.N1), i = (int)(c % d.N1);
    Geo g;
    cell_metric<MT>(d, p, b, k, j, i, g);
    double UH[9], PH[9];
    c2p_inputs<MT>(d, p, P, U, b, k, j, i, g, UH, PH, false);
    const double gam = p.adiabatic_index;
    Harm hs;
    harm_setup<MT>(UH, g, hs);
    bool ok = invert_1dvsq<MT>(UH, PH, gam, g, hs) == 0;
    count(cnt, job_of(d, b), PANGU_CNT_C2P_1DVSQ, ok);
    if (!ok) {
      ok = invert_1d<MT>(UH, PH, gam, g, hs) == 0;
      count(cnt, job_of(d, b), PANGU_CNT_C2P_1D, ok);
      count(cnt, job_of(d, b), PANGU_CNT_C2P_FAIL, !ok);
    }
    a_flag(d, flag, b)[fc - (long long)b * d.ncell] = ok ? 1.0 : 0.0;
    c2p_write(d, P, b, k, j, i, PH);
    if (fix) append(nfix, fix, !ok, fc);
  }
}

// ---------------------------------------------------------------------------
// FixRecovery (recovery_fixer.cc:12-119), two phases over the failure list.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_fixrec_scan(Dims d, pangu_params p,
                                                          const double *flag, int *count_out,
                                                          long long *list) {
  pdl_grid_wait();
  int b, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, b, k, j, i)) return;
  b = slot_of(d, b);
  const long long fc = cidx(d, b, k, j, i);
  if (a_flag(d, flag, b)[coff(d, k, j, i)] != 0) return;
  if (p.metric_type == PANGU_METRIC_CKS) {
    const double x = xc(d, b, 0, i), y = xc(d, b, 1, j), z = xc(d, b, 2, k);
    const double a2 = p.a * p.a;
    const double rad2 = x * x + y * y + z * z;
    const double sa = (rad2 - a2) * (rad2 - a2) + 4.0 * a2 * z * z;
    if (sqrt(0.5 * (rad2 - a2 + sqrt(sa))) < p.r_excise) return;
  }
  const int n = atomicAdd(count_out, 1);
  list[n] = fc;
}

__global__ void __launch_bounds__(kThreads) k_fixrec_compute(Dims d, const int *count_in,
                                                             const long long *list,
                                                             const PT *P, const double *flag,
                                                             double *vals) {
  pdl_grid_wait();
  const int n = *count_in;
  const int off2 = d.js != d.je ? 1 : 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fc = list[t];
    const long long b = fc / d.ncell;
    const long long c = fc - b * d.ncell;
    const long long sj = (long long)off2 * d.N1;
    const double *fb = a_flag(d, flag, (int)b) + c;
    auto fl = [&](long long o) { return (int)fb[o]; };
    const int pf1 = fl(sj - 1), pf2 = fl(sj), pf3 = fl(sj + 1), pf4 = fl(1);
    const int pf5 = fl(-sj + 1), pf6 = fl(-sj), pf7 = fl(-sj - 1), pf8 = fl(-1);
    for (int v = 0; v < d.NF; ++v) {
      const PT *q = a_prim(d, P, (int)b, v) + c;
      double val;
      if (pf2 && pf4 && pf6 && pf8)
        val = 0.25 * (q[sj] + q[-sj] + q[-1] + q[1]);
      else if (pf1 && pf3 && pf5 && pf7)
        val = 0.25 * (q[sj + 1] + q[sj - 1] + q[-sj + 1] + q[-sj - 1]);
      else
        val = 0.125 * (q[sj - 1] + q[sj] + q[sj + 1] + q[1] + q[-sj + 1] + q[-sj] + q[-sj - 1] +
                       q[-1]);
      vals[t * d.NF + v] = val;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_fixrec_write(Dims d, const int *count_in,
                                                           const long long *list,
                                                           const double *vals, PT *P,
                                                           double *flag,
                                                           unsigned long long *cnt) {
  pdl_grid_wait();
  const int n = *count_in;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fc = list[t];
    const long long b = fc / d.ncell;
    const long long c = fc - b * d.ncell;
    double w[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; ++v)
      if (v < d.NF) w[v] = vals[t * d.NF + v];
#pragma unroll
    for (int v = 0; v < NPRIM; ++v)
      if (v < d.NF) a_prim(d, P, (int)b, v)[c] = (v >= 2 && v < 5) ? PT(0) : (PT)w[v];
    a_flag(d, flag, (int)b)[c] = 1;
    count(cnt, job_of(d, (int)b), PANGU_CNT_FIXRECOVERY, true);
  }
}

// ---------------------------------------------------------------------------
// Physical boundary conditions (outflow / reflecting) of all faces in one
// pass. Applying the faces in the order ix1, ox1, ix2, ox2, ix3, ox3, each over
// its full transverse range, leaves every ghost cell equal to one interior
// (or exchanged) cell, reached by applying each direction's rule in turn to
// the index, with the reflections' sign flips composed. The kernel computes
// that composition directly; its sources are never written by it.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_bcs(Dims d, int enable_B, PT *P,
                                                  double *flag) {
  pdl_grid_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int bb, idx[3];
  if (!box_index(t, d.NB, 0, d.N3 - 1, 0, d.N2 - 1, 0, d.N1 - 1, bb, idx[2], idx[1], idx[0]))
    return;
  const int b = slot_of(d, bb);
  const signed char *bcf = d.bcf + 6 * b;  // -1 unless the face is a physical boundary
  const int st[3] = {d.is, d.js, d.ks}, en[3] = {d.ie, d.je, d.ke};
  int src[3] = {idx[0], idx[1], idx[2]};
  int flip[3] = {0, 0, 0};
  bool ghost = false;
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const int x = src[dir];
    int kind = -1, outer = 0;
    if (x < st[dir]) {
      kind = bcf[2 * dir];
    } else if (x > en[dir]) {
      kind = bcf[2 * dir + 1];
      outer = 1;
    }
    if (kind < 0) continue;
    ghost = true;
    if (kind == PANGU_BC_OUTFLOW) {
      src[dir] = outer ? en[dir] : st[dir];
    } else {
      src[dir] = outer ? (2 * en[dir] + 1 - x) : (2 * st[dir] - 1 - x);
      flip[dir] ^= 1;
    }
  }
  if (!ghost) return;
  const long long dc = coff(d, idx[2], idx[1], idx[0]);
  const long long sc = coff(d, src[2], src[1], src[0]);
  // every load before the first store (the sources are never written here):
  // one memory latency instead of NF in a row
  double val[NPRIM];
#pragma unroll
  for (int v = 0; v < NPRIM; ++v)
    if (v < d.NF) val[v] = a_prim(d, P, b, v)[sc];
  const bool has_flag = flag || d.tG;
  const double fl = has_flag ? a_flag(d, flag, b)[sc] : 0.0;
#pragma unroll
  for (int v = 0; v < NPRIM; ++v) {
    if (v >= d.NF) continue;
    double x = val[v];
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const bool vel = v == d.pidx[UX1] + dir;
      const bool mag = enable_B && v == d.pidx[BX1] + dir;
      if (flip[dir] && (vel || mag)) x = -x;
    }
    a_prim(d, P, b, v)[dc] = (PT)x;
  }
  if (has_flag) a_flag(d, flag, b)[dc] = fl;
}

// ---------------------------------------------------------------------------
// EstimateTimestepMesh (timestep_estimation.cc:13-102).
// ---------------------------------------------------------------------------
// Per-cell dt values are reduced as order-preserving 64-bit keys: the sign
// bit is set on non-negative doubles and every bit is flipped on negative
// ones, so unsigned comparison of keys orders the doubles (negative values
// included) and atomicMin works on them. The reference's
// "if (timestep > dt) timestep = dt" (timestep_estimation.cc:56-92) takes a
// negative dt as well and skips a NaN, which never compares below.
__device__ __forceinline__ unsigned long long dt_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dt_unkey(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

__global__ void k_dt_init(int n, unsigned long long *mins) {
  pdl_grid_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) mins[t] = dt_key(DBL_MAX);
}

// One CTA row per mesh block (blockIdx.y); warp and CTA minima, then one
// atomic per CTA and direction.
__device__ __forceinline__ void dt_reduce_cta(const Dims &d, double cfl, const double *alfven,
                                              unsigned long long *mins) {
  __shared__ unsigned long long red[3][kThreads / 32];
  const int b = slot_of(d, blockIdx.y);
  const int ni = d.ie - d.is + 1, nj = d.je - d.js + 1, nk = d.ke - d.ks + 1;
  const long long per = (long long)ni * nj * nk;
  const unsigned long long big = dt_key(DBL_MAX);
  unsigned long long m[3] = {big, big, big};
  const double cdx[3] = {MUL(cfl, dx_of(d, b, 0)), MUL(cfl, dx_of(d, b, 1)),
                         MUL(cfl, dx_of(d, b, 2))};
  const int act[3] = {d.N1 > 1, d.N2 > 1, d.N3 > 1};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < per;
       t += (long long)gridDim.x * blockDim.x) {
    int bz, k, j, i;
    box_index(t, 1, d.ks, d.ke, d.js, d.je, d.is, d.ie, bz, k, j, i);
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      if (!act[dir]) continue;
      const double dt = cdx[dir] / a_alfven(d, alfven, b, dir)[coff(d, k, j, i)];
      if (dt == dt) {
        const unsigned long long key = dt_key(dt);
        m[dir] = key < m[dir] ? key : m[dir];
      }
    }
  }
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    unsigned long long v = m[dir];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
      v = w < v ? w : v;
    }
    if ((threadIdx.x & 31) == 0) red[dir][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int dir = threadIdx.x;
    unsigned long long v = red[dir][0];
    for (int w = 1; w < kThreads / 32; ++w) v = red[dir][w] < v ? red[dir][w] : v;
    if (act[dir]) atomicMin(&mins[b * 3 + dir], v);
  }
}

__global__ void __launch_bounds__(kThreads) k_dt_reduce(Dims d, double cfl,
                                                        const double *alfven,
                                                        unsigned long long *mins) {
  pdl_grid_wait();
  dt_reduce_cta(d, cfl, alfven, mins);
}

// The minimum over the job's blocks of 1 / sum_d (1 / min_d), for jobs q =
// first, first + stride, ... (active entries jr[3q+1] .. jr[3q+2]-1 of job
// jr[3q]; the whole domain as job 0 when jr is null), written to dt_out[job].
template <class Mins>
__device__ __forceinline__ void dt_finalize_jobs(const Dims &d, int njobs, const int *jr,
                                                 Mins mins, double *dt_out, int first,
                                                 int stride) {
  for (int q = first; q < njobs; q += stride) {
    const int job = jr ? jr[3 * q] : 0;
    const int s0 = jr ? jr[3 * q + 1] : 0, s1 = jr ? jr[3 * q + 2] : d.NB;
    double gmin = DBL_MAX;
    for (int bb = s0; bb < s1; ++bb) {
      const int b = slot_of(d, bb);
      const double m0 = dt_unkey(mins[3 * b + 0]);
      const double m1 = dt_unkey(mins[3 * b + 1]);
      const double m2 = dt_unkey(mins[3 * b + 2]);
      const double bdt = 1.0 / (1.0 / m0 + 1.0 / m1 + 1.0 / m2);
      if (bdt < gmin) gmin = bdt;
    }
    dt_out[job] = gmin;
  }
}

__global__ void k_dt_finalize(Dims d, int njobs, const int *jr, const unsigned long long *mins,
                              double *dt_out) {
  pdl_grid_wait();
  if (blockIdx.x != 0) return;
  dt_finalize_jobs(d, njobs, jr, mins, dt_out, threadIdx.x, blockDim.x);
}

// The engine's dt estimate in one launch: every CTA reduces its part, and
// the CTA that finishes last (a ticket taken after a fence, no waiting)
// finalises every job, then puts the per-block minima back to DBL_MAX and the
// ticket to 0 for the next call.
__global__ void __launch_bounds__(kThreads) k_dt_reduce_final(Dims d, double cfl,
                                                              const double *alfven,
                                                              unsigned long long *mins,
                                                              unsigned int *ticket, int njobs,
                                                              const int *jr, double *dt_out,
                                                              int nmins) {
  pdl_grid_wait();
  __shared__ bool last;
  dt_reduce_cta(d, cfl, alfven, mins);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int total = gridDim.x * gridDim.y;
    last = atomicAdd(ticket, 1u) == total - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // every other CTA's atomics are complete; read the minima past L1
  const volatile unsigned long long *vm = mins;
  dt_finalize_jobs(d, njobs, jr, vm, dt_out, threadIdx.x, blockDim.x);
  __syncthreads();
  const unsigned long long big = dt_key(DBL_MAX);
  for (int t = threadIdx.x; t < nmins; t += blockDim.x) mins[t] = big;
  if (threadIdx.x == 0) *ticket = 0u;
}

__global__ void k_update_dt(int njobs, const int *jr, double *dt, const double *dt_est,
                            double factor) {
  pdl_grid_wait();
  if (blockIdx.x != 0) return;
  for (int q = threadIdx.x; q < njobs; q += blockDim.x) {
    const int job = jr ? jr[3 * q] : 0;
    const double grown = factor * dt[job];
    dt[job] = (dt_est[job] < grown) ? dt_est[job] : grown;
  }
}

// ---------------------------------------------------------------------------
// Device-side initial conditions of the benchmark problems, the same
// formulas as pangu_b200/problems.py (Orszag-Tang, Brio-Wu, and the
// Fishbone-Moncrief torus of problem_generator.cpp:103-558 with its
// MeshPostInitialization), so that jobs can start on the device.
// ---------------------------------------------------------------------------
struct GenArgs {
  int kind;
  unsigned long long seed;
  double rin, rmax, kappa, pert, beta, cut;
  double l, lnh_in;  // torus constants computed on the host
};

// SplitMix64 (Steele, Lea and Flood 2014) of seed * golden + idx, mapped to
// [-1, 1) from its top 53 bits; problems.hash_uniform gives the same values.
__device__ __forceinline__ double hash_uniform(unsigned long long seed, unsigned long long idx) {
  const unsigned long long gold = 0x9E3779B97F4A7C15ull;
  unsigned long long z = seed * gold + idx;
  z += gold;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return 2.0 * ((double)(z >> 11) * 0x1p-53) - 1.0;
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *m, double v) {
  if (v > 0.0) atomicMax(m, (unsigned long long)__double_as_longlong(v));
}

// Every cell of the job's blocks (ghosts included, as the host generator
// fills them). red[0], red[1]: torus maxima of rho and u before normalising.
template <int MT>
__global__ void __launch_bounds__(kThreads) k_gen_cells(Dims d, pangu_params p, GenArgs ga, PT *P,
                                                        unsigned long long *red) {
  pdl_grid_wait();
  int bb, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, 0, d.N3 - 1, 0, d.N2 - 1, 0, d.N1 - 1, bb, k, j, i)) return;
  const int b = slot_of(d, bb);
  const double gam = p.adiabatic_index;
  double pr[NPRIM] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double pi = 3.141592653589793;
  if (ga.kind == PANGU_PROBLEM_ORSZAG_TANG) {
    const double x = xc(d, b, 0, i), y = xc(d, b, 1, j);
    const double vx = -0.5 * sin(2 * pi * y), vy = 0.5 * sin(2 * pi * x);
    const double W = 1.0 / sqrt(1.0 - vx * vx - vy * vy);
    pr[RHO] = 25.0 / (36.0 * pi);
    pr[ENY] = 5.0 / (12.0 * pi) / (gam - 1.0);
    pr[UX1] = W * vx;
    pr[UX2] = W * vy;
    pr[BX1] = -sin(2 * pi * y) / sqrt(4 * pi);
    pr[BX2] = sin(4 * pi * x) / sqrt(4 * pi);
    pr[ENT] = (gam - 1.0) * pr[ENY] * PGK_POW(pr[RHO], -gam);
  } else if (ga.kind == PANGU_PROBLEM_BRIO_WU) {
    const bool left = xc(d, b, 0, i) < 0;
    pr[RHO] = left ? 1.0 : 0.125;
    pr[ENY] = (left ? 1.0 : 0.1) / (gam - 1.0);
    pr[BX1] = 0.5;
    pr[BX2] = left ? 1.0 : -1.0;
    pr[ENT] = (gam - 1.0) * pr[ENY] * PGK_POW(pr[RHO], -gam);
  } else if (MT == MKS) {
    const int W1 = d.N1 + 1, W2 = d.N2 + 1;
    const double *T1 = d.t1 + (long long)b * kT1Rows * W1;
    const double *T2 = d.t2 + (long long)b * 12 * W2;
    const double r = T1[i], sth = T2[j], cth = T2[W2 + j];
    const double a = p.a, a2 = a * a, l = ga.l;
    const double DD = r * r - 2.0 * r + a2;
    const double AA = (r * r + a2) * (r * r + a2) - DD * a2 * sth * sth;
    const double SS = r * r + a2 * cth * cth;
    double lnh = 0.5 * log((1.0 + sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD /
                                        (AA * sth * AA * sth))) / (SS * DD / AA)) -
                 0.5 * sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD / (AA * AA * sth * sth)) -
                 2.0 * a * r * l / AA - ga.lnh_in;
    if (!(r >= ga.rin)) lnh = 1.0;
    const double hm1 = exp(lnh) - 1.0;
    const bool inside = lnh >= 0.0 && r >= ga.rin && hm1 > 0.0;
    if (inside) {
      const double rho = PGK_POW(hm1 * (gam - 1.0) / (ga.kappa * gam), 1.0 / (gam - 1.0));
      const long long cell = ((long long)bb * d.N3 + k) * d.N2 * d.N1 + (long long)j * d.N1 + i;
      const double rnd = hash_uniform(ga.seed, (unsigned long long)cell);
      const double eint = ga.kappa * PGK_POW(rho, gam) / (gam - 1.0) * (1.0 + ga.pert * rnd);
      const double ent = (gam - 1.0) * eint * PGK_POW(rho, -gam);
      const double expm2chi = SS * SS * DD / (AA * AA * sth * sth);
      const double up1 = sqrt((-1.0 + sqrt(1.0 + 4.0 * l * l * expm2chi)) / 2.0);
      const double up_bl = 2.0 * a * r * sqrt(1.0 + up1 * up1) / sqrt(AA * SS * DD) +
                           sqrt(SS / AA) * up1 / sth;
      // Boyer-Lindquist metric entries g_00, g_03, g_33 (BL.h; the code
      // Jacobian leaves them unchanged)
      const double r2 = r * r, sth2 = sth * sth;
      const double mu = 1.0 + a2 * cth * cth / r2;
      const double irm = 1.0 / (r * mu);
      const double g00 = -1.0 + 2.0 * irm, g03 = -2.0 * a * sth2 * irm;
      const double g33 = r2 * sth2 * (1.0 + a2 / r2 + 2.0 * a2 * sth2 / (r * r2 * mu));
      const double AAq = g00, BBq = 2.0 * g03 * up_bl, CCq = 1.0 + g33 * up_bl * up_bl;
      const double u0 = (-BBq - sqrt(BBq * BBq - 4.0 * AAq * CCq)) / (2.0 * AAq);
      // BL -> KS -> code: u^r_BL = 0 leaves (u0, 0, 0, up); the weighted
      // velocity adds the shift beta^i = gcon^{0i} alpha^2 (KS code metric)
      Geo g;
      cell_metric<MT>(d, p, b, k, j, i, g);
      const double al2 = g.alpha * g.alpha;
      pr[RHO] = rho;
      pr[ENY] = eint;
      pr[UX1] = g.gcon[0][1] * al2 * u0;
      pr[UX2] = g.gcon[0][2] * al2 * u0;
      pr[UX3] = up_bl + g.gcon[0][3] * al2 * u0;
      pr[ENT] = ent;
      atomic_max_pos(&red[0], rho);
      atomic_max_pos(&red[1], eint);
    }
  }
  pr[KEL] = p.fel_0 * pr[ENT];
  const long long q = coff(d, k, j, i);
#pragma unroll
  for (int v = 0; v < NPRIM; ++v)
    if (d.pidx[v] >= 0) a_prim(d, P, b, d.pidx[v])[q] = (PT)pr[v];
}

// Torus: density and energy divided by the maximum density (all cells).
__global__ void __launch_bounds__(kThreads) k_gen_normalize(Dims d, PT *P,
                                                            const unsigned long long *red) {
  pdl_grid_wait();
  int bb, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, 0, d.N3 - 1, 0, d.N2 - 1, 0, d.N1 - 1, bb, k, j, i)) return;
  const int b = slot_of(d, bb);
  const double rhomax = __longlong_as_double((long long)red[0]);
  const long long q = coff(d, k, j, i);
  PT *p0 = a_prim(d, P, b, 0), *p1 = a_prim(d, P, b, 1);
  p0[q] = (PT)((double)p0[q] / rhomax);
  p1[q] = (PT)((double)p1[q] / rhomax);
}

// Torus field (interior cells): A_phi = max(<rho> - cut, 0) at cell corners,
// B = curl A / sqrt|g| by centred differences, and the maximum of b^2.
template <int MT>
__global__ void __launch_bounds__(kThreads) k_gen_bfield(Dims d, pangu_params p, GenArgs ga, PT *P,
                                                         unsigned long long *red) {
  pdl_grid_wait();
  int bb, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, bb, k, j, i)) return;
  const int b = slot_of(d, bb);
  const long long q = coff(d, k, j, i);
  const PT *p0 = a_prim(d, P, b, 0);
  auto rho = [&](int jj, int ii) -> double { return p0[q + (long long)(jj - j) * d.N1 + (ii - i)]; };
  auto corner = [&](int jj, int ii) -> double {
    const double avg = 0.25 * (((rho(jj, ii) + rho(jj, ii - 1)) + rho(jj - 1, ii)) + rho(jj - 1, ii - 1));
    const double v = avg - ga.cut;
    return v > 0.0 ? v : 0.0;
  };
  const double a00 = corner(j - 1, i - 1), a01 = corner(j, i - 1), a10 = corner(j - 1, i),
               a11 = corner(j, i);
  Geo g;
  cell_metric<MT>(d, p, b, k, j, i, g);
  const double b1 = -(((a00 - a01) + a10) - a11) / ((2.0 * dx_of(d, b, 1)) * g.sg);
  const double b2 = (((a00 + a01) - a10) - a11) / ((2.0 * dx_of(d, b, 0)) * g.sg);
  a_prim(d, P, b, d.pidx[BX1])[q] = (PT)b1;
  a_prim(d, P, b, d.pidx[BX2])[q] = (PT)b2;
  double pc[NPRIM];
  load_prim(d, P, b, k, j, i, pc);
  State st;
  calc_state<MT>(pc, g, st);
  atomic_max_pos(&red[2], st.bsq);
}

// Torus field normalised to the target plasma beta (interior cells).
__global__ void __launch_bounds__(kThreads) k_gen_scale(Dims d, double gam, double beta,
                                                        PT *P, const unsigned long long *red) {
  pdl_grid_wait();
  int bb, k, j, i;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!box_index(t, d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie, bb, k, j, i)) return;
  const int b = slot_of(d, bb);
  const double rhomax = __longlong_as_double((long long)red[0]);
  const double umax = __longlong_as_double((long long)red[1]);
  const double bsq_max = __longlong_as_double((long long)red[2]);
  const double beta_min = 2.0 * (gam - 1.0) * (umax / rhomax) / (bsq_max + 1.0e-30);
  const double norm = sqrt(beta_min / beta);
  const long long q = coff(d, k, j, i);
  for (int v = BX1; v <= BX3; ++v) {
    PT *pv = a_prim(d, P, b, d.pidx[v]);
    pv[q] = (PT)((double)pv[q] * norm);
  }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline int check_launch() {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PANGU_OK : PANGU_ECUDA;
}

inline long long box_count(int NB, int k0, int k1, int j0, int j1, int i0, int i1) {
  if (k1 < k0 || j1 < j0 || i1 < i0) return 0;
  return (long long)NB * (k1 - k0 + 1) * (j1 - j0 + 1) * (i1 - i0 + 1);
}

// Launch with programmatic stream serialisation: the kernel may be scheduled
// while the previous kernel of the stream drains; it waits for it in
// pdl_grid_wait() before touching memory.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl_smem(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                   cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                              Args... args) {
  return launch_pdl_smem(kernel, grid, block, 0, s, args...);
}

#define DISPATCH_MT(mt, KERNEL, grid, stream, ...)                          \
  do {                                                                      \
    switch (mt) {                                                           \
      case PANGU_METRIC_MKS: launch_pdl(KERNEL<MKS>, dim3(grid), dim3(kThreads), stream, __VA_ARGS__); break; \
      case PANGU_METRIC_BL: launch_pdl(KERNEL<BL>, dim3(grid), dim3(kThreads), stream, __VA_ARGS__); break; \
      case PANGU_METRIC_CKS: launch_pdl(KERNEL<CKS>, dim3(grid), dim3(kThreads), stream, __VA_ARGS__); break; \
      default: launch_pdl(KERNEL<MINKOWSKI>, dim3(grid), dim3(kThreads), stream, __VA_ARGS__); break; \
    }                                                                       \
  } while (0)

#define DISPATCH_MT_T(mt, KERNEL, grid, threads, stream, ...)                                 \
  do {                                                                                       \
    switch (mt) {                                                                            \
      case PANGU_METRIC_MKS: launch_pdl(KERNEL<MKS>, dim3(grid), dim3(threads), stream, __VA_ARGS__); break; \
      case PANGU_METRIC_BL: launch_pdl(KERNEL<BL>, dim3(grid), dim3(threads), stream, __VA_ARGS__); break; \
      case PANGU_METRIC_CKS: launch_pdl(KERNEL<CKS>, dim3(grid), dim3(threads), stream, __VA_ARGS__); break; \
      default: launch_pdl(KERNEL<MINKOWSKI>, dim3(grid), dim3(threads), stream, __VA_ARGS__); break; \
    }                                                                                        \
  } while (0)

// Streaming multiprocessors of the current device (148 on a B200), queried
// once per process and device.
inline int device_sms() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n;
  }
  return cached[dev];
}

inline unsigned grid_flux(long long n, int threads) {
  return (unsigned)std::max<long long>(1, (n + threads - 1) / threads);
}

// Every array a stage task may touch is given, as a contiguous array or by
// its per-(block, component) table.
bool pack_ok(const pangu_engine *e, const pangu_pack *md) {
  if (!e || !md) return false;
  auto has = [](const void *a, const void *tab) { return a || tab; };
  if (!has(md->prim, md->prim_vars) || !has(md->cons, md->cons_vars) ||
      !has(md->flux1, md->flux1_vars) || !has(md->alfven, md->alfven_vars) ||
      !has(md->efield, md->efield_vars))
    return false;
  if (e->d.ndim >= 2 && !has(md->flux2, md->flux2_vars)) return false;
  if (e->d.ndim == 3 && !has(md->flux3, md->flux3_vars)) return false;
  if (e->p.recovery == PANGU_RECOVERY_CHAINER && !has(md->flag, md->flag_vars)) return false;
  return true;
}

// True when no array of md goes through a per-(block, component) table.
inline bool contiguous(const pangu_pack *md) {
  return !md->prim_vars && !md->cons_vars && !md->flux1_vars && !md->flux2_vars &&
         !md->flux3_vars && !md->alfven_vars && !md->efield_vars && !md->flag_vars;
}

// The engine's Dims with the layout tables of md's arrays (null tables: the
// contiguous layout).
inline Dims bind(const pangu_engine *e, const pangu_pack *md) {
  Dims d = e->d;
  d.tP = reinterpret_cast<void *const *>(md->prim_vars);
  d.tU = d.tUi = md->cons_vars;
  d.tF = nullptr;
  d.tF1 = md->flux1_vars;
  d.tF2 = md->flux2_vars;
  d.tF3 = md->flux3_vars;
  d.tA = md->alfven_vars;
  d.tE = md->efield_vars;
  d.tG = md->flag_vars;
  return d;
}

// FixPrimitive; with_cons also computes the interior conserved variables
// (CalculateConservative) in the same pass (the stage path).
int run_fix_primitive(pangu_engine *e, const pangu_pack *md, bool with_cons, cudaStream_t s) {
  const Dims d = bind(e, md);
  const long long n = (long long)d.NB * d.ncell;
  // on the stage path (with_cons) the C2P retry and FixRecovery list counters
  // are zeroed here for Recovery
  DISPATCH_MT(e->p.metric_type, k_fix_primitive, grid_for(n), s, d, e->p, prim_of(md), e->d_cnt,
              md->cons, with_cons ? 1 : 0, PGK_MIXED ? 0 : 1,
              with_cons ? e->d_fail_count : nullptr, with_cons ? e->d_fix_count : nullptr);
  ++e->launches;
  return check_launch();
}

int run_fix_primitive(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  return run_fix_primitive(e, md, false, s);
}

int run_calc_cons(pangu_engine *e, const Dims &d, const pangu_pack *md, bool with_b,
                  cudaStream_t s) {
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  DISPATCH_MT(e->p.metric_type, k_calc_cons, grid_for(n), s, d, e->p, prim_of(md), md->cons,
              with_b ? 1 : 0);
  ++e->launches;
  return check_launch();
}

int run_calc_cons(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  return run_calc_cons(e, bind(e, md), md, !PGK_MIXED, s);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the runtime only).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// TMA-staged flux kernels need rows of whole 16-byte units (N1 * sizeof(PT)
// a multiple of 16) and the tensor-map encoder.
inline bool tma_ok(const pangu_engine *e) {
  return ((size_t)e->d.N1 * sizeof(PT)) % 16 == 0 && e->d.NF <= 256 &&
         tensor_map_encoder() != nullptr;
}

// Tensor map of md's primitives as a 4D array {i, j, k, slot * NF + var}
// (i fastest) with the box of the TMA-staged flux kernels of direction dir:
// x1, kTmaColsX1 x kTmaRowsX1 rows (j); x2 / x3, kTmaCols x (4 + 5) cells
// running along j / k; every component.
inline bool tma_tile_map(const pangu_engine *e, const pangu_pack *md, int dir, CUtensorMap *tm) {
  const Dims &d = e->d;
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)d.N1, (cuuint64_t)d.N2, (cuuint64_t)d.N3,
                              (cuuint64_t)e->capacity * d.NF};
  const cuuint64_t strides[3] = {(cuuint64_t)d.N1 * sizeof(PT),
                                 (cuuint64_t)d.N1 * d.N2 * sizeof(PT),
                                 (cuuint64_t)d.N1 * d.N2 * d.N3 * sizeof(PT)};
  const cuuint32_t box[4] = {(cuuint32_t)(dir == 1 ? kTmaColsX1 : kTmaCols),
                             dir == 1 ? (cuuint32_t)kTmaRowsX1 : (dir == 2 ? 9u : 1u),
                             dir == 3 ? 9u : 1u, (cuuint32_t)d.NF};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(tm, sizeof(PT) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
             4, (void *)prim_of(md), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launches the flux kernel of one direction with a given march depth
// (x2/x3) and CTA size. The TMA-staged kernels read the contiguous layout; a
// pack whose primitives come through a table runs the thread-loaded form of
// the same tile shape instead.
template <int MT, int OPT>
void launch_flux_dir(const pangu_engine *e, const pangu_pack *md, int dir, int march, int threads,
                     cudaStream_t s) {
  Dims d = bind(e, md);
  d.tF = dir == 1 ? md->flux1_vars : (dir == 2 ? md->flux2_vars : md->flux3_vars);
  if (march == kMarchTma && md->prim_vars) march = dir == 1 ? 1 : 0;
  const bool hll = e->p.riemann_solver == PANGU_RIEMANN_HLL;
  int k0 = d.ks - d.o3, k1 = d.ke + d.o3, j0 = d.js - d.o2, j1 = d.je + d.o2;
  int i0 = d.is - d.o1, i1 = d.ie + d.o1;
  if (dir == 1) { i0 = d.is; i1 = d.ie + 1; }
  if (dir == 2) { j0 = d.js; j1 = d.je + 1; }
  if (dir == 3) {  // hll.cc:293-296 narrows the transverse range
    k0 = d.ks; k1 = d.ke + 1;
    if (hll) { j0 = d.js; j1 = d.je; i0 = d.is; i1 = d.ie; }
  }
  double *F = dir == 1 ? md->flux1 : (dir == 2 ? md->flux2 : md->flux3);
  const PT *P = prim_of(md);
  if (dir == 1 && march == kMarchTma) {
    CUtensorMap tm;
    if (!tma_tile_map(e, md, 1, &tm)) return;  // pangu_set_flux_config checked tma_ok
    const int nseg = (i1 - i0 + 1 + kFacesPerWarp - 1) / kFacesPerWarp;
    const long long nt = (long long)d.NB * (k1 - k0 + 1) *
                         ((j1 - j0 + 1 + kTmaRowsX1 - 1) / kTmaRowsX1) * nseg;
    launch_pdl_smem(k_flux_x1_tma<MT, OPT>, dim3((unsigned)nt), dim3(32 * kTmaRowsX1),
                    tma_x1_smem(d.NF), s, tm, d, e->p, k0, k1, j0, j1, i0, i1, F, md->alfven,
                    e->d_err);
    return;
  }
  if (dir == 1) {
    const int nseg = (i1 - i0 + 1 + kFacesPerWarp - 1) / kFacesPerWarp;
    const long long warps = (long long)d.NB * (k1 - k0 + 1) * (j1 - j0 + 1) * nseg;
    launch_pdl_smem(k_flux_x1<MT, OPT>, dim3(grid_flux(32 * warps, threads)), dim3(threads),
                    split_faces(MT) ? 3 * NPRIM * threads * sizeof(double) : 0, s, d, e->p, k0,
                    k1, j0, j1, i0, i1, P, F, md->alfven);
    return;
  }
  const int m = dir == 2 ? (j1 - j0 + 1) : (k1 - k0 + 1);
  const int na = dir == 2 ? (k1 - k0 + 1) : (j1 - j0 + 1);
  if (march == kMarchTma) {  // TMA-staged tiles of 32 x 4 faces
    CUtensorMap tm;
    if (!tma_tile_map(e, md, dir, &tm)) return;  // pangu_set_flux_config checked tma_ok
    const long long nt = (long long)d.NB * na * ((m + 3) / 4) * ((i1 - i0 + 1 + 31) / 32);
    if (dir == 2)
      launch_pdl_smem(k_flux_tile_tma<MT, 2, 4, OPT>, dim3((unsigned)nt), dim3(128),
                      tma_tile_smem<4>(d.NF), s, tm, d, e->p, k0, k1, j0, j1, i0, i1, F,
                      md->alfven, e->d_err);
    else
      launch_pdl_smem(k_flux_tile_tma<MT, 3, 4, OPT>, dim3((unsigned)nt), dim3(128),
                      tma_tile_smem<4>(d.NF), s, tm, d, e->p, k0, k1, j0, j1, i0, i1, F,
                      md->alfven, e->d_err);
    return;
  }
  if (march == 0) {  // tiles of 32 x (threads / 32) faces
    const long long nt = (long long)d.NB * na * ((m + threads / 32 - 1) / (threads / 32)) *
                         ((i1 - i0 + 1 + 31) / 32);
#define PGK_TILE(D, TF)                                                                     \
  launch_pdl(k_flux_tile<MT, D, TF, OPT>, dim3((unsigned)nt), dim3(32 * TF), s, d, e->p, k0, k1, j0, \
             j1, i0, i1, P, F, md->alfven)
    if (dir == 2) {
      if (threads == 128) PGK_TILE(2, 4); else PGK_TILE(2, 8);
    } else {
      if (threads == 128) PGK_TILE(3, 4); else PGK_TILE(3, 8);
    }
#undef PGK_TILE
    return;
  }
  const long long n = (long long)d.NB * na * ((m + march - 1) / march) * (i1 - i0 + 1);
  const unsigned g = grid_flux(n, threads);
  const size_t msm = split_faces(MT) ? 4 * NPRIM * threads * sizeof(double) : 0;
#define PGK_MARCH(M)                                                                           \
  if (dir == 2)                                                                                \
    launch_pdl_smem(k_flux_march2<MT, M, OPT>, dim3(g), dim3(threads), msm, s, d, e->p, k0, k1, j0, \
                    j1, i0, i1, P, F, md->alfven);                                             \
  else                                                                                         \
    launch_pdl_smem(k_flux_march3<MT, M, OPT>, dim3(g), dim3(threads), msm, s, d, e->p, k0, k1, j0, \
                    j1, i0, i1, P, F, md->alfven);
  switch (march) {
    case 1: PGK_MARCH(1) break;
    case 2: PGK_MARCH(2) break;
    default: PGK_MARCH(4) break;
  }
#undef PGK_MARCH
}

template <int MT>
void launch_flux_opt(const pangu_engine *e, const pangu_pack *md, int dir, int march, int threads,
                     cudaStream_t s) {
#if PGK_MIXED
  launch_flux_dir<MT, 0>(e, md, dir, march, threads, s);  // options read at run time
#else
  const int opt = (e->p.riemann_solver == PANGU_RIEMANN_HLL ? kFluxHLL : 0) |
                  (e->p.limiter == PANGU_LIMITER_MC ? kFluxMC : 0);
  switch (opt) {
    case 0: launch_flux_dir<MT, 0>(e, md, dir, march, threads, s); break;
    case kFluxHLL: launch_flux_dir<MT, kFluxHLL>(e, md, dir, march, threads, s); break;
    case kFluxMC: launch_flux_dir<MT, kFluxMC>(e, md, dir, march, threads, s); break;
    default: launch_flux_dir<MT, kFluxHLL | kFluxMC>(e, md, dir, march, threads, s); break;
  }
#endif
}

int run_flux_dir(pangu_engine *e, const pangu_pack *md, int dir, int march, int threads,
                 cudaStream_t s) {
  switch (e->p.metric_type) {
    case PANGU_METRIC_MKS: launch_flux_opt<MKS>(e, md, dir, march, threads, s); break;
    case PANGU_METRIC_BL: launch_flux_opt<BL>(e, md, dir, march, threads, s); break;
    case PANGU_METRIC_CKS: launch_flux_opt<CKS>(e, md, dir, march, threads, s); break;
    default: launch_flux_opt<MINKOWSKI>(e, md, dir, march, threads, s); break;
  }
  ++e->launches;
  return check_launch();
}

int run_fluxes(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  for (int dir = 1; dir <= e->d.ndim; ++dir) {
    const int rc = run_flux_dir(e, md, dir, e->tune.march[dir - 1], e->tune.threads[dir - 1], s);
    if (rc) return rc;
  }
  return PANGU_OK;
}

// Times every candidate tile shape of each direction's flux kernel on the
// pack's own data (best of three launches after one untimed launch, CUDA
// events on stream s) and keeps the fastest in e->tune. The candidates
// compute every face identically, so the choice never changes results.
bool flux_tma_ok(const pangu_engine *e) { return tma_ok(e); }

int run_autotune(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  if (e->d.NB == 0) return PANGU_OK;
  cudaEvent_t ev[2];
  if (cudaEventCreate(&ev[0]) != cudaSuccess) return PANGU_ECUDA;
  if (cudaEventCreate(&ev[1]) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    return PANGU_ECUDA;
  }
  int rc = PANGU_OK;
  // candidates {march, CTA size}; march 0 is the tiled kernel (tiles of 32 x
  // CTA size / 32 faces), kMarchTma its TMA-staged form (where the rows allow)
  const int cand[9][2] = {{1, 64}, {1, 128}, {2, 64}, {2, 128}, {4, 64}, {4, 128}, {0, 128},
                          {0, 256}, {kMarchTma, 128}};
  // x1: march 1 with CTAs of 64 or 128 threads, or the TMA-staged rows
  const int x1cand[3][2] = {{1, 64}, {1, 128}, {kMarchTma, 128}};
  // Each candidate's time is the minimum over two interleaved rounds of five
  // launches after one warm-up launch, so that clock ramps and cache states
  // do not favour whichever candidate runs first. A candidate of x2 (x3) is
  // timed behind the chosen x1 (and x2) launches, as it runs in a stage, so
  // that it meets the caches those leave.
  for (int dir = 1; dir <= e->d.ndim && !rc; ++dir) {
    const int nc = dir == 1 ? (tma_ok(e) ? 3 : 2) : (tma_ok(e) ? 9 : 8);
    float t[9];
    for (int ci = 0; ci < nc; ++ci) t[ci] = 1e30f;
    for (int round = 0; round < 2 && !rc; ++round)
      for (int ci = 0; ci < nc && !rc; ++ci) {
        const int march = dir == 1 ? x1cand[ci][0] : cand[ci][0];
        const int threads = dir == 1 ? x1cand[ci][1] : cand[ci][1];
        for (int rep = 0; rep < 6 && !rc; ++rep) {
          if (cudaEventRecord(ev[0], s) != cudaSuccess) rc = PANGU_ECUDA;
          for (int lower = 1; lower < dir && !rc; ++lower)
            rc = run_flux_dir(e, md, lower, e->tune.march[lower - 1], e->tune.threads[lower - 1], s);
          if (!rc) rc = run_flux_dir(e, md, dir, march, threads, s);
          if (!rc && (cudaEventRecord(ev[1], s) != cudaSuccess ||
                      cudaEventSynchronize(ev[1]) != cudaSuccess))
            rc = PANGU_ECUDA;
          float ms = 0;
          if (!rc && cudaEventElapsedTime(&ms, ev[0], ev[1]) != cudaSuccess) rc = PANGU_ECUDA;
          if (!rc && rep > 0) t[ci] = std::min(t[ci], ms);
        }
      }
    float best = 1e30f;
    for (int ci = 0; ci < nc && !rc; ++ci)
      if (t[ci] < best) {
        best = t[ci];
        e->tune.march[dir - 1] = dir == 1 ? x1cand[ci][0] : cand[ci][0];
        e->tune.threads[dir - 1] = dir == 1 ? x1cand[ci][1] : cand[ci][1];
      }
  }
  if (!rc) e->tune.tuned = 1;
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return rc;
}


int run_ct(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  const Dims d = bind(e, md);
  const int o1 = d.N1 > 1, o2 = d.N2 > 1, o3 = d.N3 > 1;
  launch_pdl(k_ct_emf, dim3(grid_for(box_count(d.NB, d.ks, d.ke + o3, d.js, d.je + o2, d.is,
                                                d.ie + o1))),
             dim3(kThreads), s, d, md->flux1, md->flux2, md->flux3, md->efield);
  ++e->launches;
  launch_pdl(k_ct_faces, dim3(grid_for(box_count(d.NB, d.ks, d.ke + o3, d.js, d.je + o2, d.is,
                                                  d.ie + o1))),
             dim3(kThreads), s, d, md->flux1, md->flux2, md->flux3, md->efield);
  ++e->launches;
  return check_launch();
}

int run_update(pangu_engine *e, const pangu_pack *mi, const pangu_pack *m0, const pangu_pack *m1,
               double beta, const double *dt, cudaStream_t s) {
  Dims d = bind(e, m0);  // the fluxes of mc0
  d.tU = m1->cons_vars;  // written: mc1's conserved variables
  d.tUi = mi->cons_vars;  // read: the starting state's
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  launch_pdl(k_flux_div_update, dim3(grid_for(n)), dim3(kThreads), s, d, m0->flux1, m0->flux2,
             m0->flux3, mi->cons, m1->cons, beta, dt);
  ++e->launches;
  return check_launch();
}

int run_exchange_range(pangu_engine *e, const pangu_pack *md, long long off, long long n,
                       cudaStream_t s) {
  if (n == 0) return PANGU_OK;
  launch_pdl(k_exchange, dim3(grid_for(n)), dim3(kThreads), s, bind(e, md), n, e->d_xdst + off,
             e->d_xsrc + off, prim_of(md), md->flag);
  ++e->launches;
  return check_launch();
}

int run_exchange(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  return run_exchange_range(e, md, 0, e->nxch, s);
}

int run_halo_pack(pangu_engine *e, const pangu_pack *md, double *buf, cudaStream_t s) {
  const long long n = e->hsend_off.empty() ? 0 : e->hsend_off.back();
  if (n == 0) return PANGU_OK;
  launch_pdl(k_halo_pack, dim3(grid_for(n)), dim3(kThreads), s, bind(e, md), n, e->d_hsend, prim_of(md),
             md->flag, buf);
  ++e->launches;
  return check_launch();
}

int run_halo_unpack(pangu_engine *e, const pangu_pack *md, const double *buf, cudaStream_t s) {
  const long long n = e->hrecv_off.empty() ? 0 : e->hrecv_off.back();
  if (n == 0) return PANGU_OK;
  launch_pdl(k_halo_unpack, dim3(grid_for(n)), dim3(kThreads), s, bind(e, md), n, e->d_hrecv, prim_of(md),
             md->flag, buf);
  ++e->launches;
  return check_launch();
}

int run_source(pangu_engine *e, const pangu_pack *md, double beta, const double *dt,
               cudaStream_t s) {
  const Dims d = bind(e, md);
  if (e->p.metric_type == PANGU_METRIC_MINKOWSKI) return PANGU_OK;  // zero connection
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  DISPATCH_MT(e->p.metric_type, k_source, grid_for(n), s, d, e->p, prim_of(md), md->cons, beta, dt);
  ++e->launches;
  return check_launch();
}

// Recovery; with list_fix the retry pass also lists the cells FixRecovery
// repairs (the stage path).
// list_fix: the stage path, whose FixPrimitive launch has zeroed both list
// counters; otherwise the retry counter is zeroed here.
int run_recovery(pangu_engine *e, const pangu_pack *md, bool list_fix, cudaStream_t s) {
  const Dims d = bind(e, md);
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  const unsigned grid = (unsigned)((n + kRecoveryThreads - 1) / kRecoveryThreads);
  if (e->p.recovery == PANGU_RECOVERY_CHAINER && (long long)grid <= 7LL * device_sms()) {
    // one wave: the chain in the same pass; the cells the whole chain fails
    // form FixRecovery's list (the stage path)
    DISPATCH_MT_T(e->p.metric_type, k_recovery_chain, grid, kRecoveryThreads, s, d, e->p,
                  prim_of(md), md->cons, md->flag, e->d_cnt,
                  list_fix ? e->d_fix_count : nullptr, list_fix ? e->d_fix_list : nullptr);
    ++e->launches;
    return check_launch();
  }
  if (!list_fix && cudaMemsetAsync(e->d_fail_count, 0, sizeof(int), s) != cudaSuccess)
    return PANGU_ECUDA;
  DISPATCH_MT_T(e->p.metric_type, k_recovery, grid, kRecoveryThreads, s, d, e->p, prim_of(md),
                md->cons, md->flag, e->d_cnt, e->d_fail_count, e->d_fail_list);
  ++e->launches;
  if (e->p.recovery == PANGU_RECOVERY_CHAINER) {
    // one-warp CTAs: the few thousand retried cells spread over every SM
    DISPATCH_MT_T(e->p.metric_type, k_recovery_retry, 8 * 148, 32, s, d, e->p, prim_of(md),
                  md->cons, md->flag, e->d_cnt, e->d_fail_count, e->d_fail_list,
                  list_fix ? e->d_fix_count : nullptr, list_fix ? e->d_fix_list : nullptr);
    ++e->launches;
  }
  return check_launch();
}

int run_recovery(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  return run_recovery(e, md, false, s);
}

int run_heating(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  const Dims d = bind(e, md);
  if (!e->p.enable_heating) return PANGU_OK;
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  DISPATCH_MT(e->p.metric_type, k_heating, grid_for(n), s, d, e->p, prim_of(md), md->cons);
  ++e->launches;
  return check_launch();
}

// FixRecovery. listed: the failed cells were listed by the recovery retry pass
// (the stage path); otherwise a scan of the flags finds them. Both lists hold
// the same cells (in a different order, which the two-phase fix ignores).
int run_fix_recovery(pangu_engine *e, const pangu_pack *md, bool listed, cudaStream_t s) {
  const Dims d = bind(e, md);
  int *count = e->d_fix_count;
  long long *list = e->d_fix_list;
  if (!listed) {
    if (cudaMemsetAsync(count, 0, sizeof(int), s) != cudaSuccess) return PANGU_ECUDA;
    const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
    k_fixrec_scan<<<grid_for(n), kThreads, 0, s>>>(d, e->p, md->flag, count, list);
    ++e->launches;
  }
  const unsigned g = 2 * 148;
  launch_pdl(k_fixrec_compute, dim3(g), dim3(kThreads), s, d, count, list, prim_of(md), md->flag,
             e->d_fail_vals);
  launch_pdl(k_fixrec_write, dim3(g), dim3(kThreads), s, d, count, list, e->d_fail_vals,
             prim_of(md), md->flag, e->d_cnt);
  e->launches += 2;
  return check_launch();
}

int run_fix_recovery(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  return run_fix_recovery(e, md, false, s);
}

// Physical BCs of the blocks of d (all active blocks, or one job's).
int run_bcs(pangu_engine *e, const Dims &d, bool any_bc, const pangu_pack *md, cudaStream_t s) {
  if (!any_bc || d.NB == 0) return PANGU_OK;
  launch_pdl(k_bcs, dim3(grid_for((long long)d.NB * d.ncell)), dim3(kThreads), s, d, e->p.enable_B,
             prim_of(md), md->flag);
  ++e->launches;
  return check_launch();
}

int run_bcs(pangu_engine *e, const pangu_pack *md, cudaStream_t s) {
  return run_bcs(e, bind(e, md), e->any_bc, md, s);
}

int run_estimate_dt(pangu_engine *e, const pangu_pack *md, double *dt_out, cudaStream_t s) {
  const Dims d = bind(e, md);
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  const unsigned gx = (unsigned)std::min<long long>((n / std::max(1, d.NB) + kThreads - 1) / kThreads, 592);
  // d_dtmin holds the key of DBL_MAX and d_dt_ticket 0 between calls (set at pool_init)
  launch_pdl(k_dt_reduce_final, dim3(std::max(1u, gx), d.NB), dim3(kThreads), s, d,
             e->p.cfl_number, md->alfven, e->d_dtmin, e->d_dt_ticket, e->njobs_active, e->d_jr,
             dt_out, 3 * e->capacity);
  e->launches += 1;
  return check_launch();
}

template <class T>
int dalloc(T **p, size_t n) {
  return cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? PANGU_OK
                                                                                   : PANGU_ENOMEM;
}

// One RK stage of Simulator::MakeTaskCollection (ideal_grmhd.cc:23-120), in
// three parts so that a sharded mesh can move its halo messages while the
// middle part runs: the ghost cells the messages fill are read first by
// FixRecovery (neighbour means) and by the next stage.
// Part 1 (run_stage_begin) is run_stage_update followed by the ghost exchange
// at send time, whose halo cells of mc1 go to `send` (sharded only).
// run_stage_update: FixPrimitive + CalculateConservative, fluxes, CT and the
// update; reads only mc0 and mc_init, writes mc1's conserved variables.
int run_stage_update(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                     double beta, const double *dt, cudaStream_t s) {
  const pangu_pack *mc0 = stage == 1 ? base : one;
  const pangu_pack *mc1 = stage == 1 ? one : base;
  int rc;
  // FixPrimitive and CalculateConservative in one pass
  {
    TaskRange r("FixPrimitive+CalculateConservative");
    if ((rc = run_fix_primitive(e, mc0, true, s))) return rc;
  }
  {
    TaskRange r("CalculateFluxes");
    if ((rc = run_fluxes(e, mc0, s))) return rc;
  }
  if (e->p.enable_B) {
    TaskRange r("ConstraintedTransport");
    if ((rc = run_ct(e, mc0, s))) return rc;
  }
  {
    TaskRange r("FluxDivergence+UpdateIndependentData");
    if ((rc = run_update(e, base, mc0, mc1, beta, dt, s))) return rc;
  }
  return PANGU_OK;
}

int run_stage_begin(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                    double beta, const double *dt, double *send, cudaStream_t s) {
  const pangu_pack *mc1 = stage == 1 ? one : base;
  int rc = run_stage_update(e, stage, base, one, beta, dt, s);
  if (rc) return rc;
  {
    TaskRange r("GhostExchange");
    if ((rc = run_exchange(e, mc1, s))) return rc;
    if (send && (rc = run_halo_pack(e, mc1, send, s))) return rc;
  }
  return PANGU_OK;
}

// Part 2: geometric source, Recovery, electron heating (interior cells only).
int run_stage_middle(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                     double beta, const double *dt, cudaStream_t s) {
  const pangu_pack *mc1 = stage == 1 ? one : base;
  int rc;
  {
    TaskRange r("AddGeometricSource");
    if ((rc = run_source(e, mc1, beta, dt, s))) return rc;
  }
  // the retry pass of Recovery lists the cells FixRecovery repairs
  {
    TaskRange r("Recovery");
    if ((rc = run_recovery(e, mc1, true, s))) return rc;
  }
  {
    TaskRange r("ApplyElectronHeating");
    if ((rc = run_heating(e, mc1, s))) return rc;
  }
  return PANGU_OK;
}

// Part 3: halo cells from `recv` (sharded only), FixRecovery, physical BCs,
// and after the last stage the dt estimate.
int run_stage_end(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                  const double *recv, double *dt_est, cudaStream_t s) {
  const pangu_pack *mc1 = stage == 1 ? one : base;
  int rc;
  if (recv) {
    TaskRange r("GhostExchange (halo)");
    if ((rc = run_halo_unpack(e, mc1, recv, s))) return rc;
  }
  if (e->p.recovery == PANGU_RECOVERY_CHAINER) {
    TaskRange r("FixRecovery");
    if ((rc = run_fix_recovery(e, mc1, true, s))) return rc;
  }
  {
    TaskRange r("ApplyBoundaryConditions");
    if ((rc = run_bcs(e, mc1, s))) return rc;
  }
  if (stage == 2 && dt_est) {
    TaskRange r("EstimateTimestep");
    if ((rc = run_estimate_dt(e, mc1, dt_est, s))) return rc;
  }
  return PANGU_OK;
}

int run_stage(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
              double beta, const double *dt, double *dt_est, cudaStream_t s) {
  TaskRange stage_range(stage == 1 ? "pangu_stage 1" : "pangu_stage 2");
  int rc = run_stage_begin(e, stage, base, one, beta, dt, nullptr, s);
  if (!rc) rc = run_stage_middle(e, stage, base, one, beta, dt, s);
  if (!rc) rc = run_stage_end(e, stage, base, one, nullptr, dt_est, s);
  return rc;
}

// Ghost fill of a newly attached job (exchange, then physical BCs) and the
// copy of its base blocks into container "1".
int run_job_start(pangu_engine *e, int job, const pangu_pack *base, const pangu_pack *one,
                  cudaStream_t s) {
  const PoolJob &J = e->jobs[job];
  int first = 0;
  for (int q = 0; q < job; ++q)
    if (e->jobs[q].live) first += (int)e->jobs[q].slots.size();
  Dims dj = e->d;
  dj.slot = e->d_active + first;
  dj.NB = (int)J.slots.size();
  int rc = run_exchange_range(e, base, e->xoff[job], (long long)J.xdst.size(), s);
  if (!rc) rc = run_bcs(e, dj, J.any_bc, base, s);
  // the mixed form's conserved B starts from the initial primitives
  if (!rc && PGK_MIXED) rc = run_calc_cons(e, dj, base, true, s);
  if (rc) return rc;
  const size_t blk = (size_t)e->d.NF * e->d.ncell;
  for (int sl : J.slots) {
    if (cudaMemcpyAsync(prim_of(one) + sl * blk, prim_of(base) + sl * blk, blk * sizeof(PT),
                        cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(one->cons + sl * blk, base->cons + sl * blk, blk * 8,
                        cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return PANGU_ECUDA;
  }
  return PANGU_OK;
}

// problem_generator.cpp:22-35 (angular momentum of the torus at rmax).
inline double lfish_calc(double r, double a) {
  const double sr = std::sqrt(r);
  return (((a * a - 2.0 * a * sr + r * r) *
           ((-2.0 * a * r * (a * a - 2.0 * a * sr + r * r)) /
                std::sqrt(2.0 * a * sr + (-3.0 + r) * r) +
            ((a + (-2.0 + r) * sr) * (r * r * r + a * a * (2.0 + r))) /
                std::sqrt(1 + (2.0 * a) / std::pow(r, 1.5) - 3.0 / r))) /
          (r * r * r * std::sqrt(2.0 * a * sr + (-3.0 + r) * r) * (a * a + (-2.0 + r) * r)));
}

// Initial primitives of a job written into its blocks of base, on stream s;
// synchronises s to check that a torus has a bound region.
int run_generate(pangu_engine *e, int job, const pangu_problem &pb, const pangu_pack *base,
                 cudaStream_t s) {
  const PoolJob &J = e->jobs[job];
  const pangu_params &p = J.p;
  const bool torus = pb.kind == PANGU_PROBLEM_FM_TORUS;
  if (torus && p.metric_type != PANGU_METRIC_MKS) return PANGU_EINVAL;
  int first = 0;
  for (int q = 0; q < job; ++q)
    if (e->jobs[q].live) first += (int)e->jobs[q].slots.size();
  Dims dj = e->d;
  dj.slot = e->d_active + first;
  dj.NB = (int)J.slots.size();
  GenArgs ga{};
  ga.kind = pb.kind;
  ga.seed = (unsigned long long)pb.seed;
  ga.rin = pb.rin;
  ga.rmax = pb.rmax;
  ga.kappa = pb.kappa;
  ga.pert = pb.perturbation;
  ga.beta = pb.beta;
  ga.cut = pb.aphi_rho_cut;
  if (torus) {
    const double a = p.a, a2 = a * a, rin = pb.rin;
    const double l = lfish_calc(pb.rmax, a);
    const double sthin = std::sin(M_PI / 2), cthin = std::cos(M_PI / 2);
    const double DDin = rin * rin - 2.0 * rin + a2;
    const double AAin = (rin * rin + a2) * (rin * rin + a2) - DDin * a2 * sthin * sthin;
    const double SSin = rin * rin + a2 * cthin * cthin;
    ga.l = l;
    ga.lnh_in = 0.5 * std::log((1.0 + std::sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin /
                                                   (AAin * AAin * sthin * sthin))) /
                               (SSin * DDin / AAin)) -
                0.5 * std::sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin /
                                    (AAin * AAin * sthin * sthin)) -
                2.0 * a * rin * l / AAin;
  }
  if (cudaMemsetAsync(e->d_genred, 0, 3 * sizeof(unsigned long long), s) != cudaSuccess)
    return PANGU_ECUDA;
  const Dims &d = dj;
  const long long ne = (long long)d.NB * d.ncell;
  const long long ni = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  PT *P = prim_of(base);
  DISPATCH_MT(p.metric_type, k_gen_cells, grid_for(ne), s, d, p, ga, P, e->d_genred);
  ++e->launches;
  if (torus) {
    k_gen_normalize<<<grid_for(ne), kThreads, 0, s>>>(d, P, e->d_genred);
    ++e->launches;
    if (p.enable_B) {
      k_gen_bfield<MKS><<<grid_for(ni), kThreads, 0, s>>>(d, p, ga, P, e->d_genred);
      k_gen_scale<<<grid_for(ni), kThreads, 0, s>>>(d, p.adiabatic_index, pb.beta, P,
                                                    e->d_genred);
      e->launches += 2;
    }
    unsigned long long rhomax = 0;
    if (check_launch() || cudaMemcpyAsync(&rhomax, e->d_genred, 8, cudaMemcpyDeviceToHost, s) !=
                              cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return PANGU_ECUDA;
    if (rhomax == 0) return PANGU_EINVAL;  // no bound torus for these parameters
  }
  return check_launch();
}

}  // namespace PGK_NS
