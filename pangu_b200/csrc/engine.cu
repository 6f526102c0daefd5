// engine.cu -- B200 GRMHD stage engine: per-task kernels, the stage sequence
// and the C ABI of include/pangu_b200.h.
//
// Data stay where Parthenon would keep them: caller-owned FP64 arrays in
// [block][var][k][j][i] order. Every kernel maps consecutive threads to
// consecutive i so that loads and stores are coalesced in every sweep
// direction (the reference's X2/X3 loops put a strided index innermost,
// laxf.cc:185-189, 291-295).
#include "engine_impl.cuh"

#define PGK_NS pgk64
#define PGK_MIXED 0
#include "kernels.cuh"
#undef PGK_NS

using namespace pgd;
using namespace pgk64;

// The launch helpers of the other instantiations of kernels.cuh: mixed
// precision (engine_mixed.cu) and the pointer-table forms of both precisions
// (engine_tables.cu, engine_mixed_tables.cu).
#define PGK_RUN_DECLS                                                                              \
int run_fix_primitive(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                      \
int run_calc_cons(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                          \
int run_fluxes(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                             \
int run_ct(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                                 \
int run_update(pangu_engine *e, const pangu_pack *mi, const pangu_pack *m0, const pangu_pack *m1,  \
               double beta, const double *dt, cudaStream_t s);                                     \
int run_exchange(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                           \
int run_source(pangu_engine *e, const pangu_pack *md, double beta, const double *dt,               \
               cudaStream_t s);                                                                    \
int run_recovery(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                           \
int run_heating(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                            \
int run_fix_recovery(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                       \
int run_bcs(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                                \
int run_estimate_dt(pangu_engine *e, const pangu_pack *md, double *dt_out, cudaStream_t s);        \
int run_stage(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,           \
              double beta, const double *dt, double *dt_est, cudaStream_t s);                      \
int run_stage_begin(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,     \
                    double beta, const double *dt, double *send, cudaStream_t s);                  \
int run_stage_update(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,    \
                     double beta, const double *dt, cudaStream_t s);                               \
int run_stage_middle(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,    \
                     double beta, const double *dt, cudaStream_t s);                               \
int run_stage_end(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,       \
                  const double *recv, double *dt_est, cudaStream_t s);                             \
int run_halo_pack(pangu_engine *e, const pangu_pack *md, double *buf, cudaStream_t s);             \
int run_halo_unpack(pangu_engine *e, const pangu_pack *md, const double *buf, cudaStream_t s);     \
int run_job_start(pangu_engine *e, int job, const pangu_pack *base, const pangu_pack *one,         \
                  cudaStream_t s);                                                                 \
int run_autotune(pangu_engine *e, const pangu_pack *md, cudaStream_t s);                           \
bool flux_tma_ok(const pangu_engine *e);                                                           \
int run_generate(pangu_engine *e, int job, const pangu_problem &pb, const pangu_pack *base,        \
                 cudaStream_t s);

namespace pgkmx {
PGK_RUN_DECLS
}  // namespace pgkmx
namespace pgk64t {
PGK_RUN_DECLS
}  // namespace pgk64t
namespace pgkmxt {
PGK_RUN_DECLS
}  // namespace pgkmxt

// Launch helper of the engine's precision, for packs in the contiguous layout.
#define RUN(fn, ...)                                                               \
  (e->p.precision == PANGU_PRECISION_MIXED ? pgkmx::fn(__VA_ARGS__) : pgk64::fn(__VA_ARGS__))
// Launch helper of the engine's precision and of the packs' layout: tab is
// true when a pack of the call gives an array through a pointer table.
#define RUNT(tab, fn, ...)                                                                 \
  (e->p.precision == PANGU_PRECISION_MIXED                                                 \
       ? ((tab) ? pgkmxt::fn(__VA_ARGS__) : pgkmx::fn(__VA_ARGS__))                        \
       : ((tab) ? pgk64t::fn(__VA_ARGS__) : pgk64::fn(__VA_ARGS__)))


// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int pangu_num_fields(const pangu_params *p) {
  if (!p) return PANGU_EINVAL;
  return 6 + (p->enable_B ? 3 : 0) + (p->enable_heating ? 1 : 0);
}

int pangu_engine_destroy(pangu_engine *e) {
  if (!e) return PANGU_EINVAL;
  cudaFree(e->d_active);
  cudaFree(e->d_slot_job);
  cudaFree(e->d_jr);
  cudaFree(e->d_bdx);
  cudaFree(e->d_bcf);
  cudaFree(e->d_t1);
  cudaFree(e->d_ctab);
  cudaFree(e->d_ctab32);
  cudaFree(e->d_f1tab32);
  cudaFree(e->d_f2tab32);
  cudaFree(e->d_f1tab);
  cudaFree(e->d_f2tab);
  cudaFree(e->d_t2);
  cudaFree(e->d_origin);
  cudaFree(e->d_xdst);
  cudaFree(e->d_xsrc);
  cudaFree(e->d_cnt);
  cudaFree(e->d_fail_count);
  cudaFree(e->d_fail_list);
  cudaFree(e->d_fix_count);
  cudaFree(e->d_fix_list);
  cudaFree(e->d_tmp_slots);
  cudaFree(e->d_genred);
  cudaFree(e->d_fail_vals);
  cudaFree(e->d_dtmin);
  cudaFree(e->d_dt_ticket);
  cudaFree(e->d_err);
  cudaFree(e->d_hsend);
  cudaFree(e->d_hrecv);
  delete e;
  return PANGU_OK;
}

}  // extern "C"

namespace {

int validate_params(const pangu_params &p) {
  if (p.riemann_solver < 0 || p.riemann_solver > 1 || p.limiter < 0 || p.limiter > 1 ||
      p.recovery < 0 || p.recovery > 1 || p.metric_type < 0 || p.metric_type > 3 || p.model < 0 ||
      p.model > 5 || p.precision < 0 || p.precision > 1)
    return PANGU_EINVAL;
  return PANGU_OK;
}

// Block shape checks shared by single meshes, pools and jobs.
int validate_shape(const pangu_params &p, const pangu_mesh &m) {
  if (m.nx1 < 1 || m.nx2 < 1 || m.nx3 < 1 || m.ng < 0) return PANGU_EINVAL;
  const int need_ng = p.limiter == PANGU_LIMITER_PPM4 ? 3 : 2;
  if (m.ng < need_ng) return PANGU_ENGHOST;
  const int act[3] = {m.nx1 > 1, m.nx2 > 1, m.nx3 > 1};
  const int nx[3] = {m.nx1, m.nx2, m.nx3};
  for (int dd = 0; dd < 3; ++dd)
    if (act[dd] && nx[dd] < m.ng) return PANGU_EINVAL;
  return PANGU_OK;
}

int validate_mesh(const pangu_params &p, const pangu_mesh &m) {
  if (m.nbx1 < 1 || m.nbx2 < 1 || m.nbx3 < 1) return PANGU_EINVAL;
  for (int f = 0; f < 6; ++f)
    if (m.bc[f] < 0 || m.bc[f] > 2) return PANGU_EINVAL;
  return validate_shape(p, m);
}

// Allocates an empty pool of `capacity` block slots for up to `max_jobs`
// jobs with the block shape of e->m.
int pool_init(pangu_engine *e, int capacity, int max_jobs) {
  const pangu_params &p = e->p;
  pangu_mesh one = e->m;
  one.nbx1 = one.nbx2 = one.nbx3 = 1;
  const pgh::Layout L = pgh::make_layout(p, one);
  Dims &d = e->d;
  d = Dims{};
  d.N1 = L.N[0];
  d.N2 = L.N[1];
  d.N3 = L.N[2];
  d.NF = L.NF;
  d.NB = 0;
  d.o1 = L.act[0];
  d.o2 = L.act[1];
  d.o3 = L.act[2];
  d.ndim = 1 + d.o2 + d.o3;
  d.is = L.st[0]; d.ie = d.is + e->m.nx1 - 1;
  d.js = L.st[1]; d.je = d.js + e->m.nx2 - 1;
  d.ks = L.st[2]; d.ke = d.ks + e->m.nx3 - 1;
  d.ncell = (long long)d.N1 * d.N2 * d.N3;
  int n = 0;
  for (int s = 0; s < NPRIM; ++s) d.pidx[s] = -1;
  d.pidx[RHO] = n++; d.pidx[ENY] = n++;
  d.pidx[UX1] = n++; d.pidx[UX2] = n++; d.pidx[UX3] = n++;
  if (p.enable_B) { d.pidx[BX1] = n++; d.pidx[BX2] = n++; d.pidx[BX3] = n++; }
  d.pidx[ENT] = n++;
  if (p.enable_heating) d.pidx[KEL] = n++;

  e->capacity = capacity;
  e->max_jobs = max_jobs;
  e->jobs.assign(max_jobs, PoolJob{});
  e->slot_used.assign(capacity, 0);
  e->xoff.assign(max_jobs, 0);
  const size_t W1 = d.N1 + 1, W2 = d.N2 + 1;
  e->fail_cap = (long long)capacity * e->m.nx1 * e->m.nx2 * e->m.nx3;
  int rc = PANGU_OK;
  rc |= dalloc(&e->d_active, capacity);
  rc |= dalloc(&e->d_slot_job, capacity);
  rc |= dalloc(&e->d_jr, 3 * (size_t)max_jobs);
  rc |= dalloc(&e->d_bdx, 3 * (size_t)capacity);
  rc |= dalloc(&e->d_bcf, 6 * (size_t)capacity);
  rc |= dalloc(&e->d_t1, (size_t)capacity * kT1Rows * W1);
  rc |= dalloc(&e->d_t2, (size_t)capacity * 12 * W2);
  rc |= dalloc(&e->d_origin, 3 * (size_t)capacity);
  rc |= dalloc(&e->d_cnt, (size_t)max_jobs * PANGU_NCOUNTERS);
  rc |= dalloc(&e->d_fail_count, 1);
  rc |= dalloc(&e->d_fail_list, (size_t)e->fail_cap);
  rc |= dalloc(&e->d_fix_count, 1);
  rc |= dalloc(&e->d_fix_list, (size_t)e->fail_cap);
  rc |= dalloc(&e->d_fail_vals, (size_t)e->fail_cap * d.NF);
  rc |= dalloc(&e->d_dtmin, 3 * (size_t)capacity);
  rc |= dalloc(&e->d_dt_ticket, 1);
  rc |= dalloc(&e->d_err, 1);
  rc |= dalloc(&e->d_tmp_slots, capacity);
  rc |= dalloc(&e->d_genred, 3);
  // every ghost cell of a slot has at most one exchange source
  e->xch_cap = (long long)capacity * (d.ncell - (long long)e->m.nx1 * e->m.nx2 * e->m.nx3);
  rc |= dalloc(&e->d_xdst, (size_t)e->xch_cap);
  rc |= dalloc(&e->d_xsrc, (size_t)e->xch_cap);
  if (p.metric_type == PANGU_METRIC_MKS || p.metric_type == PANGU_METRIC_BL) {
    const TabLayout T = p.metric_type == PANGU_METRIC_MKS ? tab_layout(MKS) : tab_layout(BL);
    const size_t pc = (size_t)d.N2 * d.N1, p1 = (size_t)d.N2 * (d.N1 + 1),
                 p2 = (size_t)(d.N2 + 1) * d.N1;
    rc |= dalloc(&e->d_ctab, (size_t)capacity * T.ncen * pc);
    rc |= dalloc(&e->d_f1tab, (size_t)capacity * T.nmet * p1);
    rc |= dalloc(&e->d_f2tab, (size_t)capacity * T.nmet * p2);
    if (p.precision == PANGU_PRECISION_MIXED) {
      rc |= dalloc(&e->d_ctab32, (size_t)capacity * T.nconn * pc);
      rc |= dalloc(&e->d_f1tab32, (size_t)capacity * T.nmet * p1);
      rc |= dalloc(&e->d_f2tab32, (size_t)capacity * T.nmet * p2);
    }
  }
  if (rc != PANGU_OK) return PANGU_ENOMEM;
  bool ok = cudaMemset(e->d_cnt, 0, (size_t)max_jobs * PANGU_NCOUNTERS * 8) == cudaSuccess;
  ok &= cudaMemset(e->d_slot_job, 0, (size_t)capacity * sizeof(int)) == cudaSuccess;
  ok &= cudaMemset(e->d_bcf, 0xff, 6 * (size_t)capacity) == cudaSuccess;  // -1: no BC
  ok &= cudaMemset(e->d_dt_ticket, 0, sizeof(unsigned int)) == cudaSuccess;
  ok &= cudaMemset(e->d_err, 0, sizeof(int)) == cudaSuccess;
  k_dt_init<<<grid_for(3 * capacity), kThreads>>>(3 * capacity, e->d_dtmin);
  ok &= cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(0) == cudaSuccess;
  if (!ok) return PANGU_ECUDA;
  d.slot = e->d_active;
  d.slot_job = e->d_slot_job;
  d.bdx = e->d_bdx;
  d.bcf = e->d_bcf;
  d.t1 = e->d_t1;
  d.t2 = e->d_t2;
  d.origin = e->d_origin;
  d.ctab = e->d_ctab;
  d.ctab32 = e->d_ctab32;
  d.f1tab32 = e->d_f1tab32;
  d.f2tab32 = e->d_f2tab32;
  d.f1tab = e->d_f1tab;
  d.f2tab = e->d_f2tab;
  return PANGU_OK;
}

// Active block list (jobs in id order, each job's blocks in lattice order),
// per-job ranges and the concatenated exchange map, uploaded synchronously.
int pool_rebuild(pangu_engine *e) {
  std::vector<int> active, jr;
  std::vector<int64_t> xd, xs;
  e->any_bc = false;
  for (int q = 0; q < e->max_jobs; ++q) {
    const PoolJob &J = e->jobs[q];
    if (!J.live) continue;
    jr.push_back(q);
    jr.push_back((int)active.size());
    active.insert(active.end(), J.slots.begin(), J.slots.end());
    jr.push_back((int)active.size());
    e->xoff[q] = (long long)xd.size();
    xd.insert(xd.end(), J.xdst.begin(), J.xdst.end());
    xs.insert(xs.end(), J.xsrc.begin(), J.xsrc.end());
    e->any_bc = e->any_bc || J.any_bc;
  }
  if ((long long)xd.size() > e->xch_cap) return PANGU_ETOOBIG;  // cannot happen
  bool ok = true;
  if (!active.empty())
    ok &= cudaMemcpy(e->d_active, active.data(), active.size() * sizeof(int),
                     cudaMemcpyHostToDevice) == cudaSuccess;
  if (!jr.empty())
    ok &= cudaMemcpy(e->d_jr, jr.data(), jr.size() * sizeof(int), cudaMemcpyHostToDevice) ==
          cudaSuccess;
  if (!xd.empty()) {
    ok &= cudaMemcpy(e->d_xdst, xd.data(), xd.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    ok &= cudaMemcpy(e->d_xsrc, xs.data(), xs.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  }
  // a pageable upload may still be in flight when cudaMemcpy returns
  ok &= cudaStreamSynchronize(0) == cudaSuccess;
  if (!ok) return PANGU_ECUDA;
  e->d.NB = (int)active.size();
  e->nxch = (long long)xd.size();
  e->njobs_active = (int)(jr.size() / 3);
  return PANGU_OK;
}

// Places a job's blocks in free slots (lowest first) and builds their
// coordinate tables, metric tables, BC faces and exchange map. With
// block_rank non-null the job is this rank's shard of a mesh spread over
// e->nranks engines: only the blocks with block_rank[b] == e->rank are
// placed, and the exchange entries that cross ranks become the halo lists.
int pool_attach(pangu_engine *e, const pangu_mesh &m, double a, double h, int *job_out,
                int32_t *slots_out, const int32_t *block_rank = nullptr) {
  if (m.nx1 != e->m.nx1 || m.nx2 != e->m.nx2 || m.nx3 != e->m.nx3 || m.ng != e->m.ng)
    return PANGU_EINVAL;
  int rc = validate_mesh(e->p, m);
  if (rc) return rc;
  const long long nall = (long long)m.nbx1 * m.nbx2 * m.nbx3;
  std::vector<int> gb;  // lattice ids of the blocks placed here, in lattice order
  for (long long b = 0; b < nall; ++b)
    if (!block_rank || block_rank[b] == e->rank) gb.push_back((int)b);
  const long long nbl = (long long)gb.size();
  int job = -1;
  for (int q = 0; q < e->max_jobs && job < 0; ++q)
    if (!e->jobs[q].live) job = q;
  if (job < 0) return PANGU_EFULL;
  std::vector<int> slots;
  for (int sl = 0; sl < e->capacity && (long long)slots.size() < nbl; ++sl)
    if (!e->slot_used[sl]) slots.push_back(sl);
  if ((long long)slots.size() < nbl) return PANGU_EFULL;
  std::vector<long long> slot_of_block(nall, -1);
  for (long long q = 0; q < nbl; ++q) slot_of_block[gb[q]] = slots[q];

  PoolJob J;
  J.m = m;
  J.p = e->p;
  J.p.a = a;
  J.p.h = h;
  J.slots = slots;
  const pgh::Layout L = pgh::make_layout(J.p, m);
  std::vector<double> t1, t2;
  pgh::build_tables(J.p, L, t1, t2);
  std::vector<int64_t> xd, xs;
  pgh::build_exchange(m, L, xd, xs);
  const Dims &d = e->d;
  const long long nc = d.ncell;
  auto to_slot = [&](int64_t c) { return (int64_t)slot_of_block[c / nc] * nc + c % nc; };
  std::vector<std::vector<int64_t>> hsend, hrecv;
  if (block_rank) {
    std::vector<int64_t> ld, ls;
    pgh::shard_exchange(xd, xs, nc, block_rank, e->nranks, e->rank, ld, ls, hsend, hrecv);
    xd.swap(ld);
    xs.swap(ls);
  }
  for (size_t q = 0; q < xd.size(); ++q) {
    xd[q] = to_slot(xd[q]);
    xs[q] = to_slot(xs[q]);
  }
  J.xdst.swap(xd);
  J.xsrc.swap(xs);
  const size_t W1 = d.N1 + 1, W2 = d.N2 + 1;
  const size_t r1 = (size_t)kT1Rows * W1, r2 = 12 * W2;
  const int nbv[3] = {m.nbx1, m.nbx2, m.nbx3};
  const int act[3] = {d.o1, d.o2, d.o3};
  bool ok = true;
  for (long long q = 0; q < nbl; ++q) {
    const long long b = gb[q];
    const int sl = slots[q];
    const int bl[3] = {(int)(b % m.nbx1), (int)((b / m.nbx1) % m.nbx2),
                       (int)(b / ((long long)m.nbx1 * m.nbx2))};
    signed char bcf[6];
    for (int f = 0; f < 6; ++f) {
      const int dir = f / 2;
      const bool edge = (f % 2 == 0) ? bl[dir] == 0 : bl[dir] == nbv[dir] - 1;
      bcf[f] = (act[dir] && edge && m.bc[f] != PANGU_BC_PERIODIC) ? (signed char)m.bc[f] : -1;
      J.any_bc = J.any_bc || bcf[f] >= 0;
    }
    ok &= cudaMemcpy(e->d_t1 + sl * r1, &t1[b * r1], r1 * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    ok &= cudaMemcpy(e->d_t2 + sl * r2, &t2[b * r2], r2 * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    ok &= cudaMemcpy(e->d_origin + 3 * sl, &L.origin[3 * b], 24, cudaMemcpyHostToDevice) ==
          cudaSuccess;
    ok &= cudaMemcpy(e->d_bdx + 3 * sl, L.dx, 24, cudaMemcpyHostToDevice) == cudaSuccess;
    ok &= cudaMemcpy(e->d_bcf + 6 * sl, bcf, 6, cudaMemcpyHostToDevice) == cudaSuccess;
    ok &= cudaMemcpy(e->d_slot_job + sl, &job, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  ok &= cudaMemset(e->d_cnt + (size_t)job * PANGU_NCOUNTERS, 0, PANGU_NCOUNTERS * 8) == cudaSuccess;
  if (!ok) return PANGU_ECUDA;
  if (block_rank) {
    // halo lists, per peer in rank order, in slot cell offsets
    std::vector<int64_t> hs, hr;
    e->hsend_off.assign(e->nranks + 1, 0);
    e->hrecv_off.assign(e->nranks + 1, 0);
    for (int q = 0; q < e->nranks; ++q) {
      for (int64_t c : hsend[q]) hs.push_back(to_slot(c));
      for (int64_t c : hrecv[q]) hr.push_back(to_slot(c));
      e->hsend_off[q + 1] = (long long)hs.size();
      e->hrecv_off[q + 1] = (long long)hr.size();
    }
    if (dalloc(&e->d_hsend, hs.size()) || dalloc(&e->d_hrecv, hr.size())) return PANGU_ENOMEM;
    if (!hs.empty())
      ok &= cudaMemcpy(e->d_hsend, hs.data(), hs.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    if (!hr.empty())
      ok &= cudaMemcpy(e->d_hrecv, hr.data(), hr.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) return PANGU_ECUDA;
  }
  if (e->p.metric_type == PANGU_METRIC_MKS || e->p.metric_type == PANGU_METRIC_BL) {
    // static metric tables of the job's slots, with the job's a and h
    ok = cudaMemcpy(e->d_tmp_slots, slots.data(), slots.size() * sizeof(int),
                    cudaMemcpyHostToDevice) == cudaSuccess;
    Dims dj = d;
    dj.slot = e->d_tmp_slots;
    dj.NB = (int)nbl;
    const long long n = (long long)dj.NB * ((long long)d.N2 * d.N1 + (long long)d.N2 * (d.N1 + 1) +
                                            (long long)(d.N2 + 1) * d.N1);
    if (ok) {
      if (e->p.metric_type == PANGU_METRIC_MKS)
        k_build_tables<MKS><<<grid_for(n), kThreads>>>(dj, J.p, e->d_ctab, e->d_f1tab, e->d_f2tab);
      else
        k_build_tables<BL><<<grid_for(n), kThreads>>>(dj, J.p, e->d_ctab, e->d_f1tab, e->d_f2tab);
      if (e->d_ctab32) {
        const TabLayout T = e->p.metric_type == PANGU_METRIC_MKS ? tab_layout(MKS) : tab_layout(BL);
        const long long nc = (long long)dj.NB * T.nconn * d.N2 * d.N1;
        if (e->p.metric_type == PANGU_METRIC_MKS)
          k_conn_to_f32<MKS><<<grid_for(nc), kThreads>>>(dj, e->d_ctab32);
        else
          k_conn_to_f32<BL><<<grid_for(nc), kThreads>>>(dj, e->d_ctab32);
        const long long p1 = (long long)d.N2 * (d.N1 + 1), p2 = (long long)(d.N2 + 1) * d.N1;
        k_planes_to_f32<<<grid_for((long long)dj.NB * T.nmet * p1), kThreads>>>(
            dj, e->d_f1tab, e->d_f1tab32, T.nmet, p1);
        k_planes_to_f32<<<grid_for((long long)dj.NB * T.nmet * p2), kThreads>>>(
            dj, e->d_f2tab, e->d_f2tab32, T.nmet, p2);
      }
      ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(0) == cudaSuccess;
    }
    if (!ok) return PANGU_ECUDA;
  }
  J.live = true;
  for (int sl : slots) e->slot_used[sl] = 1;
  e->jobs[job] = std::move(J);
  rc = pool_rebuild(e);
  if (rc) return rc;
  *job_out = job;
  if (slots_out)
    for (long long q = 0; q < nbl; ++q) slots_out[q] = slots[q];
  return PANGU_OK;
}

int validate_ranks(const pangu_mesh &m, const int32_t *block_rank, int nranks, int rank) {
  if (!block_rank || nranks < 1 || rank < 0 || rank >= nranks) return PANGU_EINVAL;
  const long long nall = (long long)m.nbx1 * m.nbx2 * m.nbx3;
  for (long long b = 0; b < nall; ++b)
    if (block_rank[b] < 0 || block_rank[b] >= nranks) return PANGU_EINVAL;
  return PANGU_OK;
}

bool halo_sends(const pangu_engine *e) { return !e->hsend_off.empty() && e->hsend_off.back() > 0; }
bool halo_recvs(const pangu_engine *e) { return !e->hrecv_off.empty() && e->hrecv_off.back() > 0; }

}  // namespace

extern "C" {

int pangu_engine_create(const pangu_params *params, const pangu_mesh *mesh, pangu_engine **out) {
  if (!params || !mesh || !out) return PANGU_EINVAL;
  *out = nullptr;
  int rc = validate_params(*params);
  if (!rc) rc = validate_mesh(*params, *mesh);
  if (rc) return rc;
  pangu_engine *e = new (std::nothrow) pangu_engine;
  if (!e) return PANGU_ENOMEM;
  e->p = *params;
  e->m = *mesh;
  const int nb = mesh->nbx1 * mesh->nbx2 * mesh->nbx3;
  rc = pool_init(e, nb, 1);
  int job = -1;
  if (!rc) rc = pool_attach(e, *mesh, params->a, params->h, &job, nullptr);
  if (rc) {
    pangu_engine_destroy(e);
    return rc;
  }
  *out = e;
  return PANGU_OK;
}

int pangu_pool_create(const pangu_params *params, const pangu_mesh *block, int32_t capacity_blocks,
                      int32_t max_jobs, pangu_engine **out) {
  if (!params || !block || !out || capacity_blocks < 1 || max_jobs < 1) return PANGU_EINVAL;
  *out = nullptr;
  int rc = validate_params(*params);
  if (!rc) rc = validate_shape(*params, *block);
  if (rc) return rc;
  pangu_engine *e = new (std::nothrow) pangu_engine;
  if (!e) return PANGU_ENOMEM;
  e->p = *params;
  e->m = *block;
  rc = pool_init(e, capacity_blocks, max_jobs);
  if (rc) {
    pangu_engine_destroy(e);
    return rc;
  }
  *out = e;
  return PANGU_OK;
}

int pangu_job_attach(pangu_engine *e, const pangu_mesh *mesh, double a, double h, int32_t *job_out,
                     int32_t *slots_out) {
  if (!e || !mesh || !job_out) return PANGU_EINVAL;
  if (e->p.metric_type == PANGU_METRIC_CKS && (a != e->p.a || h != e->p.h)) return PANGU_EINVAL;
  int job = -1;
  const int rc = pool_attach(e, *mesh, a, h, &job, slots_out);
  if (rc) return rc;
  *job_out = job;
  return PANGU_OK;
}

int pangu_job_start(pangu_engine *e, int32_t job, const pangu_pack *base, const pangu_pack *one,
                    void *stream) {
  if (!pack_ok(e, base) || !pack_ok(e, one) || !contiguous(base) || !contiguous(one) ||
      job < 0 || job >= e->max_jobs || !e->jobs[job].live)
    return PANGU_EINVAL;
  return RUN(run_job_start, e, job, base, one, S(stream));
}

int pangu_job_detach(pangu_engine *e, int32_t job) {
  if (!e || job < 0 || job >= e->max_jobs || !e->jobs[job].live) return PANGU_EINVAL;
  for (int sl : e->jobs[job].slots) e->slot_used[sl] = 0;
  e->jobs[job] = PoolJob{};
  return pool_rebuild(e);
}

int pangu_job_counters(pangu_engine *e, int32_t job, uint64_t out[PANGU_NCOUNTERS]) {
  if (!e || !out || job < 0 || job >= e->max_jobs) return PANGU_EINVAL;
  unsigned long long tmp[PANGU_NCOUNTERS];
  if (cudaMemcpy(tmp, e->d_cnt + (size_t)job * PANGU_NCOUNTERS, sizeof(tmp),
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return PANGU_ECUDA;
  for (int i = 0; i < PANGU_NCOUNTERS; ++i) out[i] = tmp[i];
  return PANGU_OK;
}

int pangu_active_blocks(const pangu_engine *e) { return e ? e->d.NB : PANGU_EINVAL; }

#define GUARD(e, md)                      \
  if (!pack_ok(e, md)) return PANGU_EINVAL; \
  if (e->d.NB == 0) return PANGU_OK;

int pangu_fix_primitive(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_fix_primitive, e, md, S(stream));
}
int pangu_calculate_conservative(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_calc_cons, e, md, S(stream));
}
int pangu_calculate_fluxes(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_fluxes, e, md, S(stream));
}
int pangu_constrained_transport(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  if (!e->p.enable_B) return PANGU_EINVAL;
  return RUNT(!contiguous(md), run_ct, e, md, S(stream));
}
int pangu_flux_divergence_update(pangu_engine *e, const pangu_pack *mc_init, const pangu_pack *mc0,
                                 const pangu_pack *mc1, double beta, const double *dt,
                                 void *stream) {
  if (!pack_ok(e, mc_init) || !pack_ok(e, mc0) || !pack_ok(e, mc1) || !dt) return PANGU_EINVAL;
  if (e->d.NB == 0) return PANGU_OK;
  return RUNT(!contiguous(mc_init) || !contiguous(mc0) || !contiguous(mc1), run_update,
              e, mc_init, mc0, mc1, beta, dt, S(stream));
}
int pangu_exchange_ghosts(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_exchange, e, md, S(stream));
}
int pangu_add_geometric_source(pangu_engine *e, const pangu_pack *md, double beta, const double *dt,
                               void *stream) {
  GUARD(e, md);
  if (!dt) return PANGU_EINVAL;
  return RUNT(!contiguous(md), run_source, e, md, beta, dt, S(stream));
}
int pangu_recovery(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_recovery, e, md, S(stream));
}
int pangu_apply_electron_heating(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_heating, e, md, S(stream));
}
int pangu_fix_recovery(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  if (e->p.recovery != PANGU_RECOVERY_CHAINER) return PANGU_EINVAL;
  return RUNT(!contiguous(md), run_fix_recovery, e, md, S(stream));
}
int pangu_apply_boundary_conditions(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_bcs, e, md, S(stream));
}
int pangu_estimate_dt(pangu_engine *e, const pangu_pack *md, double *dt_out, void *stream) {
  GUARD(e, md);
  if (!dt_out) return PANGU_EINVAL;
  return RUNT(!contiguous(md), run_estimate_dt, e, md, dt_out, S(stream));
}

int pangu_autotune(pangu_engine *e, const pangu_pack *md, void *stream) {
  GUARD(e, md);
  return RUNT(!contiguous(md), run_autotune, e, md, S(stream));
}

int pangu_generate(pangu_engine *e, int32_t job, const pangu_problem *problem,
                   const pangu_pack *base, void *stream) {
  if (!pack_ok(e, base) || !contiguous(base) || !problem || job < 0 || job >= e->max_jobs ||
      !e->jobs[job].live || problem->kind < 0 || problem->kind > 2)
    return PANGU_EINVAL;
  if (problem->kind == PANGU_PROBLEM_FM_TORUS &&
      !(problem->kappa > 0 && problem->beta > 0 && problem->rmax > problem->rin))
    return PANGU_EINVAL;
  // the torus normalises by maxima over the whole mesh, which a shard does not hold
  if (problem->kind == PANGU_PROBLEM_FM_TORUS && e->nranks > 1) return PANGU_EINVAL;
  return RUN(run_generate, e, job, *problem, base, S(stream));
}

int pangu_flux_config(const pangu_engine *e, int32_t out[7]) {
  if (!e || !out) return PANGU_EINVAL;
  for (int d = 0; d < 3; ++d) {
    out[2 * d] = e->tune.march[d];
    out[2 * d + 1] = e->tune.threads[d];
  }
  out[6] = e->tune.tuned;
  return PANGU_OK;
}

int pangu_set_flux_config(pangu_engine *e, const int32_t cfg[6]) {
  if (!e || !cfg) return PANGU_EINVAL;
  const bool tma = RUN(flux_tma_ok, e);
  for (int d = 0; d < 3; ++d) {
    const int m = cfg[2 * d], t = cfg[2 * d + 1];
    const bool march_ok = d == 0 ? (m == 1 || (m == kMarchTma && tma))
                                 : (m == 0 || m == 1 || m == 2 || m == 4 || (m == kMarchTma && tma));
    const bool threads_ok = m == 0 ? (t == 128 || t == 256)
                                   : (m == kMarchTma ? t == 128 : (t == 64 || t == 128));
    if (!march_ok || !threads_ok) return PANGU_EINVAL;
  }
  for (int d = 0; d < 3; ++d) {
    e->tune.march[d] = cfg[2 * d];
    e->tune.threads[d] = cfg[2 * d + 1];
  }
  e->tune.tuned = 1;
  return PANGU_OK;
}

int pangu_stage(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                double beta, const double *dt, double *dt_est, void *stream) {
  if (!pack_ok(e, base) || !pack_ok(e, one) || !dt || (stage != 1 && stage != 2))
    return PANGU_EINVAL;
  if (halo_sends(e) || halo_recvs(e)) return PANGU_EINVAL;  // a shard: the three-part calls
  if (e->d.NB == 0) return PANGU_OK;
  return RUNT(!contiguous(base) || !contiguous(one), run_stage,
              e, stage, base, one, beta, dt, dt_est, S(stream));
}

// ---------------------------------------------------------------------------
// Block sharding of one mesh over several GPUs.
// ---------------------------------------------------------------------------
int pangu_shard_plan(const pangu_params *params, const pangu_mesh *mesh, const int32_t *block_rank,
                     int32_t nranks, int32_t rank, int64_t *send_counts, int64_t *recv_counts,
                     int64_t *send_cells, int64_t *recv_cells) {
  if (!params || !mesh || !send_counts || !recv_counts) return PANGU_EINVAL;
  int rc = validate_params(*params);
  if (!rc) rc = validate_mesh(*params, *mesh);
  if (!rc) rc = validate_ranks(*mesh, block_rank, nranks, rank);
  if (rc) return rc;
  const pgh::Layout L = pgh::make_layout(*params, *mesh);
  std::vector<int64_t> xd, xs, ld, ls;
  pgh::build_exchange(*mesh, L, xd, xs);
  std::vector<std::vector<int64_t>> snd, rcv;
  const int64_t nc = (int64_t)L.N[0] * L.N[1] * L.N[2];
  pgh::shard_exchange(xd, xs, nc, block_rank, nranks, rank, ld, ls, snd, rcv);
  int64_t ns = 0, nr = 0;
  for (int q = 0; q < nranks; ++q) {
    send_counts[q] = (int64_t)snd[q].size();
    recv_counts[q] = (int64_t)rcv[q].size();
    for (int64_t c : snd[q])
      if (send_cells) send_cells[ns++] = c;
    for (int64_t c : rcv[q])
      if (recv_cells) recv_cells[nr++] = c;
  }
  return PANGU_OK;
}

int pangu_shard_create(const pangu_params *params, const pangu_mesh *mesh,
                       const int32_t *block_rank, int32_t nranks, int32_t rank,
                       pangu_engine **out) {
  if (!params || !mesh || !out) return PANGU_EINVAL;
  *out = nullptr;
  int rc = validate_params(*params);
  if (!rc) rc = validate_mesh(*params, *mesh);
  if (!rc) rc = validate_ranks(*mesh, block_rank, nranks, rank);
  if (rc) return rc;
  const long long nall = (long long)mesh->nbx1 * mesh->nbx2 * mesh->nbx3;
  int nloc = 0;
  for (long long b = 0; b < nall; ++b) nloc += block_rank[b] == rank;
  if (nloc == 0) return PANGU_EINVAL;
  pangu_engine *e = new (std::nothrow) pangu_engine;
  if (!e) return PANGU_ENOMEM;
  e->p = *params;
  e->m = *mesh;
  e->nranks = nranks;
  e->rank = rank;
  rc = pool_init(e, nloc, 1);
  int job = -1;
  if (!rc) rc = pool_attach(e, *mesh, params->a, params->h, &job, nullptr, block_rank);
  if (rc) {
    pangu_engine_destroy(e);
    return rc;
  }
  *out = e;
  return PANGU_OK;
}

int pangu_halo_counts(const pangu_engine *e, int64_t *send_counts, int64_t *recv_counts) {
  if (!e || !send_counts || !recv_counts) return PANGU_EINVAL;
  for (int q = 0; q < e->nranks; ++q) {
    send_counts[q] = e->hsend_off.empty() ? 0 : e->hsend_off[q + 1] - e->hsend_off[q];
    recv_counts[q] = e->hrecv_off.empty() ? 0 : e->hrecv_off[q + 1] - e->hrecv_off[q];
  }
  return PANGU_OK;
}

int pangu_halo_pack(pangu_engine *e, const pangu_pack *md, double *send, void *stream) {
  if (!pack_ok(e, md) || (halo_sends(e) && !send)) return PANGU_EINVAL;
  return RUNT(!contiguous(md), run_halo_pack, e, md, send, S(stream));
}

int pangu_halo_unpack(pangu_engine *e, const pangu_pack *md, const double *recv, void *stream) {
  if (!pack_ok(e, md) || (halo_recvs(e) && !recv)) return PANGU_EINVAL;
  return RUNT(!contiguous(md), run_halo_unpack, e, md, recv, S(stream));
}

int pangu_stage_begin(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                      double beta, const double *dt, double *send, void *stream) {
  if (!pack_ok(e, base) || !pack_ok(e, one) || !dt || (stage != 1 && stage != 2) ||
      (halo_sends(e) && !send))
    return PANGU_EINVAL;
  if (e->d.NB == 0) return PANGU_OK;
  return RUNT(!contiguous(base) || !contiguous(one), run_stage_begin,
              e, stage, base, one, beta, dt, send, S(stream));
}

int pangu_stage_update(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                       double beta, const double *dt, void *stream) {
  if (!pack_ok(e, base) || !pack_ok(e, one) || !dt || (stage != 1 && stage != 2))
    return PANGU_EINVAL;
  if (e->d.NB == 0) return PANGU_OK;
  return RUNT(!contiguous(base) || !contiguous(one), run_stage_update,
              e, stage, base, one, beta, dt, S(stream));
}

int pangu_stage_middle(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                       double beta, const double *dt, void *stream) {
  if (!pack_ok(e, base) || !pack_ok(e, one) || !dt || (stage != 1 && stage != 2))
    return PANGU_EINVAL;
  if (e->d.NB == 0) return PANGU_OK;
  return RUNT(!contiguous(base) || !contiguous(one), run_stage_middle,
              e, stage, base, one, beta, dt, S(stream));
}

int pangu_stage_end(pangu_engine *e, int stage, const pangu_pack *base, const pangu_pack *one,
                    const double *recv, double *dt_est, void *stream) {
  if (!pack_ok(e, base) || !pack_ok(e, one) || (stage != 1 && stage != 2) ||
      (halo_recvs(e) && !recv))
    return PANGU_EINVAL;
  if (e->d.NB == 0) return PANGU_OK;
  return RUNT(!contiguous(base) || !contiguous(one), run_stage_end,
              e, stage, base, one, recv, dt_est, S(stream));
}

// ---------------------------------------------------------------------------
// dt estimate without any allocation.
//
// Some callers cannot call cudaMalloc: an application whose device memory is
// owned by a pool or a fixed budget (a Parthenon/Kokkos memory pool, or a
// serving loop that admits jobs against an HBM budget) may not allocate on
// the side, and cannot create a pangu_engine, which allocates its tables and
// scratch. pangu_estimate_dt_noalloc serves them: it needs only the caller's
// alfven array and output, and keeps its per-block scratch in the file-scope
// device array below, which every GPU that loads this library holds until
// the process exits.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocMaxBlocks = 4096;  // 3 minima per block: 96 KiB
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) unsigned long long g_noalloc_dtmin[3 * kNoAllocMaxBlocks];
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kNoAllocMaxDevices] = {};
}  // namespace

int pangu_estimate_dt_noalloc(const pangu_params *params, const pangu_mesh *mesh,
                              const double *alfven, double *dt_out, void *stream) {
  if (!params || !mesh || !alfven || !dt_out) return PANGU_EINVAL;
  const pangu_mesh &m = *mesh;
  if (m.nx1 < 1 || m.nx2 < 1 || m.nx3 < 1 || m.nbx1 < 1 || m.nbx2 < 1 || m.nbx3 < 1 || m.ng < 0)
    return PANGU_EINVAL;
  const long long nb = (long long)m.nbx1 * m.nbx2 * m.nbx3;
  if (nb > kNoAllocMaxBlocks) return PANGU_ETOOBIG;
  Dims d{};
  d.o1 = m.nx1 > 1;
  d.o2 = m.nx2 > 1;
  d.o3 = m.nx3 > 1;
  d.ndim = 1 + d.o2 + d.o3;
  d.N1 = m.nx1 + 2 * m.ng * d.o1;
  d.N2 = m.nx2 + 2 * m.ng * d.o2;
  d.N3 = m.nx3 + 2 * m.ng * d.o3;
  d.NB = (int)nb;
  d.NF = pangu_num_fields(params);
  d.is = m.ng * d.o1; d.ie = d.is + m.nx1 - 1;
  d.js = m.ng * d.o2; d.je = d.js + m.nx2 - 1;
  d.ks = m.ng * d.o3; d.ke = d.ks + m.nx3 - 1;
  d.ncell = (long long)d.N1 * d.N2 * d.N3;
  d.dx[0] = (m.x1max - m.x1min) / (double)(m.nbx1 * m.nx1);
  d.dx[1] = (m.x2max - m.x2min) / (double)(m.nbx2 * m.nx2);
  d.dx[2] = (m.x3max - m.x3min) / (double)(m.nbx3 * m.nx3);
  // Device address of the scratch array, looked up once per device with that
  // device current (the host-side name of a __device__ array is not a device
  // address).
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PANGU_ECUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return PANGU_EINVAL;
  void *ptr = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      if (cudaGetSymbolAddress(&g_noalloc_ptr[dev], g_noalloc_dtmin) != cudaSuccess) {
        g_noalloc_ptr[dev] = nullptr;
        return PANGU_ECUDA;
      }
    }
    ptr = g_noalloc_ptr[dev];
  }
  unsigned long long *mins = static_cast<unsigned long long *>(ptr);
  cudaStream_t s = S(stream);
  // The array keeps the previous call's minima: reset them first.
  k_dt_init<<<grid_for(3 * d.NB), kThreads, 0, s>>>(3 * d.NB, mins);
  const long long n = box_count(d.NB, d.ks, d.ke, d.js, d.je, d.is, d.ie);
  const unsigned gx =
      (unsigned)std::min<long long>((n / std::max(1, d.NB) + kThreads - 1) / kThreads, 592);
  k_dt_reduce<<<dim3(std::max(1u, gx), d.NB), kThreads, 0, s>>>(d, params->cfl_number, alfven,
                                                                 mins);
  k_dt_finalize<<<1, 32, 0, s>>>(d, 1, nullptr, mins, dt_out);
  return check_launch();
}

int pangu_update_dt(pangu_engine *e, double *dt, const double *dt_est, double dt_factor,
                    void *stream) {
  if (!e || !dt || !dt_est) return PANGU_EINVAL;
  if (e->njobs_active == 0) return PANGU_OK;
  launch_pdl(k_update_dt, dim3(1), dim3(128), S(stream), e->njobs_active, (const int *)e->d_jr, dt,
             dt_est, dt_factor);
  ++e->launches;
  return check_launch();
}

int pangu_counters(pangu_engine *e, uint64_t out[PANGU_NCOUNTERS]) {
  if (!e || !out) return PANGU_EINVAL;
  std::vector<unsigned long long> tmp((size_t)e->max_jobs * PANGU_NCOUNTERS);
  if (cudaMemcpy(tmp.data(), e->d_cnt, tmp.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    return PANGU_ECUDA;
  for (int i = 0; i < PANGU_NCOUNTERS; ++i) {
    out[i] = 0;
    for (int q = 0; q < e->max_jobs; ++q) out[i] += tmp[(size_t)q * PANGU_NCOUNTERS + i];
  }
  return PANGU_OK;
}

long long pangu_launches(const pangu_engine *e) { return e ? e->launches : PANGU_EINVAL; }

int pangu_device_error(const pangu_engine *e, int32_t *flag_out) {
  if (!e || !flag_out) return PANGU_EINVAL;
  int v = 0;
  if (cudaMemcpy(&v, e->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return PANGU_ECUDA;
  *flag_out = v;
  return PANGU_OK;
}

int pangu_reset_counters(pangu_engine *e, void *stream) {
  if (!e) return PANGU_EINVAL;
  return cudaMemsetAsync(e->d_cnt, 0, (size_t)e->max_jobs * PANGU_NCOUNTERS * 8, S(stream)) ==
                 cudaSuccess
             ? PANGU_OK
             : PANGU_ECUDA;
}

}  // extern "C"
