// b200_tasks.cc -- PANGU's stage tasks (the functions ideal_grmhd.cc:62-110
// registers) implemented by the B200 engine's C ABI (include/pangu_b200.h).
//
// Link this file instead of the reference's task sources
//   fixer/primitive_fixer.cc, fixer/recovery_fixer.cc,
//   riemann_solver/{conservative,laxf,hll,riemann_solver,source_term,
//                   electron_heating}.cc,
//   constrained_transport/constrained_transport.cc, recovery/invertor.cc,
//   initialization/timestep_estimation.cc
// and the task list runs unchanged: FluxDivergence, UpdateIndependentData,
// the boundary communication and ApplyBoundaryConditions stay Parthenon's.
//
// What a task does with a MeshData:
//  * its blocks become the jobs of a block pool (pangu_pool_create), one
//    single-block job per MeshBlock, so blocks need no common lattice: a
//    job's extents are its block's face coordinates at the interior bounds
//    (Xf), its metric spin and h the "metric" package's;
//  * every variable is addressed where Parthenon keeps it, through the
//    per-(block, component) pointer tables of pangu_pack: component c of a
//    variable is c * ncells past the data of MeshBlockData::Get(name), each
//    face-flux direction likewise from Get("conservative").flux[dir];
//  * the tables are uploaded once and again only when a block's arrays move
//    (e.g. after a remesh); the pool is rebuilt when the blocks' geometry or
//    count changes;
//  * the work is queued on the legacy default stream (or the one
//    b200::SetStream names) and the task returns without waiting, as a
//    Kokkos kernel launch does; EstimateTimestepMesh waits for its result.
//
// The engine computes a cell's coordinates from its job's extents, so they
// equal the MeshBlock's own where both are exact in binary (dyadic extents
// and widths); elsewhere they may differ in the last bit.
#include "b200_tasks.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "pangu_b200.h"

using parthenon::Real;

namespace {

using MD = parthenon::MeshData<Real>;

int option(const std::string &v, std::initializer_list<const char *> names, const char *what) {
  int i = 0;
  for (const char *n : names) {
    if (v == n) return i;
    ++i;
  }
  throw std::invalid_argument(std::string("unknown ") + what + ": " + v);
}

// The "core" and "metric" packages' params (package_registration.cc:21-96,
// :158-173) as the engine's parameter struct.
pangu_params params_of(const parthenon::MeshBlock &pmb) {
  auto core = pmb.packages.Get("core");
  auto metric = pmb.packages.Get("metric");
  pangu_params p{};
  p.cfl_number = core->Param<Real>("cfl_number");
  p.adiabatic_index = core->Param<Real>("adiabatic_index");
  p.riemann_solver = option(core->Param<std::string>("riemann_solver"), {"laxf", "hll"},
                            "Riemann solver");
  p.limiter = option(core->Param<std::string>("limiter"), {"ppm4", "mc"}, "limiter");
  p.density_floor = core->Param<Real>("density_floor");
  p.energy_floor = core->Param<Real>("energy_floor");
  p.density_floor_pow = core->Param<Real>("density_floor_pow");
  p.energy_floor_pow = core->Param<Real>("energy_floor_pow");
  p.enable_B = core->Param<bool>("enable_B") ? 1 : 0;
  p.recovery = option(core->Param<std::string>("recovery"), {"chainer", "robuster"}, "recovery");
  p.enable_heating = core->Param<bool>("enable_heating") ? 1 : 0;
  p.precision = PANGU_PRECISION_FP64;
  p.sigma_max = core->Param<Real>("sigma_max");
  p.lorentz_max = core->Param<Real>("lorentz_max");
  p.model = option(core->Param<std::string>("model_name"),
                   {"constant", "howes", "kawazura", "werner", "rowan", "sharma"},
                   "heating model");
  p.limit_kel = core->Param<bool>("limit_kel") ? 1 : 0;
  p.suppress_highb_heat = core->Param<bool>("suppress_highb_heat") ? 1 : 0;
  p.enforce_positive_dissipation = core->Param<bool>("enforce_positive_dissipation") ? 1 : 0;
  p.fel_constant = core->Param<Real>("fel_constant");
  p.gamma_e = core->Param<Real>("gamma_e");
  p.gamma_p = core->Param<Real>("gamma_p");
  p.ratio_min = core->Param<Real>("ratio_min");
  p.ratio_max = core->Param<Real>("ratio_max");
  p.fel_0 = core->Param<Real>("fel_0");
  // an unknown metric string is Minkowski, as in the tasks (e.g. laxf.cc:58-61)
  const std::string &mt = metric->Param<std::string>("metric_type");
  p.metric_type = mt == "bl"    ? PANGU_METRIC_BL
                  : mt == "cks" ? PANGU_METRIC_CKS
                  : mt == "mks" ? PANGU_METRIC_MKS
                                : PANGU_METRIC_MINKOWSKI;
  p.excise = metric->Param<bool>("excise") ? 1 : 0;
  p.a = metric->Param<Real>("a");
  p.h = metric->Param<Real>("h");
  p.r_excise = metric->Param<Real>("r_excise");
  p.dexcise = metric->Param<Real>("dexcise");
  p.pexcise = metric->Param<Real>("pexcise");
  return p;
}

// Face coordinate of direction d (0-based) at cell index idx of a block.
Real face(const parthenon::Coordinates &c, int d, int idx) {
  if (d == 0) return c.Xf<1, 1>(0, 0, idx);
  if (d == 1) return c.Xf<2, 2>(0, idx, 0);
  return c.Xf<3, 3>(idx, 0, 0);
}

// One block as a single-block job of the pool: interior cells, ghost width
// and extents (face coordinates at the interior bounds). The boundary
// conditions are never used: ghost exchange and physical boundaries stay
// Parthenon's.
pangu_mesh job_mesh(const parthenon::MeshBlock &pmb) {
  const parthenon::IndexShape &cb = pmb.cellbounds;
  const parthenon::IndexRange in[3] = {cb.GetBoundsI(parthenon::IndexDomain::interior),
                                       cb.GetBoundsJ(parthenon::IndexDomain::interior),
                                       cb.GetBoundsK(parthenon::IndexDomain::interior)};
  pangu_mesh m{};
  int *nx[3] = {&m.nx1, &m.nx2, &m.nx3};
  double *lo[3] = {&m.x1min, &m.x2min, &m.x3min};
  double *hi[3] = {&m.x1max, &m.x2max, &m.x3max};
  for (int d = 0; d < 3; ++d) {
    *nx[d] = in[d].e - in[d].s + 1;
    *lo[d] = face(pmb.coords, d, in[d].s);
    *hi[d] = face(pmb.coords, d, in[d].e + 1);
  }
  m.nbx1 = m.nbx2 = m.nbx3 = 1;
  m.ng = in[0].s;
  for (int f = 0; f < 6; ++f) m.bc[f] = PANGU_BC_OUTFLOW;
  return m;
}

bool same_mesh(const pangu_mesh &a, const pangu_mesh &b) {
  return a.nx1 == b.nx1 && a.nx2 == b.nx2 && a.nx3 == b.nx3 && a.ng == b.ng &&
         a.x1min == b.x1min && a.x1max == b.x1max && a.x2min == b.x2min &&
         a.x2max == b.x2max && a.x3min == b.x3min && a.x3max == b.x3max;
}

// The engine-side state of one MeshData: the pool, the device copy of the
// pointer tables and two small device arrays.
struct Binding {
  pangu_engine *e = nullptr;
  pangu_params params{};
  std::vector<pangu_mesh> blocks;
  std::vector<int> slot, job;      // [block]
  std::vector<uint64_t> table;     // host copy of the uploaded tables
  uint64_t *d_table = nullptr;     // prim, cons, flux1..3 [nb*nf]; alfven, efield [nb*3]; flag [nb]
  double *d_one = nullptr;         // [nb] 1.0: AddGeometricSource's dt[job] (beta carries dt)
  double *d_dt = nullptr;          // [nb] per-block dt estimates
  pangu_pack pack{};

  void release() {
    if (e) pangu_engine_destroy(e);
    cudaFree(d_table);
    cudaFree(d_one);
    cudaFree(d_dt);
    *this = Binding{};
  }
};

std::mutex g_mu;
std::map<const MD *, Binding> g_bind;
cudaStream_t g_stream = nullptr;

bool ok(cudaError_t rc) { return rc == cudaSuccess; }

// Builds (or rebuilds) the pool of md's blocks.
int make_pool(Binding &B, const pangu_params &p, const std::vector<pangu_mesh> &blocks) {
  B.release();
  const int nb = (int)blocks.size();
  pangu_mesh shape = blocks[0];
  int rc = pangu_pool_create(&p, &shape, nb, nb, &B.e);
  if (rc) return rc;
  B.params = p;
  B.blocks = blocks;
  B.slot.assign(nb, -1);
  B.job.assign(nb, -1);
  for (int b = 0; b < nb; ++b) {
    int32_t job = -1, slot = -1;
    rc = pangu_job_attach(B.e, &blocks[b], p.a, p.h, &job, &slot);
    if (rc) return rc;
    B.slot[b] = slot;
    B.job[b] = job;
  }
  // every job reads its own dt entry
  const std::vector<double> one(nb, 1.0);
  if (!ok(cudaMalloc(&B.d_one, nb * sizeof(double))) ||
      !ok(cudaMalloc(&B.d_dt, nb * sizeof(double))) ||
      !ok(cudaMemcpy(B.d_one, one.data(), nb * sizeof(double), cudaMemcpyHostToDevice)))
    return PANGU_ECUDA;
  return PANGU_OK;
}

// The binding of md, with its pool and pointer tables current.
int bind(MD *md, Binding *&out) {
  const int nb = md->NumBlocks();
  if (nb < 1) return PANGU_EINVAL;
  const parthenon::MeshBlock &pmb0 = *md->GetBlockData(0)->GetBlockPointer();
  const pangu_params p = params_of(pmb0);
  std::vector<pangu_mesh> blocks(nb);
  for (int b = 0; b < nb; ++b) blocks[b] = job_mesh(*md->GetBlockData(b)->GetBlockPointer());
  Binding &B = g_bind[md];
  // (pangu_params has no padding bytes: 19 doubles and 12 int32 fields)
  bool rebuild = !B.e || (int)B.blocks.size() != nb ||
                 std::memcmp(&B.params, &p, sizeof(p)) != 0;
  for (int b = 0; !rebuild && b < nb; ++b) rebuild = !same_mesh(B.blocks[b], blocks[b]);
  if (rebuild) {
    const int rc = make_pool(B, p, blocks);
    if (rc) {
      B.release();
      return rc;
    }
  }

  // pointer tables, by slot
  const int nf = pangu_num_fields(&p);
  const auto &sh = pmb0.cellbounds;
  const size_t ncell = (size_t)sh.ncellsi(parthenon::IndexDomain::entire) *
                       sh.ncellsj(parthenon::IndexDomain::entire) *
                       sh.ncellsk(parthenon::IndexDomain::entire);
  const int ndim = 1 + (blocks[0].nx2 > 1) + (blocks[0].nx3 > 1);
  const bool chainer = p.recovery == PANGU_RECOVERY_CHAINER;
  const size_t o_cons = (size_t)nb * nf, o_f1 = 2 * o_cons, o_f2 = 3 * o_cons,
               o_f3 = 4 * o_cons, o_al = 5 * o_cons, o_ef = o_al + 3 * (size_t)nb,
               o_fl = o_ef + 3 * (size_t)nb, total = o_fl + nb;
  std::vector<uint64_t> t(total, 0);
  // every array a task may touch must exist (an unallocated one has no data)
  bool absent = false;
  auto at = [&absent](Real *base, size_t c, size_t ncell) {
    absent |= base == nullptr;
    return base ? (uint64_t)(uintptr_t)(base + c * ncell) : 0;
  };
  const auto &names =
      pmb0.packages.Get("core")->Param<std::vector<std::string>>("primitive_field_names");
  for (int b = 0; b < nb; ++b) {
    auto &bd = *md->GetBlockData(b);
    const size_t s = (size_t)B.slot[b];
    size_t v = 0;
    for (const auto &n : names) {
      const auto &var = bd.Get(n);
      for (int c = 0; c < var.NumComponents(); ++c, ++v)
        if (v < (size_t)nf) t[s * nf + v] = at(var.data.data(), c, ncell);
    }
    if (v != (size_t)nf) return PANGU_EINVAL;
    const auto &cons = bd.Get("conservative");
    if (cons.NumComponents() != nf) return PANGU_EINVAL;
    for (int c = 0; c < nf; ++c) {
      t[o_cons + s * nf + c] = at(cons.data.data(), c, ncell);
      t[o_f1 + s * nf + c] = at(cons.flux[parthenon::X1DIR].data(), c, ncell);
      if (ndim >= 2) t[o_f2 + s * nf + c] = at(cons.flux[parthenon::X2DIR].data(), c, ncell);
      if (ndim == 3) t[o_f3 + s * nf + c] = at(cons.flux[parthenon::X3DIR].data(), c, ncell);
    }
    const auto &al = bd.Get("alfven");
    const auto &ef = bd.Get("electric_field");
    for (int c = 0; c < 3; ++c) {
      t[o_al + s * 3 + c] = at(al.data.data(), c, ncell);
      t[o_ef + s * 3 + c] = at(ef.data.data(), c, ncell);
    }
    if (chainer) t[o_fl + s] = at(bd.Get("flag").data.data(), 0, ncell);
  }
  if (absent) return PANGU_EINVAL;
  if (t != B.table) {
    // kernels queued earlier may still read the old tables
    if (B.d_table && !ok(cudaStreamSynchronize(g_stream))) return PANGU_ECUDA;
    if (B.table.size() != t.size()) {
      cudaFree(B.d_table);
      B.d_table = nullptr;
      if (!ok(cudaMalloc(&B.d_table, t.size() * sizeof(uint64_t)))) return PANGU_ECUDA;
    }
    if (!ok(cudaMemcpy(B.d_table, t.data(), t.size() * sizeof(uint64_t),
                       cudaMemcpyHostToDevice)))
      return PANGU_ECUDA;
    B.table = t;
    auto tab = [&](size_t off) { return reinterpret_cast<double *const *>(B.d_table + off); };
    B.pack = pangu_pack{};
    B.pack.prim_vars = tab(0);
    B.pack.cons_vars = tab(o_cons);
    B.pack.flux1_vars = tab(o_f1);
    if (ndim >= 2) B.pack.flux2_vars = tab(o_f2);
    if (ndim == 3) B.pack.flux3_vars = tab(o_f3);
    B.pack.alfven_vars = tab(o_al);
    B.pack.efield_vars = tab(o_ef);
    if (chainer) B.pack.flag_vars = tab(o_fl);
  }
  out = &B;
  return PANGU_OK;
}

// Runs fn(binding) under the lock; any failure is TaskStatus::fail.
template <class F>
parthenon::TaskStatus run(MD *md, F &&fn) {
  std::lock_guard<std::mutex> lock(g_mu);
  try {
    Binding *B = nullptr;
    if (bind(md, B) != PANGU_OK) return parthenon::TaskStatus::fail;
    return fn(*B) == PANGU_OK ? parthenon::TaskStatus::complete : parthenon::TaskStatus::fail;
  } catch (const std::exception &) {
    return parthenon::TaskStatus::fail;
  }
}

}  // namespace

parthenon::TaskStatus FixPrimitive(MD *md) {
  return run(md, [](Binding &B) { return pangu_fix_primitive(B.e, &B.pack, g_stream); });
}

parthenon::TaskStatus CalculateConservative(MD *md) {
  return run(md, [](Binding &B) { return pangu_calculate_conservative(B.e, &B.pack, g_stream); });
}

parthenon::TaskStatus CalculateFluxes(MD *md) {
  return run(md, [](Binding &B) { return pangu_calculate_fluxes(B.e, &B.pack, g_stream); });
}

parthenon::TaskStatus ConstraintedTransport(MD *md) {
  return run(md, [](Binding &B) { return pangu_constrained_transport(B.e, &B.pack, g_stream); });
}

// The engine applies beta * dt[job]; with dt[job] = 1 and beta = dt the
// product is dt exactly.
parthenon::TaskStatus AddGeometricSource(MD *md, Real dt) {
  return run(md, [dt](Binding &B) {
    return pangu_add_geometric_source(B.e, &B.pack, dt, B.d_one, g_stream);
  });
}

parthenon::TaskStatus Recovery(MD *md) {
  return run(md, [](Binding &B) { return pangu_recovery(B.e, &B.pack, g_stream); });
}

parthenon::TaskStatus ApplyElectronHeating(MD *md) {
  return run(md, [](Binding &B) { return pangu_apply_electron_heating(B.e, &B.pack, g_stream); });
}

parthenon::TaskStatus FixRecovery(MD *md) {
  return run(md, [](Binding &B) { return pangu_fix_recovery(B.e, &B.pack, g_stream); });
}

// timestep_estimation.cc:13-102: the minimum over the MeshData's blocks of
// each block's estimate (the engine reduces per job, i.e. per block). Throws
// std::runtime_error when the engine fails (the reference returns a Real).
Real EstimateTimestepMesh(MD *md) {
  Real out = 0.0;
  const auto st = run(md, [&out](Binding &B) {
    const size_t nb = B.job.size();
    int rc = pangu_estimate_dt(B.e, &B.pack, B.d_dt, g_stream);
    if (rc) return rc;
    std::vector<double> dt(nb);  // indexed by job id (0 .. nb-1 in an unshared pool)
    if (!ok(cudaMemcpyAsync(dt.data(), B.d_dt, nb * sizeof(double), cudaMemcpyDeviceToHost,
                            g_stream)) ||
        !ok(cudaStreamSynchronize(g_stream)))
      return PANGU_ECUDA;
    out = dt[B.job[0]];
    for (size_t b = 1; b < nb; ++b) out = dt[B.job[b]] < out ? dt[B.job[b]] : out;
    return PANGU_OK;
  });
  if (st != parthenon::TaskStatus::complete)
    throw std::runtime_error("EstimateTimestepMesh: the B200 engine failed");
  return out;
}

namespace b200 {

void SetStream(void *stream) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_stream = static_cast<cudaStream_t>(stream);
}

void ReleaseAll() {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto &kv : g_bind) kv.second.release();
  g_bind.clear();
}

}  // namespace b200
