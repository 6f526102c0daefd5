// driver.cc -- test driver of pangu_b200/parthenon/b200_tasks.cc (the
// reference's task functions served by the engine). It builds MeshData
// objects of the host-only Parthenon stand-in (oracle/refshim) over DEVICE
// arrays the test allocates -- one allocation per block and variable, as
// Parthenon keeps them -- and calls the shim's task functions on them, the
// way a Parthenon task list would. Test infrastructure only.
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <parthenon/package.hpp>

#include "../../pangu_b200/parthenon/b200_tasks.h"
#include "pangu_b200.h"

using parthenon::Real;

namespace {

const char *kLimiter[] = {"ppm4", "mc"};
const char *kSolver[] = {"laxf", "hll"};
const char *kRecovery[] = {"chainer", "robuster"};
const char *kMetric[] = {"minkowski", "bl", "cks", "mks"};
const char *kModel[] = {"constant", "howes", "kawazura", "werner", "rowan", "sharma"};

// Primitive variables in registration order (package_registration.cc:84-96).
std::vector<std::string> prim_names(const pangu_params &p) {
  std::vector<std::string> n = {"density", "energy", "weighted_velocity"};
  if (p.enable_B) n.push_back("magnetic_field");
  n.push_back("entropy");
  if (p.enable_heating) n.push_back("electron_entropy");
  return n;
}

// The "core" and "metric" packages with the params the tasks read
// (package_registration.cc:21-96, :158-173).
parthenon::Packages packages(const pangu_params &p) {
  auto core = std::make_shared<parthenon::StateDescriptor>();
  core->AddParam<Real>("cfl_number", p.cfl_number);
  core->AddParam<Real>("adiabatic_index", p.adiabatic_index);
  core->AddParam<std::string>("riemann_solver", kSolver[p.riemann_solver]);
  core->AddParam<std::string>("limiter", kLimiter[p.limiter]);
  core->AddParam<Real>("density_floor", p.density_floor);
  core->AddParam<Real>("energy_floor", p.energy_floor);
  core->AddParam<Real>("density_floor_pow", p.density_floor_pow);
  core->AddParam<Real>("energy_floor_pow", p.energy_floor_pow);
  core->AddParam<bool>("enable_B", p.enable_B != 0);
  core->AddParam<std::string>("recovery", kRecovery[p.recovery]);
  core->AddParam<bool>("enable_heating", p.enable_heating != 0);
  core->AddParam<Real>("sigma_max", p.sigma_max);
  core->AddParam<Real>("lorentz_max", p.lorentz_max);
  core->AddParam<std::string>("model_name", kModel[p.model]);
  core->AddParam<Real>("fel_constant", p.fel_constant);
  core->AddParam<Real>("gamma_e", p.gamma_e);
  core->AddParam<Real>("gamma_p", p.gamma_p);
  core->AddParam<bool>("limit_kel", p.limit_kel != 0);
  core->AddParam<bool>("suppress_highb_heat", p.suppress_highb_heat != 0);
  core->AddParam<bool>("enforce_positive_dissipation", p.enforce_positive_dissipation != 0);
  core->AddParam<Real>("ratio_min", p.ratio_min);
  core->AddParam<Real>("ratio_max", p.ratio_max);
  core->AddParam<Real>("fel_0", p.fel_0);
  core->AddParam<std::vector<std::string>>("primitive_field_names", prim_names(p));
  auto metric = std::make_shared<parthenon::StateDescriptor>();
  metric->AddParam<std::string>("metric_type", kMetric[p.metric_type]);
  metric->AddParam<bool>("excise", p.excise != 0);
  metric->AddParam<Real>("a", p.a);
  metric->AddParam<Real>("h", p.h);
  metric->AddParam<Real>("r_excise", p.r_excise);
  metric->AddParam<Real>("dexcise", p.dexcise);
  metric->AddParam<Real>("pexcise", p.pexcise);
  parthenon::Packages pk;
  pk.pkgs["core"] = core;
  pk.pkgs["metric"] = metric;
  return pk;
}

struct Container {
  std::shared_ptr<parthenon::Mesh> mesh;
  std::unique_ptr<parthenon::MeshData<Real>> md;
};

std::map<int, Container> g_md;
int g_next = 0;

}  // namespace

extern "C" {

// Primitive variables of a parameter set, in registration order
// (package_registration.cc:84-96), and their component counts.
int shim_num_prim_vars(const pangu_params *p) {
  return 4 + (p->enable_B ? 1 : 0) + (p->enable_heating ? 1 : 0);
}

// A MeshData over device arrays. ptrs holds, per block (lattice order, x1
// fastest), shim_num_prim_vars(p) + 7 addresses: each primitive variable's
// data (its components contiguous), then conservative, its x1/x2/x3 face
// fluxes (0 for an inactive direction), alfven, electric_field and flag (0
// for the robuster recovery). Block b's coordinates are those of block b of
// the uniform mesh m. Writes a handle for shim_run.
int shim_make(const pangu_params *p, const pangu_mesh *m, const uint64_t *ptrs, int *handle) {
  if (!p || !m || !ptrs || !handle) return -1;
  const pangu_mesh &M = *m;
  const int act[3] = {M.nx1 > 1, M.nx2 > 1, M.nx3 > 1};
  const int nx[3] = {M.nx1, M.nx2, M.nx3};
  const int N[3] = {nx[0] + 2 * M.ng * act[0], nx[1] + 2 * M.ng * act[1],
                    nx[2] + 2 * M.ng * act[2]};
  const int nb = M.nbx1 * M.nbx2 * M.nbx3;
  const int npv = shim_num_prim_vars(p), per = npv + 7;
  std::vector<std::string> pnames = prim_names(*p);
  std::vector<int> pcomp;
  for (const auto &n : pnames) pcomp.push_back(n == "weighted_velocity" || n == "magnetic_field" ? 3 : 1);
  const int nf = pangu_num_fields(p);

  auto vt = std::make_shared<parthenon::VarTable>();
  vt->nb = nb;
  vt->n1 = N[0];
  vt->n2 = N[1];
  vt->n3 = N[2];
  const size_t ncell = (size_t)N[0] * N[1] * N[2];
  auto P = [&](int b, int s) { return reinterpret_cast<Real *>(ptrs[(size_t)b * per + s]); };
  auto add = [&](const std::string &name, int slot, int ncomp, bool fluxes) {
    parthenon::VarTable::Var v;
    v.ncomp = ncomp;
    for (int b = 0; b < nb; ++b)
      for (int c = 0; c < ncomp; ++c) {
        v.data.push_back(P(b, slot) + c * ncell);
        if (fluxes)
          for (int d = 0; d < 3; ++d)
            v.flux[d].push_back(P(b, npv + 1 + d) ? P(b, npv + 1 + d) + c * ncell : nullptr);
      }
    vt->vars[name] = v;
  };
  for (int s = 0; s < npv; ++s) add(pnames[s], s, pcomp[s], false);
  add("conservative", npv, nf, true);
  add("alfven", npv + 4, 3, false);
  add("electric_field", npv + 5, 3, false);
  if (p->recovery == PANGU_RECOVERY_CHAINER) add("flag", npv + 6, 1, false);

  const double mins[3] = {M.x1min, M.x2min, M.x3min};
  const double maxs[3] = {M.x1max, M.x2max, M.x3max};
  const int nbx[3] = {M.nbx1, M.nbx2, M.nbx3};
  double dx[3];
  for (int d = 0; d < 3; ++d) dx[d] = (maxs[d] - mins[d]) / (double)(nbx[d] * nx[d]);
  Container c;
  c.mesh = std::make_shared<parthenon::Mesh>();
  c.mesh->ndim = act[0] + act[1] + act[2];
  parthenon::Packages pk = packages(*p);
  std::vector<std::shared_ptr<parthenon::MeshBlock>> blocks;
  for (int b = 0; b < nb; ++b) {
    auto pmb = std::make_shared<parthenon::MeshBlock>();
    pmb->packages = pk;
    pmb->pmy_mesh = c.mesh.get();
    const int bl[3] = {b % M.nbx1, (b / M.nbx1) % M.nbx2, b / (M.nbx1 * M.nbx2)};
    for (int d = 0; d < 3; ++d) {
      pmb->cellbounds.entire_[d] = {0, N[d] - 1};
      pmb->cellbounds.interior_[d] = {M.ng * act[d], M.ng * act[d] + nx[d] - 1};
      const double bxmin = mins[d] + (double)(bl[d] * nx[d]) * dx[d];
      pmb->coords.x0[d] = bxmin - (double)(M.ng * act[d]) * dx[d];
      pmb->coords.dx[d] = dx[d];
    }
    vt->coords.push_back(pmb->coords);
    blocks.push_back(pmb);
  }
  c.md = std::make_unique<parthenon::MeshData<Real>>(blocks, vt);
  *handle = g_next++;
  g_md[*handle] = std::move(c);
  return 0;
}

enum {
  SHIM_FIX_PRIMITIVE = 0,
  SHIM_CALCULATE_CONSERVATIVE = 1,
  SHIM_CALCULATE_FLUXES = 2,
  SHIM_CONSTRAINED_TRANSPORT = 3,
  SHIM_ADD_GEOMETRIC_SOURCE = 4,
  SHIM_RECOVERY = 5,
  SHIM_APPLY_ELECTRON_HEATING = 6,
  SHIM_FIX_RECOVERY = 7,
  SHIM_ESTIMATE_TIMESTEP = 8,
};

// Task `task` of the shim on the MeshData `handle`; dt is AddGeometricSource's
// step, EstimateTimestepMesh's result goes to *out. 0 = TaskStatus::complete,
// 1 = TaskStatus::fail, -1 = bad handle/task or an exception.
int shim_run(int handle, int task, double dt, double *out) {
  auto it = g_md.find(handle);
  if (it == g_md.end()) return -1;
  parthenon::MeshData<Real> *md = it->second.md.get();
  parthenon::TaskStatus st = parthenon::TaskStatus::complete;
  try {
    switch (task) {
      case SHIM_FIX_PRIMITIVE: st = FixPrimitive(md); break;
      case SHIM_CALCULATE_CONSERVATIVE: st = CalculateConservative(md); break;
      case SHIM_CALCULATE_FLUXES: st = CalculateFluxes(md); break;
      case SHIM_CONSTRAINED_TRANSPORT: st = ConstraintedTransport(md); break;
      case SHIM_ADD_GEOMETRIC_SOURCE: st = AddGeometricSource(md, dt); break;
      case SHIM_RECOVERY: st = Recovery(md); break;
      case SHIM_APPLY_ELECTRON_HEATING: st = ApplyElectronHeating(md); break;
      case SHIM_FIX_RECOVERY: st = FixRecovery(md); break;
      case SHIM_ESTIMATE_TIMESTEP:
        if (!out) return -1;
        *out = EstimateTimestepMesh(md);
        break;
      default: return -1;
    }
  } catch (...) {
    return -1;
  }
  return st == parthenon::TaskStatus::complete ? 0 : 1;
}

// Drops every MeshData and the shim's engines.
void shim_free_all() {
  b200::ReleaseAll();
  g_md.clear();
}

}  // extern "C"
