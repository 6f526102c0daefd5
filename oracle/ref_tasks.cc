// ref_tasks.cc -- runs the REFERENCE's own stage tasks (pangu/src/fixer,
// riemann_solver, constrained_transport, recovery, initialization) on arrays
// in the layout of include/pangu_b200.h, through the host-only Parthenon
// stand-in of oracle/refshim/parthenon/package.hpp. Built by oracle/build.py
// into oracle/_ref/ only where the reference sources are present; used by
// tests/golden/make_task_golden.py to produce task-level golden fixtures that
// pin the CPU restatement (oracle.cc) task by task. Test infrastructure only.
//
// The tasks' pow is the correctly rounded pgm::pow of pgmath.h (the
// engine's and the restatement's), selected in the stand-in Kokkos header by
// PANGU_REFSHIM_CR_POW; every other math function is the C library's. That
// isolates what these fixtures pin -- loop ranges, floors and caps, fixer
// and excision logic, the chain of C2P schemes, the dt reduction -- from the
// one-ulp pow departure, which the per-cell golden vectors pin separately.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <parthenon/package.hpp>

#include "fixer/primitive_fixer.h"
#include "fixer/recovery_fixer.h"
#include "constrained_transport/constrained_transport.h"
#include "initialization/timestep_estimation.h"
#include "pangu_b200.h"
#include "recovery/invertor.h"
#include "riemann_solver/conservative.h"
#include "riemann_solver/electron_heating.h"
#include "riemann_solver/riemann_solver.h"
#include "riemann_solver/source_term.h"

using parthenon::Real;

namespace {

const char *kLimiter[] = {"ppm4", "mc"};
const char *kSolver[] = {"laxf", "hll"};
const char *kRecovery[] = {"chainer", "robuster"};
const char *kMetric[] = {"minkowski", "bl", "cks", "mks"};
const char *kModel[] = {"constant", "howes", "kawazura", "werner", "rowan", "sharma"};

// The "core" and "metric" packages as core::Initialize / metric::Initialize
// register them (package_registration.cc:21-96, :158-173).
parthenon::Packages make_packages(const pangu_params &p) {
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
  std::vector<std::string> fnames = {"density", "energy", "weighted_velocity"};
  if (p.enable_B) fnames.push_back("magnetic_field");
  fnames.push_back("entropy");
  if (p.enable_heating) fnames.push_back("electron_entropy");
  core->AddParam<std::vector<std::string>>("primitive_field_names", fnames);

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

struct Task {
  std::shared_ptr<parthenon::Mesh> mesh;
  std::unique_ptr<parthenon::MeshData<Real>> md;
};

// A MeshData over the pack: every variable's components addressed through a
// per-(block, component) pointer table, as a Parthenon pack of per-variable
// views is.
Task make_md(const pangu_params &p, const pangu_mesh &m, const pangu_pack &pk) {
  const int act[3] = {m.nx1 > 1, m.nx2 > 1, m.nx3 > 1};
  const int nx[3] = {m.nx1, m.nx2, m.nx3};
  const int N[3] = {nx[0] + 2 * m.ng * act[0], nx[1] + 2 * m.ng * act[1],
                    nx[2] + 2 * m.ng * act[2]};
  const int nb = m.nbx1 * m.nbx2 * m.nbx3;
  const size_t ncell = (size_t)N[0] * N[1] * N[2];
  int nf = 6 + (p.enable_B ? 3 : 0) + (p.enable_heating ? 1 : 0);

  auto vt = std::make_shared<parthenon::VarTable>();
  vt->nb = nb;
  vt->n1 = N[0];
  vt->n2 = N[1];
  vt->n3 = N[2];
  // a variable of ncomp components starting at component c0 of an array of
  // nv components per block
  auto add = [&](const std::string &name, double *base, double *const flux[3], int nv, int c0,
                 int ncomp) {
    parthenon::VarTable::Var v;
    v.ncomp = ncomp;
    for (int b = 0; b < nb; ++b)
      for (int c = 0; c < ncomp; ++c) {
        const size_t off = ((size_t)b * nv + c0 + c) * ncell;
        v.data.push_back(base + off);
        for (int d = 0; d < 3; ++d)
          if (flux && flux[d]) v.flux[d].push_back(flux[d] + off);
      }
    vt->vars[name] = v;
  };
  int c = 0;
  add("density", pk.prim, nullptr, nf, c, 1); c += 1;
  add("energy", pk.prim, nullptr, nf, c, 1); c += 1;
  add("weighted_velocity", pk.prim, nullptr, nf, c, 3); c += 3;
  if (p.enable_B) { add("magnetic_field", pk.prim, nullptr, nf, c, 3); c += 3; }
  add("entropy", pk.prim, nullptr, nf, c, 1); c += 1;
  if (p.enable_heating) { add("electron_entropy", pk.prim, nullptr, nf, c, 1); c += 1; }
  double *const flux[3] = {pk.flux1, pk.flux2, pk.flux3};
  add("conservative", pk.cons, flux, nf, 0, nf);
  add("alfven", pk.alfven, nullptr, 3, 0, 3);
  add("electric_field", pk.efield, nullptr, 3, 0, 3);
  if (pk.flag) add("flag", pk.flag, nullptr, 1, 0, 1);

  const double mins[3] = {m.x1min, m.x2min, m.x3min};
  const double maxs[3] = {m.x1max, m.x2max, m.x3max};
  const int nbx[3] = {m.nbx1, m.nbx2, m.nbx3};
  double dx[3];
  for (int d = 0; d < 3; ++d) dx[d] = (maxs[d] - mins[d]) / (double)(nbx[d] * nx[d]);

  Task t;
  t.mesh = std::make_shared<parthenon::Mesh>();
  t.mesh->ndim = act[0] + act[1] + act[2];
  parthenon::Packages packages = make_packages(p);
  std::vector<std::shared_ptr<parthenon::MeshBlock>> blocks;
  for (int b = 0; b < nb; ++b) {
    auto pmb = std::make_shared<parthenon::MeshBlock>();
    pmb->packages = packages;
    pmb->pmy_mesh = t.mesh.get();
    const int bl[3] = {b % m.nbx1, (b / m.nbx1) % m.nbx2, b / (m.nbx1 * m.nbx2)};
    for (int d = 0; d < 3; ++d) {
      pmb->cellbounds.entire_[d] = {0, N[d] - 1};
      pmb->cellbounds.interior_[d] = {m.ng * act[d], m.ng * act[d] + nx[d] - 1};
      const double bxmin = mins[d] + (double)(bl[d] * nx[d]) * dx[d];
      pmb->coords.x0[d] = bxmin - (double)(m.ng * act[d]) * dx[d];
      pmb->coords.dx[d] = dx[d];
    }
    vt->coords.push_back(pmb->coords);
    blocks.push_back(pmb);
  }
  t.md = std::make_unique<parthenon::MeshData<Real>>(blocks, vt);
  return t;
}

}  // namespace

extern "C" {

// The reference task `task` on md (see the enumeration below); dt is
// AddGeometricSource's time step (the stage's beta dt). EstimateTimestepMesh
// writes its result to *out. Returns 0, or -1 when the task threw.
enum {
  REF_FIX_PRIMITIVE = 0,
  REF_CALCULATE_CONSERVATIVE = 1,
  REF_CALCULATE_FLUXES = 2,
  REF_CONSTRAINED_TRANSPORT = 3,
  REF_ADD_GEOMETRIC_SOURCE = 4,
  REF_RECOVERY = 5,
  REF_APPLY_ELECTRON_HEATING = 6,
  REF_FIX_RECOVERY = 7,
  REF_ESTIMATE_TIMESTEP = 8,
};

int ref_task(const pangu_params *p, const pangu_mesh *m, pangu_pack *md, int task, double dt,
             double *out) {
  try {
    Task t = make_md(*p, *m, *md);
    parthenon::MeshData<Real> *mdp = t.md.get();
    switch (task) {
      case REF_FIX_PRIMITIVE: FixPrimitive(mdp); break;
      case REF_CALCULATE_CONSERVATIVE: CalculateConservative(mdp); break;
      case REF_CALCULATE_FLUXES: CalculateFluxes(mdp); break;
      case REF_CONSTRAINED_TRANSPORT: ConstraintedTransport(mdp); break;
      case REF_ADD_GEOMETRIC_SOURCE: AddGeometricSource(mdp, dt); break;
      case REF_RECOVERY: Recovery(mdp); break;
      case REF_APPLY_ELECTRON_HEATING: ApplyElectronHeating(mdp); break;
      case REF_FIX_RECOVERY: FixRecovery(mdp); break;
      case REF_ESTIMATE_TIMESTEP:
        if (out) *out = EstimateTimestepMesh(mdp);
        break;
      default: return -1;
    }
  } catch (...) {
    return -1;
  }
  return 0;
}

}  // extern "C"
