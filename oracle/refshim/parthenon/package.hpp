// parthenon/package.hpp -- host-only stand-in for the part of Parthenon's API
// that PANGU's stage tasks call, so that the reference's own task sources
// (pangu/src/{fixer,riemann_solver,constrained_transport,recovery,
// initialization}/*.cc) compile with g++ from where they lie and run on
// arrays the tests own. TEST INFRASTRUCTURE ONLY (oracle/build.py links it
// into oracle/_ref/); nothing in the engine includes it.
//
// Parthenon itself is not vendored with the reference, so this header states
// the behaviour the tasks rely on, with the same conventions as the engine
// and the CPU restatement:
//  * a MeshData is a set of equal meshblocks; variables are addressed per
//    (block, component) through a table of base pointers of [N3][N2][N1]
//    arrays (i fastest), as Parthenon's packs of per-variable views are;
//    MeshBlockData::Get(name) gives one block's variable (its components
//    contiguous, as a Parthenon variable's are) and its face fluxes;
//  * IndexDomain::entire spans every cell, IndexDomain::interior the cells
//    without the ng ghost layers of each active direction;
//  * uniform Cartesian coordinates: Xc<d>(idx) = x0_d + (idx + 1/2) dx_d and
//    Xf<d, f>(k, j, i) = x0_d + idx dx_d on the face f == d (the cell centre
//    along the other directions), x0_d = block xmin - ng dx_d;
//  * par_for runs its index ranges as serial nested loops in argument order;
//    par_reduce with Kokkos::Min starts from the largest finite Real. Built
//    with PANGU_REFSHIM_OMP and OpenMP (the timing build of the reference's
//    tasks only), both spread their index ranges over the host threads, as
//    Kokkos' OpenMP backend does; the fixtures use the serial form.
#ifndef PANGU_ORACLE_REFSHIM_PARTHENON_PACKAGE_HPP
#define PANGU_ORACLE_REFSHIM_PARTHENON_PACKAGE_HPP

#include <any>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../Kokkos_Core.hpp"
#include "../basic_types.hpp"

#define PARTHENON_INSTRUMENT
#define PARTHENON_AUTO_LABEL "pangu_task"
#ifndef KOKKOS_LAMBDA
#define KOKKOS_LAMBDA [=]
#endif

template <class T>
inline T SQR(const T &x) {
  return x * x;
}

namespace Kokkos {
// Reducer of par_reduce: the result is written to the bound variable.
template <class T>
struct Min {
  T &result;
  explicit Min(T &r) : result(r) {}
};
}  // namespace Kokkos

namespace parthenon {

enum class TaskStatus { fail, complete, incomplete, iterate };
enum class IndexDomain { entire, interior };
enum CoordinateDirection { NODIR = -1, X0DIR = 0, X1DIR = 1, X2DIR = 2, X3DIR = 3 };

struct IndexRange {
  int s = 0;
  int e = 0;
};

// Index ranges of one block: entire[d] and interior[d] per direction.
struct IndexShape {
  IndexRange entire_[3], interior_[3];
  IndexRange GetBoundsI(IndexDomain d) const {
    return d == IndexDomain::entire ? entire_[0] : interior_[0];
  }
  IndexRange GetBoundsJ(IndexDomain d) const {
    return d == IndexDomain::entire ? entire_[1] : interior_[1];
  }
  IndexRange GetBoundsK(IndexDomain d) const {
    return d == IndexDomain::entire ? entire_[2] : interior_[2];
  }
  int ncellsi(IndexDomain d) const { return GetBoundsI(d).e - GetBoundsI(d).s + 1; }
  int ncellsj(IndexDomain d) const { return GetBoundsJ(d).e - GetBoundsJ(d).s + 1; }
  int ncellsk(IndexDomain d) const { return GetBoundsK(d).e - GetBoundsK(d).s + 1; }
};

struct Coordinates {
  Real x0[3] = {0.0, 0.0, 0.0};  // block xmin - ng dx (xmin on inactive directions)
  Real dx[3] = {1.0, 1.0, 1.0};
  template <int dir>
  Real Xc(const int idx) const {
    return x0[dir - 1] + ((Real)idx + 0.5) * dx[dir - 1];
  }
  template <int dir, int face>
  Real Xf(const int k, const int j, const int i) const {
    const int idx = dir == 1 ? i : (dir == 2 ? j : k);
    if (dir == face) return x0[dir - 1] + (Real)idx * dx[dir - 1];
    return Xc<dir>(idx);
  }
  template <int dir>
  Real Dx() const {
    return dx[dir - 1];
  }
};

// Named variables of one container: per block and component, the base
// pointer of an [N3][N2][N1] array, and the face-flux arrays where the
// variable has fluxes.
struct VarTable {
  int nb = 0, n1 = 1, n2 = 1, n3 = 1;
  struct Var {
    int ncomp = 1;
    std::vector<Real *> data;     // [b * ncomp + c]
    std::vector<Real *> flux[3];  // [b * ncomp + c] per direction, may be empty
  };
  std::map<std::string, Var> vars;
  std::vector<Coordinates> coords;  // [b]
};

using PackIndexMap = std::map<std::string, std::pair<int, int>>;

// Pointer table of a pack: components of the requested variables in request
// order, for every block.
struct PackTable {
  int nb = 0, nvar = 0, n1 = 1, n2 = 1, n3 = 1;
  std::vector<Real *> data;     // [b * nvar + v]
  std::vector<Real *> flux[3];  // [b * nvar + v]
  std::shared_ptr<const VarTable> src;
  Real &at(const std::vector<Real *> &t, int b, int v, int k, int j, int i) const {
    return t[(size_t)b * nvar + v][((size_t)k * n2 + j) * n1 + i];
  }
};

inline std::shared_ptr<PackTable> make_pack(const std::shared_ptr<const VarTable> &vt,
                                            const std::vector<std::string> &names,
                                            PackIndexMap *idx, bool fluxes) {
  auto p = std::make_shared<PackTable>();
  p->nb = vt->nb;
  p->n1 = vt->n1;
  p->n2 = vt->n2;
  p->n3 = vt->n3;
  p->src = vt;
  std::vector<const VarTable::Var *> sel;
  for (const auto &n : names) {
    auto it = vt->vars.find(n);
    if (it == vt->vars.end()) throw std::invalid_argument("no variable " + n);
    if (idx) (*idx)[n] = {p->nvar, p->nvar + it->second.ncomp - 1};
    p->nvar += it->second.ncomp;
    sel.push_back(&it->second);
  }
  p->data.resize((size_t)p->nb * p->nvar);
  if (fluxes)
    for (int d = 0; d < 3; ++d) p->flux[d].resize((size_t)p->nb * p->nvar, nullptr);
  for (int b = 0; b < p->nb; ++b) {
    int v = 0;
    for (const auto *var : sel)
      for (int c = 0; c < var->ncomp; ++c, ++v) {
        p->data[(size_t)b * p->nvar + v] = var->data[(size_t)b * var->ncomp + c];
        if (fluxes)
          for (int d = 0; d < 3; ++d)
            if (!var->flux[d].empty())
              p->flux[d][(size_t)b * p->nvar + v] = var->flux[d][(size_t)b * var->ncomp + c];
      }
  }
  return p;
}

// Pack of one block: (component, k, j, i).
template <class T>
class VariablePack {
 public:
  VariablePack() = default;
  VariablePack(std::shared_ptr<PackTable> p, int b) : p_(std::move(p)), b_(b) {}
  T &operator()(int v, int k, int j, int i) const { return p_->at(p_->data, b_, v, k, j, i); }
  T &flux(int dir, int v, int k, int j, int i) const {
    return p_->at(p_->flux[dir - 1], b_, v, k, j, i);
  }

 private:
  std::shared_ptr<PackTable> p_;
  int b_ = 0;
};

// Pack of every block of a MeshData: (block, component, k, j, i).
template <class T>
class MeshBlockVarPack {
 public:
  MeshBlockVarPack() = default;
  explicit MeshBlockVarPack(std::shared_ptr<PackTable> p) : p_(std::move(p)) {}
  T &operator()(int b, int v, int k, int j, int i) const {
    return p_->at(p_->data, b, v, k, j, i);
  }
  VariablePack<T> operator()(int b) const { return VariablePack<T>(p_, b); }
  const Coordinates &GetCoords(int b) const { return p_->src->coords[b]; }
  int GetNBlocks() const { return p_->nb; }

 protected:
  std::shared_ptr<PackTable> p_;
};

template <class T>
class MeshBlockVarFluxPack : public MeshBlockVarPack<T> {
 public:
  MeshBlockVarFluxPack() = default;
  explicit MeshBlockVarFluxPack(std::shared_ptr<PackTable> p)
      : MeshBlockVarPack<T>(std::move(p)) {}
};

class StateDescriptor {
 public:
  template <class T>
  void AddParam(const std::string &key, T value) {
    params_[key] = std::move(value);
  }
  template <class T>
  const T &Param(const std::string &key) const {
    auto it = params_.find(key);
    if (it == params_.end()) throw std::invalid_argument("no param " + key);
    return *std::any_cast<T>(&it->second);
  }

 private:
  std::map<std::string, std::any> params_;
};

struct Packages {
  std::map<std::string, std::shared_ptr<StateDescriptor>> pkgs;
  std::shared_ptr<StateDescriptor> Get(const std::string &name) const { return pkgs.at(name); }
};

struct Mesh {
  int ndim = 1;
};

class MeshBlock {
 public:
  Packages packages;
  IndexShape cellbounds;
  Coordinates coords;
  Mesh *pmy_mesh = nullptr;

  template <class F>
  void par_for(const char *, int b0, int b1, int k0, int k1, int j0, int j1, int i0, int i1,
               const F &f) const {
#if defined(PANGU_REFSHIM_OMP) && defined(_OPENMP)
#pragma omp parallel for collapse(4) schedule(static)
#endif
    for (int b = b0; b <= b1; ++b)
      for (int k = k0; k <= k1; ++k)
        for (int j = j0; j <= j1; ++j)
          for (int i = i0; i <= i1; ++i) f(b, k, j, i);
  }
  template <class F>
  void par_for(const char *, int k0, int k1, int j0, int j1, int i0, int i1, const F &f) const {
#if defined(PANGU_REFSHIM_OMP) && defined(_OPENMP)
#pragma omp parallel for collapse(3) schedule(static)
#endif
    for (int k = k0; k <= k1; ++k)
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) f(k, j, i);
  }
  template <class F>
  void par_reduce(const char *, int k0, int k1, int j0, int j1, int i0, int i1, const F &f,
                  Kokkos::Min<Real> red) const {
    Real acc = std::numeric_limits<Real>::max();
#if defined(PANGU_REFSHIM_OMP) && defined(_OPENMP)
#pragma omp parallel for collapse(3) schedule(static) reduction(min : acc)
#endif
    for (int k = k0; k <= k1; ++k)
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) f(k, j, i, acc);
    red.result = acc;
  }
};

// One variable of one block, as MeshBlockData::Get returns it: the
// device-side data of its components (contiguous, [comp][N3][N2][N1]) and of
// its face fluxes, flux[X1DIR..X3DIR].
struct ArrayRef {
  Real *p = nullptr;
  Real *data() const { return p; }
};
struct VariableRef {
  ArrayRef data;
  ArrayRef flux[4];
  int ncomp = 1;
  int NumComponents() const { return ncomp; }
};

template <class T>
class MeshBlockData {
 public:
  MeshBlockData(std::shared_ptr<MeshBlock> pmb, std::shared_ptr<const VarTable> vt, int b)
      : pmb_(std::move(pmb)), vt_(std::move(vt)), b_(b) {}
  std::shared_ptr<MeshBlock> GetBlockPointer() const { return pmb_; }
  VariableRef Get(const std::string &name) const {
    const VarTable::Var &v = vt_->vars.at(name);
    VariableRef r;
    r.ncomp = v.ncomp;
    r.data.p = v.data[(size_t)b_ * v.ncomp];
    for (int d = 0; d < 3; ++d)
      if (!v.flux[d].empty()) r.flux[d + 1].p = v.flux[d][(size_t)b_ * v.ncomp];
    return r;
  }
  VariablePack<T> PackVariables(const std::vector<std::string> &names, PackIndexMap &idx) {
    return VariablePack<T>(make_pack(vt_, names, &idx, false), b_);
  }

 private:
  std::shared_ptr<MeshBlock> pmb_;
  std::shared_ptr<const VarTable> vt_;
  int b_;
};

template <class T>
class MeshData {
 public:
  MeshData(std::vector<std::shared_ptr<MeshBlock>> blocks, std::shared_ptr<const VarTable> vt)
      : vt_(std::move(vt)) {
    for (size_t b = 0; b < blocks.size(); ++b)
      data_.push_back(std::make_shared<MeshBlockData<T>>(blocks[b], vt_, (int)b));
    if (!blocks.empty()) shape_ = blocks[0]->cellbounds;
  }
  std::shared_ptr<MeshBlockData<T>> &GetBlockData(int b) { return data_.at(b); }
  int NumBlocks() const { return (int)data_.size(); }
  IndexRange GetBoundsI(IndexDomain d) const { return shape_.GetBoundsI(d); }
  IndexRange GetBoundsJ(IndexDomain d) const { return shape_.GetBoundsJ(d); }
  IndexRange GetBoundsK(IndexDomain d) const { return shape_.GetBoundsK(d); }
  MeshBlockVarPack<T> PackVariables(const std::vector<std::string> &names, PackIndexMap &idx) {
    return MeshBlockVarPack<T>(make_pack(vt_, names, &idx, false));
  }
  MeshBlockVarPack<T> PackVariables(const std::vector<std::string> &names) {
    return MeshBlockVarPack<T>(make_pack(vt_, names, nullptr, false));
  }
  MeshBlockVarFluxPack<T> PackVariablesAndFluxes(const std::vector<std::string> &names,
                                                 PackIndexMap &idx) {
    return MeshBlockVarFluxPack<T>(make_pack(vt_, names, &idx, true));
  }

 private:
  std::shared_ptr<const VarTable> vt_;
  std::vector<std::shared_ptr<MeshBlockData<T>>> data_;
  IndexShape shape_;
};

namespace package {
namespace prelude {
using namespace parthenon;  // NOLINT: the prelude re-exports Parthenon's names
}  // namespace prelude
}  // namespace package

}  // namespace parthenon

#endif
