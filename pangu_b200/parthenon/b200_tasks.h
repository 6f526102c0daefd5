// b200_tasks.h -- PANGU's stage tasks served by the B200 engine.
//
// The declarations are the reference's own task signatures
// (fixer/primitive_fixer.h:12, riemann_solver/conservative.h:12,
// riemann_solver/riemann_solver.h, constrained_transport/constrained_transport.h,
// riemann_solver/source_term.h, recovery/invertor.h:11,
// riemann_solver/electron_heating.h:12, fixer/recovery_fixer.h:12,
// initialization/timestep_estimation.h:10-11): an application links
// b200_tasks.cc in place of the reference's task sources and keeps its task
// list (ideal_grmhd.cc:62-110), packages and inputfiles unchanged. Each task
// reads the MeshData's variables where Parthenon keeps them -- one allocation
// per block and variable -- through the per-(block, component) pointer tables
// of pangu_pack; nothing is copied.
#ifndef PANGU_B200_PARTHENON_TASKS_H
#define PANGU_B200_PARTHENON_TASKS_H

#include <parthenon/package.hpp>

parthenon::TaskStatus FixPrimitive(parthenon::MeshData<parthenon::Real> *md);
parthenon::TaskStatus CalculateConservative(parthenon::MeshData<parthenon::Real> *md);
parthenon::TaskStatus CalculateFluxes(parthenon::MeshData<parthenon::Real> *md);
parthenon::TaskStatus ConstraintedTransport(parthenon::MeshData<parthenon::Real> *md);
parthenon::TaskStatus AddGeometricSource(parthenon::MeshData<parthenon::Real> *md,
                                         parthenon::Real dt);
parthenon::TaskStatus Recovery(parthenon::MeshData<parthenon::Real> *md);
parthenon::TaskStatus ApplyElectronHeating(parthenon::MeshData<parthenon::Real> *md);
parthenon::TaskStatus FixRecovery(parthenon::MeshData<parthenon::Real> *md);
parthenon::Real EstimateTimestepMesh(parthenon::MeshData<parthenon::Real> *md);

namespace b200 {
// The CUDA stream (a cudaStream_t) the tasks queue their work on; NULL, the
// default, is the legacy default stream, which orders the work with the
// Kokkos default instance's (blocking) stream.
void SetStream(void *stream);
// Releases the engines and tables the tasks keep per MeshData (call before
// the device memory of the mesh goes away, e.g. at the end of the run).
void ReleaseAll();
}  // namespace b200

#endif
