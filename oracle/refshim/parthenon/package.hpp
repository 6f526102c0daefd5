// parthenon/package.hpp -- stand-in exposing parthenon::Real and the
// package prelude namespace used by recovery/constants.h.
#ifndef PANGU_ORACLE_REFSHIM_PARTHENON_PACKAGE_HPP
#define PANGU_ORACLE_REFSHIM_PARTHENON_PACKAGE_HPP
#include "../Kokkos_Core.hpp"
#include "../basic_types.hpp"
namespace parthenon {
namespace package {
namespace prelude {
using parthenon::Real;
}
}  // namespace package
}  // namespace parthenon
#endif
