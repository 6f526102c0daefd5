// basic_types.hpp -- stand-in for Parthenon's header of the same name; only
// parthenon::Real is needed by the reference's per-cell headers.
#ifndef PANGU_ORACLE_REFSHIM_BASIC_TYPES_HPP
#define PANGU_ORACLE_REFSHIM_BASIC_TYPES_HPP
#include "Kokkos_Core.hpp"
namespace parthenon {
using Real = double;
}
#endif
