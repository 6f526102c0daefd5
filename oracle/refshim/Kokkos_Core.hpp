// Kokkos_Core.hpp -- minimal host-only stand-in used ONLY to compile the
// reference's per-cell headers (metric/, physics/, interpolation/,
// recovery/scheme_*.h) with g++ into oracle/_ref/. It maps the Kokkos math
// names those headers call onto the C library, and the function-space
// macros onto plain inline functions. Test infrastructure, never shipped.
#ifndef PANGU_ORACLE_REFSHIM_KOKKOS_CORE_HPP
#define PANGU_ORACLE_REFSHIM_KOKKOS_CORE_HPP
#include <cmath>
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
namespace Kokkos {
using std::cos;
using std::exp;
using std::fabs;
using std::fmax;
using std::fmin;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
inline double abs(double x) { return std::fabs(x); }
// Kokkos::min / max are the plain comparisons below (not fmin/fmax).
template <class T>
constexpr const T &min(const T &a, const T &b) { return (b < a) ? b : a; }
template <class T>
constexpr const T &max(const T &a, const T &b) { return (a < b) ? b : a; }
}  // namespace Kokkos
#endif
