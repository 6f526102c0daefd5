// Kokkos_Core.hpp -- minimal host-only stand-in used ONLY to compile the
// reference's per-cell headers (metric/, physics/, interpolation/,
// recovery/scheme_*.h) and stage tasks with g++ into oracle/_ref/. It maps
// the Kokkos math names those sources call onto the C library, and the
// function-space macros onto plain inline functions. With
// PANGU_REFSHIM_CR_POW defined, pow is the correctly rounded pgm::pow of
// pgmath.h instead of the C library's (the task-level build). Test
// infrastructure, never shipped.
#ifndef PANGU_ORACLE_REFSHIM_KOKKOS_CORE_HPP
#define PANGU_ORACLE_REFSHIM_KOKKOS_CORE_HPP
#include <cmath>
#ifdef PANGU_REFSHIM_CR_POW
#include "pgmath.h"
#endif
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
#ifdef PANGU_REFSHIM_CR_POW
inline double pow(double x, double y) { return pgm::pow(x, y); }
#else
using std::pow;
#endif
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
