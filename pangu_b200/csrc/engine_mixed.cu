// engine_mixed.cu -- the mixed-precision instantiation of the engine's
// kernels (namespace pgkmx): primitives stored in FP32; reconstruction,
// Riemann fluxes, FixPrimitive's floors, electron heating and the geometric
// source term in FP32;
// conserved variables and the flux divergence update, C2P, the metric and CT
// in FP64.
// Built with --use_fast_math (FMA contraction, approximate FP32 division,
// square root and math functions, FP32 denormals flushed; FP64 arithmetic is
// unaffected) and the CUDA math library's pow/exp/log (the exact build,
// engine.cu, keeps --fmad=false and correctly rounded functions for
// bit-exact parity). The device helpers are compiled under
// their own namespace name so the two builds never share a definition.
#define pgd pgd_mixed
#define PGD_POW ::pow
#define PGD_EXP ::exp
#define PGD_LOG ::log
#include "engine_impl.cuh"

#define PGK_NS pgkmx
#define PGK_MIXED 1
#include "kernels.cuh"
