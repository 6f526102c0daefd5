// engine_mixed_tables.cu -- the mixed-precision kernels of engine_mixed.cu
// for packs that give arrays through per-(block, component) pointer tables
// (namespace pgkmxt). Same kernels and flags as engine_mixed.cu.
#define pgd pgd_mixed_tables
#define PGD_POW ::pow
#define PGD_EXP ::exp
#define PGD_LOG ::log
#include "engine_impl.cuh"

#define PGK_NS pgkmxt
#define PGK_MIXED 1
#define PGK_TABLES 1
#include "kernels.cuh"
