// engine_tables.cu -- the FP64 kernels for packs that give arrays through
// per-(block, component) pointer tables (namespace pgk64t): the layout of a
// Parthenon pack of per-block, per-variable views. Same kernels and flags as
// engine.cu (bit-identical results); only the address of a component
// differs, so that the contiguous kernels carry no table test.
#define pgd pgd_tables
#include "engine_impl.cuh"

#define PGK_NS pgk64t
#define PGK_MIXED 0
#define PGK_TABLES 1
#include "kernels.cuh"
