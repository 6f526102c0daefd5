// engine_impl.cuh -- engine state shared by the FP64 and mixed-precision
// translation units: the geometry every kernel receives (Dims), pool jobs and
// the engine handle behind the C ABI.
#ifndef PANGU_ENGINE_IMPL_CUH
#define PANGU_ENGINE_IMPL_CUH
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "pangu_b200.h"
#include "pangu_device.cuh"


namespace pgh {
struct Layout {
  int N[3], st[3], nx[3], act[3], nb[3], NB, ng, NF;
  double dx[3];
  std::vector<double> origin;
};
Layout make_layout(const pangu_params &p, const pangu_mesh &m);
void build_tables(const pangu_params &p, const Layout &L, std::vector<double> &t1,
                  std::vector<double> &t2);
void build_exchange(const pangu_mesh &m, const Layout &L, std::vector<int64_t> &dst,
                    std::vector<int64_t> &src);
void shard_exchange(const std::vector<int64_t> &dst, const std::vector<int64_t> &src,
                    int64_t ncell, const int32_t *block_rank, int nranks, int rank,
                    std::vector<int64_t> &ldst, std::vector<int64_t> &lsrc,
                    std::vector<std::vector<int64_t>> &send,
                    std::vector<std::vector<int64_t>> &recv);
}  // namespace pgh

// ---------------------------------------------------------------------------
// geometry passed to every kernel by value
// ---------------------------------------------------------------------------
struct Dims {
  int N1, N2, N3, NF, NB;
  int is, ie, js, je, ks, ke;
  int o1, o2, o3, ndim;
  long long ncell;  // N1 * N2 * N3
  int pidx[pgd::NPRIM];  // pack index of each slot, -1 if absent
  double dx[3];          // cell widths where bdx is null (handle-free dt estimate)
  // Block table. The launch domain is NB active blocks; active block bb lives
  // in pool slot slot[bb] (identity when null). Arrays below marked [slot]
  // are indexed by pool slot.
  const int *slot;          // [NB]
  const int *slot_job;      // [slot] owning job id (job 0 when null)
  const double *bdx;        // [slot][3] cell widths of the owning job's mesh
  const signed char *bcf;   // [slot][6] PANGU_BC_OUTFLOW/REFLECTING per face, -1 none
  const double *t1;      // [slot][10][N1 + 1]
  const double *t2;      // [slot][12][N2 + 1]
  const double *origin;  // [slot][3]
  // Static MKS/BL metric tables (built once per engine by k_build_tables):
  // component planes of [NB][comp][N2][N1] (centres), [NB][comp][N2][N1+1]
  // (x1 faces) and [NB][comp][N2+1][N1] (x2 faces); x3 faces use the centres.
  const double *ctab, *f1tab, *f2tab;
  // Mixed form only: the centre table's Christoffel planes rounded once to
  // FP32, [slot][nconn][N2][N1], read by the FP32 source term; null otherwise.
  const float *ctab32;
  // Mixed form only: the x1- and x2-face tables rounded once to FP32 (the
  // FP32 face fluxes read these); null otherwise.
  const float *f1tab32, *f2tab32;
  // Layout of the launch's arrays: when the pack they come from gives
  // per-(block, component) pointer tables (pangu_pack *_vars), the table of
  // each role; null for the contiguous layout [slot][component][N3][N2][N1].
  // Roles: prim; cons written (or read) by the task; cons read as the RK
  // starting state; the launch's flux array; the three flux arrays; alfven;
  // efield; flag.
  void *const *tP;
  double *const *tU, *const *tUi, *const *tF, *const *tF1, *const *tF2, *const *tF3;
  double *const *tA, *const *tE, *const *tG;
};

// Tile shape code of the flux kernels whose primitives are staged into
// shared memory by TMA (x1 rows; x2/x3 tiles of 32 x 4 faces); the other
// codes are march depths 1, 2, 4 and 0 for tiles loaded by the threads.
constexpr int kMarchTma = 8;

// A job: one mesh of equal meshblocks, placed in pool slots.
struct PoolJob {
  bool live = false;
  pangu_mesh m{};
  pangu_params p{};                 // the pool's params with the job's metric a, h
  std::vector<int> slots;           // slot of the job's block b (lattice order)
  std::vector<int64_t> xdst, xsrc;  // exchange map in slot cell offsets
  bool any_bc = false;              // some face is outflow / reflecting
};

struct pangu_engine {
  pangu_params p;
  pangu_mesh m;  // block shape (nx, ng); for a single-mesh engine the whole mesh
  Dims d{};      // d.NB = active blocks; d.slot = d_active
  int capacity = 0, max_jobs = 0;
  std::vector<PoolJob> jobs;
  std::vector<char> slot_used;
  int njobs_active = 0;
  bool any_bc = false;
  std::vector<long long> xoff;  // per job id: offset of its entries in the exchange map
  int *d_active = nullptr;      // [capacity] active block -> slot
  int *d_slot_job = nullptr;    // [capacity]
  int *d_jr = nullptr;          // [max_jobs][3] job id, first and end active block
  double *d_bdx = nullptr;      // [capacity][3]
  signed char *d_bcf = nullptr; // [capacity][6]
  double *d_t1 = nullptr, *d_t2 = nullptr, *d_origin = nullptr;
  double *d_ctab = nullptr, *d_f1tab = nullptr, *d_f2tab = nullptr;
  float *d_ctab32 = nullptr;  // mixed form: FP32 Christoffel planes
  float *d_f1tab32 = nullptr, *d_f2tab32 = nullptr;  // mixed form: FP32 face tables
  long long *d_xdst = nullptr, *d_xsrc = nullptr;  // [capacity x ghost cells per block]
  long long nxch = 0, xch_cap = 0;
  int *d_tmp_slots = nullptr;  // [capacity] slots of a job being attached
  unsigned long long *d_genred = nullptr;  // [3] maxima of the device generators
  unsigned long long *d_cnt = nullptr;  // [max_jobs][PANGU_NCOUNTERS]
  int *d_fail_count = nullptr;      // C2P retry list (Scheme2D failures)
  long long *d_fail_list = nullptr;
  int *d_fix_count = nullptr;       // FixRecovery list (cells the chain left failed)
  long long *d_fix_list = nullptr;
  double *d_fail_vals = nullptr;
  long long fail_cap = 0;
  int *d_err = nullptr;  // set by a kernel whose bounded wait gave up (0 otherwise)
  unsigned long long *d_dtmin = nullptr;  // [capacity][3]
  unsigned int *d_dt_ticket = nullptr;    // CTAs done in the current dt reduction
  long long launches = 0;  // kernels launched through this handle
  // Block sharding (one mesh over several GPUs): this engine holds the blocks
  // of `rank`; ghost cells whose source block is on another rank travel as
  // halo messages, per peer in rank order, each entry Nf primitives + flag.
  int nranks = 1, rank = 0;
  std::vector<long long> hsend_off, hrecv_off;       // [nranks + 1] entry offsets
  long long *d_hsend = nullptr, *d_hrecv = nullptr;  // slot cell offsets
  // Tile shapes of the flux kernels per direction: march depth (x2/x3) and
  // CTA size; set by pangu_autotune.
  struct {
    int march[3] = {1, 2, 2};
    int threads[3] = {128, 128, 128};
    int tuned = 0;
  } tune;
};

#endif  // PANGU_ENGINE_IMPL_CUH
