/*
 * pangu_b200.h -- C ABI of the B200 GRMHD stage engine.
 *
 * The engine replaces the per-RK-stage task functions of PANGU's ideal GRMHD
 * task graph (pangu/src/task_list/ideal_grmhd.cc:62-94 registers them):
 *
 *   FixPrimitive            pangu/src/fixer/primitive_fixer.h:12
 *   CalculateConservative   pangu/src/riemann_solver/conservative.h:12
 *   CalculateFluxes         pangu/src/riemann_solver/riemann_solver.h (LAXF/HLL)
 *   ConstraintedTransport   pangu/src/constrained_transport/constrained_transport.h
 *   FluxDivergence + UpdateIndependentData (Parthenon, ideal_grmhd.cc:73-76)
 *   AddGeometricSource      pangu/src/riemann_solver/source_term.h
 *   Recovery                pangu/src/recovery/invertor.h:11
 *   ApplyElectronHeating    pangu/src/riemann_solver/electron_heating.h:12
 *   FixRecovery             pangu/src/fixer/recovery_fixer.h:12
 *   EstimateTimestepMesh    pangu/src/initialization/timestep_estimation.h:10-11
 *
 * Every entry point is extern "C", never throws and never traps. It returns
 * PANGU_OK (0) or a negative PANGU_E* code. Field arrays are caller-owned device memory laid
 * out like a Parthenon MeshBlockPack with Kokkos LayoutRight:
 *   [block][variable][k][j][i]  (i fastest), over the "entire" index domain
 *   (interior plus ng ghost cells on each side of every active direction),
 * or, array by array, one allocation per (block, component) reached through
 * a pointer table (pangu_pack), as Parthenon keeps its variables.
 * The engine keeps no pointer to them past the call.
 *
 * Variable order inside prim/cons is the order of
 * package_registration.cc:84-96:
 *   density, energy, weighted_velocity[3], magnetic_field[3] (if enable_B),
 *   entropy, electron_entropy (if enable_heating).
 */
#ifndef PANGU_B200_H
#define PANGU_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PANGU_OK 0
#define PANGU_EINVAL (-1)     /* bad argument (null pointer, bad option)      */
#define PANGU_ECUDA (-2)      /* a CUDA runtime call failed                    */
#define PANGU_ENOMEM (-3)     /* engine-internal allocation failed             */
#define PANGU_ENGHOST (-4)    /* ghost width too small for the limiter         */
#define PANGU_ETOOBIG (-5)    /* size above a documented maximum               */
#define PANGU_EFULL (-6)      /* pool has no free slot or job id               */

/* ---- option enumerations (string values of the reference's params) ---- */
#define PANGU_RIEMANN_LAXF 0  /* <core>/riemann_solver = laxf */
#define PANGU_RIEMANN_HLL 1   /* <core>/riemann_solver = hll  */
#define PANGU_LIMITER_PPM4 0  /* <core>/limiter = ppm4 */
#define PANGU_LIMITER_MC 1    /* <core>/limiter = mc   */
#define PANGU_RECOVERY_CHAINER 0  /* <core>/recovery = chainer  */
#define PANGU_RECOVERY_ROBUSTER 1 /* <core>/recovery = robuster */
/* <metric>/type, christoffel.h:145-147 */
#define PANGU_METRIC_MINKOWSKI 0
#define PANGU_METRIC_BL 1
#define PANGU_METRIC_CKS 2
#define PANGU_METRIC_MKS 3
/* <electron>/model, heating_model.h:13-20 */
#define PANGU_HEAT_CONSTANT 0
#define PANGU_HEAT_HOWES 1
#define PANGU_HEAT_KAWAZURA 2
#define PANGU_HEAT_WERNER 3
#define PANGU_HEAT_ROWAN 4
#define PANGU_HEAT_SHARMA 5
/* Arithmetic of the engine (no reference counterpart; the reference is
 * FP64 throughout). MIXED stores primitives in FP32 (the pack's prim pointer
 * then addresses floats) and runs reconstruction, Riemann flux, the floors of
 * FixPrimitive, electron heating and the geometric source term (MKS/BL) in
 * FP32; conserved variables
 * and their update, C2P, the metric and CT stay FP64. The conserved magnetic field is then evolved only
 * by the FP64 CT update: CalculateConservative leaves it unchanged, and
 * pangu_job_start computes it once from the initial primitives. */
#define PANGU_PRECISION_FP64 0
#define PANGU_PRECISION_MIXED 1
/* Parthenon <parthenon/mesh> ix*_bc / ox*_bc */
#define PANGU_BC_PERIODIC 0
#define PANGU_BC_OUTFLOW 1
#define PANGU_BC_REFLECTING 2

/* Runtime parameters of the "core" and "metric" packages, with the meaning
 * and defaults of package_registration.cc:21-81 and :158-173. */
typedef struct pangu_params {
  /* <core> */
  double cfl_number;          /* 0.8 */
  double adiabatic_index;     /* 5/3 */
  int32_t riemann_solver;     /* PANGU_RIEMANN_* (laxf) */
  int32_t limiter;            /* PANGU_LIMITER_* (ppm4) */
  double density_floor;       /* 1e-6 */
  double energy_floor;        /* 1e-8 */
  double density_floor_pow;   /* -1.5 */
  double energy_floor_pow;    /* -2.5 */
  int32_t enable_B;           /* false */
  int32_t recovery;           /* PANGU_RECOVERY_* (chainer) */
  int32_t enable_heating;     /* false */
  int32_t precision;          /* PANGU_PRECISION_* (fp64); not a reference key */
  double sigma_max;           /* 50 */
  double lorentz_max;         /* 50 */
  /* <electron> */
  int32_t model;              /* PANGU_HEAT_* (constant) */
  int32_t limit_kel;          /* true */
  int32_t suppress_highb_heat;          /* false */
  int32_t enforce_positive_dissipation; /* false */
  double fel_constant;        /* 0.1 */
  double gamma_e;             /* 4/3 */
  double gamma_p;             /* 5/3 */
  double ratio_min;           /* 1e-3 */
  double ratio_max;           /* 1e3 */
  double fel_0;               /* 0.1 */
  /* <metric> */
  int32_t metric_type;        /* PANGU_METRIC_* (minkowski) */
  int32_t excise;             /* false */
  double a;                   /* 0 */
  double h;                   /* 0 */
  double r_excise;            /* 1 */
  double dexcise;             /* 1e-8 */
  double pexcise;             /* 0.333e-12 */
} pangu_params;

/* A uniform mesh cut into a regular lattice of equal meshblocks
 * (<parthenon/mesh> and <parthenon/meshblock>; refinement = none).
 * Block b sits at lattice position (b1, b2, b3) with
 * b = (b3 * nbx2 + b2) * nbx1 + b1. */
typedef struct pangu_mesh {
  int32_t nx1, nx2, nx3;      /* interior cells per meshblock */
  int32_t nbx1, nbx2, nbx3;   /* meshblocks along each direction */
  int32_t ng;                 /* ghost width of every active direction */
  int32_t reserved0;
  double x1min, x1max, x2min, x2max, x3min, x3max;
  int32_t bc[6];              /* ix1, ox1, ix2, ox2, ix3, ox3: PANGU_BC_* */
} pangu_mesh;

/* One stage container ("base" or "1") of every block, as device pointers.
 * Shapes use N1 = nx1 + 2 ng (or 1), N2, N3 likewise, NF = number of
 * prim/cons components, NB = number of blocks.
 * alfven, efield and flag are Metadata::OneCopy fields in the reference
 * (package_registration.cc:121-145): both containers point at the same
 * arrays. */
typedef struct pangu_pack {
  double *prim;    /* [NB][NF][N3][N2][N1] */
  double *cons;    /* [NB][NF][N3][N2][N1] */
  double *flux1;   /* [NB][NF][N3][N2][N1]; entry i is the face below cell i */
  double *flux2;   /* [NB][NF][N3][N2][N1]; entry j is the face below cell j */
  double *flux3;   /* [NB][NF][N3][N2][N1]; entry k is the face below cell k */
  double *alfven;  /* [NB][3][N3][N2][N1] */
  double *efield;  /* [NB][3][N3][N2][N1] */
  double *flag;    /* [NB][N3][N2][N1]; chainer only (may be NULL otherwise) */
  /* Per-(block, component) layout, the form of a Parthenon pack of
   * per-block, per-variable views (md->PackVariables, laxf.cc:37-53): a
   * non-NULL table replaces the contiguous layout of its array above (whose
   * pointer may then be NULL). Entry b * NC + c of a table is the device
   * address of component c of block b, an [N3][N2][N1] array with i fastest;
   * NC = NF for prim, cons and the fluxes, 3 for alfven and efield, 1 for
   * flag. Each table is a device array of NB * NC addresses (NB: the engine's
   * blocks, or the pool's capacity), each of an array of N3 * N2 * N1
   * elements, that must stay valid while the call's work runs (and for the
   * replays of a CUDA graph that captured it); the engine cannot check either
   * on the host. Packs with tables run separately compiled instances of the
   * kernels, so the contiguous layout pays nothing for them; FP64 results are
   * bit-identical to the contiguous layout's, mixed-precision ones agree to
   * rounding (that form is compiled with FMA contraction, whose choices may
   * differ between the two instances). The
   * per-task and stage entry points accept tables; pangu_job_start,
   * pangu_generate, the block pool and the serving loop take the contiguous
   * layout only (PANGU_EINVAL otherwise), and the TMA-staged flux kernels are
   * replaced by their thread-loaded forms for primitives given by a table.
   * A zero-initialised pack has no tables. */
  double *const *prim_vars;
  double *const *cons_vars;
  double *const *flux1_vars;
  double *const *flux2_vars;
  double *const *flux3_vars;
  double *const *alfven_vars;
  double *const *efield_vars;
  double *const *flag_vars;
} pangu_pack;

/* Hit counters of the floors and fixers (not present in the reference, which
 * has no counters; they are what makes "same floor and fixer hit counts"
 * checkable). Indices into a uint64_t[PANGU_NCOUNTERS] array. */
#define PANGU_CNT_RHO_FLOOR 0    /* FixPrimitive: density raised to the floor  */
#define PANGU_CNT_ENG_FLOOR 1    /* FixPrimitive: energy raised to the floor   */
#define PANGU_CNT_LORENTZ_CAP 2  /* FixPrimitive: velocity rescaled            */
#define PANGU_CNT_C2P_2D 3       /* Recovery: Scheme2D succeeded               */
#define PANGU_CNT_C2P_1DVSQ 4    /* Recovery: Scheme1Dvsq succeeded            */
#define PANGU_CNT_C2P_1D 5       /* Recovery: Scheme1D succeeded               */
#define PANGU_CNT_C2P_FAIL 6     /* Recovery: all three failed (flag = 0)      */
#define PANGU_CNT_FIXRECOVERY 7  /* FixRecovery: cells repaired                */
#define PANGU_CNT_KASTAUN_FAIL 8 /* Recovery (robuster): root solve failed     */
#define PANGU_CNT_EXCISED 9      /* Recovery: CKS cells inside r_excise        */
#define PANGU_NCOUNTERS 16

/* Opaque engine handle: validated parameters, mesh geometry and the device
 * tables derived from them (block origins, ghost-exchange map). */
typedef struct pangu_engine pangu_engine;

/* Number of prim/cons components for a parameter set
 * (package_registration.cc:92-96). */
int pangu_num_fields(const pangu_params *params);

/* Validates params/mesh and builds the engine on the current CUDA device.
 * Returns PANGU_ENGHOST when limiter = ppm4 and ng < 3 (PPM4 reads i-3,
 * interpolater_ppm4.h:29-67 via laxf.cc:96-101) or limiter = mc and ng < 2. */
int pangu_engine_create(const pangu_params *params, const pangu_mesh *mesh,
                        pangu_engine **out);
int pangu_engine_destroy(pangu_engine *engine);

/* ---- per-task entry points (one per reference task) ------------------- */
/* stream is a cudaStream_t passed as void*; NULL = legacy default stream. */
int pangu_fix_primitive(pangu_engine *e, const pangu_pack *md, void *stream);
int pangu_calculate_conservative(pangu_engine *e, const pangu_pack *md,
                                 void *stream);
int pangu_calculate_fluxes(pangu_engine *e, const pangu_pack *md, void *stream);
int pangu_constrained_transport(pangu_engine *e, const pangu_pack *md,
                                void *stream);
/* mc1.cons = mc_init.cons - (beta*dt) * div(mc0 fluxes) over the interior
 * (Parthenon FluxDivergence + UpdateIndependentData, ideal_grmhd.cc:73-76).
 * dt is a DEVICE pointer so a captured graph stays valid: dt[job] per job
 * (dt[0] for an engine made by pangu_engine_create). */
int pangu_flux_divergence_update(pangu_engine *e, const pangu_pack *mc_init,
                                 const pangu_pack *mc0, const pangu_pack *mc1,
                                 double beta, const double *dt, void *stream);
/* Ghost exchange of a container at send time: periodic and block-to-block
 * ghost cells of prim and flag receive the neighbour's interior values. */
int pangu_exchange_ghosts(pangu_engine *e, const pangu_pack *md, void *stream);
int pangu_add_geometric_source(pangu_engine *e, const pangu_pack *md,
                               double beta, const double *dt, void *stream);
int pangu_recovery(pangu_engine *e, const pangu_pack *md, void *stream);
int pangu_apply_electron_heating(pangu_engine *e, const pangu_pack *md,
                                 void *stream);
int pangu_fix_recovery(pangu_engine *e, const pangu_pack *md, void *stream);
/* Physical boundary conditions (outflow / reflecting) on prim and flag, in
 * the face order inner x1, outer x1, inner x2, outer x2, inner x3, outer x3. */
int pangu_apply_boundary_conditions(pangu_engine *e, const pangu_pack *md,
                                    void *stream);
/* dt estimate from the alfven field (timestep_estimation.cc:13-102),
 * written to the DEVICE array dt_out[job] of every active job. */
int pangu_estimate_dt(pangu_engine *e, const pangu_pack *md, double *dt_out,
                      void *stream);

/* ---- whole stage ------------------------------------------------------- */
/* One RK stage of Simulator::MakeTaskCollection (ideal_grmhd.cc:23-120):
 * stage = 1 or 2 of rk2, beta = integrator->beta[stage % 2],
 * mc0 = stage_name[stage-1], mc1 = stage_name[stage], mc_init = "base".
 * On the last stage the new dt estimate is written to dt_est (device). */
int pangu_stage(pangu_engine *e, int stage, const pangu_pack *base,
                const pangu_pack *one, double beta, const double *dt,
                double *dt_est, void *stream);

/* ---- one mesh over several GPUs (block sharding) ----------------------- */
/* The reference spreads a mesh's blocks over MPI ranks through Parthenon
 * (ghost exchange at ideal_grmhd.cc:78, dt reduction in
 * EstimateTimestepMesh, timestep_estimation.cc:13-102). Here rank r's
 * engine holds the blocks b with block_rank[b] == r (lattice order, x1
 * fastest). Ghost cells whose source block is on another rank travel as
 * halo messages: per peer rank q, a contiguous run of entries, each the
 * Nf primitives and the flag of one cell as FP64 (Nf + 1 doubles); the
 * k-th entry rank r sends to q is the k-th entry q receives from r. A send
 * (receive) buffer holds the messages of all peers in rank order.
 * Every stage of a shard is three calls around the message transfer:
 *   pangu_stage_begin   FixPrimitive ... update, local ghost exchange, and
 *                       the halo cells packed into `send`;
 *   (the caller moves each peer's message, e.g. NCCL send/recv)
 *   pangu_stage_middle  AddGeometricSource, Recovery, ApplyElectronHeating
 *                       (these read no ghost cell: they overlap the transfer);
 *   pangu_stage_end     the received halo cells unpacked from `recv`,
 *                       FixRecovery, physical BCs, and on stage 2 this
 *                       shard's dt estimate, which the caller reduces (min)
 *                       over the ranks before pangu_update_dt.
 * On an engine without halo entries the three calls equal pangu_stage, and
 * send / recv may be NULL; pangu_stage returns PANGU_EINVAL on a shard that
 * has halo entries. */
int pangu_shard_create(const pangu_params *params, const pangu_mesh *mesh,
                       const int32_t *block_rank, int32_t nranks, int32_t rank,
                       pangu_engine **out);
/* The halo plan of rank `rank` without a GPU: entries per peer
 * (send_counts[nranks], recv_counts[nranks]) and, when the cell arrays are
 * non-NULL, the cells in message order as offsets b * ncell + cell of the
 * whole mesh's block b (ncell = cells of one block with ghosts). */
int pangu_shard_plan(const pangu_params *params, const pangu_mesh *mesh,
                     const int32_t *block_rank, int32_t nranks, int32_t rank,
                     int64_t *send_counts, int64_t *recv_counts,
                     int64_t *send_cells, int64_t *recv_cells);
/* Entries per peer of this shard's messages ([nranks] each). */
int pangu_halo_counts(const pangu_engine *e, int64_t *send_counts,
                      int64_t *recv_counts);
/* Pack the halo cells of md into send / unpack recv into md's ghosts (the
 * initial ghost fill of a shard: pack base, transfer, unpack base, then
 * pangu_job_start, which adds the local exchange and the physical BCs). */
int pangu_halo_pack(pangu_engine *e, const pangu_pack *md, double *send,
                    void *stream);
int pangu_halo_unpack(pangu_engine *e, const pangu_pack *md,
                      const double *recv, void *stream);
int pangu_stage_begin(pangu_engine *e, int stage, const pangu_pack *base,
                      const pangu_pack *one, double beta, const double *dt,
                      double *send, void *stream);
/* The first part without its exchange: FixPrimitive + CalculateConservative,
 * fluxes, CT and the update, which read only mc0 and "base" and write mc1's
 * conserved variables. pangu_stage_update then pangu_exchange_ghosts (mc1)
 * equals pangu_stage_begin on an engine without halo entries; a caller that
 * uploads mc1's primitives and the flags can let that copy run meanwhile. */
int pangu_stage_update(pangu_engine *e, int stage, const pangu_pack *base,
                       const pangu_pack *one, double beta, const double *dt,
                       void *stream);
int pangu_stage_middle(pangu_engine *e, int stage, const pangu_pack *base,
                       const pangu_pack *one, double beta, const double *dt,
                       void *stream);
int pangu_stage_end(pangu_engine *e, int stage, const pangu_pack *base,
                    const pangu_pack *one, const double *recv,
                    double *dt_est, void *stream);

/* The dt estimate of pangu_estimate_dt without an engine handle and without
 * allocating: for callers that may not call cudaMalloc (their device memory
 * belongs to a pool or a fixed budget, so they cannot create an engine, which
 * allocates). No counterpart in the reference. Arguments: the engine's params
 * and mesh structs, the caller's alfven array ([NB][3][N3][N2][N1], device)
 * and a device double for the result. Scratch lives in a file-scope device
 * array of 3 x 4096 minima (96 KiB on every GPU that loads the library, held
 * until exit): meshes with more than 4096 blocks get PANGU_ETOOBIG. The first
 * call on a device looks the array's address up (cudaGetSymbolAddress) with
 * that device current and keeps it for the life of the process; make that
 * first call before any stream capture, and do not reset the device or its
 * primary context (cudaDeviceReset) between calls, which would leave the
 * kept address stale. Calls on the same device share the array: calls whose
 * execution overlaps (e.g. on different streams) race, so serialise them.
 * Calls on different devices are independent (each GPU holds its own copy). */
int pangu_estimate_dt_noalloc(const pangu_params *params, const pangu_mesh *mesh,
                              const double *alfven, double *dt_out, void *stream);

/* ---- measurement ------------------------------------------------------- */
/* FP64 fused multiply-add throughput of the current device (no counterpart
 * in the reference): launches `ctas` CTAs of 256 threads, each thread running
 * eight independent DFMA chains of `iters` steps; the caller times the launch
 * with CUDA events on `stream` and divides pangu_fp64_peak_flops(ctas, iters)
 * by its duration. sink: a device double[ctas] that is never written in
 * practice. This is the FP64 roofline's denominator: the stage kernels are
 * bound by FP64 issue and latency, not by HBM bandwidth. */
int pangu_fp64_peak(int ctas, int iters, double *sink, void *stream);
double pangu_fp64_peak_flops(int ctas, int iters);

/* Device dt policy applied after each cycle, per active job:
 * dt[job] = min(dt_factor*dt[job], dt_est[job]). */
int pangu_update_dt(pangu_engine *e, double *dt, const double *dt_est,
                    double dt_factor, void *stream);

/* Counters accumulated since the last reset, summed over jobs (host copy,
 * synchronous). */
int pangu_counters(pangu_engine *e, uint64_t out[PANGU_NCOUNTERS]);
int pangu_reset_counters(pangu_engine *e, void *stream);

/* Number of CUDA kernels this handle has launched so far (host-side count). */
long long pangu_launches(const pangu_engine *e);

/* 1 if a kernel of this handle gave up a bounded wait (the TMA-staged flux
 * kernels wait on an mbarrier for their copy, with a limit far beyond any
 * copy's completion) and returned without its results, else 0 (host copy,
 * synchronous). No counterpart in the reference. */
int pangu_device_error(const pangu_engine *e, int32_t *flag_out);

/* Autotuner of the flux kernels' tile shapes (no counterpart in the
 * reference): times each candidate shape of every direction -- CTA size 64
 * or 128, and for x2/x3 a march depth of 1, 2 or 4 faces per thread or a
 * shared-memory tile of 32 x 4 or 32 x 8 faces, and for every direction the
 * form whose primitives one TMA copy per CTA stages into shared memory where
 * the rows are whole 16-byte units -- on
 * the pack's own data and keeps the fastest for this engine. Every candidate
 * computes each face identically, so results never depend on the choice.
 * Overwrites the pack's fluxes and alfven (which every stage recomputes
 * before reading them), synchronises the stream, and must not be called
 * during stream capture. */
int pangu_autotune(pangu_engine *e, const pangu_pack *md, void *stream);
/* Current tile shapes: {march1, threads1, march2, threads2, march3,
 * threads3, tuned}. */
int pangu_flux_config(const pangu_engine *e, int32_t out[7]);
/* Sets the tile shapes {march1, threads1, march2, threads2, march3,
 * threads3}: march 1, 2 or 4 (x1: 1) with threads 64 or 128, or for x2 and x3
 * march 0 (tiles of 32 x threads/32 faces, each cell reconstructed once) with
 * threads 128 or 256, or march 8 with threads 128 (TMA-staged: x1 rows of 4 x
 * 31 faces, x2/x3 tiles of 32 x 4 faces; the rows of the primitives must be
 * whole 16-byte units), PANGU_EINVAL otherwise, e.g. to repeat a configuration
 * the autotuner chose elsewhere. */
int pangu_set_flux_config(pangu_engine *e, const int32_t cfg[6]);

/* ---- block pool: many jobs stepped by the same launches ---------------- */
/* No counterpart in the reference, which runs one mesh per process. A pool
 * engine owns a block table over `capacity_blocks` slots of the block shape
 * in `block` (nx1..nx3, ng; its other fields are ignored). Jobs -- meshes of
 * such blocks with their own lattice, extents, BCs and metric spin a and h --
 * are attached into free slots and detached when done; every task and
 * pangu_stage call then processes all attached jobs' blocks in one launch per
 * kernel, reading dt[job] and writing dt_est[job]. The caller owns the
 * containers: packs sized for `capacity_blocks` blocks, slot-major. Results
 * are identical to running each job alone with pangu_engine_create.
 * attach/detach need no work of this engine in flight (they rewrite the
 * block table with blocking copies on the legacy default stream, and never
 * synchronise the device or allocate); they change the launch domain, so a
 * CUDA graph captured before them must be captured again. */
int pangu_pool_create(const pangu_params *params, const pangu_mesh *block,
                      int32_t capacity_blocks, int32_t max_jobs, pangu_engine **out);
/* Places a job (mesh: the pool's nx and ng, any nbx/extents/bc) in free slots
 * (lowest first). slots_out[b] receives the slot of the job's block b (lattice
 * order, x1 fastest); job_out its id, which indexes dt/dt_est.
 * PANGU_EFULL when no id or too few slots are free. */
int pangu_job_attach(pangu_engine *e, const pangu_mesh *mesh, double a, double h,
                     int32_t *job_out, int32_t *slots_out);
/* After the caller wrote a job's interior primitives into its slots of base:
 * fills its ghosts (exchange, then physical BCs) and copies base into one for
 * its slots, as Parthenon does after the problem generator. With
 * pangu_engine_create the mesh is job 0. */
int pangu_job_start(pangu_engine *e, int32_t job, const pangu_pack *base,
                    const pangu_pack *one, void *stream);
int pangu_job_detach(pangu_engine *e, int32_t job);
/* Counters of one job since its attach (host copy, synchronous). */
int pangu_job_counters(pangu_engine *e, int32_t job, uint64_t out[PANGU_NCOUNTERS]);
/* Blocks in the launch domain (all attached jobs). */
int pangu_active_blocks(const pangu_engine *e);

/* ---- device-side initial conditions ------------------------------------ */
/* The benchmark problems' initial primitives, generated on the device into
 * a job's blocks of base (every cell; then call pangu_job_start). Same
 * formulas as the host generators of pangu_b200/problems.py: Orszag-Tang,
 * Brio-Wu, and the Fishbone-Moncrief torus of
 * fm_torus_mks/problem_generator.cpp:103-558 (MKS only; the job's metric a
 * and h), with its MeshPostInitialization (density normalisation, SANE A_phi,
 * field normalised to the target beta) computed by device reductions and a
 * counter-based random perturbation (SplitMix64 of seed and cell index).
 * Synchronises the stream for a torus and returns PANGU_EINVAL when its
 * parameters admit no bound torus. */
#define PANGU_PROBLEM_ORSZAG_TANG 0
#define PANGU_PROBLEM_BRIO_WU 1
#define PANGU_PROBLEM_FM_TORUS 2
typedef struct pangu_problem {
  int32_t kind;               /* PANGU_PROBLEM_* */
  int32_t seed;               /* <fm_torus>/seed */
  double rin, rmax, kappa, perturbation, beta, aphi_rho_cut;  /* <fm_torus> */
} pangu_problem;
int pangu_generate(pangu_engine *e, int32_t job, const pangu_problem *problem,
                   const pangu_pack *base, void *stream);

/* ---- serving: continuous batching over block pools --------------------- */
/* No counterpart in the reference. A server owns one block pool per job
 * class (parameter set + block shape), each with its containers, dt arrays,
 * stream and captured RK2-cycle graph, charged against an HBM budget (the
 * containers as allocated, the pool engine by the device memory its creation
 * takes): when the class is added (pangu_server_add_class), or, for a class
 * declared with pangu_server_declare_class, when the run admits the first job
 * that needs it; such a class is released again whenever none of its jobs is
 * running or has arrived and waits. pangu_server_run admits every submitted job once its
 * arrival time (seconds after the run starts) has passed and its class pool
 * has room (first fit in arrival order), steps the admitted jobs of each
 * class one RK2 cycle per tick of that class (classes tick independently on
 * their own streams, so their kernels overlap), copies each job's primitives
 * back and detaches it after its last cycle. A job's result is identical to
 * running it alone. */
typedef struct pangu_server pangu_server;
typedef struct pangu_server_stats {
  int64_t jobs, ticks;      /* completed jobs; class ticks                   */
  double wall_s;             /* host time of the whole run                   */
  double zone_cycles;        /* interior cells x cycles, summed over jobs    */
  double zone_cycles_per_s;  /* zone_cycles / wall_s                         */
  double p50_s, p99_s;       /* job latency (completion - arrival)           */
  uint64_t hbm_bytes;        /* device memory the classes hold after the run */
  uint64_t hbm_peak_bytes;   /* the most they held at once during the run    */
  int64_t memory_waits;      /* jobs that waited because their class's
                                memory did not fit in the budget yet          */
} pangu_server_stats;
int pangu_server_create(uint64_t hbm_budget_bytes, pangu_server **out);
int pangu_server_destroy(pangu_server *s);
/* PANGU_ENOMEM when the class's memory does not fit in the remaining budget. */
int pangu_server_add_class(pangu_server *s, const pangu_params *params,
                           const pangu_mesh *block, int32_t capacity_blocks,
                           int32_t max_jobs, double dt_factor, int32_t *class_out);
/* A class whose memory is charged only when pangu_server_run admits its first
 * job, and released while none of its jobs runs or waits: jobs of classes
 * that do not fit in the budget together take turns. pangu_server_run returns
 * PANGU_ENOMEM if an arrived job's class cannot fit even with nothing else
 * running. */
int pangu_server_declare_class(pangu_server *s, const pangu_params *params,
                               const pangu_mesh *block, int32_t capacity_blocks,
                               int32_t max_jobs, double dt_factor, int32_t *class_out);
/* prim_host: the job's initial primitives, FP64 [block][var][k][j][i] over
 * every cell of each block (ghosts are filled at admission). Copied. */
int pangu_server_submit(pangu_server *s, int32_t cls, const pangu_mesh *mesh,
                        double a, double h, double dt_init, int64_t cycles,
                        double arrival_s, const double *prim_host, int32_t *ticket_out);
/* A job whose initial state is generated on the device at admission
 * (pangu_generate) instead of uploaded. */
int pangu_server_submit_problem(pangu_server *s, int32_t cls, const pangu_mesh *mesh,
                                double a, double h, double dt_init, int64_t cycles,
                                double arrival_s, const pangu_problem *problem,
                                int32_t *ticket_out);
/* Runs until every submitted job is done. Blocks the calling thread. */
int pangu_server_run(pangu_server *s);
/* A finished job: primitives (FP64, layout of submit), times {arrival,
 * admission, completion} in seconds, and its counters. Any pointer may be
 * NULL. */
int pangu_server_result(pangu_server *s, int32_t ticket, double *prim_out,
                        double *times_out, uint64_t counters_out[PANGU_NCOUNTERS]);
int pangu_server_get_stats(const pangu_server *s, pangu_server_stats *out);
/* Cancels a job at at_s seconds after the start of the next run: a job still
 * waiting is dropped; a running one is detached at its class's next tick
 * boundary, with no result. Stats count completed jobs only. */
int pangu_server_cancel(pangu_server *s, int32_t ticket, double at_s);
/* 0 waiting, 1 running, 2 done, 3 cancelled (or a negative error). */
int pangu_server_job_state(const pangu_server *s, int32_t ticket);

#ifdef __cplusplus
}
#endif
#endif /* PANGU_B200_H */
