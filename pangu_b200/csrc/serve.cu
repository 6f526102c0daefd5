// serve.cu -- continuous-batching request loop over block pools (host code).
//
// A server holds one block pool (pangu_pool_create) per job class -- one
// parameter set and block shape -- with its containers, dt arrays, CUDA
// stream and captured RK2-cycle graph, charged against the server's HBM
// budget: at class creation (pangu_server_add_class), or, for a class
// declared with pangu_server_declare_class, when the first job that needs it
// is admitted -- a job of a class whose memory does not fit in what is left of
// the budget waits until retiring jobs and released classes free enough --
// and released again when none of the class's jobs is running or waiting.
// Submitted jobs wait until their arrival
// time; a job is admitted as soon as its class pool has a free job id and
// enough free block slots (first fit in arrival order; of jobs that arrive
// together, the one with the most work first) and then runs one RK2
// cycle per tick of its class together with every other admitted job of the
// class (one graph launch per tick). Classes tick independently, each on its
// own stream, so their kernels overlap and a class of small jobs is not held
// to the pace of a class of large ones. A job is copied out and detached
// after its last cycle. Latency = completion - arrival, on the host clock.
//
// No counterpart in the reference, which runs one mesh per process.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "pangu_b200.h"

namespace {

struct Arena {
  pangu_pack base{}, one{};
  double *dt = nullptr, *dt_est = nullptr;
  std::vector<void *> allocs;
};

// Cycles a class keeps queued on its stream ahead of the host loop, so that
// the host's work for other classes (admission, retirement, graph capture)
// does not leave this class's stream idle. Never more than any of its
// running jobs still needs.
constexpr int kQueue = 4;

struct SClass {
  pangu_params p{};
  pangu_mesh block{};
  int capacity = 0, max_jobs = 0, nf = 0;
  long long ncell = 0, interior = 0;  // cells per block (entire, interior)
  size_t prim_bytes = 8;
  double dt_factor = 2.0;
  pangu_engine *e = nullptr;
  Arena a;
  cudaStream_t stream = nullptr;
  // one event per queued cycle, a ring of kQueue: ev[head] is the oldest
  cudaEvent_t ev[kQueue] = {};
  int queued = 0, head = 0;
  cudaGraphExec_t graph = nullptr;
  bool dirty = true, tuned = false;
  int running = 0;
  bool lazy = false;       // allocated at admission, released when idle
  bool allocated = false;  // engine, arena, stream and event exist
  uint64_t bytes = 0;      // device memory charged to the budget while allocated
  uint64_t need = 0;       // bytes an allocation of the class took (0: unknown)
};

struct SJob {
  int cls = 0;
  pangu_mesh mesh{};
  double a = 0, h = 0, dt_init = 0, arrival = 0;
  long long cycles = 0, done_cycles = 0;
  std::vector<double> prim;  // initial state (unless generated), then the result
  bool generated = false;    // initial state generated on the device
  pangu_problem problem{};
  int state = 0;             // 0 waiting, 1 running, 2 done, 3 cancelled
  double cancel_at = 1e300;  // seconds after the start of the run
  int job = -1;
  std::vector<int32_t> slots;
  double t_admit = 0, t_done = 0;
  bool waited_for_memory = false;  // its class's memory did not fit at some point
  uint64_t counters[PANGU_NCOUNTERS] = {};
};

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct pangu_server {
  uint64_t budget = 0, used = 0, peak = 0;
  std::vector<SClass> classes;
  std::vector<SJob> jobs;
  pangu_server_stats stats{};
};

namespace {

template <class T>
int salloc(pangu_server *s, SClass &c, T **p, size_t n) {
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  if (s->used + bytes > s->budget) return PANGU_ENOMEM;
  if (cudaMalloc((void **)p, bytes) != cudaSuccess) return PANGU_ENOMEM;
  c.a.allocs.push_back(*p);
  s->used += bytes;
  c.bytes += bytes;
  if (cudaMemset(*p, 0, bytes) != cudaSuccess) return PANGU_ECUDA;
  return PANGU_OK;
}

// Frees a class's device resources and returns its bytes to the budget; the
// class keeps its parameters and can be allocated again.
void release(pangu_server *s, SClass &c) {
  if (c.graph) cudaGraphExecDestroy(c.graph);
  if (c.e) pangu_engine_destroy(c.e);
  for (void *p : c.a.allocs) cudaFree(p);
  for (cudaEvent_t &ev : c.ev)
    if (ev) cudaEventDestroy(ev);
  if (c.stream) cudaStreamDestroy(c.stream);
  s->used -= std::min(s->used, c.bytes);
  c.graph = nullptr;
  c.e = nullptr;
  c.a = Arena{};
  for (cudaEvent_t &ev : c.ev) ev = nullptr;
  c.queued = c.head = 0;
  c.stream = nullptr;
  c.bytes = 0;
  c.allocated = false;
  c.dirty = true;
  c.tuned = false;
  c.running = 0;
}

// Creates a class's pool engine, containers, dt arrays, stream and event,
// charging the budget: the containers as allocated, the engine by the device
// memory its creation took (tables, block table, exchange map, lists).
int allocate(pangu_server *s, SClass &c) {
  size_t free0 = 0, free1 = 0, total = 0;
  if (cudaMemGetInfo(&free0, &total) != cudaSuccess) return PANGU_ECUDA;
  int rc = pangu_pool_create(&c.p, &c.block, c.capacity, c.max_jobs, &c.e);
  if (rc) return rc;
  if (cudaMemGetInfo(&free1, &total) != cudaSuccess) return PANGU_ECUDA;
  const uint64_t eng = free0 > free1 ? free0 - free1 : 0;
  if (s->used + eng > s->budget) {
    pangu_engine_destroy(c.e);
    c.e = nullptr;
    return PANGU_ENOMEM;
  }
  s->used += eng;
  c.bytes = eng;
  const int act[3] = {c.block.nx1 > 1, c.block.nx2 > 1, c.block.nx3 > 1};
  const size_t nv = (size_t)c.capacity * c.nf * c.ncell;
  const size_t na = (size_t)c.capacity * 3 * c.ncell;
  Arena &a = c.a;
  double *alfven = nullptr, *efield = nullptr, *flag = nullptr;
  rc = salloc(s, c, &alfven, na);
  if (!rc) rc = salloc(s, c, &efield, na);
  if (!rc) rc = salloc(s, c, &flag, (size_t)c.capacity * c.ncell);
  pangu_pack *packs[2] = {&a.base, &a.one};
  for (pangu_pack *pk : packs) {
    if (rc) break;
    if (c.prim_bytes == 4) {
      float *pf = nullptr;
      rc = salloc(s, c, &pf, nv);
      pk->prim = reinterpret_cast<double *>(pf);
    } else {
      rc = salloc(s, c, &pk->prim, nv);
    }
    if (!rc) rc = salloc(s, c, &pk->cons, nv);
    if (!rc) rc = salloc(s, c, &pk->flux1, nv);
    if (!rc && act[1]) rc = salloc(s, c, &pk->flux2, nv);
    if (!rc && act[2]) rc = salloc(s, c, &pk->flux3, nv);
    pk->alfven = alfven;
    pk->efield = efield;
    pk->flag = flag;
  }
  if (!rc) rc = salloc(s, c, &a.dt, c.max_jobs);
  if (!rc) rc = salloc(s, c, &a.dt_est, c.max_jobs);
  if (!rc && cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = PANGU_ECUDA;
  for (cudaEvent_t &ev : c.ev)
    if (!rc && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      rc = PANGU_ECUDA;
  if (rc) {
    release(s, c);
    return rc;
  }
  c.allocated = true;
  c.need = c.bytes;
  s->peak = std::max(s->peak, s->used);
  return PANGU_OK;
}

int init_class(SClass &c, const pangu_params *params, const pangu_mesh *block,
               int32_t capacity_blocks, int32_t max_jobs, double dt_factor) {
  c.p = *params;
  c.block = *block;
  c.capacity = capacity_blocks;
  c.max_jobs = max_jobs;
  c.dt_factor = dt_factor;
  c.nf = pangu_num_fields(params);
  if (c.nf <= 0) return PANGU_EINVAL;
  c.prim_bytes = params->precision == PANGU_PRECISION_MIXED ? 4 : 8;
  const int act[3] = {block->nx1 > 1, block->nx2 > 1, block->nx3 > 1};
  const int nx[3] = {block->nx1, block->nx2, block->nx3};
  c.ncell = 1;
  c.interior = 1;
  for (int d = 0; d < 3; ++d) {
    c.ncell *= nx[d] + 2 * block->ng * act[d];
    c.interior *= nx[d];
  }
  return PANGU_OK;
}

// Captures one RK2 cycle of the class pool (both stages and the dt policy).
int capture(SClass &c) {
  if (c.graph) {
    cudaGraphExecDestroy(c.graph);
    c.graph = nullptr;
  }
  if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return PANGU_ECUDA;
  int rc = pangu_stage(c.e, 1, &c.a.base, &c.a.one, 0.5, c.a.dt, nullptr, c.stream);
  if (!rc) rc = pangu_stage(c.e, 2, &c.a.base, &c.a.one, 1.0, c.a.dt, c.a.dt_est, c.stream);
  if (!rc) rc = pangu_update_dt(c.e, c.a.dt, c.a.dt_est, c.dt_factor, c.stream);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(c.stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ec != cudaSuccess) return PANGU_ECUDA;
  const cudaError_t ei = cudaGraphInstantiate(&c.graph, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return PANGU_ECUDA;
  c.dirty = false;
  return PANGU_OK;
}

// Places a job in its class pool and uploads its initial state. Needs the
// class idle (no cycle in flight).
int admit(SClass &c, SJob &j) {
  const long long nb = (long long)j.mesh.nbx1 * j.mesh.nbx2 * j.mesh.nbx3;
  j.slots.assign(nb, -1);
  int32_t job = -1;
  int rc = pangu_job_attach(c.e, &j.mesh, j.a, j.h, &job, j.slots.data());
  if (rc) return rc;
  j.job = job;
  // uploads are ordered on the class stream before the job's first kernels;
  // a pageable source is consumed before cudaMemcpyAsync returns
  const size_t blk = (size_t)c.nf * c.ncell;
  std::vector<float> tmp;
  for (long long b = 0; b < nb; ++b) {
    const int sl = j.slots[b];
    if (j.generated) {
      if (cudaMemsetAsync(c.a.base.cons + (size_t)sl * blk, 0, blk * 8, c.stream) != cudaSuccess ||
          cudaMemsetAsync(c.a.base.flag + (size_t)sl * c.ncell, 0, c.ncell * 8, c.stream) !=
              cudaSuccess)
        return PANGU_ECUDA;
      continue;
    }
    const double *src = j.prim.data() + b * blk;
    char *dst = (char *)c.a.base.prim + (size_t)sl * blk * c.prim_bytes;
    cudaError_t ec;
    if (c.prim_bytes == 4) {
      tmp.assign(src, src + blk);
      ec = cudaMemcpyAsync(dst, tmp.data(), blk * 4, cudaMemcpyHostToDevice, c.stream);
    } else {
      ec = cudaMemcpyAsync(dst, src, blk * 8, cudaMemcpyHostToDevice, c.stream);
    }
    if (ec != cudaSuccess ||
        cudaMemsetAsync(c.a.base.cons + (size_t)sl * blk, 0, blk * 8, c.stream) != cudaSuccess ||
        cudaMemsetAsync(c.a.base.flag + (size_t)sl * c.ncell, 0, c.ncell * 8, c.stream) !=
            cudaSuccess)
      return PANGU_ECUDA;
  }
  if (cudaMemcpyAsync(c.a.dt + job, &j.dt_init, 8, cudaMemcpyHostToDevice, c.stream) !=
      cudaSuccess)
    return PANGU_ECUDA;
  if (j.generated && (rc = pangu_generate(c.e, job, &j.problem, &c.a.base, c.stream))) return rc;
  rc = pangu_job_start(c.e, job, &c.a.base, &c.a.one, c.stream);
  if (rc) return rc;
  c.dirty = true;
  ++c.running;
  return PANGU_OK;
}

// Detaches a cancelled job without copying anything back. Needs the class
// idle.
int drop(SClass &c, SJob &j) {
  const int rc = pangu_job_detach(c.e, j.job);
  if (rc) return rc;
  c.dirty = true;
  --c.running;
  return PANGU_OK;
}

// Copies a finished job's primitives and counters back and detaches it.
// Needs the class idle.
int retire(SClass &c, SJob &j) {
  const size_t blk = (size_t)c.nf * c.ncell;
  j.prim.resize(j.slots.size() * blk);
  std::vector<float> tmp(c.prim_bytes == 4 ? blk : 0);
  for (size_t b = 0; b < j.slots.size(); ++b) {
    const char *src = (const char *)c.a.base.prim + (size_t)j.slots[b] * blk * c.prim_bytes;
    double *dst = j.prim.data() + b * blk;
    if (c.prim_bytes == 4) {
      if (cudaMemcpy(tmp.data(), src, blk * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PANGU_ECUDA;
      for (size_t q = 0; q < blk; ++q) dst[q] = tmp[q];
    } else if (cudaMemcpy(dst, src, blk * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      return PANGU_ECUDA;
    }
  }
  int rc = pangu_job_counters(c.e, j.job, j.counters);
  if (!rc) rc = pangu_job_detach(c.e, j.job);
  if (rc) return rc;
  c.dirty = true;
  --c.running;
  return PANGU_OK;
}

}  // namespace

extern "C" {

int pangu_server_create(uint64_t hbm_budget_bytes, pangu_server **out) {
  if (!out || hbm_budget_bytes == 0) return PANGU_EINVAL;
  *out = new (std::nothrow) pangu_server;
  if (!*out) return PANGU_ENOMEM;
  (*out)->budget = hbm_budget_bytes;
  return PANGU_OK;
}

int pangu_server_destroy(pangu_server *s) {
  if (!s) return PANGU_EINVAL;
  for (SClass &c : s->classes)
    if (c.stream) cudaStreamSynchronize(c.stream);
  for (SClass &c : s->classes) release(s, c);
  delete s;
  return PANGU_OK;
}

int pangu_server_add_class(pangu_server *s, const pangu_params *params, const pangu_mesh *block,
                           int32_t capacity_blocks, int32_t max_jobs, double dt_factor,
                           int32_t *class_out) {
  if (!s || !params || !block || !class_out || capacity_blocks < 1 || max_jobs < 1)
    return PANGU_EINVAL;
  SClass c;
  int rc = init_class(c, params, block, capacity_blocks, max_jobs, dt_factor);
  if (!rc) rc = allocate(s, c);
  if (rc) return rc;
  *class_out = (int32_t)s->classes.size();
  s->classes.push_back(c);
  return PANGU_OK;
}

int pangu_server_declare_class(pangu_server *s, const pangu_params *params,
                               const pangu_mesh *block, int32_t capacity_blocks,
                               int32_t max_jobs, double dt_factor, int32_t *class_out) {
  if (!s || !params || !block || !class_out || capacity_blocks < 1 || max_jobs < 1)
    return PANGU_EINVAL;
  SClass c;
  const int rc = init_class(c, params, block, capacity_blocks, max_jobs, dt_factor);
  if (rc) return rc;
  c.lazy = true;
  *class_out = (int32_t)s->classes.size();
  s->classes.push_back(c);
  return PANGU_OK;
}

int pangu_server_submit(pangu_server *s, int32_t cls, const pangu_mesh *mesh, double a, double h,
                        double dt_init, int64_t cycles, double arrival_s, const double *prim_host,
                        int32_t *ticket_out) {
  if (!s || !mesh || !prim_host || !ticket_out || cls < 0 || cls >= (int)s->classes.size() ||
      cycles < 1)
    return PANGU_EINVAL;
  const SClass &c = s->classes[cls];
  if (mesh->nx1 != c.block.nx1 || mesh->nx2 != c.block.nx2 || mesh->nx3 != c.block.nx3 ||
      mesh->ng != c.block.ng)
    return PANGU_EINVAL;
  const long long nb = (long long)mesh->nbx1 * mesh->nbx2 * mesh->nbx3;
  if (nb < 1 || nb > c.capacity) return PANGU_ETOOBIG;
  SJob j;
  j.cls = cls;
  j.mesh = *mesh;
  j.a = a;
  j.h = h;
  j.dt_init = dt_init;
  j.cycles = cycles;
  j.arrival = arrival_s;
  j.prim.assign(prim_host, prim_host + (size_t)nb * c.nf * c.ncell);
  *ticket_out = (int32_t)s->jobs.size();
  s->jobs.push_back(std::move(j));
  return PANGU_OK;
}

int pangu_server_submit_problem(pangu_server *s, int32_t cls, const pangu_mesh *mesh, double a,
                                double h, double dt_init, int64_t cycles, double arrival_s,
                                const pangu_problem *problem, int32_t *ticket_out) {
  if (!s || !mesh || !problem || !ticket_out || cls < 0 || cls >= (int)s->classes.size() ||
      cycles < 1)
    return PANGU_EINVAL;
  const SClass &c = s->classes[cls];
  if (mesh->nx1 != c.block.nx1 || mesh->nx2 != c.block.nx2 || mesh->nx3 != c.block.nx3 ||
      mesh->ng != c.block.ng)
    return PANGU_EINVAL;
  const long long nb = (long long)mesh->nbx1 * mesh->nbx2 * mesh->nbx3;
  if (nb < 1 || nb > c.capacity) return PANGU_ETOOBIG;
  SJob j;
  j.cls = cls;
  j.mesh = *mesh;
  j.a = a;
  j.h = h;
  j.dt_init = dt_init;
  j.cycles = cycles;
  j.arrival = arrival_s;
  j.generated = true;
  j.problem = *problem;
  *ticket_out = (int32_t)s->jobs.size();
  s->jobs.push_back(std::move(j));
  return PANGU_OK;
}

int pangu_server_run(pangu_server *s) {
  if (!s) return PANGU_EINVAL;
  std::vector<int> order(s->jobs.size());
  for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
  // admission order: arrival time; among jobs that arrive together, the one
  // with the most work (cells x cycles) first, so that a long job does not
  // start last and set the makespan (longest processing time first)
  auto work = [&](const SJob &j) {
    return (double)j.cycles * j.mesh.nbx1 * j.mesh.nbx2 * j.mesh.nbx3;
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const SJob &a = s->jobs[x], &b = s->jobs[y];
    if (a.arrival != b.arrival) return a.arrival < b.arrival;
    return work(a) > work(b);
  });
  size_t done = 0;
  for (const SJob &j : s->jobs) done += j.state == 2;
  pangu_server_stats &st = s->stats;
  st = pangu_server_stats{};
  const auto t0 = std::chrono::steady_clock::now();
  int rc = PANGU_OK;
  // Every class advances on its own stream. Its finished cycles are credited
  // to its running jobs; with none of its cycles in flight, finished and
  // cancelled jobs are copied out and detached and arrived jobs admitted
  // (both rewrite the block table that queued kernels read); then cycles are
  // queued, up to kQueue and never past any running job's last cycle. An
  // admissible waiting job lets the queue drain instead.
  while (done < s->jobs.size()) {
    bool busy = false, starved = false, released = false;
    for (int ci = 0; ci < (int)s->classes.size(); ++ci) {
      SClass &c = s->classes[ci];
      while (c.queued > 0) {
        const cudaError_t q = cudaEventQuery(c.ev[c.head]);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) return PANGU_ECUDA;
        c.head = (c.head + 1) % kQueue;
        --c.queued;
        ++st.ticks;
        for (SJob &j : s->jobs) {
          if (j.state != 1 || j.cls != ci) continue;
          ++j.done_cycles;
          st.zone_cycles += (double)c.interior * j.slots.size();
        }
      }
      if (c.queued > 0) busy = true;
      const double t = now_s(t0);
      if (c.queued == 0) {
        for (SJob &j : s->jobs) {
          if (j.state != 1 || j.cls != ci) continue;
          if (t >= j.cancel_at && j.done_cycles < j.cycles) {  // cancelled while running
            if ((rc = drop(c, j))) return rc;
            j.state = 3;
            j.t_done = t;
            ++done;
            continue;
          }
          if (j.done_cycles < j.cycles) continue;
          if ((rc = retire(c, j))) return rc;
          j.state = 2;
          j.t_done = now_s(t0);
          ++done;
        }
      }
      bool waiting = false, admissible = false;
      const int free_blocks = c.allocated ? c.capacity - pangu_active_blocks(c.e) : c.capacity;
      for (int q : order) {  // first fit in arrival order
        SJob &j = s->jobs[q];
        if (j.cls != ci || j.state != 0) continue;
        if (t >= j.cancel_at) {  // cancelled before admission
          j.state = 3;
          j.t_done = t;
          ++done;
          continue;
        }
        if (j.arrival > t) continue;
        waiting = true;
        const long long nb = (long long)j.mesh.nbx1 * j.mesh.nbx2 * j.mesh.nbx3;
        if (nb <= free_blocks && c.running < c.max_jobs) admissible = true;
        if (c.queued > 0) continue;  // admitted once the queue has drained
        if (!c.allocated) {
          // the class's memory is charged at its first admission; a class
          // that does not fit yet waits for retiring work to free the budget
          rc = c.need && s->used + c.need > s->budget ? PANGU_ENOMEM : allocate(s, c);
          if (rc == PANGU_ENOMEM) {
            j.waited_for_memory = true;
            starved = true;
            break;
          }
          if (rc) return rc;
        }
        rc = admit(c, j);
        if (rc == PANGU_EFULL) continue;
        if (rc) return rc;
        j.state = 1;
        j.t_admit = now_s(t0);
      }
      if (!c.running) {
        // an idle lazily allocated class with no arrived job waiting gives its
        // memory back
        if (c.lazy && c.allocated && c.queued == 0 && !waiting) {
          release(s, c);
          released = true;
        }
        continue;
      }
      bool cancelling = false;  // a running job to drop once the queue drains
      for (const SJob &j : s->jobs)
        cancelling |= j.state == 1 && j.cls == ci && t >= j.cancel_at;
      if ((admissible || cancelling) && c.queued > 0) continue;  // drain first
      if (c.queued == 0) {
        if (!c.tuned) {
          // flux tile shapes, tuned once on the class's first jobs, with the
          // device to itself: the other classes' queued cycles would make the
          // timings (and so the choice) depend on what else was running
          if (cudaDeviceSynchronize() != cudaSuccess) return PANGU_ECUDA;
          if ((rc = pangu_autotune(c.e, &c.a.base, c.stream))) return rc;
          c.tuned = true;
        }
        if (c.dirty && (rc = capture(c))) return rc;
      }
      long long room = kQueue - c.queued;
      for (const SJob &j : s->jobs)
        if (j.state == 1 && j.cls == ci)
          room = std::min(room, j.cycles - j.done_cycles - c.queued);
      for (long long n = 0; n < room; ++n) {
        if (cudaGraphLaunch(c.graph, c.stream) != cudaSuccess ||
            cudaEventRecord(c.ev[(c.head + c.queued) % kQueue], c.stream) != cudaSuccess)
          return PANGU_ECUDA;
        ++c.queued;
      }
      if (c.queued > 0) busy = true;
    }
    if (!busy && starved && !released) {
      // nothing runs, so nothing will free memory: an arrived job's class does
      // not fit in the budget even with every idle class released
      return PANGU_ENOMEM;
    }
    if (!busy && done < s->jobs.size()) {
      // nothing on the device: sleep until the next arrival
      const double t = now_s(t0);
      double next = -1;
      for (int q : order)
        if (s->jobs[q].state == 0) {
          next = s->jobs[q].arrival;
          break;
        }
      for (int q : order)  // a pending cancellation may come first
        if (s->jobs[q].state == 0 && s->jobs[q].cancel_at < next) next = s->jobs[q].cancel_at;
      if (next > t) std::this_thread::sleep_for(std::chrono::duration<double>(next - t));
    }
  }
  st.wall_s = now_s(t0);
  // lazily allocated classes give their memory back once the run is over
  for (SClass &c : s->classes)
    if (c.lazy && c.allocated) {
      if (cudaStreamSynchronize(c.stream) != cudaSuccess) return PANGU_ECUDA;
      c.queued = 0;
      release(s, c);
    }
  std::vector<double> lat;
  for (const SJob &j : s->jobs)
    if (j.state == 2) lat.push_back(j.t_done - j.arrival);
  std::sort(lat.begin(), lat.end());
  if (!lat.empty()) {
    auto pct = [&](double f) {
      const double pos = f * (lat.size() - 1);
      const size_t lo = (size_t)pos;
      const size_t hi = std::min(lo + 1, lat.size() - 1);
      return lat[lo] + (pos - lo) * (lat[hi] - lat[lo]);
    };
    st.p50_s = pct(0.50);
    st.p99_s = pct(0.99);
  }
  st.jobs = (int64_t)lat.size();
  for (const SJob &j : s->jobs) st.memory_waits += j.waited_for_memory;
  st.zone_cycles_per_s = st.wall_s > 0 ? st.zone_cycles / st.wall_s : 0;
  st.hbm_bytes = s->used;
  st.hbm_peak_bytes = s->peak;
  return PANGU_OK;
}

int pangu_server_result(pangu_server *s, int32_t ticket, double *prim_out, double *times_out,
                        uint64_t counters_out[PANGU_NCOUNTERS]) {
  if (!s || ticket < 0 || ticket >= (int)s->jobs.size()) return PANGU_EINVAL;
  const SJob &j = s->jobs[ticket];
  if (j.state != 2) return PANGU_EINVAL;
  if (prim_out) std::memcpy(prim_out, j.prim.data(), j.prim.size() * 8);
  if (times_out) {
    times_out[0] = j.arrival;
    times_out[1] = j.t_admit;
    times_out[2] = j.t_done;
  }
  if (counters_out)
    for (int q = 0; q < PANGU_NCOUNTERS; ++q) counters_out[q] = j.counters[q];
  return PANGU_OK;
}

int pangu_server_cancel(pangu_server *s, int32_t ticket, double at_s) {
  if (!s || ticket < 0 || ticket >= (int)s->jobs.size()) return PANGU_EINVAL;
  SJob &j = s->jobs[ticket];
  if (j.state >= 2) return PANGU_EINVAL;
  j.cancel_at = at_s;
  return PANGU_OK;
}

int pangu_server_job_state(const pangu_server *s, int32_t ticket) {
  if (!s || ticket < 0 || ticket >= (int)s->jobs.size()) return PANGU_EINVAL;
  return s->jobs[ticket].state;
}

int pangu_server_get_stats(const pangu_server *s, pangu_server_stats *out) {
  if (!s || !out) return PANGU_EINVAL;
  *out = s->stats;
  return PANGU_OK;
}

}  // extern "C"
