// Request server: continuous admission of Poisson solves of different sizes.
//
// No counterpart in the reference, whose solver serves one simulation's
// time step at a time (PoissonSolver::solve, source/Poisson/Base.h:12).
// Here independent callers submit solves against meshes they registered
// once; the server keeps each mesh's assembled operator and vectors resident
// on the device while the memory budget allows (least-recently-used idle
// meshes are evicted first), and a worker thread admits requests as solve
// slots and memory free up.  Every admitted request runs as its own
// persistent solve of `team` CTAs on its slot's stream, so requests that
// arrive while others are running overlap with them on the device.  A solve
// is deterministic for a given team size, so a request's result does not
// depend on what else is running.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/cup2d_poisson.h"
#include "handle_view.hpp"
#include "kernels.hpp"

using namespace cup2d;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Mesh {
  int32_t bpdx, bpdy, level_max, px, py;
  double extent;
  std::vector<int32_t> level, bx, by;
  cup2d_poisson* h = nullptr;  // resident operator and vectors, or null
  int64_t bytes = 0;           // device bytes while resident
  int team = 0;                // CTAs of its solves
  bool busy = false;           // a request of this mesh is on the device
  bool assembling = false;     // queued for, or in, assembly
  bool solved = false;         // the resident x holds a solution (warm starts)
  int error = CUP2D_OK;        // assembly failed: its requests fail with this
  uint64_t last_used = 0;

  cup2d_forest forest() const {
    cup2d_forest f{};
    f.bpdx = bpdx;
    f.bpdy = bpdy;
    f.level_max = level_max;
    f.periodic_x = px;
    f.periodic_y = py;
    f.extent = extent;
    f.nblocks = (int64_t)level.size();
    f.level = level.data();
    f.bx = bx.data();
    f.by = by.data();
    return f;
  }
  int64_t estimate_bytes() const {
    // vectors (FP64 and FP32 Krylov, staging) and operator per block, the
    // dense leaf tables, and per-handle fixed buffers (P^-1, reduction
    // partials); replaced by the measured size once resident
    return (int64_t)level.size() * 9216 + leaf_table_entries(bpdx, bpdy, level_max) * 4 + (256 << 10);
  }
};

struct Request {
  int64_t mesh;
  const double* b;
  double* x;
  int32_t flags;
  Clock::time_point submitted, finished;
  Clock::time_point blocked_since{};  // first time it did not fit the free CTAs
  bool blocked = false;
  bool done = false;
  int status = CUP2D_PENDING;
  cup2d_solve_stats stats{};
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr, done = nullptr;
  void* raw = nullptr;  // pinned statistics record
  int64_t request = -1; // -1: free
  int ctas = 0;         // CTAs of the solve it runs
};

}  // namespace

// Host threads work for the callers: the scheduler (run) completes and
// admits requests; assemblers build operators for meshes that are not
// resident, so that an assembly, whose kernels may wait for SMs held by
// running solves, never holds up admissions.  Solves in flight are kept a
// little below the number of solve CTAs the device holds at once
// (cta_cap), which leaves room for assembly kernels and copies.
struct cup2d_server {
  cup2d_server_opts opts{};
  int device = 0;
  int64_t budget = 0;
  int cta_cap = 0, ctas_inflight = 0;
  std::vector<Slot> slots;
  std::map<int64_t, Mesh> meshes;
  std::map<int64_t, Request> requests;
  std::deque<int64_t> pending;
  std::deque<int64_t> to_assemble;  // mesh ids
  int64_t next_mesh = 1, next_request = 1;
  uint64_t tick = 0;
  int64_t resident_bytes = 0;
  cup2d_server_counters counters{};
  std::mutex mu;
  std::condition_variable work_cv;  // new submissions, finished assemblies
  std::condition_variable done_cv;  // completions
  std::condition_variable asm_cv;   // meshes to assemble
  std::thread worker;
  std::vector<std::thread> assemblers;
  // one assembly stream per assembler thread, at the highest priority, made
  // once: a handle created per request would otherwise make (and destroy)
  // a stream and two events every time, which under load took as long as
  // the assembly itself; the handles of a thread assemble on its stream
  std::vector<cudaStream_t> asm_streams;
  std::deque<int64_t> completed_q;  // finished requests not yet taken
  static constexpr int kAssemblers = 8;
  bool stop = false;
  int fatal = CUP2D_OK;  // a CUDA error that stopped the worker

  void run();
  void run_assembler(cudaStream_t stream);
  bool complete_slots();  // mu held
  bool admit();           // mu held
  int assemble(Mesh& m, std::unique_lock<std::mutex>& lk, cudaStream_t stream);
  int launch(Slot& s, int64_t rid, Request& r, Mesh& m);
  // CTAs of a mesh's solves: opts.team, or by size when it is 0
  int team_for(int64_t nb) const {
    const int t = opts.team > 0
                      ? opts.team
                      : (int)std::min<int64_t>(128, std::max<int64_t>(2, (nb + opts.blocks_per_cta / 2) /
                                                                                  opts.blocks_per_cta));
    return std::min(t, cta_cap);
  }
  static constexpr std::chrono::milliseconds kMaxBypass{100};
};

namespace {

int server_error(cup2d_server* S, int st) {
  if (!S->fatal) S->fatal = st;
  return st;
}

}  // namespace

// Makes m resident: evicts idle meshes (least recently used first) until it
// fits the budget, then assembles it with the lock released.  Returns
// CUP2D_QUEUE_FULL when the memory is held by meshes in use.
int cup2d_server::assemble(Mesh& m, std::unique_lock<std::mutex>& lk, cudaStream_t stream) {
  const int64_t need = m.estimate_bytes();
  if (need > budget) return CUP2D_OOM;
  while (resident_bytes + need > budget) {
    Mesh* victim = nullptr;
    for (auto& kv : meshes) {
      Mesh& c = kv.second;
      if (c.h && !c.busy && (!victim || c.last_used < victim->last_used)) victim = &c;
    }
    if (!victim) return CUP2D_QUEUE_FULL;
    handle_destroy_idle(victim->h);  // idle: its last solve has completed
    victim->h = nullptr;
    victim->solved = false;
    resident_bytes -= victim->bytes;
    victim->bytes = 0;
    ++counters.evictions;
  }
  const cup2d_forest f = m.forest();
  cup2d_solve_opts o = opts.solve;
  const int team = team_for((int64_t)m.level.size());
  cup2d_poisson* h = nullptr;
  resident_bytes += need;  // reserved while assembling
  lk.unlock();
  const Clock::time_point t_asm = Clock::now();
  int st = handle_create(&f, &o, stream, true, &h);
  if (st == CUP2D_OK) st = cup2d_poisson_set_grid(h, team);
  double* db = nullptr;
  double* dx = nullptr;
  if (st == CUP2D_OK) st = handle_stage(h, &db, &dx);
  lk.lock();
  resident_bytes -= need;
  if (st != CUP2D_OK) {
    if (h) handle_destroy_idle(h);
    return st;
  }
  m.h = h;
  m.team = team;
  m.bytes = handle_bytes(h);
  resident_bytes += m.bytes;
  m.solved = false;
  m.last_used = ++tick;
  ++counters.assemblies;
  counters.assembly_us += (int64_t)(ms_between(t_asm, Clock::now()) * 1000.0);
  return CUP2D_OK;
}

void cup2d_server::run_assembler(cudaStream_t stream) {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    if (to_assemble.empty()) {
      asm_cv.wait_for(lk, std::chrono::milliseconds(5));
      continue;
    }
    const int64_t id = to_assemble.front();
    to_assemble.pop_front();
    Mesh& m = meshes.at(id);
    const int st = assemble(m, lk, stream);
    if (st == CUP2D_QUEUE_FULL) {
      // the budget is held by meshes in use: retry after a completion
      to_assemble.push_back(id);
      done_cv.wait_for(lk, std::chrono::milliseconds(2));
      continue;
    }
    m.assembling = false;
    if (st != CUP2D_OK) m.error = st;
    work_cv.notify_all();
  }
}

int cup2d_server::launch(Slot& s, int64_t rid, Request& r, Mesh& m) {
  double* db = nullptr;
  double* dx = nullptr;
  int st = handle_stage(m.h, &db, &dx);
  if (st) return st;
  const size_t bytes = sizeof(double) * (size_t)m.level.size() * kBLEN;
  const bool warm = (r.flags & CUP2D_SUBMIT_WARM_START) && m.solved;
  if (cudaMemcpyAsync(db, r.b, bytes, cudaMemcpyHostToDevice, s.stream) != cudaSuccess) return CUP2D_CUDA_ERROR;
  if (!warm) {
    if (r.flags & CUP2D_SUBMIT_WARM_START) {
      if (cudaMemsetAsync(dx, 0, bytes, s.stream) != cudaSuccess) return CUP2D_CUDA_ERROR;
    } else if (cudaMemcpyAsync(dx, r.x, bytes, cudaMemcpyHostToDevice, s.stream) != cudaSuccess) {
      return CUP2D_CUDA_ERROR;
    }
  }
  if (cudaEventRecord(s.t0, s.stream) != cudaSuccess) return CUP2D_CUDA_ERROR;
  if ((st = handle_solve_async(m.h, db, dx, s.stream, s.raw))) return st;
  if (cudaEventRecord(s.t1, s.stream) != cudaSuccess ||
      cudaMemcpyAsync(r.x, dx, bytes, cudaMemcpyDeviceToHost, s.stream) != cudaSuccess ||
      cudaEventRecord(s.done, s.stream) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

bool cup2d_server::complete_slots() {
  bool any = false;
  for (Slot& s : slots) {
    if (s.request < 0) continue;
    const cudaError_t q = cudaEventQuery(s.done);
    if (q == cudaErrorNotReady) continue;
    Request& r = requests.at(s.request);
    Mesh& m = meshes.at(r.mesh);
    if (q != cudaSuccess) {
      r.status = CUP2D_CUDA_ERROR;
      server_error(this, CUP2D_CUDA_ERROR);
    } else {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, s.t0, s.t1);
      handle_stats_from_raw(s.raw, ms, &r.stats);
      r.status = r.stats.status;
      m.solved = r.status == CUP2D_OK || r.status == CUP2D_NOT_CONVERGED || r.status == CUP2D_BREAKDOWN_LIMIT;
    }
    r.finished = Clock::now();
    r.done = true;
    completed_q.push_back(s.request);
    m.busy = false;
    ctas_inflight -= s.ctas;
    s.request = -1;
    s.ctas = 0;
    --counters.inflight;
    if (r.status == CUP2D_OK) ++counters.completed;
    else ++counters.failed;
    any = true;
  }
  return any;
}

// Admits pending requests in submission order while slots and CTAs are
// free; a request whose mesh is running or not resident yet stays queued
// (its mesh is handed to the assembler) without blocking the ones behind
// it; one that does not fit the free CTAs is overtaken by smaller ones for
// at most kMaxBypass, after which admission waits for it.  Called
// with mu held by the scheduler, the only thread that removes from
// `pending` or touches the slots; the lock is released around launches.
bool cup2d_server::admit() {
  bool any = false;
  std::unique_lock<std::mutex> lk(mu, std::adopt_lock);
  const std::vector<int64_t> snapshot(pending.begin(), pending.end());
  std::vector<int64_t> leaving;
  for (const int64_t rid : snapshot) {
    Request& r = requests.at(rid);
    Mesh& m = meshes.at(r.mesh);
    int st = m.error;
    if (st == CUP2D_OK) {
      if (m.busy || m.assembling) continue;
      if (!m.h) {
        m.assembling = true;
        to_assemble.push_back(r.mesh);
        asm_cv.notify_one();
        continue;
      }
      if (ctas_inflight + m.team > cta_cap) {
        // does not fit the free CTAs: later requests that fit may go first
        // (backfill), until this one has waited kMaxBypass; then admission
        // stops until running solves have freed enough CTAs for it
        const Clock::time_point now = Clock::now();
        if (!r.blocked) {
          r.blocked = true;
          r.blocked_since = now;
        }
        if (now - r.blocked_since > kMaxBypass) break;
        continue;
      }
      Slot* free_slot = nullptr;
      for (Slot& s : slots)
        if (s.request < 0) { free_slot = &s; break; }
      if (!free_slot) break;
      m.busy = true;
      free_slot->request = rid;
      free_slot->ctas = m.team;
      ctas_inflight += m.team;
      m.last_used = ++tick;
      lk.unlock();
      st = launch(*free_slot, rid, r, m);
      lk.lock();
      if (st != CUP2D_OK) {
        m.busy = false;
        ctas_inflight -= free_slot->ctas;
        free_slot->request = -1;
        free_slot->ctas = 0;
      }
    }
    if (st != CUP2D_OK) {
      r.status = st;
      r.done = true;
      r.finished = Clock::now();
      completed_q.push_back(rid);
      ++counters.failed;
      if (st == CUP2D_CUDA_ERROR) server_error(this, st);
    } else {
      ++counters.admitted;
      ++counters.inflight;
    }
    --counters.queued;
    leaving.push_back(rid);
    any = true;
  }
  if (!leaving.empty())
    pending.erase(std::remove_if(pending.begin(), pending.end(),
                                 [&](int64_t id) {
                                   return std::find(leaving.begin(), leaving.end(), id) != leaving.end();
                                 }),
                  pending.end());
  lk.release();
  return any;
}

void cup2d_server::run() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    const bool completed = complete_slots();
    const bool admitted = admit();
    if (completed || admitted) done_cv.notify_all();
    if (fatal) break;
    if (completed || admitted) continue;
    if (counters.inflight > 0) {
      // solves on the device: poll their completion events closely
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(20));
      lk.lock();
    } else {
      work_cv.wait_for(lk, std::chrono::milliseconds(5));
    }
  }
  done_cv.notify_all();
}

extern "C" {

void cup2d_server_default_opts(cup2d_server_opts* o) {
  if (!o) return;
  o->max_inflight = 24;
  o->team = 16;
  o->blocks_per_cta = 320;
  o->solve_share = 0.9;
  o->hbm_budget_bytes = 0;
  cup2d_default_opts(&o->solve);
}

int cup2d_server_destroy(cup2d_server* S) {
  if (!S) return CUP2D_OK;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->work_cv.notify_all();
  S->asm_cv.notify_all();
  S->done_cv.notify_all();
  if (S->worker.joinable()) S->worker.join();
  for (std::thread& t : S->assemblers)
    if (t.joinable()) t.join();
  cudaSetDevice(S->device);
  for (Slot& s : S->slots) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.t0) cudaEventDestroy(s.t0);
    if (s.t1) cudaEventDestroy(s.t1);
    if (s.done) cudaEventDestroy(s.done);
    if (s.raw) cudaFreeHost(s.raw);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  for (auto& kv : S->meshes)
    if (kv.second.h) handle_destroy_idle(kv.second.h);  // every slot stream is synchronised
  for (cudaStream_t st : S->asm_streams)  // after the handles that assembled on them
    if (st) cudaStreamDestroy(st);
  delete S;
  return CUP2D_OK;
}

int cup2d_server_create(const cup2d_server_opts* opts, cup2d_server** out) {
  if (!out) return CUP2D_INVALID_ARGUMENT;
  *out = nullptr;
  cup2d_server_opts o;
  cup2d_server_default_opts(&o);
  if (opts) o = *opts;
  if (o.max_inflight < 1 || o.max_inflight > 256 || o.team < 0 || o.team > 1024 || o.blocks_per_cta < 1 ||
      o.hbm_budget_bytes < 0 || !(o.solve_share > 0.0 && o.solve_share <= 1.0))
    return CUP2D_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CUP2D_NO_DEVICE;
  }
  auto* S = new (std::nothrow) cup2d_server();
  if (!S) return CUP2D_OOM;
  S->opts = o;
  cudaGetDevice(&S->device);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    delete S;
    return CUP2D_CUDA_ERROR;
  }
  S->budget = o.hbm_budget_bytes > 0 ? std::min<int64_t>(o.hbm_budget_bytes, (int64_t)free_b)
                                     : (int64_t)(0.8 * (double)free_b);
  S->counters.budget_bytes = S->budget;
  S->slots.resize(o.max_inflight);
  for (Slot& s : S->slots) {
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s.t0) != cudaSuccess || cudaEventCreate(&s.t1) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&s.raw, handle_stats_bytes()) != cudaSuccess) {
      cup2d_server_destroy(S);
      return CUP2D_CUDA_ERROR;
    }
  }
  const int grid_max = o.solve.precision == CUP2D_PREC_MIXED ? max_coop_grid_mixed(S->device, true)
                                                              : max_coop_grid_fp64(S->device, true);
  if (grid_max <= 0) {
    cup2d_server_destroy(S);
    return CUP2D_CUDA_ERROR;
  }
  S->cta_cap = std::max(1, (int)(o.solve_share * grid_max));
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  S->asm_streams.assign(cup2d_server::kAssemblers, nullptr);
  for (cudaStream_t& st : S->asm_streams)
    if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
      st = nullptr;
      cup2d_server_destroy(S);
      return CUP2D_CUDA_ERROR;
    }
  S->worker = std::thread([S] { S->run(); });
  for (int i = 0; i < cup2d_server::kAssemblers; ++i) {
    cudaStream_t st = S->asm_streams[i];
    S->assemblers.emplace_back([S, st] { S->run_assembler(st); });
  }
  *out = S;
  return CUP2D_OK;
}

int cup2d_server_add_mesh(cup2d_server* S, const cup2d_forest* f, int64_t* mesh_id) {
  if (!S || !f || !mesh_id || f->nblocks <= 0 || !f->level || !f->bx || !f->by) return CUP2D_INVALID_ARGUMENT;
  Mesh m;
  m.bpdx = f->bpdx;
  m.bpdy = f->bpdy;
  m.level_max = f->level_max;
  m.px = f->periodic_x;
  m.py = f->periodic_y;
  m.extent = f->extent;
  m.level.assign(f->level, f->level + f->nblocks);
  m.bx.assign(f->bx, f->bx + f->nblocks);
  m.by.assign(f->by, f->by + f->nblocks);
  std::lock_guard<std::mutex> g(S->mu);
  const int64_t id = S->next_mesh++;
  S->meshes.emplace(id, std::move(m));
  *mesh_id = id;
  return CUP2D_OK;
}

int cup2d_server_submit(cup2d_server* S, int64_t mesh_id, const double* b, double* x, int32_t flags,
                        int64_t* request_id) {
  if (!S || !b || !x || !request_id) return CUP2D_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(S->mu);
  if (S->fatal) return S->fatal;
  if (!S->meshes.count(mesh_id)) return CUP2D_INVALID_ARGUMENT;
  const int64_t id = S->next_request++;
  Request r;
  r.mesh = mesh_id;
  r.b = b;
  r.x = x;
  r.flags = flags;
  r.submitted = Clock::now();
  S->requests.emplace(id, r);
  S->pending.push_back(id);
  ++S->counters.submitted;
  ++S->counters.queued;
  *request_id = id;
  S->work_cv.notify_one();
  return CUP2D_OK;
}

namespace {
int finish(cup2d_server* S, std::map<int64_t, Request>::iterator it, cup2d_solve_stats* stats, double* latency_ms) {
  Request& r = it->second;
  if (stats) {
    *stats = r.stats;
    stats->status = r.status;
  }
  if (latency_ms) *latency_ms = ms_between(r.submitted, r.finished);
  const int st = r.status;
  // collected: no longer reported by take_completed
  auto q = std::find(S->completed_q.begin(), S->completed_q.end(), it->first);
  if (q != S->completed_q.end()) S->completed_q.erase(q);
  S->requests.erase(it);
  return st;
}
}  // namespace

int cup2d_server_poll(cup2d_server* S, int64_t request_id, cup2d_solve_stats* stats, double* latency_ms) {
  if (!S) return CUP2D_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->requests.find(request_id);
  if (it == S->requests.end()) return CUP2D_INVALID_ARGUMENT;
  if (!it->second.done) return CUP2D_PENDING;
  return finish(S, it, stats, latency_ms);
}

int cup2d_server_wait(cup2d_server* S, int64_t request_id, int32_t timeout_ms, cup2d_solve_stats* stats,
                      double* latency_ms) {
  if (!S || timeout_ms < 0) return CUP2D_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->requests.find(request_id);
  if (it == S->requests.end()) return CUP2D_INVALID_ARGUMENT;
  const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms);
  while (!it->second.done) {
    if (S->fatal) return S->fatal;  // the worker has stopped
    if (S->done_cv.wait_until(lk, deadline) == std::cv_status::timeout && !it->second.done) return CUP2D_PENDING;
  }
  return finish(S, it, stats, latency_ms);
}

int cup2d_server_take_completed(cup2d_server* S, int64_t* ids, int32_t max_ids, int32_t timeout_ms, int32_t* n) {
  if (!S || !ids || max_ids < 1 || timeout_ms < 0 || !n) return CUP2D_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  *n = 0;
  if (S->completed_q.empty() && timeout_ms > 0)
    S->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [S] { return !S->completed_q.empty() || S->fatal; });
  while (*n < max_ids && !S->completed_q.empty()) {
    ids[(*n)++] = S->completed_q.front();
    S->completed_q.pop_front();
  }
  return S->fatal ? S->fatal : CUP2D_OK;
}

int cup2d_server_get_counters(cup2d_server* S, cup2d_server_counters* out) {
  if (!S || !out) return CUP2D_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(S->mu);
  *out = S->counters;
  int64_t resident = 0;
  for (auto& kv : S->meshes) resident += kv.second.h ? 1 : 0;
  out->resident_meshes = resident;
  out->resident_bytes = S->resident_bytes;
  return CUP2D_OK;
}

}  // extern "C"
