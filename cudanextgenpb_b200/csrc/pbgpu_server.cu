// PB solve server: continuous batching of requests of different molecule sizes
// on one GPU.  No counterpart in the reference, whose driver
// (src/poisson_boltzmann.cpp:192-299) runs one molecule per process.
//
// A tick of pbgpu_server_progress:
//   1. launches one persistent step of the multi-system solver over the
//      members (pbgpu_batch_launch), which holds the matrices and Krylov
//      states of all members on the device;
//   2. meanwhile admits queued requests (FIFO) while the member cap, the
//      per-tick admission cap and the HBM budget allow, and sets each one up
//      (inputs, markers, density map, SELL system) on its own context and
//      stream from its own host thread;
//   3. waits for the persistent step;
//   4. retires the members that converged: energies on their context, result
//      returned, context back to the idle pool;
//   5. adds the set-up requests to the batch; they start with the next tick.
// The persistent kernel is limited to blocks_per_sm resident blocks so the
// set-up kernels of (2) run beside it.
// Admission counts the device bytes every context holds (idle ones included,
// their buffers are kept for reuse) plus an estimate for the request; idle
// contexts are destroyed, largest first, when the budget needs the room.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pbgpu_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

struct Pending {
  int64_t id;
  pbgpu_request req;
  Clock::time_point t_submit;
};

struct Running {
  int64_t id;
  int64_t tag;
  int slot;
  pbgpu_ctx* ctx;
  int64_t n_atoms;
  Clock::time_point t_submit, t_admit;
};

int64_t ctx_bytes(pbgpu_ctx* c) { return c ? c->c.dev_bytes : 0; }

// A converged member out of the batch whose energy is still to compute.
struct Retire {
  Running r;
  pbgpu_solve_stats stats;
  pbgpu_energy_out energy;
  int st;
};

}  // namespace

struct pbgpu_server {
  int device = 0;
  pbgpu_server_opts opts{};
  pbgpu_batch* batch = nullptr;
  // concurrent mode: worker threads, each with its own context and stream
  std::vector<std::thread> workers;
  std::vector<pbgpu_ctx*> worker_ctx;
  std::mutex mu;
  std::condition_variable cv_job, cv_done;
  std::deque<Pending> jobs;
  std::deque<pbgpu_result> finished;
  int in_flight = 0;
  bool stop = false;
  std::deque<Pending> queue;
  std::vector<Running> running;
  std::vector<Retire> finishing;  // batched mode: energies of the next tick
  std::vector<pbgpu_ctx*> idle;
  int64_t next_id = 1;
  bool in_session = false;
  std::string err;
  int64_t admitted = 0, completed = 0, rejected = 0;
  int64_t retired_launches = 0;  // kernels of contexts the server has destroyed
  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
};

// Inputs (the mesh set or built), markers, density map and SELL system of one
// request on `ctx`.
static int setup_request(pbgpu_server* s, pbgpu_ctx* ctx, const pbgpu_request& r) {
  int st;
  if (r.mesh) {
    if ((st = pbgpu_set_mesh(ctx, r.mesh)) != PBGPU_OK) return st;
    for (int a = 0; a < 3; ++a)
      if ((st = pbgpu_set_rays(ctx, a, &r.rays[a])) != PBGPU_OK) return st;
  } else if ((st = pbgpu_build_mesh(ctx, r.build)) != PBGPU_OK) {
    return st;
  }
  if ((st = pbgpu_set_atoms(ctx, r.n_atoms, r.pos, r.charge)) != PBGPU_OK) return st;
  if ((st = pbgpu_set_model(ctx, r.model)) != PBGPU_OK) return st;
  if ((st = pbgpu_create_markers(ctx)) != PBGPU_OK) return st;
  if ((st = pbgpu_create_density_map(ctx)) != PBGPU_OK) return st;
  pbgpu_sell_opts so{32, 2048, 4};
  return pbgpu_assemble(ctx, &so);
  (void)s;
}

// Concurrent mode: a worker takes dispatched requests one at a time and runs
// the whole path for each on its own context (and stream).
static void worker_loop(pbgpu_server* s, int w) {
  pbgpu_ctx* ctx = s->worker_ctx[w];
  while (true) {
    Pending p;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_job.wait(lk, [s] { return s->stop || !s->jobs.empty(); });
      if (s->jobs.empty()) return;
      p = s->jobs.front();
      s->jobs.pop_front();
    }
    pbgpu_result o;
    std::memset(&o, 0, sizeof(o));
    o.id = p.id;
    o.user_tag = p.req.user_tag;
    o.queue_ms = ms_since(p.t_submit);
    int st = setup_request(s, ctx, p.req);
    if (st == PBGPU_OK) st = pbgpu_solve(ctx, &s->opts.solver, &o.stats);
    if (st == PBGPU_OK) st = pbgpu_energy(ctx, s->opts.energy_fast, &o.energy);
    o.status = st;
    o.latency_ms = ms_since(p.t_submit);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->finished.push_back(o);
      --s->in_flight;
    }
    s->cv_done.notify_one();
  }
}

// The result of a request that can never fit the budget.
static pbgpu_result rejection(const Pending& p) {
  pbgpu_result o;
  std::memset(&o, 0, sizeof(o));
  o.id = p.id;
  o.user_tag = p.req.user_tag;
  o.status = PBGPU_REJECTED;
  o.latency_ms = ms_since(p.t_submit);
  o.queue_ms = o.latency_ms;
  return o;
}

extern "C" {

int64_t pbgpu_request_bytes_estimate(const pbgpu_request* r) {
  if (!r || (!r->mesh && !r->build)) return 0;
  if (!r->mesh) {
    // Mesh still to build: every refinement level above the initial octree
    // splits surface octants into 8; measured, each surface level multiplies
    // the octant count by at most ~3.5 (the refined shell is thin), and nodes
    // and hanging nodes stay below 0.8 and 0.7 per octant.  Bound the final
    // octants by 4x per level.
    const pbgpu_mesh_build* b = r->build;
    int top = 0;
    for (int64_t i = 0; i < b->n_oct; ++i) top = std::max(top, (int)b->oct_level[i]);
    const int levels = b->refine ? std::max(0, b->maxlevel - top) : 0;
    double no = (double)b->n_oct;
    for (int l = 0; l < levels; ++l) no *= 4.0;
    return (int64_t)(1120.0 * no + 1000.0 * (double)b->n_spheres) + ((int64_t)64 << 20);
  }
  const double no = (double)r->mesh->n_oct, n = (double)r->mesh->n_nodes, nh = (double)r->mesh->n_hang;
  // mesh, incidence lists, per-octant local coefficients (assembly scratch),
  // SELL matrix (~11 nonzeros per row, 12 B each), Krylov vectors (FP64 and
  // FP32), energy scratch; per unit of each size.  Measured on B200 after
  // set-up, a mixed-precision batch solve, energy and pot_field, contexts
  // held 810-860 B per octant (nodes ~0.7 and hanging nodes ~0.55 per
  // octant) before the assembly kept 9 B per node more and, while it runs,
  // 336 B per node of row lines (freed at its end); these coefficients give
  // 1,120 B per octant, an upper bound that includes the lines.
  return (int64_t)(500.0 * no + 850.0 * n + 40.0 * nh) + ((int64_t)64 << 20);
}

void pbgpu_default_server_opts(pbgpu_server_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->hbm_budget_bytes = 160e9;
  o->max_members = 64;
  o->steps_per_tick = 32;
  o->blocks_per_sm = 2;
  o->admit_per_tick = 16;
  o->mode = 0;
  o->workers = 8;
  pbgpu_default_solver_opts(&o->solver);
  o->solver.method = PBGPU_CG;
  o->solver.precond = PBGPU_PRECOND_JACOBI;
  o->solver.precision = PBGPU_MIXED;
  o->solver.tol = 1e-8;
  o->solver.inner_tol = 1e-4;
  o->solver.max_iter = 50000;
  o->energy_fast = 0;
}

int pbgpu_server_create(pbgpu_server** out, int device, const pbgpu_server_opts* opts) {
  if (!out) return PBGPU_ERR_ARG;
  *out = nullptr;
  pbgpu_server* s = new (std::nothrow) pbgpu_server();
  if (!s) return PBGPU_ERR_OOM;
  s->device = device;
  if (opts)
    s->opts = *opts;
  else
    pbgpu_default_server_opts(&s->opts);
  if (s->opts.max_members <= 0) s->opts.max_members = 64;
  if (s->opts.steps_per_tick <= 0) s->opts.steps_per_tick = 32;
  if (!(s->opts.hbm_budget_bytes > 0)) s->opts.hbm_budget_bytes = 160e9;
  if (s->opts.mode == 1) {
    const int nw = s->opts.workers > 0 ? s->opts.workers : 8;
    for (int w = 0; w < nw; ++w) {
      pbgpu_ctx* c = nullptr;
      const int st = pbgpu_ctx_create(&c, device, nullptr);
      if (st != PBGPU_OK) {
        for (pbgpu_ctx* x : s->worker_ctx) pbgpu_ctx_destroy(x);
        delete s;
        return st;
      }
      s->worker_ctx.push_back(c);
    }
    for (int w = 0; w < nw; ++w) s->workers.emplace_back(worker_loop, s, w);
    *out = s;
    return PBGPU_OK;
  }
  int st = pbgpu_batch_create(&s->batch, device, nullptr);
  if (st != PBGPU_OK) {
    delete s;
    return st;
  }
  pbgpu_batch_set_blocks_per_sm(s->batch, s->opts.blocks_per_sm);
  *out = s;
  return PBGPU_OK;
}

void pbgpu_server_destroy(pbgpu_server* s) {
  if (!s) return;
  if (!s->workers.empty()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
      s->jobs.clear();
    }
    s->cv_job.notify_all();
    for (std::thread& t : s->workers) t.join();
    for (pbgpu_ctx* c : s->worker_ctx) pbgpu_ctx_destroy(c);
  }
  if (s->batch) pbgpu_batch_destroy(s->batch);
  for (Running& r : s->running) pbgpu_ctx_destroy(r.ctx);
  for (Retire& x : s->finishing) pbgpu_ctx_destroy(x.r.ctx);
  for (pbgpu_ctx* c : s->idle) pbgpu_ctx_destroy(c);
  delete s;
}

const char* pbgpu_server_last_error(const pbgpu_server* s) { return s ? s->err.c_str() : "null server"; }

int pbgpu_server_submit(pbgpu_server* s, const pbgpu_request* req, int64_t* id) {
  if (!s || !req || (!req->mesh && !req->build) || !req->model || req->n_atoms < 0 ||
      (req->n_atoms > 0 && (!req->pos || !req->charge)))
    return PBGPU_ERR_ARG;
  Pending p{s->next_id++, *req, Clock::now()};
  s->queue.push_back(p);
  if (id) *id = p.id;
  return PBGPU_OK;
}

int pbgpu_server_stats(const pbgpu_server* sc, int64_t* admitted, int64_t* completed, int64_t* rejected,
                       int64_t* launches) {
  if (!sc) return PBGPU_ERR_ARG;
  pbgpu_server* s = const_cast<pbgpu_server*>(sc);
  std::lock_guard<std::mutex> lk(s->mu);
  if (admitted) *admitted = s->admitted;
  if (completed) *completed = s->completed;
  if (rejected) *rejected = s->rejected;
  if (launches) {
    int64_t l = s->retired_launches + (s->batch ? pbgpu::batch_launch_count(s->batch) : 0);
    for (pbgpu_ctx* c : s->worker_ctx) l += c->c.launches;
    for (const Running& r : s->running) l += r.ctx->c.launches;
    for (const Retire& x : s->finishing) l += x.r.ctx->c.launches;
    for (pbgpu_ctx* c : s->idle) l += c->c.launches;
    *launches = l;
  }
  return PBGPU_OK;
}

int pbgpu_server_pending(const pbgpu_server* sc, int* queued, int* running, int64_t* device_bytes) {
  if (!sc) return PBGPU_ERR_ARG;
  pbgpu_server* s = const_cast<pbgpu_server*>(sc);
  if (s->opts.mode == 1) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int)(s->queue.size() + s->jobs.size());
    if (running) *running = s->in_flight - (int)s->jobs.size() + (int)s->finished.size();
    if (device_bytes) {
      int64_t b = 0;
      for (pbgpu_ctx* c : s->worker_ctx) b += ctx_bytes(c);
      *device_bytes = b;
    }
    return PBGPU_OK;
  }
  if (queued) *queued = (int)s->queue.size();
  if (running) *running = (int)(s->running.size() + s->finishing.size());
  if (device_bytes) {
    int64_t b = 0;
    for (const Running& r : s->running) b += ctx_bytes(r.ctx);
    for (const Retire& x : s->finishing) b += ctx_bytes(x.r.ctx);
    for (pbgpu_ctx* c : s->idle) b += ctx_bytes(c);
    *device_bytes = b;
  }
  return PBGPU_OK;
}


static int64_t held_bytes(const pbgpu_server* s) {
  int64_t b = 0;
  for (const Running& r : s->running) b += ctx_bytes(r.ctx);
  for (const Retire& x : s->finishing) b += ctx_bytes(x.r.ctx);
  for (pbgpu_ctx* c : s->idle) b += ctx_bytes(c);
  return b;
}

// Concurrent mode: dispatch queued requests to the workers while the budget
// allows, then hand back the finished ones (waiting briefly when work is in
// flight and nothing has finished yet).
static int progress_concurrent(pbgpu_server* s, pbgpu_result* out, int cap, int* n_out) {
  std::unique_lock<std::mutex> lk(s->mu);
  const int nw = (int)s->workers.size();
  int64_t held = 0, largest = 0;
  for (pbgpu_ctx* c : s->worker_ctx) {
    held += ctx_bytes(c);
    largest = std::max(largest, ctx_bytes(c));
  }
  while (!s->queue.empty() && s->in_flight < nw) {
    const int64_t need = pbgpu_request_bytes_estimate(&s->queue.front().req);
    if ((double)need > s->opts.hbm_budget_bytes) {
      // alone it already exceeds the budget: reject instead of admitting
      s->finished.push_back(rejection(s->queue.front()));
      s->queue.pop_front();
      ++s->rejected;
      continue;
    }
    // a worker may grow to this request's size: at worst all of them do
    if (held - largest + (int64_t)nw * std::max(largest, need) > (int64_t)s->opts.hbm_budget_bytes &&
        s->in_flight > 0)
      break;
    s->jobs.push_back(s->queue.front());
    s->queue.pop_front();
    ++s->in_flight;
    ++s->admitted;
  }
  s->cv_job.notify_all();
  if (s->finished.empty() && s->in_flight > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(2), [s] { return !s->finished.empty(); });
  while (!s->finished.empty() && *n_out < cap) {
    out[(*n_out)++] = s->finished.front();
    s->finished.pop_front();
    ++s->completed;
  }
  return PBGPU_OK;
}

int pbgpu_server_progress(pbgpu_server* s, pbgpu_result* out, int cap, int* n_out) {
  if (!s || (cap > 0 && !out)) return PBGPU_ERR_ARG;
  if (n_out) *n_out = 0;
  if (s->opts.mode == 1) {
    int dummy = 0;
    return progress_concurrent(s, out, cap, n_out ? n_out : &dummy);
  }
  int st;
  if (!s->in_session) {
    if ((st = pbgpu_batch_begin(s->batch, &s->opts.solver)) != PBGPU_OK)
      return s->fail(st, std::string("server: ") + pbgpu_batch_last_error(s->batch));
    s->in_session = true;
  }
  // 1. the members of the previous ticks advance on the batch stream ...
  const bool launched = !s->running.empty();
  if (launched && (st = pbgpu_batch_launch(s->batch, s->opts.steps_per_tick)) != PBGPU_OK)
    return s->fail(st, std::string("server: ") + pbgpu_batch_last_error(s->batch));
  // 2. ... while admitted requests are set up on their own contexts, one host
  //    thread each (their host waits overlap)
  struct Admit {
    Pending p;
    pbgpu_ctx* ctx;
    Clock::time_point t_admit;
    int st;
  };
  std::vector<Admit> adm;
  const int room = s->opts.max_members - (int)s->running.size();
  const int max_new = std::min(room, s->opts.admit_per_tick > 0 ? s->opts.admit_per_tick : room);
  int64_t held = held_bytes(s);
  while (!s->queue.empty() && (int)adm.size() < max_new) {
    const Pending& p = s->queue.front();
    const int64_t need = pbgpu_request_bytes_estimate(&p.req);
    if ((double)need > s->opts.hbm_budget_bytes) {
      // alone it already exceeds the budget: reject instead of admitting (it
      // waits in the queue for the next tick if the output array is full)
      if (*n_out >= cap) break;
      out[(*n_out)++] = rejection(p);
      s->queue.pop_front();
      ++s->rejected;
      continue;
    }
    // the idle context whose buffers are closest above the need, else the largest
    int pick = -1;
    for (size_t k = 0; k < s->idle.size(); ++k) {
      const int64_t b = ctx_bytes(s->idle[k]);
      if (pick < 0) {
        pick = (int)k;
        continue;
      }
      const int64_t bp = ctx_bytes(s->idle[pick]);
      const bool fits = b >= need, fits_p = bp >= need;
      if ((fits && (!fits_p || b < bp)) || (!fits && !fits_p && b > bp)) pick = (int)k;
    }
    const int64_t reuse = pick >= 0 ? ctx_bytes(s->idle[pick]) : 0;
    int64_t after = held - reuse + std::max(reuse, need);
    // free idle contexts (largest first, never the picked one) until it fits
    while (after > (int64_t)s->opts.hbm_budget_bytes) {
      int big = -1;
      for (size_t k = 0; k < s->idle.size(); ++k)
        if ((int)k != pick && (big < 0 || ctx_bytes(s->idle[k]) > ctx_bytes(s->idle[big]))) big = (int)k;
      if (big < 0) break;
      after -= ctx_bytes(s->idle[big]);
      held -= ctx_bytes(s->idle[big]);
      s->retired_launches += s->idle[big]->c.launches;
      pbgpu_ctx_destroy(s->idle[big]);
      s->idle.erase(s->idle.begin() + big);
      if (pick > big) --pick;
    }
    if (after > (int64_t)s->opts.hbm_budget_bytes && !(s->running.empty() && adm.empty())) break;
    pbgpu_ctx* ctx = nullptr;
    if (pick >= 0) {
      ctx = s->idle[pick];
      s->idle.erase(s->idle.begin() + pick);
    } else if ((st = pbgpu_ctx_create(&ctx, s->device, nullptr)) != PBGPU_OK) {
      if (launched) pbgpu_batch_wait(s->batch, nullptr);
      return s->fail(st, "server: context creation failed");
    }
    held += std::max(reuse, need) - reuse;
    adm.push_back(Admit{p, ctx, Clock::now(), PBGPU_OK});
    s->queue.pop_front();
  }
  //    and the members that converged last tick compute their energies (as
  //    many as the output array holds), also one host thread each
  const size_t n_fin = std::min(s->finishing.size(), (size_t)std::max(cap - *n_out, 0));
  auto energy_of = [s](Retire& x) {
    if (x.st == PBGPU_OK) x.st = pbgpu_energy(x.r.ctx, s->opts.energy_fast, &x.energy);
  };
  // at most `workers` host threads: a thread waiting in a stream
  // synchronisation spins, and one thread per job oversubscribes the host
  std::vector<std::function<void()>> jobs;
  jobs.reserve(adm.size() + n_fin);
  for (Admit& a : adm) jobs.emplace_back([s, &a] { a.st = setup_request(s, a.ctx, a.p.req); });
  for (size_t k = 0; k < n_fin; ++k) jobs.emplace_back([&energy_of, s, k] { energy_of(s->finishing[k]); });
  if (!jobs.empty()) {
    std::atomic<size_t> next{0};
    auto run = [&jobs, &next] {
      for (size_t k; (k = next.fetch_add(1)) < jobs.size();) jobs[k]();
    };
    const size_t nth = std::min(jobs.size(), (size_t)std::max(1, s->opts.workers));
    std::vector<std::thread> th;
    th.reserve(nth - 1);
    for (size_t t = 1; t < nth; ++t) th.emplace_back(run);
    run();
    for (std::thread& t : th) t.join();
  }
  for (size_t k = 0; k < n_fin; ++k) {
    Retire& x = s->finishing[k];
    pbgpu_result& o = out[(*n_out)++];
    std::memset(&o, 0, sizeof(o));
    o.id = x.r.id;
    o.user_tag = x.r.tag;
    o.status = x.st;
    o.stats = x.stats;
    o.energy = x.energy;
    o.latency_ms = ms_since(x.r.t_submit);
    o.queue_ms = std::chrono::duration<double, std::milli>(x.r.t_admit - x.r.t_submit).count();
    s->idle.push_back(x.r.ctx);
    ++s->completed;
  }
  s->finishing.erase(s->finishing.begin(), s->finishing.begin() + n_fin);
  // 3. the batch launch completes
  int active = 0;
  if (launched && (st = pbgpu_batch_wait(s->batch, &active)) != PBGPU_OK)
    return s->fail(st, std::string("server: ") + pbgpu_batch_last_error(s->batch));
  // 4. converged members leave the batch with their potentials; their
  //    energies run during the next tick
  for (size_t k = 0; k < s->running.size();) {
    Running& r = s->running[k];
    int done = 0;
    pbgpu_solve_stats stats{};
    if ((st = pbgpu_batch_member(s->batch, r.slot, &done, &stats)) != PBGPU_OK)
      return s->fail(st, std::string("server: ") + pbgpu_batch_last_error(s->batch));
    if (!done) {
      ++k;
      continue;
    }
    s->finishing.push_back(Retire{r, stats, pbgpu_energy_out{}, stats.status});
    pbgpu_batch_remove(s->batch, r.slot);
    s->running.erase(s->running.begin() + k);
  }
  // 5. the newly set-up requests join the batch (they start next tick)
  for (Admit& a : adm) {
    Running r{a.p.id, a.p.req.user_tag, -1, a.ctx, a.p.req.n_atoms, a.p.t_submit, a.t_admit};
    int stt = a.st;
    if (stt == PBGPU_OK) stt = pbgpu_batch_add(s->batch, a.ctx, &r.slot);
    if (stt != PBGPU_OK) {
      // the request fails alone: report it (if there is room), keep serving
      if (n_out && *n_out < cap) {
        pbgpu_result& o = out[(*n_out)++];
        std::memset(&o, 0, sizeof(o));
        o.id = a.p.id;
        o.user_tag = a.p.req.user_tag;
        o.status = stt;
        o.latency_ms = ms_since(a.p.t_submit);
      }
      s->idle.push_back(a.ctx);
      continue;
    }
    s->running.push_back(r);
    ++s->admitted;
  }
  (void)active;
  return PBGPU_OK;
}

}  // extern "C"
