// Serving: a request loop over the public C-ABI (fe_engine_*, fe_batch_*).
// No counterpart in the reference, which runs one solve per process
// (felbm_gpu_main.cu). One host thread owns the batch:
//  * admission: queued solves are admitted while a slot is free and their
//    footprint fits the budget; creator threads then make them resident
//    (engine created, state uploaded) and hands them to the loop;
//  * scheduling: each chunk runs the resident solves with the least
//    remaining work, up to fill_sites sites, as one batch (the GPU's
//    throughput saturates at a few million sites, so adding more solves to a
//    chunk only slows every member's step rate);
//  * overlap: a prep thread builds the order parameter of each initial state
//    on the host ahead of admission (the device builds the equilibrium
//    state from it), creator threads build engines and a finisher thread
//    reads back retired solves, all on their engines' own streams while
//    chunks run, so the loop thread only launches chunks and changes batch
//    membership; retired engines are freed by the loop after a chunk
//    (freeing device memory waits for the GPU);
//  * retirement: after the step count, or the convergence test.
// Submission and polling only touch the queues under a mutex.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  fe_request r;               // arrays are held by the owned vectors below
  std::vector<uint8_t> solid;
  std::vector<double> h0, g0;  // a given initial state, or
  std::vector<double> c0;      // the order parameter of the built one (equilibrium at rest, init_p)
  int64_t sites = 0;
  double t_submit = 0.0;
  bool ready = false;         // initial state present (given, or built by the prep thread)
  bool preparing = false;
  int prep_status = FE_OK;
  std::string prep_message;
};

struct Live {
  Req q;
  fe_engine* e = nullptr;
  int64_t done = 0;
  double t_admit = 0.0;
  double mass0 = 0.0;
  double last_u = NAN;
  double bytes = 0.0;         // footprint charged to the budget
  bool in_batch = false;
  int status = FE_OK;         // nonzero: failed, report it
};

// mean bytes of an h and a g population
double pop_bytes(int storage) {
  if (storage == FE_F64) return 8;
  if (storage == FE_F32) return 4;
  return (storage == FE_F16G || storage == FE_BF16G) ? 3 : 2;
}
size_t fld_bytes(int storage) { return storage == FE_F64 ? 8 : 4; }

// Device bytes of one resident solve: two buffers of h and g (one with the
// in-place layout), the
// three per-site momentum fields, the stencil fields on the node grid (c, p,
// mu, lap(mu) and the (c', p') pairs: six values a node; the lattice rounded
// up to bricks plus a two-node ring, bounded here by 20 more nodes per axis),
// the FP64 transfer buffer (upload/download), and the site/brick tables
// (generous per-site bound).
double footprint(int64_t n, int nx, int ny, int nz, int storage, int pop_layout = FE_POP_TWO_BUFFERS) {
  const double bufs = pop_layout == FE_POP_IN_PLACE ? 2.0 : 4.0;  // h and g, one or two buffers each
  const double per = bufs * 19 * pop_bytes(storage) + 3.0 * fld_bytes(storage) + 2.0 * 19 * 8 + 64;
  const double cells = (double)(nx + 20) * (double)(ny + 20) * (double)(nz == 1 ? 1 : nz + 20);
  return (double)n * per + 6.0 * cells * (double)fld_bytes(storage) + (double)(64 << 20);
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t lo = (size_t)std::floor(pos), hi = std::min(v.size() - 1, lo + 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

struct fe_server {
  fe_server_config cfg{};
  fe_batch* batch = nullptr;
  Clock::time_point t0;
  std::thread th, finisher;
  std::vector<std::thread> preps, creators;  // host work of several solves at once
  std::mutex mu;
  std::condition_variable cv;       // loop: a prepared solve is queued, a solve was created or read back / stop
  std::condition_variable cv_prep;  // a solve needs its initial state / stop
  std::condition_variable cv_make;  // creator: an admitted solve waits for its engine / stop
  std::condition_variable cv_read;  // finisher: a retired solve waits to be read back / stop
  std::condition_variable cv_idle;  // queue and resident set drained
  std::deque<Req> queue;
  std::vector<Live> live;           // resident solves in the loop (loop thread only)
  std::deque<Live> to_create;       // admitted, engine not built yet (under mu)
  std::vector<Live> created;        // engine built, not yet in the loop (under mu)
  std::deque<Live> to_read;         // stepped out, results not read back yet (under mu)
  std::vector<Live> to_free;        // read back; engines freed after the chunk (under mu)
  int64_t holding = 0;              // admitted solves whose memory is not released (under mu)
  std::vector<fe_result> finished;
  bool stop = false;
  double budget = 0.0, committed = 0.0, reserve = 0.0;
  // statistics (under mu)
  int64_t submitted = 0, admitted = 0, completed = 0, active = 0, peak_active = 0, site_steps = 0;
  double busy = 0.0;
  std::vector<double> ttr;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  void report(fe_result& r, bool ok) {
    std::lock_guard<std::mutex> g(mu);
    finished.push_back(r);
    if (ok) ttr.push_back(r.t_done - r.t_submit);
    ++completed;
    --active;
  }

  fe_result base_result(const Live& L) const {
    fe_result r{};
    r.id = L.q.r.id;
    r.sites = L.q.sites;
    r.steps_done = L.done;
    r.t_submit = L.q.t_submit;
    r.t_admit = L.t_admit;
    r.mass0 = L.mass0;
    return r;
  }

  void release(Live& L) {
    if (L.e) fe_engine_destroy(L.e);  // leaves the batch first
    L.e = nullptr;
    std::lock_guard<std::mutex> g(mu);
    committed -= L.bytes;
    L.bytes = 0.0;
    --holding;
  }

  void fail(Live& L, int status) {
    fe_result r = base_result(L);
    r.status = status;
    std::snprintf(r.message, sizeof(r.message), "%s", fe_last_error());
    release(L);
    r.t_done = now();
    report(r, false);
  }

  // Results of a retired solve (its engine is out of the batch).
  void read_back(Live& L) {
    fe_result r = base_result(L);
    int rc = fe_flow_stats(L.e, r.stats);
    if (!rc) rc = fe_current_mass(L.e, &r.mass_final);
    if (!rc && L.q.r.want_fields) {
      const size_t nb = std::max<size_t>((size_t)L.q.sites * sizeof(double), 8);
      double** dst[6] = {&r.rho, &r.c, &r.ux, &r.uy, &r.uz, &r.p};
      for (double** d : dst) {
        *d = static_cast<double*>(std::malloc(nb));
        if (!*d) rc = FE_ERR_MEMORY;
      }
      fe_fields f{r.rho, r.c, r.ux, r.uy, r.uz, r.p, nullptr};
      if (!rc) rc = fe_download_fields(L.e, &f);
    }
    if (rc) {
      r.status = rc;
      std::snprintf(r.message, sizeof(r.message), "%s", fe_last_error());
    }
    r.t_done = now();
    report(r, rc == FE_OK);
  }

  // Creates the engine of an admitted solve and uploads its state.
  bool make_resident(Live& L) {
    Req& q = L.q;
    fe_params p = q.r.params;
    p.storage = cfg.storage;
    p.pop_layout = cfg.pop_layout;
    if (q.prep_status) {
      fail(L, fe_fail(q.prep_status, q.prep_message));
      return false;
    }
    int rc = fe_engine_create(&p, q.r.nx, q.r.ny, q.r.nz, q.solid.data(), cfg.device, &L.e);
    if (rc) { fail(L, rc); return false; }
    if (!q.c0.empty())  // built on the device from c (n values across the link, not 38n)
      rc = fe_upload_equilibrium(L.e, q.c0.data(), nullptr, q.r.init_p, q.sites);
    else
      rc = fe_upload_state(L.e, q.h0.data(), q.g0.data(), 19 * q.sites);
    if (rc) { fail(L, rc); return false; }
    std::vector<double>().swap(q.h0);  // the state lives on the device now
    std::vector<double>().swap(q.g0);
    std::vector<double>().swap(q.c0);
    std::vector<uint8_t>().swap(q.solid);
    if (p.correct_op_mass && (rc = fe_record_target_mass(L.e))) { fail(L, rc); return false; }
    if ((rc = fe_current_mass(L.e, &L.mass0))) { fail(L, rc); return false; }
    return true;
  }

  // Builds the order parameter of queued solves' initial states (oldest
  // first) on the host, ahead of their admission; the creator thread uploads
  // it and the device builds the equilibrium state from it. Queue elements
  // stay in place: the loop pops only ready ones.
  void prep_loop() {
    for (;;) {
      Req* q = nullptr;
      {
        std::unique_lock<std::mutex> g(mu);
        auto next = [&]() -> Req* {
          for (Req& r : queue)
            if (!r.ready && !r.preparing) return &r;
          return nullptr;
        };
        cv_prep.wait(g, [&] { return stop || next() != nullptr; });
        if (stop) return;
        q = next();
        q->preparing = true;
      }
      std::vector<double> c(q->sites);
      const int rc = fe_init_order_parameter(q->solid.data(), q->r.nx, q->r.ny, q->r.nz, q->r.init_kind,
                                             q->r.init_a, q->r.init_width, c.data());
      std::lock_guard<std::mutex> g(mu);
      q->c0.swap(c);
      q->prep_status = rc;
      if (rc) q->prep_message = fe_last_error();
      q->preparing = false;
      q->ready = true;
      cv.notify_all();
    }
  }

  bool fits(const Req& q) {  // under mu
    if (cfg.max_active > 0 && holding >= cfg.max_active) return false;
    const double need = footprint(q.sites, q.r.nx, q.r.ny, q.r.nz, cfg.storage, cfg.pop_layout);
    if (committed + need > budget) return false;
    size_t fr = 0, tot = 0;  // memory other users took since the server started
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return (double)fr - need >= reserve;
  }

  // Admits queued solves (oldest first) while they fit: their memory is
  // charged and the creator thread builds their engines. Under mu.
  void admit_locked() {
    while (!stop && !queue.empty() && queue.front().ready) {
      // with nothing held, the oldest solve is admitted even if its estimate
      // exceeds the budget: engine creation then reports an out-of-memory
      // failure for it instead of a queue that never moves
      if (!fits(queue.front()) && holding > 0) return;
      Live L;
      L.q = std::move(queue.front());
      queue.pop_front();
      ++admitted;
      ++active;
      peak_active = std::max(peak_active, active);
      L.t_admit = now();
      L.bytes = footprint(L.q.sites, L.q.r.nx, L.q.r.ny, L.q.r.nz, cfg.storage, cfg.pop_layout);
      committed += L.bytes;
      ++holding;
      to_create.push_back(std::move(L));
      cv_make.notify_all();
    }
  }

  void creator_loop() {
    cudaSetDevice(cfg.device);
    for (;;) {
      Live L;
      {
        std::unique_lock<std::mutex> g(mu);
        cv_make.wait(g, [&] { return stop || !to_create.empty(); });
        if (stop) return;
        L = std::move(to_create.front());
        to_create.pop_front();
      }
      if (make_resident(L)) {
        std::lock_guard<std::mutex> g(mu);
        created.push_back(std::move(L));
        cv.notify_all();
      } else {
        std::lock_guard<std::mutex> g(mu);
        cv.notify_all();
      }
    }
  }

  void finisher_loop() {
    cudaSetDevice(cfg.device);
    for (;;) {
      Live L;
      {
        std::unique_lock<std::mutex> g(mu);
        cv_read.wait(g, [&] { return stop || !to_read.empty(); });
        if (stop) return;
        L = std::move(to_read.front());
        to_read.pop_front();
      }
      read_back(L);
      std::lock_guard<std::mutex> g(mu);
      to_free.push_back(std::move(L));
      cv.notify_all();
    }
  }

  // Engines of read-back solves (loop thread, outside a running chunk).
  void free_retired() {
    std::vector<Live> v;
    {
      std::lock_guard<std::mutex> g(mu);
      v.swap(to_free);
    }
    for (Live& L : v) release(L);
  }

  // The chunk's running set: least remaining work first, up to fill_sites.
  // latency_first also caps it at the sites that keep the step of the solve
  // with the least remaining work within twice its step alone: a step costs
  // about a launch floor plus sites / rate, the floor worth STEP_FLOOR_SITES
  // sites on a B200 (about 25 us at 5 G site updates a second), so that cap
  // is 2 s1 + STEP_FLOOR_SITES. Small requests then finish at about their
  // own step rate instead of a large member's; a backlog of many solves
  // submitted at once loses throughput to the smaller chunks.
  static constexpr int64_t STEP_FLOOR_SITES = 131072;
  std::vector<int> choose() {
    std::vector<int> idx(live.size());
    for (size_t q = 0; q < live.size(); ++q) idx[q] = (int)q;
    auto work = [&](int q) { return (double)live[q].q.sites * (double)(live[q].q.r.steps - live[q].done); };
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return work(a) < work(b); });
    std::vector<int> run;
    int64_t sites = 0, cap = cfg.fill_sites;
    if (cfg.latency_first && cap > 0 && !idx.empty())
      cap = std::min<int64_t>(cap, 2 * live[idx[0]].q.sites + STEP_FLOOR_SITES);
    for (int q : idx) {
      if (!run.empty() && cap > 0 && sites + live[q].q.sites > cap) continue;
      run.push_back(q);
      sites += live[q].q.sites;
    }
    return run;
  }

  void loop() {
    cudaSetDevice(cfg.device);
    {
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) cudaGetLastError();
      std::lock_guard<std::mutex> g(mu);
      reserve = cfg.hbm_reserve_frac * (double)tot;
      budget = (double)fr - reserve;
    }
    for (;;) {
      free_retired();
      {
        std::unique_lock<std::mutex> g(mu);
        if (stop) break;
        admit_locked();
        for (Live& L : created) live.push_back(std::move(L));
        created.clear();
        if (live.empty()) {
          if (queue.empty() && to_create.empty() && to_read.empty() && active == 0) cv_idle.notify_all();
          cv.wait(g, [&] {
            return stop || !created.empty() || !to_free.empty() ||
                   (!queue.empty() && queue.front().ready && (holding == 0 || fits(queue.front())));
          });
          continue;
        }
      }
      // batch membership of this chunk
      const std::vector<int> run = choose();
      std::vector<char> sel(live.size(), 0);
      for (int q : run) sel[q] = 1;
      for (size_t q = 0; q < live.size(); ++q)
        if (live[q].in_batch && !sel[q]) {
          fe_batch_remove(batch, live[q].e);
          live[q].in_batch = false;
        }
      int64_t chunk = cfg.chunk_steps, sites = 0;
      for (int q : run) {
        Live& L = live[q];
        if (!L.in_batch) {
          const int rc = fe_batch_add(batch, L.e);
          if (rc) L.status = rc;
          else L.in_batch = true;
        }
        chunk = std::min(chunk, L.q.r.steps - L.done);
        sites += L.q.sites;
      }
      chunk = std::max<int64_t>(chunk, 1);
      const double tb = now();
      int rc = fe_batch_launch(batch, (int)chunk);
      {  // while the chunk runs: admit what fits now
        std::lock_guard<std::mutex> g(mu);
        admit_locked();
      }
      if (!rc) rc = fe_batch_wait(batch);
      const double te = now();
      if (rc) {  // the batch failed: report every solve of the chunk
        for (int q : run) live[q].status = rc;
      } else {
        std::lock_guard<std::mutex> g(mu);
        busy += te - tb;
        site_steps += sites * chunk;
      }
      std::vector<Live> keep;
      for (size_t q = 0; q < live.size(); ++q) {
        Live& L = live[q];
        if (L.status) {
          fail(L, L.status);
          continue;
        }
        bool ret = false;
        if (sel[q]) {
          L.done += chunk;
          ret = L.done >= L.q.r.steps;
          if (!ret && L.q.r.conv_tol > 0.0) {
            double st[6];
            if (fe_flow_stats(L.e, st) == FE_OK) {
              const double u = std::sqrt(st[0] * st[0] + st[1] * st[1] + st[2] * st[2]) / (double)L.q.sites;
              if (std::isfinite(L.last_u) &&
                  std::fabs(u - L.last_u) <= L.q.r.conv_tol * std::max(std::fabs(u), 1e-300))
                ret = true;
              L.last_u = u;
            }
          }
        }
        if (ret) {
          fe_batch_remove(batch, L.e);
          L.in_batch = false;
          std::lock_guard<std::mutex> g(mu);
          to_read.push_back(std::move(L));
          cv_read.notify_all();
        } else {
          keep.push_back(std::move(L));
        }
      }
      live.swap(keep);
    }
    for (Live& L : live) {
      if (L.in_batch) fe_batch_remove(batch, L.e);
      release(L);
    }
    live.clear();
    std::lock_guard<std::mutex> g(mu);
    cv_idle.notify_all();
  }
};

extern "C" {

int fe_server_create(const fe_server_config* cfg, fe_server** out) {
  if (!cfg || !out) return fe_fail(FE_ERR_ARG, "fe_server_create: bad arguments");
  if (cfg->chunk_steps < 1) return fe_fail(FE_ERR_ARG, "chunk_steps must be > 0");
  if (cfg->storage < FE_F64 || cfg->storage > FE_BF16G) return fe_fail(FE_ERR_ARG, "unknown storage");
  if (cfg->pop_layout == FE_POP_IN_PLACE && cfg->storage != FE_F64 && cfg->storage != FE_F32)
    return fe_fail(FE_ERR_ARG, "the in-place population layout takes FE_F64 or FE_F32 storage");
  if (cfg->pop_layout != FE_POP_TWO_BUFFERS && cfg->pop_layout != FE_POP_IN_PLACE)
    return fe_fail(FE_ERR_ARG, "unknown pop_layout");
  if (cfg->hbm_reserve_frac < 0.0 || cfg->hbm_reserve_frac >= 1.0)
    return fe_fail(FE_ERR_ARG, "hbm_reserve_frac must be in [0, 1)");
  *out = nullptr;
  fe_server* s = new (std::nothrow) fe_server();
  if (!s) return fe_fail(FE_ERR_MEMORY, "host allocation");
  s->cfg = *cfg;
  const int rc = fe_batch_create(cfg->device, &s->batch);
  if (rc) {
    delete s;
    return rc;
  }
  s->t0 = Clock::now();
  s->th = std::thread([s] { s->loop(); });
  for (int k = 0; k < 1; ++k) s->preps.emplace_back([s] { s->prep_loop(); });
  for (int k = 0; k < 1; ++k) s->creators.emplace_back([s] { s->creator_loop(); });
  s->finisher = std::thread([s] { s->finisher_loop(); });
  *out = s;
  return FE_OK;
}

int fe_server_submit(fe_server* s, const fe_request* r) {
  if (!s || !r) return fe_fail(FE_ERR_ARG, "fe_server_submit: bad arguments");
  if (!r->solid || r->nx < 1 || r->ny < 1 || r->nz < 1 || r->steps < 1)
    return fe_fail(FE_ERR_ARG, "fe_server_submit: bad request");
  if ((r->h0 == nullptr) != (r->g0 == nullptr)) return fe_fail(FE_ERR_ARG, "give both h0 and g0, or neither");
  Req q;
  q.r = *r;
  const size_t nodes = (size_t)r->nx * r->ny * r->nz;
  q.solid.assign(r->solid, r->solid + nodes);
  int64_t n = 0;
  const int rc = fe_geom_sites(q.solid.data(), r->nx, r->ny, r->nz, &n, nullptr);
  if (rc) return rc;
  if (n == 0) return fe_fail(FE_ERR_ARG, "request geometry has no fluid site");
  q.sites = n;
  if (r->h0) {
    q.h0.assign(r->h0, r->h0 + 19 * n);
    q.g0.assign(r->g0, r->g0 + 19 * n);
    q.ready = true;
  }
  q.r.solid = nullptr;  // the copies above are used
  q.r.h0 = q.r.g0 = nullptr;
  std::lock_guard<std::mutex> g(s->mu);
  q.t_submit = s->now();
  s->queue.push_back(std::move(q));
  ++s->submitted;
  s->cv.notify_all();
  s->cv_prep.notify_all();
  return FE_OK;
}

int fe_server_poll(fe_server* s, fe_result* out, int max, int* n) {
  if (!s || !n || (max > 0 && !out)) return fe_fail(FE_ERR_ARG, "fe_server_poll: bad arguments");
  std::lock_guard<std::mutex> g(s->mu);
  const int k = std::max(0, std::min<int>(max, (int)s->finished.size()));
  for (int q = 0; q < k; ++q) out[q] = s->finished[q];
  s->finished.erase(s->finished.begin(), s->finished.begin() + k);
  *n = k;
  return FE_OK;
}

int fe_server_free_result(fe_result* r) {
  if (!r) return FE_OK;
  double** f[6] = {&r->rho, &r->c, &r->ux, &r->uy, &r->uz, &r->p};
  for (double** d : f) {
    std::free(*d);
    *d = nullptr;
  }
  return FE_OK;
}

int fe_server_wait_idle(fe_server* s, double timeout_s) {
  if (!s) return fe_fail(FE_ERR_ARG, "null server");
  std::unique_lock<std::mutex> g(s->mu);
  const bool ok = s->cv_idle.wait_for(g, std::chrono::duration<double>(timeout_s),
                                      [&] { return s->queue.empty() && s->active == 0; });
  return ok ? FE_OK : fe_fail(FE_ERR_STATE, "fe_server_wait_idle: timeout");
}

int fe_server_get_stats(fe_server* s, fe_server_stats* st) {
  if (!s || !st) return fe_fail(FE_ERR_ARG, "fe_server_get_stats: bad arguments");
  std::lock_guard<std::mutex> g(s->mu);
  *st = fe_server_stats{};
  st->submitted = s->submitted;
  st->admitted = s->admitted;
  st->completed = s->completed;
  st->queued = (int64_t)s->queue.size();
  st->active = s->active;
  st->peak_active = s->peak_active;
  st->site_steps = s->site_steps;
  st->busy_seconds = s->busy;
  st->elapsed_seconds = s->now();
  st->mlups_busy = s->busy > 0 ? (double)s->site_steps / s->busy / 1e6 : 0.0;
  st->mlups_wall = st->elapsed_seconds > 0 ? (double)s->site_steps / st->elapsed_seconds / 1e6 : 0.0;
  st->ttr_p50 = percentile(s->ttr, 0.50);
  st->ttr_p99 = percentile(s->ttr, 0.99);
  st->ttr_max = s->ttr.empty() ? 0.0 : *std::max_element(s->ttr.begin(), s->ttr.end());
  return FE_OK;
}

int fe_server_destroy(fe_server* s) {
  if (!s) return FE_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->cv.notify_all();
    s->cv_prep.notify_all();
    s->cv_make.notify_all();
    s->cv_read.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  for (std::thread& t : s->preps) t.join();
  for (std::thread& t : s->creators) t.join();
  if (s->finisher.joinable()) s->finisher.join();
  // solves caught between the threads at shutdown
  for (Live& L : s->created) s->release(L);
  for (Live& L : s->to_read) s->release(L);
  for (Live& L : s->to_free) s->release(L);
  for (fe_result& r : s->finished) fe_server_free_result(&r);
  fe_batch_destroy(s->batch);
  delete s;
  return FE_OK;
}

}  // extern "C"
