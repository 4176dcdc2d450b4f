// server.cu -- the solve server: continuous batching of scattering solves.
//
// The reference solves one system per blocking call (examples/
// scattering_film.jl:58-61); this server takes solve requests of any self
// volume as they arrive and keeps the GPU busy with all of them:
//
//  * one scheduler thread owns every batch (solver.h): per volume shape a
//    set of right-hand-side slots on its own CUDA stream, with the shape's
//    ComplexF64 / ComplexF32 operators and the Krylov vectors resident;
//  * a request joins its shape's batch at the next Krylov-cycle boundary as
//    soon as a slot is free (continuous batching); batches of different
//    shapes overlap on their streams;
//  * admission is by device memory: a shape's operators and batch are
//    allocated only when they fit the HBM budget; idle batches and operators
//    of shapes nobody is waiting for are freed, least recently used first;
//  * operators are built on the GPU by a builder thread so that the
//    scheduler never stalls on a kernel build.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"
#include "solver.h"

namespace gila {
namespace {

using Clock = std::chrono::steady_clock;

struct ShapeKey {
  int64_t v[9];  // cells, scale numerators, scale denominators
  bool operator<(const ShapeKey& o) const { return std::lexicographical_compare(v, v + 9, o.v, o.v + 9); }
};

struct Request {
  uint64_t ticket = 0;
  ShapeKey key{};
  gila_vol vol{};
  const void* chi = nullptr;
  const void* b = nullptr;
  void* x = nullptr;
  SlotOpts so;
  Clock::time_point t0;
};

struct Ticket {
  bool done = false;
  gila_status status = GILA_OK;
  std::string err;
  gila_solve_info info{};
  double latency_ms = 0.0;
};

enum class OpState { None, Building, Ready, Failed };

struct Shape {
  ShapeKey key{};
  gila_vol vol{};
  OpState op = OpState::None;  // guarded by Server::mu
  std::string err;
  std::shared_ptr<Core> g64, g32;
  size_t op_bytes = 0;    // estimate charged while building, then the real size
  size_t build_tmp = 0;   // transient bytes of the build
  std::unique_ptr<LsBatch> batch;
  size_t batch_bytes = 0;
  std::map<int, Request> slot_req;
  Clock::time_point last_use;
};

size_t self_op_bytes(const gila_vol& v, bool mixed) {
  size_t k = 48;  // 8 branches x 6 components
  for (int d = 0; d < 3; ++d) {
    const int64_t n = v.cel[d];
    k *= (size_t)std::max<int64_t>((n + 1) / 2 + (n % 2 == 0 ? 1 : 0), 2);
  }
  return k * (16 + (mixed ? 8 : 0));
}

// Stream priority of a shape's batch: volumes of at most 2^17 cells get the
// device's highest priority, up to 2^19 cells the next one, larger volumes
// the default, which they share.  A small request's Krylov cycle (tens of
// microseconds of kernels) then waits for free SMs, not behind a large
// batch's queued kernels; large shapes are not ranked among themselves (a
// large shape below another one would starve: its cycles are long and the
// other's never stop).  GILA_SERVER_PRIORITY=0 gives every batch the default
// priority.
int shape_priority(const gila_vol& v) {
  static const bool on = [] {
    const char* e = getenv("GILA_SERVER_PRIORITY");
    return !(e && e[0] == '0');
  }();
  if (!on) return 0;
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  double cells = 1.0;
  for (int d = 0; d < 3; ++d) cells *= (double)v.cel[d];
  if (cells > (double)(1 << 19)) return least;
  const int p = greatest + (cells > (double)(1 << 17) ? 1 : 0);
  return p > least ? least : p;
}

size_t build_tmp_bytes(const gila_vol& v) {
  size_t p = 1, c = 1;
  for (int d = 0; d < 3; ++d) {
    p *= (size_t)(2 * v.cel[d]);
    c *= (size_t)v.cel[d];
  }
  return 6 * p * 16 + 6 * c * 16 + (64ull << 20);
}

}  // namespace

struct Server {
  gila_ctx* ctx = nullptr;
  int device = 0;
  gila_server_opts o{};
  BatchCfg cfg;
  gila_kopt kopt{};
  size_t budget = 0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_build;
  std::deque<Request> incoming;         // submitted, not yet taken by the scheduler
  std::map<uint64_t, Ticket> tickets;
  std::deque<Shape*> build_q;
  uint64_t next_ticket = 1;
  bool stop = false;
  int64_t n_submitted = 0, n_completed = 0;
  size_t used = 0;                      // charged device bytes (operators, builds, batches)

  // scheduler-thread state (shapes are also read by the builder via build_q)
  std::deque<Request> pending;
  std::map<ShapeKey, std::unique_ptr<Shape>> shapes;
  int64_t running = 0;
  // copies of the scheduler's counts for gila_server_stats_get (guarded by mu)
  int64_t c_pending = 0, c_running = 0, c_batches = 0, c_ops = 0;

  std::thread th_sched, th_build;

  void builder() {
    cudaSetDevice(device);
    for (;;) {
      Shape* sh = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_build.wait(lk, [&] { return stop || !build_q.empty(); });
        if (stop) return;
        sh = build_q.front();
        build_q.pop_front();
      }
      std::shared_ptr<Core> g64, g32;
      gila_status s = init_core(ctx, &sh->vol, nullptr, &kopt, GILA_C128, g64);
      if (s == GILA_OK) s = build_kernel(*g64);
      if (s == GILA_OK && cfg.mixed) s = cast_core(ctx, *g64, GILA_C64, g32);
      // launch shapes timed here, off the scheduler thread; the tuning
      // workspaces are released (batches own theirs)
      for (Core* c : {g64.get(), g32.get()})
        if (s == GILA_OK && c) {
          s = ensure_tuned(*c, 1);
          release_work(*c);
        }
      std::string err = s == GILA_OK ? "" : std::string(gila_last_error());
      {
        std::lock_guard<std::mutex> lk(mu);
        used -= sh->build_tmp;
        sh->build_tmp = 0;
        if (s == GILA_OK) {
          used -= sh->op_bytes;
          sh->op_bytes = g64->ker_bytes + (g32 ? g32->ker_bytes : 0);
          used += sh->op_bytes;
          sh->g64 = g64;
          sh->g32 = g32;
          sh->op = OpState::Ready;
        } else {
          used -= sh->op_bytes;
          sh->op_bytes = 0;
          sh->op = OpState::Failed;
          sh->err = err;
        }
      }
      cv_work.notify_all();
    }
  }

  void complete(const Request& rq, gila_status st, const std::string& err, const gila_solve_info& inf) {
    const double ms = std::chrono::duration<double, std::milli>(Clock::now() - rq.t0).count();
    {
      std::lock_guard<std::mutex> lk(mu);
      Ticket& t = tickets[rq.ticket];
      t.done = true;
      t.status = st;
      t.err = err;
      t.info = inf;
      t.latency_ms = ms;
      ++n_completed;
    }
    cv_done.notify_all();
  }

  // free idle batches and unused operators until `need` more bytes fit;
  // shapes that requests older than `upto` wait for are kept (first come,
  // first served)
  bool make_room(size_t need, const Shape* keep, std::deque<Request>::iterator upto) {
    for (;;) {
      {
        std::lock_guard<std::mutex> lk(mu);
        if (used + need <= budget) return true;
      }
      Shape* victim = nullptr;
      for (auto& kv : shapes) {
        Shape* s = kv.second.get();
        if (s == keep || !s->slot_req.empty()) continue;
        if (s->batch && s->batch->in_flight()) continue;
        bool wanted = false;
        for (auto r = pending.begin(); r != upto; ++r) wanted |= !(r->key < s->key) && !(s->key < r->key);
        if (wanted) continue;
        std::lock_guard<std::mutex> lk(mu);
        if (s->op == OpState::Building) continue;
        if (!s->batch && s->op != OpState::Ready) continue;
        if (!victim || s->last_use < victim->last_use) victim = s;
      }
      if (!victim) return false;
      std::lock_guard<std::mutex> lk(mu);
      if (victim->batch) {
        victim->batch.reset();
        used -= victim->batch_bytes;
        victim->batch_bytes = 0;
      } else {
        victim->g64.reset();
        victim->g32.reset();
        used -= victim->op_bytes;
        victim->op_bytes = 0;
        victim->op = OpState::None;
      }
    }
  }

  // place pending requests into free slots (FIFO within each shape)
  void admit() {
    for (auto it = pending.begin(); it != pending.end();) {
      Request& rq = *it;
      auto& up = shapes[rq.key];
      if (!up) {
        up = std::make_unique<Shape>();
        up->key = rq.key;
        up->vol = rq.vol;
        up->last_use = Clock::now();
      }
      Shape* sh = up.get();
      OpState ops;
      {
        std::lock_guard<std::mutex> lk(mu);
        ops = sh->op;
      }
      if (ops == OpState::Failed) {
        gila_solve_info inf{};
        complete(rq, GILA_ERR_ARG, "operator build failed: " + sh->err, inf);
        it = pending.erase(it);
        continue;
      }
      if (ops == OpState::None) {
        const size_t est = self_op_bytes(rq.vol, cfg.mixed != 0), tmp = build_tmp_bytes(rq.vol);
        if (!make_room(est + tmp, sh, it)) {
          ++it;
          continue;
        }
        std::lock_guard<std::mutex> lk(mu);
        sh->op = OpState::Building;
        sh->op_bytes = est;
        sh->build_tmp = tmp;
        used += est + tmp;
        build_q.push_back(sh);
        cv_build.notify_one();
        ++it;
        continue;
      }
      if (ops == OpState::Building) {
        ++it;
        continue;
      }
      if (!sh->batch) {
        // largest slot count that fits the budget
        int S = o.slots;
        size_t need = 0;
        for (; S >= 1; S /= 2) {
          need = ls_batch_bytes(*sh->g64, sh->g32.get(), S, cfg);
          if (make_room(need, sh, it)) break;
        }
        if (S < 1) {
          ++it;
          continue;
        }
        std::unique_ptr<LsBatch> b;
        BatchCfg bc = cfg;
        bc.priority = shape_priority(sh->vol);
        const gila_status s = make_ls_batch(*sh->g64, sh->g32.get(), S, bc, b);
        if (s != GILA_OK) {
          gila_solve_info inf{};
          complete(rq, s, gila_last_error(), inf);
          it = pending.erase(it);
          continue;
        }
        sh->batch = std::move(b);
        sh->batch_bytes = need;
        std::lock_guard<std::mutex> lk(mu);
        used += need;
      }
      if (sh->batch->in_flight()) {
        ++it;
        continue;
      }
      const int slot = sh->batch->free_slot();
      if (slot < 0) {
        ++it;
        continue;
      }
      const gila_status s = sh->batch->assign(slot, rq.chi, rq.b, rq.x, rq.so, rq.ticket);
      if (s != GILA_OK) {
        gila_solve_info inf{};
        complete(rq, s, gila_last_error(), inf);
        it = pending.erase(it);
        continue;
      }
      sh->slot_req[slot] = rq;
      sh->last_use = Clock::now();
      ++running;
      it = pending.erase(it);
    }
  }

  void scheduler() {
    cudaSetDevice(device);
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        if (stop) break;
        while (!incoming.empty()) {
          pending.push_back(incoming.front());
          incoming.pop_front();
        }
      }
      bool progressed = false;
      // finished steps: digest, report released slots, enqueue the next step
      for (auto& kv : shapes) {
        Shape* sh = kv.second.get();
        if (!sh->batch || !sh->batch->ready()) continue;
        bool enq = false;
        const gila_status s = sh->batch->advance(&enq);
        for (const SlotResult& r : sh->batch->take_finished()) {
          auto f = sh->slot_req.find(r.slot);
          if (f == sh->slot_req.end()) continue;
          gila_solve_info inf{};
          inf.iters = r.cycles;
          inf.outer = r.updates;
          inf.rel_res = r.rel_res;
          inf.converged = r.converged;
          inf.breakdowns = r.broke;
          complete(f->second, r.converged ? GILA_OK : GILA_ERR_NOTCONV, "", inf);
          sh->slot_req.erase(f);
          --running;
          progressed = true;
        }
        if (s != GILA_OK) {
          // a failed step: every request of the batch fails, the batch goes
          const std::string err = gila_last_error();
          for (auto& q : sh->slot_req) {
            gila_solve_info inf{};
            complete(q.second, s, err, inf);
            --running;
          }
          sh->slot_req.clear();
          sh->batch.reset();
          std::lock_guard<std::mutex> lk(mu);
          used -= sh->batch_bytes;
          sh->batch_bytes = 0;
          continue;
        }
        progressed |= enq;
      }
      // new requests join at step boundaries
      if (!pending.empty()) {
        const size_t before = pending.size();
        admit();
        progressed |= pending.size() != before;
        for (auto& kv : shapes) {
          Shape* sh = kv.second.get();
          if (!sh->batch || sh->batch->in_flight()) continue;
          bool enq = false;
          if (sh->batch->advance(&enq) == GILA_OK && enq) progressed = true;
        }
      }
      {
        int64_t nb = 0, nops = 0;
        for (auto& kv : shapes) nb += kv.second->batch ? 1 : 0;
        std::lock_guard<std::mutex> lk(mu);
        for (auto& kv : shapes) nops += kv.second->op == OpState::Ready ? 1 : 0;
        c_pending = (int64_t)pending.size();
        c_running = running;
        c_batches = nb;
        c_ops = nops;
      }
      if (!progressed) {
        std::unique_lock<std::mutex> lk(mu);
        bool busy = false;
        for (auto& kv : shapes) busy |= kv.second->batch && kv.second->batch->in_flight();
        if (busy)
          cv_work.wait_for(lk, std::chrono::microseconds(50));
        else
          cv_work.wait_for(lk, std::chrono::milliseconds(5), [&] { return stop || !incoming.empty(); });
      }
    }
    // shutdown: let every batch's stream drain
    for (auto& kv : shapes)
      if (kv.second->batch) kv.second->batch->wait();
  }
};

}  // namespace gila

using namespace gila;

struct gila_server {
  Server* impl;
};

extern "C" {

gila_status gila_server_create(gila_ctx* ctx, const gila_server_opts* opts, gila_server** out) {
  if (!ctx || !out) return fail(GILA_ERR_ARG, "null argument");
  GILA_CUDA_TRY(cudaSetDevice(ctx->impl->device));
  auto* sv = new Server;
  sv->ctx = ctx;
  sv->device = ctx->impl->device;
  if (opts) sv->o = *opts;
  if (sv->o.slots <= 0) sv->o.slots = 8;
  sv->cfg.ell = sv->o.ell > 0 ? sv->o.ell : 2;
  sv->cfg.mixed = sv->o.mixed != 0;
  sv->cfg.graph = 1;
  sv->cfg.chi_shared = 0;
  if (sv->cfg.ell > 4) {
    delete sv;
    return fail(GILA_ERR_ARG, "BiCGStab(l) degree must be 1..4");
  }
  sv->kopt.frq_re = (sv->o.frq_re == 0.0 && sv->o.frq_im == 0.0) ? 1.0 : sv->o.frq_re;
  sv->kopt.frq_im = sv->o.frq_im;
  sv->kopt.int_ord = sv->o.int_ord > 0 ? sv->o.int_ord : 32;
  sv->kopt.dev_mod = 1;
  if (sv->o.hbm_budget > 0) {
    sv->budget = (size_t)sv->o.hbm_budget;
  } else {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    sv->budget = fr > (4ull << 30) ? fr - (4ull << 30) : fr / 2;
  }
  sv->th_build = std::thread([sv] { sv->builder(); });
  sv->th_sched = std::thread([sv] { sv->scheduler(); });
  auto* h = new gila_server;
  h->impl = sv;
  *out = h;
  return GILA_OK;
}

gila_status gila_server_destroy(gila_server* srv) {
  if (!srv) return GILA_OK;
  Server* sv = srv->impl;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  sv->cv_build.notify_all();
  sv->th_sched.join();
  sv->th_build.join();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (auto& kv : sv->tickets)
      if (!kv.second.done) {
        kv.second.done = true;
        kv.second.status = GILA_ERR_ARG;
        kv.second.err = "server destroyed";
      }
  }
  sv->cv_done.notify_all();
  sv->shapes.clear();
  delete sv;
  delete srv;
  return GILA_OK;
}

gila_status gila_server_submit(gila_server* srv, const gila_vol* vol, const void* chi, const void* b, void* x,
                               const gila_solve_opts* opts, uint64_t* ticket) {
  if (!srv || !vol || !chi || !b || !x || !ticket) return fail(GILA_ERR_ARG, "null argument");
  Server* sv = srv->impl;
  Request rq;
  rq.vol = *vol;
  for (int d = 0; d < 3; ++d) {
    if (vol->cel[d] <= 0) return fail(GILA_ERR_ARG, "cell counts must be positive");
    if (vol->scl_den[d] == 0 || vol->scl_num[d] <= 0) return fail(GILA_ERR_ARG, "cell scales must be positive");
    const Rat r = rat(vol->scl_num[d], vol->scl_den[d]);
    rq.key.v[d] = vol->cel[d];
    rq.key.v[3 + d] = r.n;
    rq.key.v[6 + d] = r.d;
    rq.vol.org_num[d] = 0;
    rq.vol.org_den[d] = 1;
    rq.vol.grd_num[d] = r.n;
    rq.vol.grd_den[d] = r.d;
  }
  {
    const int64_t V = vol->cel[0] * vol->cel[1] * vol->cel[2];
    gila_status s = check_finite(chi, V, "The medium (chi)");
    if (s == GILA_OK) s = check_finite(b, 3 * V, "The incident field (b)");
    if (s != GILA_OK) return s;
  }
  rq.chi = chi;
  rq.b = b;
  rq.x = x;
  if (opts) {
    if (opts->tol > 0) rq.so.tol = opts->tol;
    if (opts->max_matvecs > 0) rq.so.max_mv = opts->max_matvecs;
    if (opts->max_restarts > 0) rq.so.max_restarts = opts->max_restarts;
    if (opts->delta > 0) rq.so.delta = opts->delta;
    rq.so.x0 = opts->x0 != 0;
  }
  rq.t0 = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return fail(GILA_ERR_ARG, "server stopped");
    rq.ticket = sv->next_ticket++;
    sv->tickets[rq.ticket] = Ticket{};
    sv->incoming.push_back(rq);
    ++sv->n_submitted;
  }
  sv->cv_work.notify_all();
  *ticket = rq.ticket;
  return GILA_OK;
}

gila_status gila_server_wait(gila_server* srv, uint64_t ticket, int64_t timeout_ms, gila_solve_info* info,
                             double* latency_ms) {
  if (!srv) return fail(GILA_ERR_ARG, "null server");
  Server* sv = srv->impl;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->tickets.find(ticket);
  if (it == sv->tickets.end()) return fail(GILA_ERR_ARG, "unknown ticket");
  auto pred = [&] { return sv->tickets[ticket].done; };
  if (timeout_ms < 0)
    sv->cv_done.wait(lk, pred);
  else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
    return fail(GILA_ERR_TIMEOUT, "request not finished");
  Ticket t = sv->tickets[ticket];
  sv->tickets.erase(ticket);
  lk.unlock();
  if (info) *info = t.info;
  if (latency_ms) *latency_ms = t.latency_ms;
  if (t.status == GILA_ERR_NOTCONV)
    return fail(GILA_ERR_NOTCONV, "the solve stopped at relative residual " + std::to_string(t.info.rel_res));
  if (t.status != GILA_OK) return fail(t.status, t.err);
  return GILA_OK;
}

gila_status gila_server_stats_get(gila_server* srv, gila_server_stats* out) {
  if (!srv || !out) return fail(GILA_ERR_ARG, "null argument");
  Server* sv = srv->impl;
  std::lock_guard<std::mutex> lk(sv->mu);
  memset(out, 0, sizeof(*out));
  out->submitted = sv->n_submitted;
  out->completed = sv->n_completed;
  out->running = sv->c_running;
  out->queued = (int64_t)sv->incoming.size() + sv->c_pending;
  out->batches = sv->c_batches;
  out->operators = sv->c_ops;
  out->bytes_in_use = (int64_t)sv->used;
  out->hbm_budget = (int64_t)sv->budget;
  return GILA_OK;
}

}  // extern "C"
