// Serving engine: GMRES-IR requests of mixed sizes and kinds on one GPU.
//
// The reference solves one system per GmresLDLIR object, one call at a time:
// Compute (gmres_ir.hpp:323) then Solve (gmres_ir.hpp:534-634), with
// QDLDL_etree / QDLDL_factor / QDLDL_solve (qdldl.hpp:48-432) underneath.
// This engine takes a stream of such requests and keeps what one request
// leaves behind for the next:
//
//   patterns  a request names its pattern (pattern_key) and its values
//             (values_key).  An unknown pattern is analysed on the host (the
//             ordering and symbolic analysis) and its plan uploaded once;
//   factors   a factor is kept per (pattern, values) while memory allows:
//             a request on a resident factor is only a solve, one with new
//             values on a known pattern a refactorization from the pattern's
//             plan, and a solve;
//   admission every plan, factor and batch-buffer growth is charged its
//             device bytes against the budget before it reaches the device
//             (plans and batch growth best effort, factors strictly); what
//             does not fit evicts idle factors (then
//             idle plans): those no queued request names first, least
//             recently used first, then those the queue needs last (freed
//             before the job waits or tries again), and a request whose
//             exceeds the whole budget, or that finds no room while no other
//             job runs on or within two minutes, is refused with
//             MPIR_ERR_NOMEM;
//   batching  worker threads, each driving its own CUDA stream, take the
//             oldest request whose pattern and factor are idle, together with
//             every queued request on the same factor (up to max_batch): those
//             are solved in lockstep by one batched GMRES-IR whose
//             preconditioner applications are several-vector triangular
//             solves (gmres_batch.cu, solve_multi.cu);
//   overlap   requests on different factors run on different streams at the
//             same time, and the host analysis of a new pattern runs on its
//             worker's thread while the GPU serves the others.
// Each result is the solve the request would get alone: the same analysis,
// factor and GMRES-IR control flow; a batched solve differs from a lone one
// only by the rounding of the several-vector triangular solves.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "server.hpp"
#include "symbolic.hpp"

namespace mpir {

static double now_s() {
  using C = std::chrono::steady_clock;
  return std::chrono::duration<double>(C::now().time_since_epoch()).count();
}

struct Server::Impl {
  ServerConfig cfg;

  struct Pattern {
    std::shared_ptr<Plan> plan;
    bool                  busy     = true;   // being analysed, uploaded or offloaded
    bool                  resident = false;  // plan arrays on the device
    size_t                bytes    = 0;
    double                last    = 0;
    int                   factors = 0;  // resident factors on this plan
  };
  struct Factor {
    std::unique_ptr<Solver> solver;
    bool                    busy  = false;
    bool                    valid = false;
    size_t                  bytes = 0;
    double                  last  = 0;
  };
  using FKey = std::pair<uint64_t, uint64_t>;

  struct Job {
    enum Kind { kNone, kAnalyse, kFactor, kSolve } kind = kNone;
    std::vector<ServerRequest> reqs;
  };

  std::mutex                           mu;
  std::condition_variable              cv_work, cv_done;
  std::deque<ServerRequest>            queue;
  std::map<uint64_t, Pattern>          patterns;
  std::map<FKey, Factor>               factors;
  std::unordered_map<int64_t, ServerResult> done;
  // Host analyses of every pattern seen (host memory, never evicted).
  std::map<uint64_t, std::shared_ptr<const Symbolic>> sym_cache;
  std::vector<std::thread>             workers;
  ServerStats                          st{};
  size_t                               used    = 0;
  int                                  running = 0;
  int                                  waiting_room = 0;  // jobs waiting in admission
  // A factor that finds no room for this long is refused (MPIR_ERR_NOMEM).
  static constexpr double              kAdmitWaitSeconds = 120.0;
  int64_t                              next_id = 1;
  bool                                 stop    = false;

  // ---- scheduling (under mu) -------------------------------------------------
  // Moves the queued requests on factor key k (at most `room`) into out.
  void take_same(const FKey &k, size_t room, std::vector<ServerRequest> &out) {
    for (auto it = queue.begin(); it != queue.end() && out.size() < room;) {
      if (it->pattern_key == k.first && it->values_key == k.second) {
        out.push_back(*it);
        it = queue.erase(it);
      } else {
        ++it;
      }
    }
  }

  // The oldest request that can run now, except that one on a pattern not
  // seen before goes first: its host analysis is the start of the longest
  // chain of work in the queue (analysis, factorization, solves), and every
  // queued request on that pattern waits for it.  (A pattern whose plan was
  // evicted keeps its place: preferring those too re-uploaded plans that
  // evicted others, whose requests were then preferred in turn.)
  bool pick(Job &job) {
    auto choice = queue.end();
    for (int pass = 0; pass < 2 && choice == queue.end(); pass++)
      for (auto it = queue.begin(); it != queue.end(); ++it) {
        auto p = patterns.find(it->pattern_key);
        if (p != patterns.end() && p->second.busy) continue;  // being analysed
        auto f = factors.find(FKey{it->pattern_key, it->values_key});
        if (f != factors.end() && f->second.busy) continue;   // in use
        if (pass == 0 && p != patterns.end()) continue;
        choice = it;
        break;
      }
    if (choice == queue.end()) return false;
    const ServerRequest r = *choice;
    const FKey          k{r.pattern_key, r.values_key};
    auto                p = patterns.find(r.pattern_key);
    auto                f = factors.find(k);
    queue.erase(choice);
    job.reqs.clear();
    job.reqs.push_back(r);
    take_same(k, static_cast<size_t>(cfg.max_batch), job.reqs);
    if (p == patterns.end() || !p->second.resident) {
      if (p == patterns.end()) {
        Pattern np;
        np.last = now_s();
        p       = patterns.emplace(r.pattern_key, std::move(np)).first;
      }
      p->second.busy = true;
      job.kind       = Job::kAnalyse;
    } else if (f != factors.end() && f->second.valid) {
      job.kind = Job::kSolve;
    } else {
      job.kind = Job::kFactor;
    }
    Factor &fe = factors[k];  // placeholder while it is built
    fe.busy    = true;
    running++;
    return true;
  }

  // Frees room for `need` bytes by evicting idle factors, then idle plans
  // without factors.  The victim is the one whose next use in the queue is
  // furthest away: first those no queued request names (least recently used
  // among them), then the rest by the position of their first queued
  // request.  Returns false when it cannot (the evicted solvers are handed
  // back to be destroyed outside the lock).
  bool make_room(size_t need, std::vector<std::unique_ptr<Solver>> &graveyard,
                 std::vector<std::shared_ptr<Plan>> &plan_graveyard) {
    if (used + need <= static_cast<size_t>(cfg.budget_bytes)) return true;
    constexpr size_t                none = static_cast<size_t>(-1);
    std::map<FKey, size_t>          next_f;
    std::map<uint64_t, size_t>      next_p;
    size_t                          pos = 0;
    for (const ServerRequest &q : queue) {
      next_f.emplace(FKey{q.pattern_key, q.values_key}, pos);
      next_p.emplace(q.pattern_key, pos);
      pos++;
    }
    auto later = [none](size_t a, double la, size_t b, double lb) {
      // true when a use at a (last used at la) should be evicted before b
      if (a != b) return a == none || (b != none && a > b);
      return la < lb;
    };
    while (used + need > static_cast<size_t>(cfg.budget_bytes)) {
      auto   victim = factors.end();
      size_t vnext  = 0;
      for (auto it = factors.begin(); it != factors.end(); ++it) {
        if (it->second.busy || !it->second.solver) continue;
        const auto   nf = next_f.find(it->first);
        const size_t nx = nf == next_f.end() ? none : nf->second;
        if (victim == factors.end() || later(nx, it->second.last, vnext, victim->second.last)) {
          victim = it;
          vnext  = nx;
        }
      }
      if (victim != factors.end()) {
        used -= victim->second.bytes;
        auto p = patterns.find(victim->first.first);
        if (p != patterns.end()) p->second.factors--;
        graveyard.push_back(std::move(victim->second.solver));
        factors.erase(victim);
        st.evictions++;
        continue;
      }
      auto   pv     = patterns.end();
      size_t pvnext = 0;
      for (auto it = patterns.begin(); it != patterns.end(); ++it) {
        if (it->second.busy || it->second.factors != 0 || !it->second.resident) continue;
        bool referenced = false;  // by the placeholder factor of a running job
        for (auto &f : factors)
          if (f.first.first == it->first) referenced = true;
        if (referenced) continue;
        const auto   np = next_p.find(it->first);
        const size_t nx = np == next_p.end() ? none : np->second;
        if (pv == patterns.end() || later(nx, it->second.last, pvnext, pv->second.last)) {
          pv     = it;
          pvnext = nx;
        }
      }
      if (pv == patterns.end()) return false;
      // The plan leaves the device; its host side (analysis and tables)
      // stays, so it comes back by an upload.  The arrays are freed outside
      // the lock, the pattern busy until then.
      used -= pv->second.bytes;
      pv->second.bytes    = 0;
      pv->second.resident = false;
      pv->second.busy     = true;
      plan_graveyard.push_back(pv->second.plan);
      st.evictions++;
    }
    return true;
  }

  // Charges `need` bytes once they fit the budget (lk held on entry and on
  // return): evicts as make_room does, frees what it evicted before waiting
  // or trying again, and waits while other jobs run on.  Returns "" when
  // admitted, else why the job is refused (no other job runs on that could
  // free memory, or the wait passed kAdmitWaitSeconds).
  std::string admit(size_t need, std::unique_lock<std::mutex> &lk,
                    std::vector<std::unique_ptr<Solver>> &graveyard,
                    std::vector<std::shared_ptr<Plan>> &plan_graveyard) {
    const double t_wait = now_s();
    for (;;) {
      if (make_room(need, graveyard, plan_graveyard)) {
        used += need;
        st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
        return "";
      }
      if (!graveyard.empty() || !plan_graveyard.empty()) {
        // What was evicted leaves the device before this job waits or tries
        // again (the budget already counts it as free).
        lk.unlock();
        graveyard.clear();
        release_plans(plan_graveyard);
        lk.lock();
        continue;
      }
      // Memory comes free only from jobs that run on: none other than those
      // waiting for room themselves (or the wait ran too long).
      if (running - waiting_room <= 1) return "admission budget held by resident plans";
      if (now_s() - t_wait > kAdmitWaitSeconds) return "admission wait exceeded";
      waiting_room++;
      cv_done.wait_for(lk, std::chrono::milliseconds(20));
      waiting_room--;
    }
  }

  // ---- work (outside mu) ------------------------------------------------------
  // Frees the device arrays of plans evicted by make_room and clears their
  // patterns' busy flags.
  void release_plans(std::vector<std::shared_ptr<Plan>> &plans) {
    for (auto &pl : plans) pl->release_device();
    if (!plans.empty()) {
      std::lock_guard<std::mutex> lk(mu);
      for (auto &pl : plans)
        for (auto &pt : patterns)
          if (pt.second.plan == pl) pt.second.busy = false;
    }
    plans.clear();
    cv_work.notify_all();
  }

  void finish(const ServerRequest &r, int status, int path, int batch, double t0,
              const Report &rep, const std::string &msg) {
    ServerResult res{};
    res.id         = r.id;
    res.status     = status;
    res.path       = path;
    res.batch      = batch;
    const double t = now_s();
    res.latency_ms = 1e3 * (t - r.t_submit);
    res.queue_ms   = 1e3 * (t0 - r.t_submit);
    res.service_ms = 1e3 * (t - t0);
    res.report     = rep;
    res.message    = msg;
    std::lock_guard<std::mutex> lk(mu);
    done[r.id] = res;
    st.completed++;
    if (status != 0) st.failed++;
  }

  void run(Job &job) {
    const double               t0 = now_s();
    const ServerRequest       &r  = job.reqs.front();
    const FKey                 k{r.pattern_key, r.values_key};
    int                        path = job.kind == Job::kAnalyse ? 2 : job.kind == Job::kFactor ? 1 : 0;
    std::shared_ptr<Plan>      plan;
    Solver                    *sv = nullptr;
    std::vector<std::unique_ptr<Solver>> graveyard;
    std::vector<std::shared_ptr<Plan>>   plan_graveyard;
    size_t                               reserved = 0;  // admitted bytes not yet counted as a plan's or factor's
    // Plans evicted on this job's behalf leave the device however the job
    // ends (after every lock of this function is released).
    struct ReleaseAtExit {
      Impl                               *self;
      std::vector<std::shared_ptr<Plan>> *plans;
      ~ReleaseAtExit() { self->release_plans(*plans); }
    } release_at_exit{this, &plan_graveyard};
    auto fail_all = [&](int code, const std::string &msg) {
      for (const ServerRequest &q : job.reqs) finish(q, code, path, 1, t0, Report{}, msg);
    };
    // A plan's device arrays are charged before they are uploaded, after
    // evicting what makes room for them if anything can go (best effort: a
    // plan is small, and waiting for room here would hold every queued
    // request on its pattern).
    auto load_plan = [&](const std::shared_ptr<Plan> &pl) -> bool {
      const size_t pb = pl->upload_bytes();
      {
        std::lock_guard<std::mutex> lk(mu);
        make_room(pb, graveyard, plan_graveyard);
        used += pb;
        reserved      = pb;
        st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
      }
      graveyard.clear();
      release_plans(plan_graveyard);
      cudaStream_t s = nullptr;
      MPIR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      try {
        pl->upload_all(s);
      } catch (...) {
        cudaStreamDestroy(s);
        throw;
      }
      cudaStreamDestroy(s);
      return true;
    };
    try {
      MPIR_CUDA(cudaSetDevice(cfg.device));
      if (job.kind == Job::kAnalyse) {
        // A pattern whose plan was evicted uploads its kept host tables
        // again; one seen before without them takes its host analysis from
        // the cache and only builds its plan again.
        std::shared_ptr<Plan> kept;
        {
          std::lock_guard<std::mutex> lk(mu);
          auto pt = patterns.find(r.pattern_key);
          if (pt != patterns.end() && pt->second.plan && !pt->second.plan->on_device)
            kept = pt->second.plan;
        }
        if (kept) {
          const double tu = now_s();
          if (!load_plan(kept)) return;
          plan = kept;
          std::lock_guard<std::mutex> lk(mu);
          Pattern &p = patterns[r.pattern_key];
          p.busy     = false;
          p.resident = true;
          p.bytes    = plan->device_bytes();
          p.last     = now_s();
          used       = used - reserved + p.bytes;
          reserved   = 0;
          st.plan_uploads++;
          st.plan_ms += 1e3 * (p.last - tu);
          st.plan_upload_ms += plan->upload_ms;
          st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
        }
      }
      if (job.kind == Job::kAnalyse && !plan) {
        std::vector<int8_t> sign(r.n, 0);
        for (int64_t j = 0; j < r.n; j++)
          for (int64_t p = r.Ap[j]; p < r.Ap[j + 1]; p++)
            if (r.Ai[p] == j && r.Ax[p] > 0) sign[j] = 1;
        std::shared_ptr<const Symbolic> cached;
        {
          std::lock_guard<std::mutex> lk(mu);
          auto it = sym_cache.find(r.pattern_key);
          if (it != sym_cache.end()) cached = it->second;
        }
        const double ta = now_s();
        Symbolic    S;
        std::string err;
        int         rc = kOk;
        if (cached) {
          S = *cached;
        } else {
          rc = analyze(r.n, r.Ap, r.Ai, sign.data(), Ordering::Auto, S, err);
          if (rc == kOk) {
            auto keep = std::make_shared<const Symbolic>(S);
            std::lock_guard<std::mutex> lk(mu);
            sym_cache[r.pattern_key] = std::move(keep);
          }
        }
        const double tb = now_s();
        if (rc != kOk) {
          {
            std::lock_guard<std::mutex> lk(mu);
            patterns.erase(r.pattern_key);
            factors.erase(k);
            st.analyses++;
          }
          fail_all(rc, err.empty() ? "analysis failed" : err);
          return;
        }
        plan = std::make_shared<Plan>();
        plan->build(std::move(S), nullptr, false);  // host tables; uploaded once admitted
        if (!load_plan(plan)) return;
        std::lock_guard<std::mutex> lk(mu);
        const size_t pb = plan->device_bytes();
        Pattern &p = patterns[r.pattern_key];
        p.plan     = plan;
        p.busy     = false;
        p.resident = true;
        p.bytes    = pb;
        p.last     = now_s();
        used       = used - reserved + pb;
        reserved   = 0;
        st.analyses++;
        if (cached) st.analysis_reuses++;
        st.analysis_ms += 1e3 * (tb - ta);
        st.plan_ms += 1e3 * (p.last - tb);
        st.plan_upload_ms += plan->upload_ms;
        st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
      } else {
        std::lock_guard<std::mutex> lk(mu);
        plan = patterns.at(r.pattern_key).plan;
      }
      if (job.kind != Job::kSolve) {
        const int    width = job.reqs.size() > 1 ? multi_width(static_cast<int>(job.reqs.size())) : 1;
        const size_t need  = Solver::bytes_for(*plan, cfg.max_gmres_iterations, width, cfg.uf);
        {
          std::unique_lock<std::mutex> lk(mu);
          if (need > static_cast<size_t>(cfg.budget_bytes)) {
            factors.erase(k);
            lk.unlock();
            fail_all(-4, "factor footprint " + std::to_string(need) +
                             " bytes exceeds the admission budget");
            std::lock_guard<std::mutex> lk2(mu);
            st.refused += static_cast<int64_t>(job.reqs.size());
            return;
          }
          const std::string why = admit(need, lk, graveyard, plan_graveyard);
          if (!why.empty()) {
            factors.erase(k);
            lk.unlock();
            fail_all(-4, why);
            std::lock_guard<std::mutex> lk2(mu);
            st.refused += static_cast<int64_t>(job.reqs.size());
            return;
          }
          reserved = need;  // charged; corrected to the measured bytes below
        }
        graveyard.clear();
        release_plans(plan_graveyard);
        const double tf     = now_s();
        auto solver = std::make_unique<Solver>(cfg.uf, kF64, cfg.ur, cfg.device);
        solver->ir_iter    = cfg.max_ir_iterations;
        solver->gmres_iter = cfg.max_gmres_iterations;
        solver->tol        = cfg.tolerance;
        solver->update_engine = cfg.update;
        solver->adopt(plan);
        const double t_setup = now_s();
        const int fr = solver->factor(r.Ax);
        const double sv_factor_ms = solver->last_factor_ms;
        // A resident factor keeps only what the solves read.
        MPIR_CUDA(cudaStreamSynchronize(solver->stream()));
        const double t_trim = now_s();
        solver->trim();
        const double t_end = now_s();
        {
          std::lock_guard<std::mutex> lk(mu);
          Factor &f = factors[k];
          f.bytes   = solver->device_bytes();
          used      = used - need + f.bytes;
          reserved  = 0;
          f.solver  = std::move(solver);
          f.valid   = fr == kOk;
          f.last    = now_s();
          patterns[r.pattern_key].factors++;
          st.factorizations++;
          st.factor_ms += 1e3 * (now_s() - tf);
          st.factor_device_ms += sv_factor_ms;
          st.setup_ms += 1e3 * (t_setup - tf);
          st.trim_ms += 1e3 * (t_end - t_trim);
          st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
          sv = f.solver.get();
        }
        if (fr != kOk) {
          fail_all(fr, fr == -5 ? "a bounded device wait ran out" : "zero pivot");
          std::lock_guard<std::mutex> lk(mu);
          factors[k].busy = false;
          return;
        }
      } else {
        {
          // A lockstep batch wider than the factor's buffers grows them:
          // that growth is charged before the solve, after evicting what
          // makes room for it if anything can go (best effort, as plans).
          std::lock_guard<std::mutex> lk(mu);
          sv = factors.at(k).solver.get();
          if (job.reqs.size() > 1) {
            const size_t grow = sv->batch_growth(multi_width(static_cast<int>(job.reqs.size())));
            if (grow > 0) {
              make_room(grow, graveyard, plan_graveyard);
              used += grow;
              reserved      = grow;
              st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
            }
          }
        }
        graveyard.clear();
        release_plans(plan_graveyard);
      }
      // Solve the batch: one request alone, several in lockstep.
      const double  ts = now_s();
      const int64_t n  = plan->S.n;
      const int     nb = static_cast<int>(job.reqs.size());
      std::vector<Report> reps(nb);
      int                 rc = kOk;
      if (nb == 1) {
        rc = sv->solve(r.b, r.x, &reps[0]);
      } else {
        std::vector<double> B(static_cast<size_t>(n) * nb), X(static_cast<size_t>(n) * nb);
        for (int q = 0; q < nb; q++)
          std::copy(job.reqs[q].b, job.reqs[q].b + n, B.begin() + static_cast<size_t>(q) * n);
        rc = sv->solve_batch(nb, B.data(), X.data(), reps.data());
        for (int q = 0; q < nb; q++)
          std::copy(X.begin() + static_cast<size_t>(q) * n, X.begin() + static_cast<size_t>(q + 1) * n,
                    job.reqs[q].x);
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        Factor &f = factors[k];
        // the batch buffers may have grown (their growth was reserved)
        const size_t b = f.solver->device_bytes();
        used           = used - f.bytes - reserved + b;
        reserved       = 0;
        f.bytes        = b;
        f.last         = now_s();
        patterns[r.pattern_key].last = f.last;
        st.solves++;
        st.solve_ms += 1e3 * (now_s() - ts);
        st.solve_device_ms += reps[0].solve_ms;  // a batch reports its whole time in each
        if (nb > 1) {
          st.batched_solves++;
          st.batched_rhs += nb;
        }
        st.peak_bytes = std::max<int64_t>(st.peak_bytes, used);
      }
      for (int q = 0; q < nb; q++)
        finish(job.reqs[q], rc, path, nb, t0, reps[q], rc == kOk ? "" : "solve failed");
      std::lock_guard<std::mutex> lk(mu);
      factors[k].busy = false;
    } catch (const std::exception &e) {
      const bool oom = dynamic_cast<const CudaError *>(&e) &&
                       static_cast<const CudaError &>(e).code == cudaErrorMemoryAllocation;
      {
        std::lock_guard<std::mutex> lk(mu);
        used -= reserved;
        auto f = factors.find(k);
        if (f != factors.end()) {
          if (f->second.solver) {
            used -= f->second.bytes;
            patterns[k.first].factors--;
            graveyard.push_back(std::move(f->second.solver));
          }
          factors.erase(f);
        }
        auto p = patterns.find(k.first);
        if (p != patterns.end() && p->second.busy) patterns.erase(p);
      }
      fail_all(oom ? -4 : -3, e.what());
    }
  }

  void worker_main() {
    cudaSetDevice(cfg.device);
    set_thread_pool(false);  // see memory.cu
    for (;;) {
      Job job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || pick(job); });
        if (job.kind == Job::kNone) return;  // stopping, nothing left to pick
      }
      run(job);
      {
        std::lock_guard<std::mutex> lk(mu);
        running--;
      }
      cv_work.notify_all();
      cv_done.notify_all();
    }
  }
};

Server::Server(const ServerConfig &cfg) : impl_(new Impl) {
  impl_->cfg = cfg;
  if (impl_->cfg.workers < 1) impl_->cfg.workers = 1;
  impl_->cfg.max_batch = std::max(1, std::min(impl_->cfg.max_batch, Solver::kMaxBatch));
  for (int w = 0; w < impl_->cfg.workers; w++)
    impl_->workers.emplace_back([this] { impl_->worker_main(); });
}

Server::~Server() {
  drain();
  {
    std::lock_guard<std::mutex> lk(impl_->mu);
    impl_->stop = true;
  }
  impl_->cv_work.notify_all();
  for (auto &t : impl_->workers) t.join();
  cudaSetDevice(impl_->cfg.device);
  impl_->factors.clear();
  impl_->patterns.clear();
  device_cache_flush(impl_->cfg.device);  // the workers' idle blocks
}

int64_t Server::submit(ServerRequest r) {
  std::lock_guard<std::mutex> lk(impl_->mu);
  r.id       = impl_->next_id++;
  r.t_submit = now_s();
  impl_->queue.push_back(r);
  impl_->st.submitted++;
  impl_->cv_work.notify_one();
  return r.id;
}

bool Server::wait(int64_t id, ServerResult *out) {
  std::unique_lock<std::mutex> lk(impl_->mu);
  impl_->cv_done.wait(lk, [&] { return impl_->done.count(id) != 0; });
  if (out) *out = impl_->done[id];
  impl_->done.erase(id);
  return true;
}

void Server::drain() {
  std::unique_lock<std::mutex> lk(impl_->mu);
  impl_->cv_done.wait(lk, [&] { return impl_->queue.empty() && impl_->running == 0; });
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(impl_->mu);
  ServerStats s       = impl_->st;
  s.bytes_in_use      = static_cast<int64_t>(impl_->used);
  s.resident_factors  = 0;
  for (auto &f : impl_->factors) s.resident_factors += f.second.solver ? 1 : 0;
  s.resident_patterns = static_cast<int64_t>(impl_->patterns.size());
  s.queued            = static_cast<int64_t>(impl_->queue.size());
  return s;
}

}  // namespace mpir
