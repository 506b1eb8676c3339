// server.cu -- request loop over resident systems (thp_server_*).
//
// Registered systems keep a host copy of their topology and parameters.  A
// request names a system and carries positions; worker threads take requests
// in arrival order, skipping ones whose system is busy with an earlier
// request.  A system on the device keeps its context (parameters, list, last
// dipoles) between requests, so a repeat is warm-started.  Admission is by
// footprint against the budget: idle systems are evicted least recently used
// first, and their contexts go to a pool from which the next new system takes
// one (thp_ctx_reset keeps every buffer that is large enough), so serving
// does not free device memory -- cudaFree waits for the whole device, which
// would stall every other request in flight.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "thp.h"

namespace thp {
int plan_prefetch(int device, const int nfft[3], int mixed);
int upload_positions(thp_ctx* h, const double* x, const double* y, const double* z, bool host_check);
struct SystemImage;
int image_create(const thp_config& cfg, const double* polarity, const double* thole, const double* pdamp,
                 const int* const* off, const int* const* idx, const double* scales, const double* pole,
                 const int* zaxis, const int* xaxis, const int* axt, SystemImage** out);
void image_free(SystemImage* img);
int image_load(thp_ctx* h, const SystemImage* img);
}

namespace {

using Clock = std::chrono::steady_clock;

// context set-up calls the driver's allocator and the FFT planner, which
// serialise across threads; more than two at once only slows every request
constexpr int kMaxSetups = 2;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// A registered system: its configuration and its inputs prepared for fast
// loading onto a context (thp::SystemImage, pinned host memory).
struct SysRec {
  thp_config cfg{};
  thp::SystemImage* img = nullptr;
  size_t footprint = 0;
  ~SysRec() { thp::image_free(img); }
};

struct Req {
  unsigned long long ticket = 0, key = 0;
  const double *x = nullptr, *y = nullptr, *z = nullptr;  // the caller's, read when the request starts
  double* uind = nullptr;
  double* uinp = nullptr;
  Clock::time_point submitted, started;
  thp_result res{};
  bool done = false;
};

struct Resident {
  thp_ctx* ctx = nullptr;
  size_t bytes = 0;
  bool busy = false;
  bool solved = false;
  unsigned long long last_use = 0;
};

struct Pooled {
  thp_ctx* ctx;
  size_t bytes;
};

}  // namespace

struct thp_server {
  thp_server_config cfg{};
  std::mutex m;
  std::condition_variable cv_work, cv_done, cv_room;
  std::deque<Req*> queue;
  std::map<unsigned long long, std::unique_ptr<Req>> reqs;
  std::map<unsigned long long, std::shared_ptr<SysRec>> systems;
  std::map<unsigned long long, Resident> resident;
  std::vector<Pooled> pool;
  std::vector<std::thread> threads;
  size_t used = 0;
  unsigned long long next_ticket = 1, clock = 0;
  bool stopping = false;
  bool paused = false;  // workers take no new request (those in flight finish)
  int setups_active = 0;
  std::condition_variable cv_setup;
  long completed = 0, failed = 0, created = 0, reused = 0, evicted = 0;
  std::vector<double> latencies;

  void worker();
  int acquire(std::unique_lock<std::mutex>& lk, unsigned long long key, const SysRec& sys, Resident*& slot,
              bool& fresh, thp_ctx*& reuse);
  int load_system(thp_ctx* h, const SysRec& sys);
};

namespace {

thp_config server_cfg(const thp_server_config& s, const thp_config& sys) {
  thp_config k = sys;
  k.precision = s.precision;
  k.poleps = s.poleps;
  k.politer = s.politer;
  k.device = s.device;
  return k;
}

}  // namespace

// Sets every system input of a fresh or re-targeted context.
int thp_server::load_system(thp_ctx* h, const SysRec& sys) { return thp::image_load(h, sys.img); }

// Under the lock: makes the system resident and marks it busy.  On return
// with THP_OK, slot is its entry; fresh is true when the caller must load
// the system into slot->ctx, which is then either a pooled context to
// re-target (reuse) or null (create one).  Waits while the budget is held
// by busy systems.
int thp_server::acquire(std::unique_lock<std::mutex>& lk, unsigned long long key, const SysRec& sys,
                        Resident*& slot, bool& fresh, thp_ctx*& reuse) {
  reuse = nullptr;
  fresh = false;
  for (;;) {
    auto it = resident.find(key);
    if (it != resident.end()) {
      if (!it->second.busy) {
        it->second.busy = true;
        it->second.last_use = ++clock;
        slot = &it->second;
        return THP_OK;
      }
      cv_room.wait(lk);
      continue;
    }
    // a pooled context large enough for this system, the smallest such
    int best = -1;
    for (size_t q = 0; q < pool.size(); ++q)
      if (pool[q].bytes >= sys.footprint && (best < 0 || pool[q].bytes < pool[(size_t)best].bytes)) best = (int)q;
    if (best >= 0) {
      reuse = pool[(size_t)best].ctx;
      Resident r;
      r.ctx = reuse;
      r.bytes = pool[(size_t)best].bytes;
      r.busy = true;
      r.last_use = ++clock;
      pool.erase(pool.begin() + best);
      slot = &(resident[key] = r);
      fresh = true;
      return THP_OK;
    }
    const bool crowded = cfg.max_resident > 0 && (int)resident.size() >= cfg.max_resident;
    if (!crowded && used + sys.footprint <= cfg.budget_bytes) {
      Resident r;
      r.bytes = sys.footprint;
      r.busy = true;
      r.last_use = ++clock;
      used += sys.footprint;
      slot = &(resident[key] = r);
      fresh = true;
      return THP_OK;
    }
    // make room: free a pooled context that is too small, else move the
    // least recently used idle system's context to the pool
    if (!pool.empty() && !crowded) {
      auto big = std::max_element(pool.begin(), pool.end(),
                                  [](const Pooled& a, const Pooled& b) { return a.bytes < b.bytes; });
      thp_ctx* dead = big->ctx;
      used -= big->bytes;
      pool.erase(big);
      lk.unlock();
      thp_ctx_destroy(dead);
      lk.lock();
      continue;
    }
    auto victim = resident.end();
    for (auto r = resident.begin(); r != resident.end(); ++r)
      if (!r->second.busy && r->second.ctx && (victim == resident.end() || r->second.last_use < victim->second.last_use))
        victim = r;
    if (victim != resident.end()) {
      pool.push_back(Pooled{victim->second.ctx, victim->second.bytes});
      resident.erase(victim);
      ++evicted;
      continue;
    }
    cv_room.wait(lk);
  }
}

void thp_server::worker() {
  std::unique_lock<std::mutex> lk(m);
  for (;;) {
    // first queued request whose system is not busy with an earlier one
    Req* r = nullptr;
    for (;;) {
      // a paused server still drains its queue once it is being destroyed
      for (auto it = queue.begin(); (!paused || stopping) && it != queue.end(); ++it) {
        auto res = resident.find((*it)->key);
        if (res == resident.end() || !res->second.busy) {
          r = *it;
          queue.erase(it);
          break;
        }
      }
      if (r || (stopping && queue.empty())) break;
      cv_work.wait(lk);
    }
    if (!r) return;
    r->started = Clock::now();
    std::shared_ptr<SysRec> sys = systems[r->key];
    Resident* slot = nullptr;
    bool fresh = false;
    thp_ctx* reuse = nullptr;
    int st = acquire(lk, r->key, *sys, slot, fresh, reuse);
    thp_ctx* h = slot->ctx;
    const bool warm = !fresh && slot->solved;
    lk.unlock();
    const Clock::time_point t_acq = Clock::now();
    const thp_config k = server_cfg(cfg, sys->cfg);
    size_t bytes_now = 0;
    bool loaded = !fresh;
    if (fresh) {  // at most kMaxSetups threads create or re-target contexts at once
      lk.lock();
      cv_setup.wait(lk, [this] { return setups_active < kMaxSetups; });
      ++setups_active;
      lk.unlock();
    }
    if (!st && fresh) {
      if (reuse) {
        st = thp_ctx_reset(reuse, &k);
        h = reuse;
      } else {
        st = thp_ctx_create(&k, &h);
      }
      if (!st) st = load_system(h, *sys);
      loaded = st == THP_OK;
      if (h) bytes_now = thp_ctx_footprint(h);
    }
    if (fresh) {
      lk.lock();
      --setups_active;
      cv_setup.notify_one();
      lk.unlock();
    }
    const Clock::time_point t_setup = Clock::now();
    thp_solve_info info{};
    if (!st) st = thp::upload_positions(h, r->x, r->y, r->z, false);
    if (!st) {
      st = thp_solve(h, warm ? THP_GUESS_PREVIOUS : THP_GUESS_DIRECT, &info);
      if (st == THP_E_NOT_CONVERGED) st = THP_OK;  // reported through info.converged
    }
    if (!st && (r->uind || r->uinp)) st = thp_get_dipoles(h, r->uind, r->uinp);
    const Clock::time_point end = Clock::now();
    lk.lock();
    if (fresh) {
      if (reuse) ++reused;
      else if (h) ++created;
    }
    if (h && fresh) {
      slot->ctx = h;
      // a re-targeted context may have grown, a new one is exactly its size
      if (bytes_now > slot->bytes) {
        used += bytes_now - slot->bytes;
        slot->bytes = bytes_now;
      }
    }
    if (!h) {  // creation failed: give the reservation back
      used -= slot->bytes;
      resident.erase(r->key);
    } else if (!loaded) {  // the system never made it onto the context: keep the context for reuse
      pool.push_back(Pooled{h, slot->bytes});
      resident.erase(r->key);
    } else {
      slot->busy = false;
      slot->solved = st == THP_OK;  // a failed solve leaves no dipoles to start the next one from
      slot->last_use = ++clock;
    }
    r->res.status = st;
    r->res.niter = info.niter;
    r->res.warm = warm ? 1 : 0;
    r->res.epol = info.epol;
    r->res.queue_ms = ms_between(r->submitted, r->started);
    r->res.latency_ms = ms_between(r->submitted, end);
    r->res.wait_ms = ms_between(r->started, t_acq);
    r->res.setup_ms = ms_between(t_acq, t_setup);
    r->res.solve_ms = ms_between(t_setup, end);
    r->done = true;
    if (st == THP_OK) {
      ++completed;
      latencies.push_back(r->res.latency_ms);
    } else {
      ++failed;
    }
    cv_done.notify_all();
    cv_room.notify_all();
    cv_work.notify_all();
  }
}

extern "C" {

int thp_server_create(const thp_server_config* cfg, thp_server** out) {
  if (!cfg || !out || cfg->workers <= 0 || cfg->budget_bytes == 0 || cfg->poleps <= 0 || cfg->politer <= 0 ||
      cfg->max_resident < 0 ||
      (cfg->precision != THP_FP64 && cfg->precision != THP_MIXED))
    return THP_E_INVALID;
  thp_server* s = new thp_server();
  s->cfg = *cfg;
  for (int w = 0; w < cfg->workers; ++w) s->threads.emplace_back([s] { s->worker(); });
  *out = s;
  return THP_OK;
}

int thp_server_register(thp_server* s, unsigned long long key, const thp_system* sys) {
  if (!s || !sys || !sys->polarity || !sys->thole || !sys->pdamp || !sys->conn_off || !sys->conn_idx ||
      !sys->scales || !sys->pole || !sys->zaxis || !sys->xaxis || !sys->axt || sys->cfg.n <= 0)
    return THP_E_INVALID;
  auto rec = std::make_shared<SysRec>();
  const size_t n = sys->cfg.n;
  rec->cfg = sys->cfg;
  for (int q = 0; q < 8; ++q) {
    const int* off = sys->conn_off[q];
    if (!off) continue;
    const int m = off[n];
    if (m < 0 || (m > 0 && !sys->conn_idx[q])) return THP_E_INVALID;
  }
  int st = thp::image_create(sys->cfg, sys->polarity, sys->thole, sys->pdamp, sys->conn_off, sys->conn_idx,
                             sys->scales, sys->pole, sys->zaxis, sys->xaxis, sys->axt, &rec->img);
  if (st) return st;
  const thp_config k = server_cfg(s->cfg, sys->cfg);
  rec->footprint = thp_footprint(&k);
  // the FFT plan of this shape is made now, not by the first request: a new
  // shape can take tens of milliseconds to plan (a missing device only
  // means the requests will report it)
  thp::plan_prefetch(k.device, k.nfft, k.precision == THP_MIXED);
  std::lock_guard<std::mutex> g(s->m);
  s->systems[key] = rec;  // requests already queued keep the record they were given
  return THP_OK;
}

int thp_server_submit(thp_server* s, unsigned long long key, const double* x, const double* y, const double* z,
                      double* uind, double* uinp, unsigned long long* ticket) {
  if (!s || !x || !y || !z || !ticket) return THP_E_INVALID;
  std::lock_guard<std::mutex> g(s->m);
  auto it = s->systems.find(key);
  if (it == s->systems.end() || s->stopping) return THP_E_INVALID;
  if (it->second->footprint > s->cfg.budget_bytes) return THP_E_OOM_ADMISSION;
  auto r = std::make_unique<Req>();
  const size_t n = it->second->cfg.n;
  r->ticket = s->next_ticket++;
  r->key = key;
  r->x = x;
  r->y = y;
  r->z = z;
  r->uind = uind;
  r->uinp = uinp;
  r->submitted = Clock::now();
  *ticket = r->ticket;
  s->queue.push_back(r.get());
  s->reqs[r->ticket] = std::move(r);
  s->cv_work.notify_one();
  return THP_OK;
}

int thp_server_warm(thp_server* s, int count) {
  if (!s || count < 0) return THP_E_INVALID;
  std::shared_ptr<SysRec> big;
  {
    std::lock_guard<std::mutex> g(s->m);
    for (auto& kv : s->systems)
      if (!big || kv.second->footprint > big->footprint) big = kv.second;
  }
  if (!big) return THP_E_STATE;
  const thp_config k = server_cfg(s->cfg, big->cfg);
  for (int q = 0; q < count; ++q) {
    {
      std::lock_guard<std::mutex> g(s->m);
      if (s->used + big->footprint > s->cfg.budget_bytes) break;
      s->used += big->footprint;  // reserved before the slow creation
    }
    thp_ctx* h = nullptr;
    const int st = thp_ctx_create(&k, &h);
    std::lock_guard<std::mutex> g(s->m);
    if (st) {
      s->used -= big->footprint;
      return st;
    }
    s->pool.push_back(Pooled{h, big->footprint});
    ++s->created;
  }
  s->cv_room.notify_all();
  return THP_OK;
}

int thp_server_wait(thp_server* s, unsigned long long ticket, thp_result* res) {
  if (!s) return THP_E_INVALID;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return THP_E_INVALID;
  Req* r = it->second.get();
  s->cv_done.wait(lk, [r] { return r->done; });
  if (res) *res = r->res;
  s->reqs.erase(it);
  return THP_OK;
}

int thp_server_wait_for(thp_server* s, unsigned long long ticket, double timeout_ms, thp_result* res) {
  if (!s || !(timeout_ms >= 0.0)) return THP_E_INVALID;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return THP_E_INVALID;
  Req* r = it->second.get();
  const auto limit = std::chrono::duration<double, std::milli>(timeout_ms);
  if (!s->cv_done.wait_for(lk, limit, [r] { return r->done; })) return THP_E_TIMEOUT;  // the ticket stays valid
  if (res) *res = r->res;
  s->reqs.erase(it);
  return THP_OK;
}

int thp_server_pause(thp_server* s, int paused) {
  if (!s) return THP_E_INVALID;
  {
    std::lock_guard<std::mutex> g(s->m);
    s->paused = paused != 0;
  }
  s->cv_work.notify_all();
  return THP_OK;
}

int thp_server_query(thp_server* s, thp_server_stats* out) {
  if (!s || !out) return THP_E_INVALID;
  std::lock_guard<std::mutex> g(s->m);
  thp_server_stats st{};
  st.completed = s->completed;
  st.failed = s->failed;
  std::vector<double> lat = s->latencies;
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) {  // linear interpolation between order statistics
      const double pos = p * (double)(lat.size() - 1);
      const size_t lo = (size_t)pos;
      const size_t hi = std::min(lo + 1, lat.size() - 1);
      return lat[lo] + (pos - (double)lo) * (lat[hi] - lat[lo]);
    };
    st.p50_ms = pct(0.50);
    st.p99_ms = pct(0.99);
  }
  st.resident = (int)s->resident.size();
  st.pooled = (int)s->pool.size();
  st.created = s->created;
  st.reused = s->reused;
  st.evicted = s->evicted;
  st.bytes = s->used;
  *out = st;
  return THP_OK;
}

int thp_server_destroy(thp_server* s) {
  if (!s) return THP_E_INVALID;
  {
    std::lock_guard<std::mutex> g(s->m);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->threads) t.join();
  for (auto& kv : s->resident)
    if (kv.second.ctx) thp_ctx_destroy(kv.second.ctx);
  for (auto& p : s->pool) thp_ctx_destroy(p.ctx);
  delete s;
  return THP_OK;
}

}  // extern "C"
