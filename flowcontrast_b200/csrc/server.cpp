// Served solves (include/fslbm.h, fslbm_server_*): a request queue, admission by device
// footprint under an HBM budget, and continuous batching on a worker thread. The reference has
// no counterpart: it runs one pipe per process (FSLBM.cu:489-905).
//
// The worker owns its own context (one device, one stream) and uses only the public solve and
// batch calls. A round is: launch min(quantum, most steps left) batched steps for every storage
// type present, each member stopping at its own step budget (fslbm_batch_set_stop); while those
// run, create and initialise the solves of requests that fit the budget (their set-up is
// queued on the same stream, behind the round); wait for the round; hand finished results
// back and free their memory. Client calls only touch the request table under the mutex, so
// they are thread-safe and never wait for the GPU.
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

#include <nvtx3/nvToolsExt.h>

#include "../../include/fslbm.h"

int fslbm_set_error(int code, const char* fmt, ...);

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  fslbm_request req{};
  std::vector<uint8_t> mask;      // copy of req.domain.mask
  std::vector<float> init;        // copy of the host start, 4 * cells, if given
  fslbm_result res{};
  fslbm_solve* solve = nullptr;   // worker-owned while running
  int64_t left = 0;
  bool has_out = false;
  bool in_round = false;          // worker-only: advanced by the current round
};

using ReqPtr = std::shared_ptr<Request>;

struct Group {
  int dtype = 0;
  std::vector<int64_t> ids;       // the members' request ids: the group's identity
  std::vector<fslbm_solve*> members;
  std::vector<int64_t> stops;     // each member's total step count
  fslbm_batch* batch = nullptr;
};

}  // namespace

struct fslbm_server {
  int device = 0;
  fslbm_ctx* ctx = nullptr;
  fslbm_server_config cfg{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<ReqPtr> queue;                 // waiting for admission, arrival order
  std::map<int64_t, ReqPtr> table;          // every request not yet released
  int64_t next_id = 1;
  fslbm_server_stats st{};
  Clock::time_point t0;
  // worker-only
  std::vector<ReqPtr> active;
  std::vector<Group> groups;
};

namespace {

double since(const fslbm_server* S) {
  return std::chrono::duration<double>(Clock::now() - S->t0).count();
}

void finish(fslbm_server* S, const ReqPtr& r, int status, int error) {
  std::lock_guard<std::mutex> lk(S->mu);
  r->res.status = status;
  r->res.error = error;
  r->res.t_done = since(S);
  S->st.bytes_resident -= r->res.bytes_device;
  S->st.resident -= 1;
  if (status == FSLBM_REQ_DONE) {
    S->st.completed += 1;
    S->st.cell_steps += double(r->res.cells) * double(r->req.nsteps);
  } else {
    S->st.failed += 1;
  }
  S->cv_done.notify_all();
}

// Creates and initialises the solve of an admitted request (queued behind the running round).
int start_request(fslbm_server* S, const ReqPtr& r) {
  fslbm_domain dom = r->req.domain;
  dom.mask = r->mask.empty() ? nullptr : r->mask.data();
  fslbm_solve* s = nullptr;
  int rc = fslbm_solve_create(S->ctx, &dom, &r->req.params, fslbm_dtype(r->req.dtype), &s);
  if (rc) return rc;
  if (!r->init.empty()) {
    const size_t n = size_t(r->res.cells);
    const float* f = r->init.data();
    rc = fslbm_solve_set_fields(s, FSLBM_F32, f, f + n, f + 2 * n, f + 3 * n);
  } else {
    const fslbm_init_spec& q = r->req.init_spec;
    rc = fslbm_solve_init_poiseuille(s, q.umax, q.noise, q.modes, q.mode_amp, q.seed);
  }
  if (rc) {
    fslbm_solve_destroy(s);
    return rc;
  }
  r->solve = s;
  r->left = r->req.nsteps;
  return FSLBM_OK;
}

// Hands a finished request's result back and frees its device memory.
void retire(fslbm_server* S, const ReqPtr& r) {
  int rc = FSLBM_OK;
  if (r->has_out)
    rc = fslbm_solve_get_fields(r->solve, FSLBM_F32, r->req.out[0], r->req.out[1], r->req.out[2],
                                r->req.out[3]);
  if (!rc) rc = fslbm_solve_sync(r->solve);
  fslbm_monitor m{};
  if (!rc && fslbm_solve_monitor(r->solve, &m) == FSLBM_OK) r->res.last = m;
  fslbm_solve_destroy(r->solve);
  r->solve = nullptr;
  finish(S, r, rc ? FSLBM_REQ_FAILED : FSLBM_REQ_DONE, rc);
}

// Admits queued requests in arrival order while they fit; returns the admitted ones.
std::vector<ReqPtr> take_admissible(fslbm_server* S) {
  std::vector<ReqPtr> out;
  std::lock_guard<std::mutex> lk(S->mu);
  while (!S->queue.empty()) {
    const ReqPtr& r = S->queue.front();
    if (S->st.bytes_resident + r->res.bytes_device > S->cfg.hbm_budget) break;
    if (S->cfg.max_resident > 0 && S->st.resident >= S->cfg.max_resident) break;
    S->st.bytes_resident += r->res.bytes_device;
    S->st.bytes_peak = std::max(S->st.bytes_peak, S->st.bytes_resident);
    S->st.resident += 1;
    S->st.queued -= 1;
    r->res.status = FSLBM_REQ_RUNNING;
    r->res.t_admit = since(S);
    out.push_back(r);
    S->queue.pop_front();
  }
  return out;
}

// Creates the admitted requests' solves (their set-up is queued on the worker's stream) and
// returns those with steps to take; requests of zero steps are retired at once.
void add_time(fslbm_server* S, double fslbm_server_stats::*field, Clock::time_point t) {
  const double d = std::chrono::duration<double>(Clock::now() - t).count();
  std::lock_guard<std::mutex> lk(S->mu);
  S->st.*field += d;
}

std::vector<ReqPtr> admit(fslbm_server* S, const std::vector<ReqPtr>& adm) {
  const auto t = Clock::now();
  std::vector<ReqPtr> started;
  for (const ReqPtr& r : adm) {
    const int rc = start_request(S, r);
    if (rc) {
      finish(S, r, FSLBM_REQ_FAILED, rc);
      continue;
    }
    if (r->left == 0) retire(S, r);
    else started.push_back(r);
  }
  add_time(S, &fslbm_server_stats::t_admit, t);
  return started;
}

// The resident requests a round advances: all of them, or (least-work policy) those with the
// least work left, in that order, up to round_cells box cells and at least one.
std::vector<ReqPtr> round_set(const fslbm_server* S) {
  if (S->cfg.policy != FSLBM_SERVE_LEAST_WORK) return S->active;
  std::vector<ReqPtr> order = S->active;
  std::stable_sort(order.begin(), order.end(), [](const ReqPtr& a, const ReqPtr& b) {
    return double(a->res.cells) * double(a->left) < double(b->res.cells) * double(b->left);
  });
  std::vector<ReqPtr> out;
  int64_t cells = 0;
  for (const ReqPtr& r : order) {
    if (!out.empty() && cells + r->res.cells > S->cfg.round_cells) break;
    out.push_back(r);
    cells += r->res.cells;
  }
  return out;
}

// Rebuilds the per-dtype groups of the round's requests whose membership changed.
int regroup(fslbm_server* S, const std::vector<ReqPtr>& round) {
  std::vector<Group> next;
  for (const ReqPtr& r : round) {
    auto it = std::find_if(next.begin(), next.end(), [&](const Group& g) { return g.dtype == r->req.dtype; });
    if (it == next.end()) {
      next.push_back(Group{});
      next.back().dtype = r->req.dtype;
      it = next.end() - 1;
    }
    it->ids.push_back(r->id);
    it->members.push_back(r->solve);
    it->stops.push_back(r->req.nsteps);
  }
  // A batch is reused only for the same requests. Solve addresses are no identity: a solve
  // created after another was destroyed can reuse its address, and a batch kept for it would
  // step the new solve with the old one's work items and stop step.
  for (Group& g : next) {
    auto old = std::find_if(S->groups.begin(), S->groups.end(), [&](const Group& o) {
      return o.dtype == g.dtype && o.ids == g.ids && o.members == g.members && o.batch;
    });
    if (old != S->groups.end()) {
      g.batch = old->batch;
      old->batch = nullptr;
    } else {
      int rc = fslbm_batch_create(S->ctx, g.members.data(), int(g.members.size()), &g.batch);
      for (int i = 0; !rc && i < int(g.members.size()); ++i)
        rc = fslbm_batch_set_stop(g.batch, i, g.stops[i]);
      if (rc) {
        for (Group& o : next)
          if (o.batch) fslbm_batch_destroy(o.batch);
        for (Group& o : next) o.batch = nullptr;
        return rc;
      }
    }
  }
  for (Group& o : S->groups)
    if (o.batch) fslbm_batch_destroy(o.batch);
  S->groups = std::move(next);
  return FSLBM_OK;
}

void fail_active(fslbm_server* S, int rc) {
  for (Group& g : S->groups)
    if (g.batch) fslbm_batch_destroy(g.batch);
  S->groups.clear();
  for (const ReqPtr& r : S->active) {
    fslbm_solve_destroy(r->solve);
    r->solve = nullptr;
    finish(S, r, FSLBM_REQ_FAILED, rc);
  }
  S->active.clear();
}

void run(fslbm_server* S) {
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->active.empty())
        S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
      if (S->stop) break;
    }
    if (S->active.empty()) {
      S->active = admit(S, take_admissible(S));
      continue;
    }
    const auto tg = Clock::now();
    struct RoundRange {              // NVTX range over the round (header-only NVTX v3)
      RoundRange() { nvtxRangePushA("fslbm_server_round"); }
      ~RoundRange() { nvtxRangePop(); }
    } range;
    const std::vector<ReqPtr> round = round_set(S);
    for (const ReqPtr& r : round) r->in_round = true;
    const int rg = regroup(S, round);
    add_time(S, &fslbm_server_stats::t_regroup, tg);
    if (rg) {
      fail_active(S, rg);
      continue;
    }
    int64_t most = 0;
    for (const ReqPtr& r : round) most = std::max(most, r->left);
    const int64_t k = std::min<int64_t>(S->cfg.quantum, most);
    const auto tr = Clock::now();
    int rc = FSLBM_OK;
    for (Group& g : S->groups)
      if (!rc) rc = fslbm_batch_step(g.batch, k, 1);
    add_time(S, &fslbm_server_stats::t_launch, tr);
    // set-up of new arrivals overlaps the round; they join the next one
    std::vector<ReqPtr> started = rc ? std::vector<ReqPtr>{} : admit(S, take_admissible(S));
    const auto tw = Clock::now();
    for (Group& g : S->groups)
      if (!rc) rc = fslbm_batch_sync(g.batch);
    add_time(S, &fslbm_server_stats::t_wait, tw);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->st.busy_seconds += std::chrono::duration<double>(Clock::now() - tr).count();
      S->st.rounds += 1;
    }
    if (rc) {
      fail_active(S, rc);
      S->active = started;
      continue;
    }
    std::vector<ReqPtr> still;
    const auto tt = Clock::now();
    for (const ReqPtr& r : S->active) {
      if (!r->in_round) {            // waits for a later round
        still.push_back(r);
        continue;
      }
      r->in_round = false;
      const int64_t took = std::min(k, r->left);
      r->left -= took;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        r->res.steps_done += took;
      }
      if (r->left == 0) retire(S, r);
      else still.push_back(r);
    }
    add_time(S, &fslbm_server_stats::t_retire, tt);
    still.insert(still.end(), started.begin(), started.end());
    S->active.swap(still);
  }
  fail_active(S, FSLBM_ERR_STATE);
  for (Group& g : S->groups)
    if (g.batch) fslbm_batch_destroy(g.batch);
  S->groups.clear();
}

}  // namespace

extern "C" int fslbm_server_create(int device, const fslbm_server_config* cfg, fslbm_server** out) {
  if (!out) return fslbm_set_error(FSLBM_ERR_ARG, "server_create: null output");
  auto* S = new fslbm_server;
  S->device = device;
  if (cfg) S->cfg = *cfg;
  if (S->cfg.hbm_budget <= 0) S->cfg.hbm_budget = int64_t(150e9);
  if (S->cfg.quantum <= 0) S->cfg.quantum = 50;
  if (S->cfg.round_cells <= 0) S->cfg.round_cells = int64_t(48) << 20;
  if (S->cfg.policy != FSLBM_SERVE_ALL && S->cfg.policy != FSLBM_SERVE_LEAST_WORK) {
    delete S;
    return fslbm_set_error(FSLBM_ERR_ARG, "server_create: unknown policy %d", cfg->policy);
  }
  if (int rc = fslbm_ctx_create(device, &S->ctx)) {
    delete S;
    return rc;
  }
  S->t0 = Clock::now();
  S->worker = std::thread(run, S);
  *out = S;
  return FSLBM_OK;
}

extern "C" int fslbm_server_destroy(fslbm_server* S) {
  if (!S) return FSLBM_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    for (const ReqPtr& r : S->queue) {
      r->res.status = FSLBM_REQ_FAILED;
      r->res.error = FSLBM_ERR_STATE;
    }
    S->queue.clear();
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  S->cv_done.notify_all();
  fslbm_ctx_destroy(S->ctx);
  delete S;
  return FSLBM_OK;
}

extern "C" int fslbm_server_submit(fslbm_server* S, const fslbm_request* req, int64_t* id) {
  if (!S || !req || !id) return fslbm_set_error(FSLBM_ERR_ARG, "server_submit: null argument");
  const fslbm_domain& d = req->domain;
  if (d.lx < 3 || d.ly < 3 || d.lz < 1 || req->nsteps < 0)
    return fslbm_set_error(FSLBM_ERR_ARG, "server_submit: bad domain or step count");
  const bool some_init = req->init[0] || req->init[1] || req->init[2] || req->init[3];
  const bool all_init = req->init[0] && req->init[1] && req->init[2] && req->init[3];
  const bool some_out = req->out[0] || req->out[1] || req->out[2] || req->out[3];
  const bool all_out = req->out[0] && req->out[1] && req->out[2] && req->out[3];
  if (some_init != all_init || some_out != all_out)
    return fslbm_set_error(FSLBM_ERR_ARG, "server_submit: give all four init (out) arrays or none");
  auto r = std::make_shared<Request>();
  r->req = *req;
  r->res.cells = int64_t(d.lx) * d.ly * d.lz;
  r->has_out = all_out;
  int64_t bytes = 0;
  if (int rc = fslbm_solve_footprint(&d, fslbm_dtype(req->dtype), &bytes)) return rc;
  // host start in or fields out go through a staging buffer (4 FP32 fields) unless the state is
  // FP32 without pitch padding
  if ((all_out || all_init) && (req->dtype != FSLBM_F32 || d.lx % 8 != 0)) bytes += 16 * r->res.cells;
  r->res.bytes_device = bytes;
  if (bytes > S->cfg.hbm_budget)
    return fslbm_set_error(FSLBM_ERR_BUDGET, "server_submit: footprint %lld B exceeds the budget %lld B",
                           (long long)bytes, (long long)S->cfg.hbm_budget);
  if (d.mask) r->mask.assign(d.mask, d.mask + size_t(d.lx) * d.ly);
  r->req.domain.mask = nullptr;
  if (all_init) {
    const size_t n = size_t(r->res.cells);
    r->init.resize(4 * n);
    for (int f = 0; f < 4; ++f) std::memcpy(r->init.data() + f * n, req->init[f], n * sizeof(float));
    for (int f = 0; f < 4; ++f) r->req.init[f] = nullptr;
  }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return fslbm_set_error(FSLBM_ERR_STATE, "server_submit: server is stopping");
    r->id = S->next_id++;
    r->res.status = FSLBM_REQ_QUEUED;
    r->res.t_submit = since(S);
    S->table[r->id] = r;
    S->queue.push_back(r);
    S->st.submitted += 1;
    S->st.queued += 1;
    *id = r->id;
  }
  S->cv_work.notify_one();
  return FSLBM_OK;
}

extern "C" int fslbm_server_poll(fslbm_server* S, int64_t id, fslbm_result* out) {
  if (!S || !out) return fslbm_set_error(FSLBM_ERR_ARG, "server_poll: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->table.find(id);
  if (it == S->table.end()) return fslbm_set_error(FSLBM_ERR_NOTFOUND, "server_poll: no request %lld", (long long)id);
  *out = it->second->res;
  return FSLBM_OK;
}

extern "C" int fslbm_server_wait(fslbm_server* S, int64_t id, double timeout_s, fslbm_result* out) {
  if (!S) return fslbm_set_error(FSLBM_ERR_ARG, "server_wait: null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->table.find(id);
  if (it == S->table.end()) return fslbm_set_error(FSLBM_ERR_NOTFOUND, "server_wait: no request %lld", (long long)id);
  ReqPtr r = it->second;
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    return r->res.status == FSLBM_REQ_DONE || r->res.status == FSLBM_REQ_FAILED;
  });
  if (out) *out = r->res;
  if (!ok) return fslbm_set_error(FSLBM_ERR_TIMEOUT, "server_wait: request %lld not done", (long long)id);
  return FSLBM_OK;
}

extern "C" int fslbm_server_drain(fslbm_server* S, double timeout_s) {
  if (!S) return fslbm_set_error(FSLBM_ERR_ARG, "server_drain: null server");
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    return S->st.completed + S->st.failed == S->st.submitted;
  });
  if (!ok) return fslbm_set_error(FSLBM_ERR_TIMEOUT, "server_drain: requests still pending");
  return FSLBM_OK;
}

extern "C" int fslbm_server_release(fslbm_server* S, int64_t id) {
  if (!S) return fslbm_set_error(FSLBM_ERR_ARG, "server_release: null server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->table.find(id);
  if (it == S->table.end()) return fslbm_set_error(FSLBM_ERR_NOTFOUND, "server_release: no request %lld", (long long)id);
  const int st = it->second->res.status;
  if (st != FSLBM_REQ_DONE && st != FSLBM_REQ_FAILED)
    return fslbm_set_error(FSLBM_ERR_STATE, "server_release: request %lld is not finished", (long long)id);
  S->table.erase(it);
  return FSLBM_OK;
}

extern "C" int fslbm_server_stats_get(fslbm_server* S, fslbm_server_stats* out) {
  if (!S || !out) return fslbm_set_error(FSLBM_ERR_ARG, "server_stats: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->st;
  return FSLBM_OK;
}
