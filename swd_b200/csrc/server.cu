// Served request loop: misfit and gradient requests of any survey size, admitted by HBM
// footprint and run concurrently on one GPU.
//
// Each admitted request owns a gradient engine (its own stream, memory and CUDA graphs) and
// runs on a worker thread, so the kernels of requests in flight overlap on the device.  A
// request that arrives while others run is admitted as soon as a slot is free and the
// memory its engine plans fits beside the engines in use; requests are admitted in arrival
// order.  A finished request's engine stays resident, keyed by the caller's survey key, so
// the next request on the same survey (the next inversion iteration, or a line-search
// misfit) reuses its device memory, Radon tables and captured time loops; idle engines are
// freed, least recently used first, when a new request needs their memory.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "fd_host.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  uint64_t id = 0;
  uint64_t key = 0;
  int kind = SWD_REQ_GRADIENT;
  swd_survey sv{};
  std::vector<int> sx, sz, shot_no;
  std::vector<double> wavelet, vp, vs, cr0_r, cr0_l;
  // results
  std::vector<double> dk, res_r, res_l, crp_r, crp_l;
  double residual = 0.0;
  int status = SWD_OK;
  std::string err;
  bool done = false, cancelled = false, reused = false;
  bool cancel_running = false;  // cancelled after it started: its engine's time loops are told to stop
  swd_engine* eng = nullptr;    // the engine running it (set by its worker, under the server lock)
  size_t bytes = 0;
  Clock::time_point t_submit, t_start, t_done;
};

struct Idle {
  uint64_t key;
  swd_survey sv;  // pointers cleared; compared field by field before reuse
  swd_engine* eng;
  size_t bytes;
};

bool same_survey(const swd_survey& a, const swd_survey& b) {
  swd_survey x = a, y = b;
  x.sx = y.sx = nullptr;
  x.sz = y.sz = nullptr;
  x.shot_no = y.shot_no = nullptr;
  return std::memcmp(&x, &y, sizeof(x)) == 0;
}

}  // namespace

struct swd_server {
  swd_server_opts opt{};
  size_t budget = 0, in_use = 0;
  int inflight = 0;
  uint64_t next_id = 1;
  bool stopping = false;
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<uint64_t, std::shared_ptr<Request>> reqs;
  std::list<Idle> idle;  // front = most recently used
  std::thread sched;  // workers are detached; destroy waits for inflight == 0
  swd_server_stats_t st{};
};

namespace swd {

static void free_idle(swd_server* S, std::list<Idle>::iterator it) {
  swd_engine_destroy(it->eng);
  S->in_use -= it->bytes;
  S->idle.erase(it);
}

static int run_request(swd_server* S, Request& r, swd_engine* eng) {
  SWD_TRY(swd_engine_set_source(eng, r.wavelet.data()));
  SWD_TRY(swd_engine_set_observed(eng, r.cr0_r.data(), r.cr0_l.data()));
  const int ns = r.sv.ns;
  const size_t np2 = r.cr0_r.size() / (size_t)ns;
  r.res_r.assign(ns, 0.0);
  r.res_l.assign(ns, 0.0);
  r.crp_r.assign(np2 * ns, 0.0);
  r.crp_l.assign(np2 * ns, 0.0);
  if (r.kind == SWD_REQ_MISFIT)
    return swd_engine_misfit(eng, r.vp.data(), r.vs.data(), r.res_r.data(), r.res_l.data(), r.crp_r.data(),
                             r.crp_l.data(), &r.residual);
  r.dk.assign(r.vp.size(), 0.0);
  swd_gradient_out o{};
  o.dk_vs = r.dk.data();
  o.res_r = r.res_r.data();
  o.res_l = r.res_l.data();
  o.cr_pre_r = r.crp_r.data();
  o.cr_pre_l = r.crp_l.data();
  const int rc = swd_engine_gradient(eng, r.vp.data(), r.vs.data(), &o);
  r.residual = o.residual;
  (void)S;
  return rc;
}

// One admitted request on its own thread; the engine goes back to the idle list afterwards.
static void worker(swd_server* S, std::shared_ptr<Request> r, swd_engine* eng) {
  int rc = cudaSetDevice(S->opt.device) == cudaSuccess ? SWD_OK : SWD_ERR_CUDA;
  if (rc == SWD_OK && !eng) {
    swd_engine_opts o{};
    o.hbm_budget = r->bytes;
    o.use_graphs = 1;
    o.device = S->opt.device;
    rc = swd_engine_create(&r->sv, &o, &eng);
  }
  if (rc == SWD_OK) {
    std::lock_guard<std::mutex> lk(S->mu);
    r->eng = eng;
    if (r->cancel_running) rc = swd_engine_cancel(eng);  // cancelled while its engine was being built
  }
  if (rc == SWD_OK) rc = run_request(S, *r, eng);
  std::string err = rc == SWD_OK ? "" : swd_last_error();
  std::lock_guard<std::mutex> lk(S->mu);
  if (r->cancel_running && eng) {
    // cancelled while running: a cancel that landed after the engine's call had finished is
    // still pending on the engine; withdraw it so that it cannot cancel the next request, and
    // report this one as cancelled either way
    const int crc = swd_engine_cancel_clear(eng);
    if (rc == SWD_OK || rc == SWD_ERR_CANCELLED) {
      rc = crc == SWD_OK ? SWD_ERR_CANCELLED : crc;
      err = crc == SWD_OK ? "request cancelled while running" : swd_last_error();
    }
  }
  r->status = rc;
  r->err = err;
  r->t_done = Clock::now();
  r->done = true;
  r->eng = nullptr;
  S->inflight--;
  S->st.completed++;
  // a cancelled call leaves its engine ready for the next one (the cancel word is cleared)
  if (eng && (rc == SWD_OK || rc == SWD_ERR_CANCELLED) && r->key != 0 && S->opt.keep_engines) {
    Idle d{r->key, r->sv, eng, r->bytes};
    d.sv.sx = d.sv.sz = nullptr;
    d.sv.shot_no = nullptr;
    S->idle.push_front(d);
  } else {
    if (eng) swd_engine_destroy(eng);
    S->in_use -= r->bytes;
  }
  S->cv_done.notify_all();
  S->cv_sched.notify_all();
}

// Admission in arrival order: the head request starts when a slot is free and its engine's
// planned bytes fit beside the engines in use (idle engines are freed to make room).
static void scheduler(swd_server* S) {
  std::unique_lock<std::mutex> lk(S->mu);
  while (true) {
    S->cv_sched.wait(lk, [&] { return S->stopping || (!S->queue.empty() && S->inflight < S->opt.max_inflight); });
    if (S->stopping) break;
    auto r = S->queue.front();
    if (r->cancelled) { S->queue.pop_front(); continue; }
    // an idle engine of the same survey: no new memory
    swd_engine* eng = nullptr;
    if (r->key != 0) {
      for (auto it = S->idle.begin(); it != S->idle.end(); ++it)
        if (it->key == r->key && same_survey(it->sv, r->sv)) {
          eng = it->eng;
          r->bytes = it->bytes;
          r->reused = true;
          S->idle.erase(it);
          break;
        }
    }
    if (!eng) {
      // plan against the per-request cap; wait for memory if it does not fit yet
      const size_t cap = S->budget / (size_t)S->opt.max_inflight;
      swd_engine_opts o{};
      o.hbm_budget = cap;
      o.device = S->opt.device;
      swd_engine_info_t inf{};
      swd_survey sv = r->sv;
      sv.sx = r->sx.data();
      sv.sz = r->sz.data();
      sv.shot_no = r->shot_no.empty() ? nullptr : r->shot_no.data();
      const int rc = swd_engine_plan(&sv, &o, &inf);
      if (rc != SWD_OK) {  // cannot run at all: fail it
        r->status = rc;
        r->err = swd_last_error();
        r->done = true;
        r->t_start = r->t_done = Clock::now();
        S->queue.pop_front();
        S->cv_done.notify_all();
        continue;
      }
      r->bytes = std::min(cap, inf.bytes + (inf.bytes >> 5));
      while (S->in_use + r->bytes > S->budget && !S->idle.empty()) free_idle(S, std::prev(S->idle.end()));
      if (S->in_use + r->bytes > S->budget && S->inflight == 0) {  // larger than the whole budget
        r->status = SWD_ERR_OOM;
        r->err = "request needs more device memory than the server's budget";
        r->done = true;
        r->t_start = r->t_done = Clock::now();
        S->queue.pop_front();
        S->cv_done.notify_all();
        continue;
      }
      if (S->in_use + r->bytes > S->budget) {
        S->st.waits_for_memory++;
        S->cv_sched.wait(lk);  // a request finishes and frees memory
        continue;
      }
      S->in_use += r->bytes;
    }
    S->queue.pop_front();
    S->inflight++;
    S->st.admitted++;
    S->st.peak_inflight = std::max(S->st.peak_inflight, S->inflight);
    S->st.peak_bytes = std::max(S->st.peak_bytes, S->in_use);
    r->t_start = Clock::now();
    // the request keeps its survey pointers valid through its own vectors
    r->sv.sx = r->sx.data();
    r->sv.sz = r->sz.data();
    r->sv.shot_no = r->shot_no.empty() ? nullptr : r->shot_no.data();
    std::thread(worker, S, r, eng).detach();
  }
}

}  // namespace swd

using namespace swd;

extern "C" {

int swd_server_create(const swd_server_opts* o, swd_server** out) {
  clear_error();
  SWD_CHECK(out, "null argument");
  *out = nullptr;
  auto S = std::make_unique<swd_server>();
  if (o) S->opt = *o;
  if (S->opt.max_inflight <= 0) S->opt.max_inflight = 4;
  SWD_CUDA(cudaSetDevice(S->opt.device));
  S->budget = S->opt.hbm_budget;
  if (S->budget == 0) {
    size_t fr = 0, tot = 0;
    SWD_CUDA(cudaMemGetInfo(&fr, &tot));
    S->budget = (size_t)(fr * 0.85);
  }
  S->sched = std::thread(scheduler, S.get());
  *out = S.release();
  return SWD_OK;
}

int swd_server_submit(swd_server* S, const swd_request* q, uint64_t* id) {
  clear_error();
  SWD_CHECK(S && q && q->survey && id, "null argument");
  const swd_survey& s = *q->survey;
  SWD_CHECK(s.ns >= 1 && s.sx && s.sz && s.nz >= 1 && s.nx >= 1, "survey needs ns >= 1 shots and a grid");
  SWD_CHECK(q->vp && q->vs && q->cr0_r && q->cr0_l && q->npair >= 1, "request needs vp, vs, cr0_r, cr0_l, npair");
  SWD_CHECK(q->kind == SWD_REQ_GRADIENT || q->kind == SWD_REQ_MISFIT, "kind must be SWD_REQ_GRADIENT or _MISFIT");
  auto r = std::make_shared<Request>();
  r->key = q->survey_key;
  r->kind = q->kind;
  r->sv = s;
  r->sx.assign(s.sx, s.sx + s.ns);
  r->sz.assign(s.sz, s.sz + s.ns);
  if (s.shot_no) r->shot_no.assign(s.shot_no, s.shot_no + s.ns);
  const size_t n = (size_t)s.nz * s.nx, c = (size_t)q->npair * s.ns;
  r->vp.assign(q->vp, q->vp + n);
  r->vs.assign(q->vs, q->vs + n);
  r->cr0_r.assign(q->cr0_r, q->cr0_r + c);
  r->cr0_l.assign(q->cr0_l, q->cr0_l + c);
  SWD_CHECK(q->wavelet, "request needs its source wavelet (nt samples)");
  r->wavelet.assign(q->wavelet, q->wavelet + s.nt);
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(S->mu);
  SWD_CHECK(!S->stopping, "server is shutting down");
  r->id = S->next_id++;
  S->reqs[r->id] = r;
  S->queue.push_back(r);
  S->st.submitted++;
  *id = r->id;
  S->cv_sched.notify_all();
  return SWD_OK;
}

int swd_server_wait(swd_server* S, uint64_t id, int timeout_ms, swd_request_result* out) {
  clear_error();
  SWD_CHECK(S && out, "null argument");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  SWD_CHECK(it != S->reqs.end(), "unknown request id %llu", (unsigned long long)id);
  auto r = it->second;
  auto ready = [&] { return r->done || r->cancelled; };
  if (timeout_ms < 0) S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    set_error("request %llu still running", (unsigned long long)id);
    return SWD_ERR_TIMEOUT;
  }
  S->reqs.erase(it);
  if (r->cancelled) {
    set_error("request %llu was cancelled", (unsigned long long)id);
    return SWD_ERR_CANCELLED;
  }
  out->status = r->status;
  out->residual = r->residual;
  out->queue_ms = ms_between(r->t_submit, r->t_start);
  out->run_ms = ms_between(r->t_start, r->t_done);
  out->total_ms = ms_between(r->t_submit, r->t_done);
  out->reused_engine = r->reused ? 1 : 0;
  out->engine_bytes = r->bytes;
  if (r->status != SWD_OK) {
    set_error("%s", r->err.c_str());
    return r->status;
  }
  if (out->dk_vs && !r->dk.empty()) std::memcpy(out->dk_vs, r->dk.data(), r->dk.size() * sizeof(double));
  if (out->res_r) std::memcpy(out->res_r, r->res_r.data(), r->res_r.size() * sizeof(double));
  if (out->res_l) std::memcpy(out->res_l, r->res_l.data(), r->res_l.size() * sizeof(double));
  if (out->cr_pre_r) std::memcpy(out->cr_pre_r, r->crp_r.data(), r->crp_r.size() * sizeof(double));
  if (out->cr_pre_l) std::memcpy(out->cr_pre_l, r->crp_l.data(), r->crp_l.size() * sizeof(double));
  return SWD_OK;
}

int swd_server_cancel(swd_server* S, uint64_t id) {
  clear_error();
  SWD_CHECK(S, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  SWD_CHECK(it != S->reqs.end(), "unknown request id %llu", (unsigned long long)id);
  auto& r = it->second;
  if (r->done) {
    set_error("request %llu already finished", (unsigned long long)id);
    return SWD_ERR_INVALID;
  }
  S->st.cancelled++;
  if (r->t_start != Clock::time_point{}) {
    // running: its engine's FD launches return at once from here on, and the call reports
    // SWD_ERR_CANCELLED to swd_server_wait; an engine still being built is told when it is ready
    r->cancel_running = true;
    if (r->eng) SWD_TRY(swd_engine_cancel(r->eng));
    return SWD_OK;
  }
  r->cancelled = true;
  S->cv_done.notify_all();
  S->cv_sched.notify_all();
  return SWD_OK;
}

int swd_server_stats(swd_server* S, swd_server_stats_t* out) {
  clear_error();
  SWD_CHECK(S && out, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->st;
  out->bytes_in_use = S->in_use;
  out->budget = S->budget;
  out->idle_engines = (int)S->idle.size();
  return SWD_OK;
}

int swd_server_destroy(swd_server* S) {
  clear_error();
  if (!S) return SWD_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
    for (auto& r : S->queue) r->cancelled = true;
    S->queue.clear();
    S->cv_sched.notify_all();
    S->cv_done.notify_all();
  }
  if (S->sched.joinable()) S->sched.join();
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->inflight == 0; });
  }
  for (auto& d : S->idle) swd_engine_destroy(d.eng);
  delete S;
  return SWD_OK;
}

}  // extern "C"
