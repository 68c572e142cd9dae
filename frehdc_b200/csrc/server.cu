// Continuous-batching server (include/frehd_b200.h, frehd_server_*): the served
// form's request loop in native code.
//
// One host thread owns a frehd_batch and steps it for as long as it holds
// domains.  Callers prepare a domain on their own thread (create, geometry,
// series, init: all on the domain's own stream, so preparing overlaps the
// stepping) and submit it with a step count.  Between two batch steps the
// thread admits waiting domains in submission order while the memory budget
// and the batched CG's CTA capacity allow (a request that does not fit waits
// for room; one that cannot fit an empty batch completes with
// FREHD_ERR_NOMEM), steps, and releases every domain that has run its steps
// into the completion queue that frehd_server_poll drains.  At most two steps
// are in flight on the device, so a domain admitted now joins within two steps
// instead of behind a long queue of launches.
//
// A domain whose step fails on the device (CFL > 20, where the reference
// exits, nsfunctions.c:1225-1231; a device wait that gave up) is evicted as
// soon as the server has waited for that step: it completes with the failure
// status and the steps it ran, and its slot and memory go to waiting requests
// at once.  A domain whose solves stopped at maxIter completes normally with
// FREHD_ERR_CG_NOCONVERGE as a warning.
//
// A domain's result does not depend on what shares the batch with it (the
// batch's guarantee), so the server only changes when results arrive.  The
// caller owns every domain throughout: the server neither creates nor
// destroys one, and a domain must not be touched between its submit and the
// poll that returns it.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "domain_host.h"
#include "frehd_internal.h"

using namespace frehd;

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  long long ticket = 0;
  frehd_domain *d = nullptr;
  int t0 = 1, nsteps = 0, taken = 0, slot = -1;
  double submitted = 0, admitted = -1;
};

constexpr int kInFlight = 2;  // batch steps queued on the device at most

}  // namespace

struct frehd_server {
  int device = 0;
  frehd_batch *batch = nullptr;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req> waiting;
  std::map<int, Req> active;  // by batch slot
  std::deque<frehd_server_done> done;
  bool stop = false;
  int fatal = FREHD_OK;
  char fatal_msg[256] = {0};
  long long next_ticket = 1, submitted = 0, completed = 0, cell_steps = 0, steps = 0;
  int max_active = 0;
  cudaEvent_t ev[kInFlight] = {};
  std::thread th;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void finish(frehd_server *s, const Req &r, int status, int steps) {
  frehd_server_done o;
  std::memset(&o, 0, sizeof(o));
  o.ticket = r.ticket;
  o.domain = r.d;
  o.status = status;
  o.steps = steps;
  o.t_submit = r.submitted;
  o.t_admit = r.admitted;
  o.t_done = s->now();
  s->done.push_back(o);
  ++s->completed;
}

// Record a failure of the batch itself: every request still held completes
// with it, and the thread stops.
void fail_all(frehd_server *s, int rc) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->fatal = rc;
  std::snprintf(s->fatal_msg, sizeof(s->fatal_msg), "%s", frehd_last_error());
  for (auto &kv : s->active) {
    frehd_batch_release(s->batch, kv.first, nullptr);
    finish(s, kv.second, rc, kv.second.taken);
  }
  s->active.clear();
  for (const Req &r : s->waiting) finish(s, r, rc, 0);
  s->waiting.clear();
  s->stop = true;
  s->cv_done.notify_all();
}

void loop(frehd_server *s) {
  if (cudaSetDevice(s->device) != cudaSuccess) {
    fail_all(s, fail(FREHD_ERR_CUDA, "server thread: cudaSetDevice failed"));
    return;
  }
  long long issued = 0;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->waiting.empty() || !s->active.empty(); });
      if (s->stop) return;
      // admission in submission order while there is room
      while (!s->waiting.empty()) {
        Req &r = s->waiting.front();
        int slot = -1;
        const int rc = frehd_batch_admit(s->batch, r.d, r.t0, &slot);
        if (rc == FREHD_ERR_NOMEM && !s->active.empty()) break;  // wait for room
        if (rc != FREHD_OK) {  // cannot fit even an empty batch, or a bad domain
          finish(s, r, rc, 0);
          s->waiting.pop_front();
          s->cv_done.notify_all();
          continue;
        }
        r.slot = slot;
        r.admitted = s->now();
        s->active[slot] = r;
        s->waiting.pop_front();
      }
      if ((int)s->active.size() > s->max_active) s->max_active = (int)s->active.size();
      if (s->active.empty()) continue;
    }
    // one step of every admitted domain; at most kInFlight steps queued
    cudaEvent_t &e = s->ev[issued % kInFlight];
    if (issued >= kInFlight) {
      if (cudaEventSynchronize(e) != cudaSuccess) {
        fail_all(s, fail(FREHD_ERR_CUDA, "server thread: step event failed"));
        return;
      }
      // evict the domains whose step failed on the device; their later queued
      // steps are skipped on the device, and the release waits for them
      std::lock_guard<std::mutex> lk(s->mu);
      bool any = false;
      for (auto it = s->active.begin(); it != s->active.end();) {
        const int st = batch_slot_status(s->batch, it->first);
        if (st == FREHD_OK) {
          ++it;
          continue;
        }
        Req &r = it->second;
        frehd_domain *d = nullptr;
        const int rr = frehd_batch_release(s->batch, it->first, &d);
        // the failing step is the last one the domain completed or began
        const int ran = rr ? r.taken : r.d->last.step - r.t0 + 1;
        s->cell_steps -= (long long)(r.taken - ran) * r.d->gr.nx * r.d->gr.ny;
        finish(s, r, rr ? rr : st, ran);
        any = true;
        it = s->active.erase(it);
      }
      if (any) s->cv_done.notify_all();
      if (any && s->active.empty()) continue;  // nothing left to step: admit first

    }
    int rc = frehd_batch_step(s->batch);
    void *stream = nullptr;
    if (!rc) rc = frehd_batch_stream(s->batch, &stream);
    if (!rc && cudaEventRecord(e, (cudaStream_t)stream) != cudaSuccess)
      rc = fail(FREHD_ERR_CUDA, "server thread: cudaEventRecord failed");
    if (rc) {
      fail_all(s, rc);
      return;
    }
    ++issued;
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->steps;
    bool any = false;
    for (auto it = s->active.begin(); it != s->active.end();) {
      Req &r = it->second;
      ++r.taken;
      s->cell_steps += (long long)r.d->gr.nx * r.d->gr.ny;
      if (r.taken < r.nsteps) {
        ++it;
        continue;
      }
      // release waits for the queued steps; the domain's last status comes with it
      frehd_domain *d = nullptr;
      const int rr = frehd_batch_release(s->batch, it->first, &d);
      int st = rr ? rr : r.d->last.status;
      if (st == FREHD_OK && domain_take_noconv(r.d) > 0) st = FREHD_ERR_CG_NOCONVERGE;
      finish(s, r, st, rr ? r.taken : r.d->last.step - r.t0 + 1);
      any = true;
      it = s->active.erase(it);
    }
    if (any) s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" int frehd_server_create(int device, long long hbm_budget_bytes, double cells_per_cta,
                                   frehd_server **out) {
  clear_error();
  if (!out) return fail(FREHD_ERR_INVALID, "null argument");
  *out = nullptr;
  frehd_server *s = new frehd_server();
  s->device = device;
  s->t0 = Clock::now();
  int rc = frehd_batch_create(device, hbm_budget_bytes, cells_per_cta, &s->batch);
  for (int k = 0; k < kInFlight && !rc; ++k)
    if (cudaEventCreateWithFlags(&s->ev[k], cudaEventDisableTiming) != cudaSuccess)
      rc = fail(FREHD_ERR_CUDA, "cudaEventCreate failed");
  if (rc) {
    for (cudaEvent_t &e : s->ev)
      if (e) cudaEventDestroy(e);
    if (s->batch) frehd_batch_destroy(s->batch);
    delete s;
    return rc;
  }
  s->th = std::thread(loop, s);
  *out = s;
  return FREHD_OK;
}

extern "C" int frehd_server_submit(frehd_server *s, frehd_domain *d, int t0, int nsteps,
                                   long long *ticket) {
  clear_error();
  if (!s || !d || !ticket || nsteps < 1) return fail(FREHD_ERR_INVALID, "bad argument");
  if (!d->ready) return fail(FREHD_ERR_STATE, "domain has no state (init or upload first)");
  if (d->in_batch) return fail(FREHD_ERR_STATE, "domain is already in a batch");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(s->fatal ? s->fatal : FREHD_ERR_STATE, "server stopped: %s", s->fatal_msg);
  for (const Req &r : s->waiting)
    if (r.d == d) return fail(FREHD_ERR_STATE, "domain already submitted");
  for (const auto &kv : s->active)
    if (kv.second.d == d) return fail(FREHD_ERR_STATE, "domain already submitted");
  Req r;
  r.ticket = s->next_ticket++;
  r.d = d;
  r.t0 = t0;
  r.nsteps = nsteps;
  r.submitted = s->now();
  s->waiting.push_back(r);
  ++s->submitted;
  *ticket = r.ticket;
  s->cv_work.notify_one();
  return FREHD_OK;
}

extern "C" int frehd_server_poll(frehd_server *s, frehd_server_done *out, int cap, int timeout_ms,
                                 int *n) {
  clear_error();
  if (!s || !n || cap < 0 || (cap > 0 && !out)) return fail(FREHD_ERR_INVALID, "bad argument");
  std::unique_lock<std::mutex> lk(s->mu);
  if (timeout_ms > 0 && s->done.empty())
    s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty(); });
  int k = 0;
  while (k < cap && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  *n = k;
  return FREHD_OK;
}

extern "C" int frehd_server_info(frehd_server *s, frehd_server_info_t *out) {
  if (!s || !out) return fail(FREHD_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->waiting = (int)s->waiting.size();
  out->active = (int)s->active.size();
  out->max_active = s->max_active;
  out->batch_steps = s->steps;
  out->cell_steps = s->cell_steps;
  out->clock = s->now();
  out->status = s->fatal;
  return FREHD_OK;
}

extern "C" int frehd_server_destroy(frehd_server *s) {
  if (!s) return FREHD_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->th.joinable()) s->th.join();
  // requests still held go back to their owners unfinished
  for (auto &kv : s->active) frehd_batch_release(s->batch, kv.first, nullptr);
  s->active.clear();
  if (s->batch) frehd_batch_destroy(s->batch);
  for (cudaEvent_t &e : s->ev)
    if (e) cudaEventDestroy(e);
  delete s;
  return FREHD_OK;
}
