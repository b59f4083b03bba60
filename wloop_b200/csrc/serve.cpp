// serve.cpp -- request loop for Wilson-loop measurements with continuous
// batching.  No counterpart in the reference (ms10 processes a fixed list of
// configurations one after the other, main/ms10.c:701-742).
//
// Requests (a lattice, its boundary condition, the loop parameters, the
// precision, and either a host gauge field or a synthetic-field seed) enter a
// FIFO queue.  max_inflight worker threads each repeatedly take the oldest
// pending request that fits, together with further pending requests of the
// same precision (any lattices and loop parameters; up to max_batch), as long
// as their device footprint fits both the server's memory budget (a fraction
// of the HBM free at start, counting the batch pool's idle memory, minus what
// the batches in flight reserve) and what cudaMemGetInfo reports free now.
// A request at the head of the queue that does not fit yet does not block
// the ones behind it: later requests that fit are admitted around it, until
// the head has waited longer than the bypass limit; from then on nothing
// else starts until the head has started, so a large request cannot starve.
// The group becomes one wlg_batch on the worker's own stream (a batch holds
// lattices of any sizes, each measured exactly as it would be alone):
// requests that arrive while others run are admitted as soon as a worker and
// memory free up, and the batches of different workers overlap on the
// device.  Each request's latency is measured from submission to the moment
// its result is on the host.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/wloop_b200.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Req {
  long long id = 0;
  wlg_request r;
  std::vector<double> links;  // host copy of the field, if one was given
  std::vector<double> wl;
  int state = 0;  // 0 pending, 1 running, 2 done, 3 failed
  std::string err;
  double t_submit = 0, t_start = 0, t_done = 0;
  long long bytes = 0;
  int batch_size = 0;
};

thread_local std::string g_serve_err;

}  // namespace

struct wlg_server {
  int dev = 0;
  long long budget = 0;
  long long reserved = 0;
  int max_batch = 8;
  double bypass_ms = 5000.0;  // how long the head of the queue may be bypassed
  std::vector<std::thread> workers;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<long long> pending;
  std::map<long long, Req*> reqs;
  long long next_id = 1;
  bool stop = false;
  long long completed = 0, failed = 0, batches = 0;
  double t_first_submit = -1, t_last_done = 0;
  std::vector<double> latencies;
};

namespace {

long long footprint(const wlg_request& r) {
  return wlg_batch_estimate_bytes(1, r.n, &r.bc, &r.parms, r.precision);
}

// requests that can share one batch: a batch has one precision
bool batchable(const wlg_request& a, const wlg_request& b) { return a.precision == b.precision; }

void fail_locked(wlg_server* s, Req* q, const std::string& msg) {
  q->state = 3;
  q->err = msg;
  q->t_done = now_ms();
  s->failed++;
}

void worker(wlg_server* s) {
  cudaSetDevice(s->dev);
  std::unique_lock<std::mutex> lk(s->m);
  while (true) {
    // ---- admission: oldest request plus same-shape followers that fit ----
    std::vector<Req*> group;
    long long need = 0;
    while (group.empty()) {
      if (s->stop && s->pending.empty()) return;
      if (s->pending.empty()) {
        s->cv_work.wait(lk);
        continue;
      }
      // requests that can never fit the budget fail at once, wherever they are
      bool failed_one = false;
      for (auto it = s->pending.begin(); it != s->pending.end();) {
        Req* q = s->reqs[*it];
        if (q->bytes > s->budget) {
          char buf[160];
          snprintf(buf, sizeof(buf), "request needs %.2f GB, more than the server budget %.2f GB",
                   q->bytes / 1e9, s->budget / 1e9);
          fail_locked(s, q, buf);
          it = s->pending.erase(it);
          failed_one = true;
        } else {
          ++it;
        }
      }
      if (failed_one) s->cv_done.notify_all();
      if (s->pending.empty()) continue;
      Req* head = s->reqs[s->pending.front()];
      size_t fr0 = 0, tot = 0;
      cudaMemGetInfo(&fr0, &tot);
      // free for a batch: the device's free memory plus what the batch pool
      // keeps idle from earlier batches
      const long long fr = (long long)fr0 + wlg_batch_pool_idle_bytes(s->dev);
      auto fits = [&](const Req* q, long long extra) {
        return s->reserved + extra + q->bytes <= s->budget && extra + q->bytes <= fr;
      };
      if (!fits(head, 0) && s->reserved == 0 && fr < head->bytes) {
        // nothing of ours is in flight: the device is full for other reasons
        s->pending.pop_front();
        fail_locked(s, head, "not enough free device memory");
        s->cv_done.notify_all();
        continue;
      }
      // the oldest request that fits; the head is bypassed only while it has
      // waited less than the bypass limit
      const bool head_may_wait = now_ms() - head->t_submit < s->bypass_ms;
      auto first = s->pending.end();
      for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
        if (fits(s->reqs[*it], 0)) {
          first = it;
          break;
        }
        if (!head_may_wait) break;  // only the head may start now
      }
      if (first == s->pending.end()) {
        // wait for a batch in flight to release memory (or for the head's
        // bypass window to close)
        s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        continue;
      }
      for (auto it = first; it != s->pending.end() && (int)group.size() < s->max_batch;) {
        Req* q = s->reqs[*it];
        if (group.empty() || (batchable(group[0]->r, q->r) && fits(q, need))) {
          group.push_back(q);
          need += q->bytes;
          it = s->pending.erase(it);
        } else {
          ++it;
        }
        if (!head_may_wait) break;  // a starving head starts alone
      }
    }
    s->reserved += need;
    double t0 = now_ms();
    for (Req* q : group) {
      q->state = 1;
      q->t_start = t0;
      q->batch_size = (int)group.size();
    }
    s->batches++;
    lk.unlock();

    // ---- one batch on this worker's stream ----
    const int k = (int)group.size();
    std::vector<int> dims(4 * k), bcs(k);
    std::vector<wlg_wloop_parms> parms(k);
    std::vector<uint64_t> seeds(k);
    std::vector<double> eps(k);
    for (int i = 0; i < k; i++) {
      memcpy(&dims[4 * i], group[i]->r.n, sizeof(int) * 4);
      bcs[i] = group[i]->r.bc;
      parms[i] = group[i]->r.parms;
      seeds[i] = group[i]->r.seed;
      eps[i] = group[i]->r.eps;
    }
    std::string err;
    wlg_batch* b = nullptr;
    if (wlg_batch_create(k, dims.data(), bcs.data(), parms.data(), group[0]->r.precision, s->dev,
                         &b)) {
      err = wlg_last_error();
    } else {
      wlg_batch_use_graph(b, 0);  // each batch runs once
      bool any_synth = false;
      for (int i = 0; i < k && err.empty(); i++) {
        if (!group[i]->links.empty()) {
          if (wlg_batch_upload(b, i, group[i]->links.data())) err = wlg_last_error();
        } else {
          any_synth = true;
        }
      }
      if (err.empty() && any_synth) {
        // generate synthetic fields for the requests without a host field
        // (those with one are uploaded again afterwards)
        if (wlg_batch_generate(b, seeds.data(), eps.data())) err = wlg_last_error();
        for (int i = 0; i < k && err.empty(); i++)
          if (!group[i]->links.empty() && wlg_batch_upload(b, i, group[i]->links.data()))
            err = wlg_last_error();
      }
      if (err.empty() && wlg_batch_run(b)) err = wlg_last_error();
      if (err.empty())
        for (int i = 0; i < k; i++) {
          const wlg_wloop_parms& p = group[i]->r.parms;
          group[i]->wl.resize((size_t)p.msl * p.msl * p.mwlt * p.mwlr * group[i]->r.n[0]);
          wlg_batch_result(b, i, group[i]->wl.data());
        }
      wlg_batch_destroy(b);
    }

    lk.lock();
    s->reserved -= need;
    double t1 = now_ms();
    for (Req* q : group) {
      if (err.empty()) {
        q->state = 2;
        q->t_done = t1;
        s->completed++;
        s->latencies.push_back(q->t_done - q->t_submit);
        s->t_last_done = std::max(s->t_last_done, t1);
      } else {
        fail_locked(s, q, err);
      }
      q->links.clear();
      q->links.shrink_to_fit();
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  double x = p / 100.0 * (v.size() - 1);
  size_t i = (size_t)x;
  double f = x - i;
  if (i + 1 >= v.size()) return v.back();
  return v[i] * (1 - f) + v[i + 1] * f;
}

}  // namespace

extern "C" {

int wlg_server_create(int device, double mem_fraction, int max_inflight, int max_batch,
                      wlg_server** out) {
  if (!out || max_inflight < 1 || max_batch < 1 || mem_fraction <= 0.0 || mem_fraction > 1.0)
    return -1;
  if (wlg_device_count() <= device || device < 0) return -1;
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return -1;
  wlg_server* s = new wlg_server();
  s->dev = device;
  // free for batches: the device's free memory and what the batch pool keeps
  // idle from earlier batches of this process
  s->budget = (long long)(mem_fraction * ((double)fr + (double)wlg_batch_pool_idle_bytes(device)));
  s->max_batch = max_batch;
  for (int i = 0; i < max_inflight; i++) s->workers.emplace_back(worker, s);
  *out = s;
  return 0;
}

int wlg_server_destroy(wlg_server* s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
  return 0;
}

long long wlg_server_submit(wlg_server* s, const wlg_request* r) {
  if (!s || !r) return -1;
  long long bytes = footprint(*r);
  if (bytes < 0) return -1;
  Req* q = new Req();
  q->r = *r;
  q->bytes = bytes;
  if (r->links) {
    long long vol = (long long)r->n[0] * r->n[1] * r->n[2] * r->n[3];
    q->links.assign(r->links, r->links + 4 * 18 * vol);
    q->r.links = nullptr;
  }
  q->t_submit = now_ms();
  std::lock_guard<std::mutex> lk(s->m);
  q->id = s->next_id++;
  if (s->t_first_submit < 0) s->t_first_submit = q->t_submit;
  s->reqs[q->id] = q;
  s->pending.push_back(q->id);
  s->cv_work.notify_one();
  return q->id;
}

int wlg_server_wait(wlg_server* s, long long id, double* wl_mat, double* latency_ms,
                    int* batch_size) {
  if (!s) return -1;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return -1;
  Req* q = it->second;
  s->cv_done.wait(lk, [&] { return q->state >= 2; });
  if (q->state == 3) {
    g_serve_err = q->err;
    return -1;
  }
  if (wl_mat) memcpy(wl_mat, q->wl.data(), q->wl.size() * sizeof(double));
  if (latency_ms) *latency_ms = q->t_done - q->t_submit;
  if (batch_size) *batch_size = q->batch_size;
  return 0;
}

int wlg_server_release(wlg_server* s, long long id) {
  if (!s) return -1;
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second->state < 2) return -1;
  delete it->second;
  s->reqs.erase(it);
  return 0;
}

const char* wlg_server_error(void) { return g_serve_err.c_str(); }

int wlg_server_stats(wlg_server* s, long long* completed, long long* failed, long long* batches,
                     double* p50_ms, double* p99_ms, double* throughput) {
  if (!s) return -1;
  std::lock_guard<std::mutex> lk(s->m);
  if (completed) *completed = s->completed;
  if (failed) *failed = s->failed;
  if (batches) *batches = s->batches;
  if (p50_ms) *p50_ms = percentile(s->latencies, 50.0);
  if (p99_ms) *p99_ms = percentile(s->latencies, 99.0);
  if (throughput) {
    double span = s->t_last_done - s->t_first_submit;
    *throughput = (span > 0 && s->completed > 0) ? s->completed / (span * 1e-3) : 0.0;
  }
  return 0;
}

long long wlg_server_budget(wlg_server* s) { return s ? s->budget : -1; }

int wlg_server_set_limits(wlg_server* s, long long budget_bytes, double bypass_ms) {
  if (!s) return -1;
  std::lock_guard<std::mutex> lk(s->m);
  if (budget_bytes > 0) s->budget = budget_bytes;
  if (bypass_ms >= 0.0) s->bypass_ms = bypass_ms;
  s->cv_work.notify_all();
  return 0;
}

}  // extern "C"
