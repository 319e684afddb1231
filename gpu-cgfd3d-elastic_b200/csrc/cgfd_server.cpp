// cgfd_server.cpp -- serving loop: continuous admission of forward simulations onto one GPU.
//
// Requests (problem descriptions with their own sources) are queued by cgfd_server_submit from
// any thread. Two threads own the CUDA calls:
//   - admission (scheduler thread), in submission order, whenever a slot and HBM budget are
//     free: the request at the head of the queue is grouped with the queued requests on the
//     SAME grid (same model arrays and run parameters; only the sources differ), up to
//     max_batch, sized beforehand by cgfd_problem_bytes (its build high-water mark is reserved
//     from the budget) and handed to the builder thread;
//   - build (builder thread): cgfd_batch_create, i.e. the model upload and setup, which takes
//     tens to hundreds of milliseconds for a large grid; the ready problem goes back to the
//     scheduler. The scheduler never waits for a build, so resident problems keep their
//     slices queued while a new grid uploads;
//   - progress: every resident problem gets its time steps in slices of steps_per_slice, at
//     most two slices queued on its own stream, so problems of different grids and media run
//     side by side on the device and a newly admitted one starts while others are mid-run;
//   - retirement: when a problem's last slice completes, its seismograms are copied out per
//     request, the problem is destroyed (memory returns to the budget) and the next requests
//     are admitted at once.
// Latency = submit -> results ready (host steady clock); p50/p99 over completed requests.
// No counterpart in the reference (one simulation per process there).
#include <cuda_runtime.h>

#include <algorithm>
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

#include "cgfd_b200.h"
#include "cgfd_setup.h"

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { PENDING = 0, RUNNING = 1, DONE = 2, FAILED = 3 };

struct Request {
  long long id = 0;
  cgfd_problem_desc desc{};
  // owned copies of the source and station arrays (the model arrays stay the caller's)
  std::vector<float> loc, t_start, coefs, cmp, cmp_values, sta_loc;
  std::vector<int> wavelet, flag_coord, flag_depth;
  int state = PENDING;
  int rc = CGFD_OK;
  std::string err;
  std::vector<float> seis;  // [nsta][9][nt_total]
  int nsta = 0;
  Clock::time_point t_submit, t_done;
  double cell_stages = 0.0, source_steps = 0.0;
};

// requests on the same grid (same model arrays and run parameters) batch together
bool same_grid(const cgfd_problem_desc &a, const cgfd_problem_desc &b) {
  if (a.ni != b.ni || a.nj != b.nj || a.nk != b.nk || a.medium_type != b.medium_type) return false;
  if (a.medium_type == CGFD_MEDIUM_VISCO_ISO) return false;  // visco-elastic problems run one shot each
  if (a.coord != b.coord || a.metric != b.metric || a.medium != b.medium) return false;
  if (memcmp(a.pml, b.pml, sizeof(a.pml)) != 0) return false;
  if (a.free_top != b.free_top || a.dt != b.dt || a.t0 != b.t0 || a.nt_total != b.nt_total) return false;
  if (a.precision != b.precision || a.device != b.device) return false;
  if (a.sta.num != b.sta.num) return false;
  for (int n = 0; n < a.sta.num; n++) {
    if (a.sta.flag_coord[n] != b.sta.flag_coord[n] || a.sta.flag_depth[n] != b.sta.flag_depth[n]) return false;
    for (int c = 0; c < 3; c++)
      if (a.sta.loc[3 * n + c] != b.sta.loc[3 * n + c]) return false;
  }
  return true;
}

struct Slot {
  cgfd_problem *p = nullptr;
  std::vector<std::shared_ptr<Request>> reqs;
  int nt_total = 0, enqueued = 0;
  size_t bytes = 0;     // resident bytes once built
  size_t reserved = 0;  // budget held while building (the build's high-water mark)
  std::deque<std::pair<cudaEvent_t, int>> inflight;  // (event after a slice, steps up to it)
  int done_steps = 0;
};

}  // namespace

struct cgfd_server {
  cgfd_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::shared_ptr<Request>> pending;
  std::map<long long, std::shared_ptr<Request>> all;
  long long next_id = 1;
  bool stop = false;
  std::thread th;
  // scheduler-owned
  std::vector<Slot> slots;
  size_t in_use = 0;       // budget held by resident and building problems
  int building = 0;        // problems handed to the builder and not yet back
  // builder hand-off (under mu): groups to build, built problems (or failures) to take back
  std::deque<Slot> to_build, built;
  std::thread builder;
  // statistics (under mu)
  size_t peak = 0;
  long long batches = 0, completed = 0, failed = 0;
  std::vector<double> lat_ms;
  double work_cells = 0.0, work_sources = 0.0;
  bool any_start = false;
  Clock::time_point t_first, t_last;
  std::string fatal;

  void fail(const std::shared_ptr<Request> &r, int rc, const std::string &msg) {
    std::lock_guard<std::mutex> g(mu);
    r->state = FAILED;
    r->rc = rc;
    r->err = msg;
    r->t_done = Clock::now();
    failed++;
    cv.notify_all();
  }

  // admit queued requests while a slot and budget are free (scheduler thread)
  void admit() {
    while ((int)slots.size() + building < opts.max_active) {
      std::vector<std::shared_ptr<Request>> group;
      {
        std::lock_guard<std::mutex> g(mu);
        if (pending.empty()) return;
        group.push_back(pending.front());
        for (size_t n = 1; n < pending.size() && (int)group.size() < opts.max_batch; n++)
          if (same_grid(pending[n]->desc, group[0]->desc)) group.push_back(pending[n]);
      }
      std::vector<cgfd_source_desc> shots;
      for (auto &r : group) shots.push_back(r->desc.src);
      size_t resident = 0, peak_b = 0;
      int rc = cgfd_problem_bytes(&group[0]->desc, (int)group.size(), shots.data(), &resident, &peak_b);
      if (rc != CGFD_OK) {  // cannot happen for validated requests; fail the head only
        remove_pending({group[0]});
        fail(group[0], rc, cgfd_last_error());
        continue;
      }
      if (in_use + peak_b > opts.hbm_budget) {
        if (!slots.empty() || building > 0) return;  // wait for memory to free up (order kept)
        if (group.size() > 1) {      // try the head alone
          group.resize(1);
          shots.resize(1);
          rc = cgfd_problem_bytes(&group[0]->desc, 1, shots.data(), &resident, &peak_b);
        }
        if (rc != CGFD_OK || peak_b > opts.hbm_budget) {
          remove_pending({group[0]});
          fail(group[0], CGFD_ERR_NOMEM,
               "request needs " + std::to_string(peak_b) + " device bytes, budget " + std::to_string(opts.hbm_budget));
          continue;
        }
      }
      remove_pending(group);
      Slot s;
      s.reqs = group;
      s.nt_total = group[0]->desc.nt_total;
      s.reserved = peak_b;
      in_use += peak_b;
      building++;
      {
        std::lock_guard<std::mutex> g(mu);
        for (auto &r : group) r->state = RUNNING;
        batches++;
        peak = std::max(peak, in_use);
        if (!any_start) { any_start = true; t_first = Clock::now(); }
        to_build.push_back(std::move(s));
      }
      cv.notify_all();
    }
  }

  // builder thread: one batched problem at a time, off the scheduler's path
  void build_loop() {
    cudaSetDevice(opts.device);
    for (;;) {
      Slot s;
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return stop || !to_build.empty(); });
        if (stop) return;
        s = std::move(to_build.front());
        to_build.pop_front();
      }
      std::vector<cgfd_source_desc> shots;
      for (auto &r : s.reqs) shots.push_back(r->desc.src);
      const int rc = cgfd_batch_create(&s.reqs[0]->desc, (int)s.reqs.size(), shots.data(), &s.p);
      if (rc != CGFD_OK) {
        const std::string m = cgfd_last_error();
        for (auto &r : s.reqs) fail(r, rc, m);
        s.p = nullptr;
      } else {
        s.bytes = cgfd_device_bytes(s.p);
      }
      std::lock_guard<std::mutex> g(mu);
      built.push_back(std::move(s));
    }
  }

  // scheduler: take built problems back (the reservation becomes the resident size)
  void collect_built() {
    std::deque<Slot> ready;
    {
      std::lock_guard<std::mutex> g(mu);
      ready.swap(built);
    }
    for (Slot &s : ready) {
      building--;
      in_use -= s.reserved;
      if (!s.p) continue;  // failed build: its requests were failed by the builder
      in_use += s.bytes;
      slots.push_back(std::move(s));
    }
  }

  void remove_pending(const std::vector<std::shared_ptr<Request>> &g) {
    std::lock_guard<std::mutex> lk(mu);
    for (auto &r : g) {
      auto it = std::find(pending.begin(), pending.end(), r);
      if (it != pending.end()) pending.erase(it);
    }
  }

  // queue more slices, retire finished problems; returns true if anything progressed
  bool progress() {
    bool moved = false;
    for (size_t n = 0; n < slots.size();) {
      Slot &s = slots[n];
      // completed slices
      while (!s.inflight.empty()) {
        cudaError_t q = cudaEventQuery(s.inflight.front().first);
        if (q == cudaErrorNotReady) break;
        cudaEventDestroy(s.inflight.front().first);
        s.done_steps = s.inflight.front().second;
        s.inflight.pop_front();
        moved = true;
        if (q != cudaSuccess) { s.done_steps = -1; break; }
      }
      bool dead = s.done_steps < 0;
      // keep two slices queued
      while (!dead && s.enqueued < s.nt_total && s.inflight.size() < 2) {
        int k = std::min(opts.steps_per_slice, s.nt_total - s.enqueued);
        int rc = cgfd_enqueue_steps(s.p, k);
        cudaEvent_t e;
        if (rc != CGFD_OK || cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) { dead = true; break; }
        cudaEventRecord(e, (cudaStream_t)cgfd_stream(s.p));
        s.enqueued += k;
        s.inflight.emplace_back(e, s.enqueued);
        moved = true;
      }
      if (dead || s.done_steps >= s.nt_total) {
        retire(s, dead);
        slots.erase(slots.begin() + n);
        moved = true;
        continue;
      }
      n++;
    }
    return moved;
  }

  void retire(Slot &s, bool dead) {
    for (auto &ev : s.inflight) cudaEventDestroy(ev.first);
    s.inflight.clear();
    int rc = dead ? CGFD_ERR_CUDA : cgfd_synchronize(s.p);
    std::string msg = rc == CGFD_OK ? "" : (dead ? std::string("device error during the run") : cgfd_last_error());
    const int nsta = cgfd_num_stations(s.p), nsh = (int)s.reqs.size();
    std::vector<float> all_seis;
    if (rc == CGFD_OK && nsta > 0) {
      all_seis.resize((size_t)nsh * nsta * 9 * s.nt_total);
      rc = cgfd_get_seismograms(s.p, all_seis.data());
      if (rc != CGFD_OK) msg = cgfd_last_error();
    }
    cgfd_problem_destroy(s.p);
    s.p = nullptr;
    in_use -= s.bytes;
    const size_t per = (size_t)nsta * 9 * s.nt_total;
    for (int n = 0; n < nsh; n++) {
      auto &r = s.reqs[n];
      if (rc != CGFD_OK) { fail(r, rc, msg); continue; }
      std::lock_guard<std::mutex> g(mu);
      r->nsta = nsta;
      r->seis.assign(all_seis.begin() + per * n, all_seis.begin() + per * (n + 1));
      r->state = DONE;
      r->t_done = Clock::now();
      lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
      work_cells += r->cell_stages;
      work_sources += r->source_steps;
      completed++;
      t_last = r->t_done;
    }
    std::lock_guard<std::mutex> g(mu);
    cv.notify_all();
  }

  void loop() {
    if (cudaSetDevice(opts.device) != cudaSuccess) {
      std::lock_guard<std::mutex> g(mu);
      fatal = "cudaSetDevice failed";
    }
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu);
        if (stop) break;
        if (slots.empty() && pending.empty() && built.empty()) cv.wait_for(g, std::chrono::milliseconds(20));
        if (stop) break;
        if (!fatal.empty()) {
          for (auto &r : pending) { r->state = FAILED; r->rc = CGFD_ERR_CUDA; r->err = fatal; failed++; }
          pending.clear();
          cv.notify_all();
          continue;
        }
      }
      collect_built();
      admit();
      if (!progress()) std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    // shutdown: finish nothing further, release device state
    if (builder.joinable()) builder.join();
    collect_built();
    for (auto &s : slots) {
      for (auto &ev : s.inflight) cudaEventDestroy(ev.first);
      cgfd_synchronize(s.p);
      cgfd_problem_destroy(s.p);
      for (auto &r : s.reqs) {
        std::lock_guard<std::mutex> g(mu);
        if (r->state == RUNNING) { r->state = FAILED; r->rc = CGFD_ERR_BUSY; r->err = "server destroyed"; }
      }
    }
    slots.clear();
  }
};

namespace {
int fail_call(int rc, const std::string &m) {
  cgfd::set_last_error(m);
  return rc;
}
}  // namespace

extern "C" {

int cgfd_server_create(const cgfd_server_opts *opts, cgfd_server **out) {
  if (!out) return fail_call(CGFD_ERR_INVALID, "out is NULL");
  *out = nullptr;
  cgfd_server_opts o{};
  if (opts) o = *opts;
  if (o.max_active <= 0) o.max_active = 4;
  if (o.max_batch <= 0) o.max_batch = 8;
  if (o.steps_per_slice <= 0) o.steps_per_slice = 50;
  if (cudaSetDevice(o.device) != cudaSuccess) return fail_call(CGFD_ERR_CUDA, "cudaSetDevice failed (no GPU?)");
  if (o.hbm_budget == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return fail_call(CGFD_ERR_CUDA, "cudaMemGetInfo failed");
    o.hbm_budget = (size_t)(0.85 * (double)fr);
  }
  cgfd_server *s = new cgfd_server;
  s->opts = o;
  s->builder = std::thread([s] { s->build_loop(); });
  s->th = std::thread([s] { s->loop(); });
  *out = s;
  return CGFD_OK;
}

int cgfd_server_submit(cgfd_server *s, const cgfd_problem_desc *desc, long long *request_id) {
  if (!s || !desc || !request_id) return fail_call(CGFD_ERR_INVALID, "invalid argument");
  auto r = std::make_shared<Request>();
  r->desc = *desc;
  try {
    cgfd::validate_desc(desc);
  } catch (cgfd::Error &e) {
    return fail_call(e.code, e.what());
  }
  // own the source and station arrays
  const cgfd_source_desc &sd = desc->src;
  const int n = sd.num;
  if (n > 0) {
    r->loc.assign(sd.loc, sd.loc + 3 * n);
    r->t_start.assign(sd.t_start, sd.t_start + n);
    if (sd.stf_given == 0) {
      r->wavelet.assign(sd.wavelet, sd.wavelet + n);
      if (sd.wavelet_coefs) r->coefs.assign(sd.wavelet_coefs, sd.wavelet_coefs + 10 * n);
      r->cmp.assign(sd.cmp, sd.cmp + 9 * n);
    } else {
      r->cmp_values.assign(sd.cmp_values, sd.cmp_values + (size_t)9 * n * sd.stf_nt);
    }
  }
  cgfd_source_desc &od = r->desc.src;
  od.loc = r->loc.empty() ? nullptr : r->loc.data();
  od.t_start = r->t_start.empty() ? nullptr : r->t_start.data();
  od.wavelet = r->wavelet.empty() ? nullptr : r->wavelet.data();
  od.wavelet_coefs = r->coefs.empty() ? nullptr : r->coefs.data();
  od.cmp = r->cmp.empty() ? nullptr : r->cmp.data();
  od.cmp_values = r->cmp_values.empty() ? nullptr : r->cmp_values.data();
  const cgfd_station_desc &st = desc->sta;
  if (st.num > 0) {
    r->flag_coord.assign(st.flag_coord, st.flag_coord + st.num);
    r->flag_depth.assign(st.flag_depth, st.flag_depth + st.num);
    r->sta_loc.assign(st.loc, st.loc + 3 * st.num);
    r->desc.sta.flag_coord = r->flag_coord.data();
    r->desc.sta.flag_depth = r->flag_depth.data();
    r->desc.sta.loc = r->sta_loc.data();
  }
  if (desc->device != s->opts.device) return fail_call(CGFD_ERR_INVALID, "request device differs from the server's");
  r->cell_stages = (double)desc->ni * desc->nj * desc->nk * 4.0 * desc->nt_total;
  r->source_steps = (double)desc->nt_total;
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> g(s->mu);
  r->id = s->next_id++;
  s->pending.push_back(r);
  s->all[r->id] = r;
  *request_id = r->id;
  s->cv.notify_all();
  return CGFD_OK;
}

int cgfd_server_poll(cgfd_server *s, long long request_id, float *seismo_out, int *nsta) {
  if (!s) return fail_call(CGFD_ERR_INVALID, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->all.find(request_id);
  if (it == s->all.end()) return fail_call(CGFD_ERR_INVALID, "unknown request id");
  Request &r = *it->second;
  if (r.state == PENDING || r.state == RUNNING) return CGFD_ERR_BUSY;
  if (r.state == FAILED) return fail_call(r.rc, r.err);
  if (nsta) *nsta = r.nsta;
  if (seismo_out) {
    if (!r.seis.empty()) memcpy(seismo_out, r.seis.data(), r.seis.size() * sizeof(float));
    s->all.erase(it);  // results delivered: release them
  }
  return CGFD_OK;
}

int cgfd_server_wait(cgfd_server *s, long long request_id, double timeout_s) {
  if (!s) return fail_call(CGFD_ERR_INVALID, "server is NULL");
  std::unique_lock<std::mutex> g(s->mu);
  auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
  for (;;) {
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return fail_call(CGFD_ERR_INVALID, "unknown request id");
    if (it->second->state == DONE) return CGFD_OK;
    if (it->second->state == FAILED) return fail_call(it->second->rc, it->second->err);
    if (timeout_s >= 0 && Clock::now() >= deadline) return CGFD_ERR_BUSY;
    s->cv.wait_for(g, std::chrono::milliseconds(10));
  }
}

int cgfd_server_get_stats(cgfd_server *s, cgfd_server_stats *out) {
  if (!s || !out) return fail_call(CGFD_ERR_INVALID, "invalid argument");
  std::lock_guard<std::mutex> g(s->mu);
  cgfd_server_stats o{};
  o.submitted = s->next_id - 1;
  o.completed = s->completed;
  o.failed = s->failed;
  o.pending = (long long)s->pending.size();
  o.active = (long long)std::count_if(s->all.begin(), s->all.end(),
                                      [](const std::pair<const long long, std::shared_ptr<Request>> &e) {
                                        return e.second->state == RUNNING;
                                      });
  o.batches = s->batches;
  o.hbm_budget = s->opts.hbm_budget;
  o.hbm_in_use = s->in_use;
  o.hbm_peak = s->peak;
  if (!s->lat_ms.empty()) {
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)(f * (v.size() - 1) + 0.5))]; };
    o.p50_ms = q(0.50);
    o.p99_ms = q(0.99);
    double m = 0;
    for (double x : v) m += x;
    o.mean_ms = m / v.size();
    const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
    if (span > 0) {
      o.cell_stages_per_s = s->work_cells / span;
      o.source_steps_per_s = s->work_sources / span;
    }
  }
  *out = o;
  return CGFD_OK;
}

int cgfd_server_destroy(cgfd_server *s) {
  if (!s) return CGFD_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    for (auto &r : s->pending) { r->state = FAILED; r->rc = CGFD_ERR_BUSY; r->err = "server destroyed"; }
    s->pending.clear();
    for (auto &b : s->to_build)
      for (auto &r : b.reqs) { r->state = FAILED; r->rc = CGFD_ERR_BUSY; r->err = "server destroyed"; }
    s->to_build.clear();
    s->cv.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  if (s->builder.joinable()) s->builder.join();
  delete s;
  return CGFD_OK;
}

}  // extern "C"
