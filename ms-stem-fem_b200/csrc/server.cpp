// msf_server: a request loop with continuous batching over slot lanes.
//
// Submission copies the request into a FIFO and returns a ticket.  A worker
// thread owns the lanes and loops:
//   1. admit waiting requests in arrival order whose estimated device bytes
//      fit the budget (the oldest is always admitted when nothing runs or
//      builds); a request that does not fit lets later, smaller ones past
//      it until it has waited kBackfillWindow seconds, after which it holds
//      them back until memory frees up for it; admitted requests go to the
//      builder thread;
//   2. hand the probes of every request the builder finished to the lane of
//      its grid size (created on first use);
//   3. step every lane that has work and a free table in its ring (no
//      blocking, so a lane of small grids is not paced by a lane of large
//      ones; the lanes' streams overlap on the GPU);
//   4. finish the rasters whose completion event has fired (FEM statistics
//      on the host), publish their results and latency, free their memory.
// The builder thread builds specimens and raster plans on a context and
// stream of its own, so those set-up kernels overlap the lanes' steps
// instead of holding the worker; it takes the smallest admitted request
// first (unless one has waited kBackfillWindow seconds).  A request that
// arrives while others run joins the running launches as soon as slots of
// its grid size free up: lanes refill slots fairly across their rasters,
// and lanes of smaller grids run on higher-priority streams, so a small
// request is not queued behind the launches of a large one.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "lanes.hpp"
#include "msf.h"

namespace msf {
namespace {

// Seconds a request that does not fit the budget lets later requests be
// admitted (or built) before it.
constexpr double kBackfillWindow = 5.0;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Results of a finished request, owned by the server until polled.
struct Stored {
  msf_status status = MSF_OK;
  std::string error;
  int32_t nx = 0, ny = 0;  // the request's grid (latency by grid size)
  int64_t n_probes = 0;
  int32_t n_k = 0;
  std::vector<double> adf, k_lower, v[6], mean_a, mean_i, ring_a, ring_i;
  std::vector<int32_t> counts;
  int64_t probe_slices = 0, launches = 0;
  double seconds_setup = 0, seconds_raster = 0, latency = 0;
};

struct Request {
  uint64_t ticket = 0;
  msf_grid grid{};
  std::vector<double> q, xp, yp, mtf, mtf_domain_sqr;
  std::vector<uint32_t> z;
  msf_optics optics{};
  msf_detect det{};  // its MTF pointers are set to the copies above at admission
  double t_submit = 0;
};

struct Running {
  uint64_t ticket = 0;
  double t_submit = 0, t_admit = 0;
  std::unique_ptr<msf_specimen> spec;
  std::unique_ptr<SlotJob> job;
  Lane* lane = nullptr;
  double setup_s = 0;
};

// A request between admission and its lane: built on the builder thread.
struct Pending {
  Request r;
  Running run;
  int64_t need = 0;  // estimated device bytes, held against the budget
  msf_status status = MSF_OK;
  std::string error;
};

int64_t estimate_bytes(const Request& r) {
  const int64_t plane = (int64_t)r.grid.nx * r.grid.ny;
  double zlo = 0, zhi = 0;
  for (size_t k = 0; k < r.z.size(); ++k) {
    const double z = r.q[3 * k + 2];
    if (k == 0 || z < zlo) zlo = z;
    if (k == 0 || z > zhi) zhi = z;
  }
  const int dz = std::max(1, r.grid.dupe_z);
  const double span = (zhi - zlo) + (dz - 1) * r.grid.zperiod;
  const int64_t slices = (int64_t)(span / std::max(r.grid.min_slice, 1e-3)) + 2;
  // specimen: tau + propagators; plan: vacuum table, probe, sums; set-up
  // scratch (LUTs, FP64 slice) while building
  return 8 * plane * slices * 2 + 8 * (r.grid.nx + r.grid.ny) * slices + 64 * plane +
         (int64_t)(r.xp.size() * r.yp.size()) * 8 * (r.grid.nx + 4);
}

}  // namespace
}  // namespace msf

using namespace msf;

struct msf_server {
  msf_options opt{};
  msf_context* ctx = nullptr;   // lanes (worker thread)
  msf_context* bctx = nullptr;  // specimens and raster plans (builder thread)
  std::thread builder;
  std::condition_variable cv_build;
  std::deque<Pending> to_build, built;  // guarded by mu
  int64_t building_bytes = 0;
  int slots = 0;  // per lane; 0: by grid size (lane_slots)
  int64_t budget = 0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stopping = false;
  uint64_t next_ticket = 1;
  std::deque<Request> waiting;
  std::map<uint64_t, Stored> done;
  std::set<uint64_t> cancelled;  // admitted requests whose results are discarded
  std::set<uint64_t> live;       // submitted, not yet finished
  std::vector<double> latencies;
  std::map<std::pair<int, int>, std::vector<double>> latencies_by_grid;
  int64_t submitted = 0, completed = 0, failed = 0, running_n = 0, probe_slices = 0;
  double t_first = -1, t_last = 0;
  int64_t held_bytes = 0;
  // worker-only
  std::map<std::pair<int, int>, std::unique_ptr<Lane>> lanes;
  std::vector<Running> running;
  uint64_t order = 0;

  void publish(uint64_t ticket, Stored&& s) {
    std::lock_guard<std::mutex> lk(mu);
    live.erase(ticket);
    if (cancelled.erase(ticket)) {
      s = Stored();
      s.status = MSF_ERR_CANCELLED;
      s.error = "request " + std::to_string(ticket) + " was cancelled";
    }
    if (s.status == MSF_OK) {
      ++completed;
      latencies.push_back(s.latency);
      latencies_by_grid[{s.nx, s.ny}].push_back(s.latency);
      probe_slices += s.probe_slices;
      t_last = now_s();
    } else {
      ++failed;
    }
    done[ticket] = std::move(s);
    cv_done.notify_all();
  }

  // Builder thread: the specimen and the raster plan, on bctx's stream
  // (both end synchronised, so the lanes may read them at once).
  msf_status build(Request& r, Running* out) {
    out->ticket = r.ticket;
    out->t_submit = r.t_submit;
    out->t_admit = now_s();
    msf_atoms atoms;
    atoms.n_atoms = (int64_t)r.z.size();
    atoms.q = r.q.data();
    atoms.z = r.z.data();
    out->spec = std::make_unique<msf_specimen>();
    msf_status st = build_specimen(bctx, &r.grid, &atoms, out->spec.get());
    if (st != MSF_OK) return st;
    out->setup_s = out->spec->seconds_setup;
    out->job = std::make_unique<SlotJob>();
    msf_raster raster;
    raster.n_x = (int32_t)r.xp.size();
    raster.n_y = (int32_t)r.yp.size();
    raster.x_p = r.xp.data();
    raster.y_p = r.yp.data();
    r.det.mtf = r.mtf.empty() ? nullptr : r.mtf.data();
    r.det.mtf_domain_sqr = r.mtf_domain_sqr.empty() ? nullptr : r.mtf_domain_sqr.data();
    return plan_raster(bctx, out->spec.get(), &r.optics, &raster, &r.det, &out->job->plan);
  }

  void build_loop() {
    cudaSetDevice(bctx->device);
    for (;;) {
      Pending p;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_build.wait(lk, [&] { return stopping_builder || !to_build.empty(); });
        if (to_build.empty()) return;
        // smallest first, unless the oldest has waited the backfill window
        auto pick = to_build.begin();
        if (now_s() - pick->r.t_submit < kBackfillWindow)
          for (auto it = to_build.begin(); it != to_build.end(); ++it)
            if (it->need < pick->need) pick = it;
        p = std::move(*pick);
        to_build.erase(pick);
      }
      p.status = build(p.r, &p.run);
      if (p.status != MSF_OK) p.error = last_error_copy();
      {
        std::lock_guard<std::mutex> lk(mu);
        built.push_back(std::move(p));
      }
      cv_work.notify_one();
    }
  }
  bool stopping_builder = false;

  // Worker thread: a built request joins the lane of its grid size.
  msf_status join_lane(const Request& r, Running* out) {
    out->job->order = order++;
    msf_status st;
    const std::pair<int, int> key{r.grid.nx, r.grid.ny};
    auto it = lanes.find(key);
    if (it == lanes.end()) {
      const int64_t plane = (int64_t)r.grid.nx * r.grid.ny;
      const int b = lane_slots(slots, plane, (int)lanes.size() + 1, 1 << 30);
      // smaller grids on higher-priority streams: one step per 4x the pixels
      int least = 0, greatest = 0;
      cudaDeviceGetStreamPriorityRange(&least, &greatest);
      int lg = 0;
      while ((int64_t(1) << (lg + 1)) <= plane) ++lg;
      const int prio = std::min(least, std::max(greatest, greatest + (lg - 16) / 2));
      auto lane = std::make_unique<Lane>(ctx, r.grid.nx, r.grid.ny, b, prio, true);
      st = lane->init();
      if (st != MSF_OK) return st;
      it = lanes.emplace(key, std::move(lane)).first;
    }
    out->lane = it->second.get();
    return out->lane->add(out->job.get());
  }

  void finish(Running& r) {
    Stored s;
    const RasterPlan& P = r.job->plan;
    s.nx = r.lane->nx();
    s.ny = r.lane->ny();
    s.n_probes = P.n_probes;
    s.n_k = P.n_k;
    s.adf.assign(P.n_probes, 0.0);
    const int cap = std::max(1, P.n_k);
    s.k_lower.assign(cap, 0.0);
    s.counts.assign(cap, 0);
    for (auto& v : s.v) v.assign(cap, 0.0);
    if (P.pix_modes) {
      s.mean_a.assign(P.plane, 0.0);
      s.mean_i.assign(P.plane, 0.0);
    }
    if (P.fem) {
      s.ring_a.assign((size_t)P.n_probes * cap, 0.0);
      s.ring_i.assign((size_t)P.n_probes * cap, 0.0);
    }
    msf_results res{};
    res.adf_image = s.adf.data();
    res.cap_k = cap;
    res.k_lower = s.k_lower.data();
    res.bin_counts = s.counts.data();
    res.v_omega = s.v[0].data();
    res.vbar_r = s.v[1].data();
    res.v_re = s.v[2].data();
    res.omega_vimage = s.v[3].data();
    res.v_gt17 = s.v[4].data();
    res.v_rbar = s.v[5].data();
    if (P.pix_modes) {
      res.mean_amplitude = s.mean_a.data();
      res.mean_intensity = s.mean_i.data();
    }
    if (P.fem) {
      res.ring_amplitude = s.ring_a.data();
      res.ring_intensity = s.ring_i.data();
    }
    s.status = finish_raster(ctx, P, ctx->stream, &res);
    if (s.status == MSF_OK) s.status = r.lane->check_error();
    if (s.status != MSF_OK) s.error = last_error_copy();
    s.probe_slices = P.n_probes * P.S;
    s.launches = P.setup_launches + r.lane->launches();
    s.seconds_setup = r.setup_s;
    s.latency = now_s() - r.t_submit;
    s.seconds_raster = now_s() - r.t_admit;
    publish(r.ticket, std::move(s));
  }

  static std::string last_error_copy();

  void loop() {
    cudaSetDevice(ctx->device);
    for (;;) {
      bool worked = false;
      // 1. admission: to the builder
      {
        std::unique_lock<std::mutex> lk(mu);
        const double t = now_s();
        for (auto it = waiting.begin(); it != waiting.end();) {
          const int64_t need = estimate_bytes(*it);
          const bool idle = running.empty() && to_build.empty() && built.empty();
          if (!idle && ctx->allocated() + bctx->allocated() + building_bytes + need > budget) {
            // does not fit: later requests may pass it while it is young
            if (t - it->t_submit >= kBackfillWindow) break;
            ++it;
            continue;
          }
          Pending p;
          p.r = std::move(*it);
          p.need = need;
          it = waiting.erase(it);
          ++running_n;
          building_bytes += need;
          to_build.push_back(std::move(p));
          cv_build.notify_one();
          worked = true;
        }
      }
      // 2. built requests join their lanes
      for (;;) {
        Pending p;
        {
          std::lock_guard<std::mutex> lk(mu);
          if (built.empty()) break;
          p = std::move(built.front());
          built.pop_front();
          building_bytes -= p.need;
        }
        worked = true;
        msf_status st = p.status;
        if (st == MSF_OK) st = join_lane(p.r, &p.run);
        if (st != MSF_OK) {
          Stored s;
          s.status = st;
          s.error = p.status != MSF_OK ? p.error : last_error_copy();
          s.latency = now_s() - p.r.t_submit;
          {
            std::lock_guard<std::mutex> lk(mu);
            --running_n;
          }
          publish(p.r.ticket, std::move(s));
          continue;
        }
        running.push_back(std::move(p.run));
      }
      // 3. one step of every lane that can take one without waiting
      for (auto it = lanes.begin(); it != lanes.end();) {
        Lane* lane = it->second.get();
        if (!lane->busy() || !lane->ready()) {
          ++it;
          continue;
        }
        msf_status st = lane->step();
        worked = true;
        if (st == MSF_OK) {
          ++it;
          continue;
        }
        // fail every raster of this lane, then drop the lane (its slots
        // still point at the rasters) before their memory goes
        const std::string err = last_error_copy();
        it = lanes.erase(it);
        for (auto& r : running)
          if (r.lane == lane && r.job) {
            Stored s;
            s.status = st;
            s.error = err;
            s.latency = now_s() - r.t_submit;
            publish(r.ticket, std::move(s));
            r.job.reset();
          }
      }
      // 4. completions
      for (size_t i = 0; i < running.size();) {
        Running& r = running[i];
        const bool gone = !r.job;
        const bool fin = !gone && r.job->complete &&
                         cudaEventQuery(r.job->finished) == cudaSuccess;
        if (fin) finish(r);
        if (gone || fin) {
          worked = true;
          running.erase(running.begin() + i);
          std::lock_guard<std::mutex> lk(mu);
          --running_n;
          held_bytes = ctx->allocated() + bctx->allocated();
          continue;
        }
        ++i;
      }
      {
        std::unique_lock<std::mutex> lk(mu);
        held_bytes = ctx->allocated() + bctx->allocated();
        const bool empty =
            waiting.empty() && running.empty() && to_build.empty() && built.empty();
        if (stopping && empty) break;
        if (!worked) {
          if (empty)
            cv_work.wait_for(lk, std::chrono::milliseconds(50));
          else
            cv_work.wait_for(lk, std::chrono::microseconds(50));
        }
      }
    }
    for (auto& kv : lanes) kv.second->synchronize();
  }
};

std::string msf_server::last_error_copy() { return std::string(msf_last_error()); }

extern "C" {

msf_status msf_server_create(const msf_options* opt, int32_t slots, msf_server** out) {
  if (!out) return MSF_ERR_ARG;
  *out = nullptr;
  msf_options o{};
  if (opt) o = *opt;
  o.precision = MSF_FP32;
  msf_server* s = new msf_server;
  s->opt = o;
  msf_status st = msf_context_create(&o, &s->ctx);
  if (st != MSF_OK) {
    delete s;
    return st;
  }
  st = msf_context_create(&o, &s->bctx);
  if (st != MSF_OK) {
    msf_context_destroy(s->ctx);
    delete s;
    return st;
  }
  s->slots = slots > 0 ? slots : 0;
  if (o.hbm_budget > 0) {
    s->budget = o.hbm_budget;
  } else {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = (int64_t)(0.8 * (double)free_b);
  }
  s->ctx->budget = 0;  // admission enforces the budget; allocations may overshoot briefly
  s->bctx->budget = 0;
  s->builder = std::thread([s] { s->build_loop(); });
  s->worker = std::thread([s] { s->loop(); });
  *out = s;
  return MSF_OK;
}

msf_status msf_server_submit(msf_server* s, const msf_request* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return MSF_ERR_ARG;
  if (req->atoms.n_atoms < 0 || (req->atoms.n_atoms > 0 && (!req->atoms.q || !req->atoms.z)) ||
      req->raster.n_x <= 0 || req->raster.n_y <= 0 || !req->raster.x_p || !req->raster.y_p) {
    set_error("request: missing atoms or raster");
    return MSF_ERR_ARG;
  }
  Request r;
  r.grid = req->grid;
  r.q.assign(req->atoms.q, req->atoms.q + 3 * req->atoms.n_atoms);
  r.z.assign(req->atoms.z, req->atoms.z + req->atoms.n_atoms);
  r.xp.assign(req->raster.x_p, req->raster.x_p + req->raster.n_x);
  r.yp.assign(req->raster.y_p, req->raster.y_p + req->raster.n_y);
  r.optics = req->optics;
  r.det = req->detect;
  if (r.det.n_mtf > 0 && r.det.mtf && r.det.mtf_domain_sqr) {
    r.mtf.assign(r.det.mtf, r.det.mtf + r.det.n_mtf);
    r.mtf_domain_sqr.assign(r.det.mtf_domain_sqr, r.det.mtf_domain_sqr + r.det.n_mtf);
  } else {
    r.det.n_mtf = 0;
  }
  r.det.mtf = r.det.mtf_domain_sqr = nullptr;
  r.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) {
      set_error("server is stopping");
      return MSF_ERR_CANCELLED;
    }
    r.ticket = s->next_ticket++;
    *ticket = r.ticket;
    ++s->submitted;
    s->live.insert(r.ticket);
    if (s->t_first < 0) s->t_first = r.t_submit;
    s->waiting.push_back(std::move(r));
  }
  s->cv_work.notify_one();
  return MSF_OK;
}

msf_status msf_server_poll(msf_server* s, uint64_t ticket, int32_t wait_ms, msf_results* res) {
  if (!s || !res) return MSF_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (ticket == 0 || ticket >= s->next_ticket) {
    set_error("unknown ticket");
    return MSF_ERR_ARG;
  }
  auto ready = [&] { return s->done.count(ticket) > 0; };
  if (!ready() && wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  auto it = s->done.find(ticket);
  if (it == s->done.end()) return MSF_ERR_BUSY;
  Stored& d = it->second;
  if (d.status != MSF_OK) {
    set_error(d.error);
    const msf_status st = d.status;
    s->done.erase(it);
    return st;
  }
  if (d.n_k > res->cap_k && (res->k_lower || res->bin_counts || res->v_omega || res->vbar_r ||
                             res->v_re || res->omega_vimage || res->v_gt17 || res->v_rbar ||
                             res->ring_amplitude || res->ring_intensity)) {
    set_error("results.cap_k is smaller than the number of k bins (" + std::to_string(d.n_k) +
              ")");
    return MSF_ERR_ARG;
  }
  const size_t nk = (size_t)d.n_k;
  if (res->adf_image) std::memcpy(res->adf_image, d.adf.data(), d.adf.size() * 8);
  if (res->k_lower) std::memcpy(res->k_lower, d.k_lower.data(), nk * 8);
  if (res->bin_counts) std::memcpy(res->bin_counts, d.counts.data(), nk * 4);
  double* outs[6] = {res->v_omega, res->vbar_r, res->v_re, res->omega_vimage, res->v_gt17,
                     res->v_rbar};
  for (int m = 0; m < 6; ++m)
    if (outs[m]) std::memcpy(outs[m], d.v[m].data(), nk * 8);
  if (res->mean_amplitude && !d.mean_a.empty())
    std::memcpy(res->mean_amplitude, d.mean_a.data(), d.mean_a.size() * 8);
  if (res->mean_intensity && !d.mean_i.empty())
    std::memcpy(res->mean_intensity, d.mean_i.data(), d.mean_i.size() * 8);
  const size_t cap_src = std::max<size_t>(1, nk);
  for (int64_t p = 0; p < d.n_probes && !d.ring_a.empty(); ++p) {
    if (res->ring_amplitude)
      std::memcpy(res->ring_amplitude + p * res->cap_k, d.ring_a.data() + p * cap_src, nk * 8);
    if (res->ring_intensity)
      std::memcpy(res->ring_intensity + p * res->cap_k, d.ring_i.data() + p * cap_src, nk * 8);
  }
  res->n_k = d.n_k;
  res->probe_slices = d.probe_slices;
  res->kernel_launches = d.launches;
  res->seconds_setup = d.seconds_setup;
  res->seconds_raster = d.seconds_raster;
  s->done.erase(it);
  return MSF_OK;
}

msf_status msf_server_stats_get(msf_server* s, msf_server_stats* out) {
  if (!s || !out) return MSF_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  msf_server_stats st{};
  st.submitted = s->submitted;
  st.completed = s->completed;
  st.failed = s->failed;
  st.running = s->running_n;
  st.waiting = (int64_t)s->waiting.size();
  st.probe_slices = s->probe_slices;
  st.device_bytes = s->held_bytes;
  std::vector<double> l = s->latencies;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto q = [&](double f) {
      const size_t k = (size_t)std::min<double>((double)l.size() - 1, f * (double)l.size());
      return l[k];
    };
    st.p50_s = q(0.50);
    st.p99_s = q(0.99);
    st.max_s = l.back();
  }
  if (s->t_first >= 0 && s->t_last > s->t_first)
    st.probe_slices_per_s = (double)s->probe_slices / (s->t_last - s->t_first);
  *out = st;
  return MSF_OK;
}

int32_t msf_server_grid_stats_get(msf_server* s, msf_server_grid_stats* out, int32_t cap) {
  if (!s) return 0;
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<std::pair<int64_t, std::pair<int, int>>> grids;
  for (const auto& kv : s->latencies_by_grid)
    grids.push_back({(int64_t)kv.first.first * kv.first.second, kv.first});
  std::sort(grids.begin(), grids.end());
  for (int32_t k = 0; k < (int32_t)grids.size() && k < cap && out; ++k) {
    std::vector<double> l = s->latencies_by_grid[grids[k].second];
    std::sort(l.begin(), l.end());
    auto q = [&](double f) {
      const size_t i = (size_t)std::min<double>((double)l.size() - 1, f * (double)l.size());
      return l[i];
    };
    msf_server_grid_stats g{};
    g.nx = grids[k].second.first;
    g.ny = grids[k].second.second;
    g.completed = (int64_t)l.size();
    g.p50_s = q(0.50);
    g.p99_s = q(0.99);
    g.max_s = l.back();
    out[k] = g;
  }
  return (int32_t)grids.size();
}

msf_status msf_server_cancel(msf_server* s, uint64_t ticket) {
  if (!s) return MSF_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  const std::string why = "request " + std::to_string(ticket) + " was cancelled";
  auto fin = s->done.find(ticket);
  if (fin != s->done.end() && fin->second.status == MSF_OK) {
    fin->second = Stored();  // it ran (the statistics keep it); its results go
    fin->second.status = MSF_ERR_CANCELLED;
    fin->second.error = why;
    return MSF_OK;
  }
  if (!s->live.count(ticket) || s->cancelled.count(ticket)) {
    set_error("unknown, delivered or already cancelled ticket");
    return MSF_ERR_ARG;
  }
  for (auto it = s->waiting.begin(); it != s->waiting.end(); ++it)
    if (it->ticket == ticket) {
      s->waiting.erase(it);
      s->live.erase(ticket);
      Stored d;
      d.status = MSF_ERR_CANCELLED;
      d.error = why;
      ++s->failed;
      s->done[ticket] = std::move(d);
      s->cv_done.notify_all();
      return MSF_OK;
    }
  s->cancelled.insert(ticket);  // admitted: discarded when it finishes
  return MSF_OK;
}

msf_status msf_server_destroy(msf_server* s) {
  if (!s) return MSF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping_builder = true;
  }
  s->cv_build.notify_all();
  if (s->builder.joinable()) s->builder.join();
  s->running.clear();
  s->lanes.clear();
  msf_context_destroy(s->ctx);
  msf_context_destroy(s->bctx);
  delete s;
  return MSF_OK;
}

}  // extern "C"
