// msf_run_batch: several rasters through slot lanes, one lane per grid size.
#include <algorithm>
#include <chrono>
#include <thread>
#include <map>
#include <memory>
#include <string>
#include <utility>

#include "engine.hpp"
#include "lanes.hpp"

namespace msf {

namespace {

#define MSF_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) +      \
                " at " + __FILE__ + ":" + std::to_string(__LINE__));        \
      return MSF_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

#define MSF_TRY(call)                \
  do {                               \
    msf_status s_ = (call);          \
    if (s_ != MSF_OK) return s_;     \
  } while (0)

}  // namespace

// Slots of a lane: `want`, or about 2 GiB of FP32 wavefields, clamped to
// [16, 256] (measured on B200: 256 slots at 512^2 and 1024^2, 64 at 2048^2;
// larger sets of wavefields run slower), bounded by the lane's probes and by
// half the free memory shared among `lanes` lanes.
int lane_slots(int want, int64_t plane, int lanes, int64_t probes) {
  if (want > 0) return want;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const int64_t cap = (int64_t)(0.5 * (double)free_b / std::max(1, lanes)) / (8 * plane);
  const int64_t footprint = std::max<int64_t>(16, std::min<int64_t>(256, (2LL << 30) / (8 * plane)));
  return (int)std::max<int64_t>(1, std::min<int64_t>({cap, footprint, probes}));
}

msf_status run_batch(msf_context* ctx, int n, const msf_specimen* const* specs,
                     const msf_optics* optics, const msf_raster* rasters,
                     const msf_detect* detects, msf_results* results, int slots) {
  if (n <= 0 || !specs || !optics || !rasters || !detects || !results) {
    set_error("null argument or empty batch");
    return MSF_ERR_ARG;
  }
  if (ctx->fp64) {
    set_error("slot batches run FP32 wavefields: create the context with MSF_FP32");
    return MSF_ERR_UNSUPPORTED;
  }
  for (int i = 0; i < n; ++i)
    if (!specs[i] || specs[i]->ctx != ctx) {
      set_error("specimen " + std::to_string(i) + " does not belong to this context");
      return MSF_ERR_ARG;
    }
  MSF_CUDA(cudaSetDevice(ctx->device));
  std::vector<std::unique_ptr<SlotJob>> jobs(n);
  for (int i = 0; i < n; ++i) {
    jobs[i] = std::make_unique<SlotJob>();
    jobs[i]->order = (uint64_t)i;
    MSF_TRY(plan_raster(ctx, specs[i], &optics[i], &rasters[i], &detects[i], &jobs[i]->plan));
  }
  // one lane per grid size, rasters in submission order
  std::map<std::pair<int, int>, std::vector<int>> groups;
  for (int i = 0; i < n; ++i) groups[{specs[i]->g.nx, specs[i]->g.ny}].push_back(i);
  std::vector<std::unique_ptr<Lane>> lanes;
  std::vector<int> lane_of(n);
  for (auto& kv : groups) {
    int64_t probes = 0;
    for (int i : kv.second) probes += jobs[i]->plan.n_probes;
    const int b = lane_slots(slots, (int64_t)kv.first.first * kv.first.second,
                             (int)groups.size(), probes);
    lanes.push_back(std::make_unique<Lane>(ctx, kv.first.first, kv.first.second, b));
    MSF_TRY(lanes.back()->init());
    for (int i : kv.second) {
      MSF_TRY(lanes.back()->add(jobs[i].get()));
      lane_of[i] = (int)lanes.size() - 1;
    }
  }
  // start events (timing), then round-robin steps over the lanes
  std::vector<cudaEvent_t> start(lanes.size());
  for (size_t l = 0; l < lanes.size(); ++l) {
    MSF_CUDA(cudaEventCreate(&start[l]));
    MSF_CUDA(cudaEventRecord(start[l], lanes[l]->stream()));
  }
  std::vector<cudaEvent_t> stop(n);
  for (int i = 0; i < n; ++i) MSF_CUDA(cudaEventCreate(&stop[i]));
  std::vector<bool> stamped(n, false);
  msf_status st = MSF_OK;
  bool any = true;
  while (any && st == MSF_OK) {
    // step every lane that can take a step without waiting, so that a lane
    // of small grids is not paced by one of large grids
    any = false;
    bool stepped = false;
    for (auto& lane : lanes) {
      if (!lane->busy()) continue;
      any = true;
      if (!lane->ready()) continue;
      st = lane->step();
      stepped = true;
      if (st != MSF_OK) break;
    }
    if (any && !stepped) std::this_thread::sleep_for(std::chrono::microseconds(20));
    for (int i = 0; i < n && st == MSF_OK; ++i)
      if (jobs[i]->complete && !stamped[i]) {
        cudaError_t e = cudaEventRecord(stop[i], lanes[lane_of[i]]->stream());
        if (e != cudaSuccess) {
          set_error(std::string("cudaEventRecord: ") + cudaGetErrorString(e));
          st = MSF_ERR_CUDA;
        }
        stamped[i] = true;
      }
  }
  for (auto& lane : lanes) {
    msf_status s2 = lane->synchronize();
    if (st == MSF_OK) st = s2;
    if (st == MSF_OK) st = lane->check_error();
  }
  for (int i = 0; i < n && st == MSF_OK; ++i) {
    const RasterPlan& P = jobs[i]->plan;
    Lane& lane = *lanes[lane_of[i]];
    float ms = 0;
    cudaEventElapsedTime(&ms, start[lane_of[i]], stop[i]);
    results[i].seconds_raster = 1e-3 * ms;
    results[i].seconds_setup = 0;
    results[i].probe_slices = P.n_probes * P.S;
    results[i].kernel_launches = P.setup_launches + lane.launches();
    st = finish_raster(ctx, P, lane.stream(), &results[i]);
  }
  for (auto e : start) cudaEventDestroy(e);
  for (auto e : stop) cudaEventDestroy(e);
  return st;
}

}  // namespace msf
