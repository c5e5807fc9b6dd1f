// Slot lanes: continuous batching of probes from several rasters.
//
// A lane owns `slots` FP32 wavefields of one grid size.  Every step runs one
// row pass and one column pass over all slots, each slot at its own slice of
// its own raster (specimen, probe, shift), then the detection of the slots
// that just finished their last slice.  A finished slot is refilled at the
// next step with the next waiting probe of any raster of that grid size, so
// rasters that arrive while others run join the same launches.
//
// Per step the host writes one table (SlotPass per slot, then the
// detection entries) into a pinned ring and copies it to a fixed device
// table; the launches of a step read only that table, so they are captured
// once as two CUDA graphs (the passes; the detection, replayed only on steps
// where some slot finishes) and replayed.
//
// The active slots of a step fall into groups: runs of neighbouring slots
// whose probes belong to one raster and are at one slice (probes that
// start together advance together, and refills hand each raster a
// contiguous run of slots).  A step of at most kMaxGroups groups runs each
// group through the batched passes of msf_run over its wavefields, with
// the probes' shifts from the step's table: the same arithmetic
// (bit-identical) without the per-slot table reads.  Steps more fragmented
// than that run the slot passes.
#pragma once
#include <cuda_runtime.h>

#include <deque>
#include <memory>
#include <vector>

#include "engine.hpp"
#include "kernels.h"

namespace msf {

// One raster taking part in slot batches.
struct SlotJob {
  RasterPlan plan;
  uint64_t order = 0;          // admission order: detection entries sort by it
  int64_t next_probe = 0;      // next probe to start
  int64_t started = 0, done = 0;
  cudaEvent_t finished = nullptr;  // recorded after the last detection
  bool complete = false;       // `finished` has been recorded
  ~SlotJob() {
    if (finished) cudaEventDestroy(finished);
  }
};

class Lane {
 public:
  // `priority`: the CUDA stream priority of the lane's launches (0: the
  // default; lower numbers are scheduled first).  `fair`: an idle slot takes
  // the next probe of the raster with the fewest probes in flight (oldest
  // first among equals), so a raster that arrives while a large one runs
  // gets its share of the slots at once; otherwise the oldest raster's
  // probes go first.  Neither changes any result: a probe's arithmetic does
  // not depend on its slot, and each raster's probes still start, finish
  // and are detected in probe order.
  Lane(msf_context* ctx, int nx, int ny, int slots, int priority = 0, bool fair = false);
  ~Lane();
  Lane(const Lane&) = delete;
  Lane& operator=(const Lane&) = delete;

  msf_status init();
  // The job's probes join the lane's queue (the job must outlive the lane's
  // use of it: until it is complete and the lane has synchronised).
  msf_status add(SlotJob* job);
  bool busy() const { return active_ > 0 || !queue_.empty(); }
  // True when step() would not wait for a free table in the ring.
  bool ready() const {
    return cudaEventQuery(ring_ev_[steps_ % kRing]) != cudaErrorNotReady;
  }
  // Plans and enqueues one step; no-op when idle.
  msf_status step();
  msf_status synchronize();
  // 0, or 1 when a pipelined pass gave up on a tile copy (bounded wait).
  msf_status check_error();
  cudaStream_t stream() const { return stream_; }
  int nx() const { return nx_; }
  int ny() const { return ny_; }
  int slots() const { return B_; }
  int64_t steps() const { return steps_; }
  int64_t launches() const { return launches_; }
  // steps that ran the batched passes per group of slots
  int64_t grouped_steps() const { return grouped_steps_; }

 private:
  struct Slot {
    SlotJob* job = nullptr;
    int64_t probe = -1;
    int s = 0;
  };
  msf_status capture_passes();
  msf_status capture_detect();
  msf_status launch_passes();
  msf_status launch_group(const SlotJob* job, int s, int base, int nb);
  msf_status launch_detect();
  msf_status grow_chunks(int n_chunks);

  msf_context* ctx_;
  int nx_, ny_, B_;
  int priority_ = 0;
  bool fair_ = false;
  int64_t plane_;
  cudaStream_t stream_ = nullptr;
  DevBuf psi_, table_, partial_, err_;
  int max_chunks_ = 0;
  bool pipe_col_ = false;
  // removed-column skipping: on while every raster the lane was given has
  // the same removed columns (the first one's); off for good otherwise
  bool skip_ = false, skip_decided_ = false;
  std::vector<int32_t> h_live_;
  std::vector<uint8_t> h_dead_cols_;  // [ny] 1: removed while skipping
  DevBuf dead_bits_, live_groups_;
  alignas(64) unsigned char col_map_[128];
  PassArgs row_, col_;
  size_t table_bytes_ = 0;
  size_t shift_off_ = 0;  // [B][2] int32 probe shifts after the detection part
  int64_t grouped_steps_ = 0, slot_steps_ = 0;
  static constexpr int kMaxGroups = 8;
  bool groups_ok_ = true;
  static constexpr int kRing = 4;
  unsigned char* host_ring_ = nullptr;  // kRing pinned tables
  cudaEvent_t ring_ev_[kRing] = {};
  cudaGraphExec_t graph_pass_ = nullptr;    // row + column pass
  cudaGraphExec_t graph_detect_ = nullptr;  // detection of finished slots
  std::vector<Slot> slot_;
  std::deque<SlotJob*> queue_;
  int active_ = 0;
  int64_t steps_ = 0, launches_ = 0;
  bool any_pixel_jobs_ = false;
};

}  // namespace msf
