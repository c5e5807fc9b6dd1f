// Slot lanes (see lanes.hpp).
#include "lanes.hpp"

#include <algorithm>
#include <cstdlib>
#include <string>

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

constexpr size_t round_up(size_t n, size_t a) { return (n + a - 1) / a * a; }

}  // namespace

Lane::Lane(msf_context* ctx, int nx, int ny, int slots, int priority, bool fair)
    : ctx_(ctx), nx_(nx), ny_(ny), B_(slots), priority_(priority), fair_(fair),
      plane_((int64_t)nx * ny) {}

Lane::~Lane() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (graph_pass_) cudaGraphExecDestroy(graph_pass_);
  if (graph_detect_) cudaGraphExecDestroy(graph_detect_);
  for (auto& e : ring_ev_)
    if (e) cudaEventDestroy(e);
  if (host_ring_) cudaFreeHost(host_ring_);
  psi_.release();
  table_.release();
  partial_.release();
  err_.release();
  if (stream_) cudaStreamDestroy(stream_);
}

msf_status Lane::init() {
  if (ctx_->fp64) {
    set_error("slot batches run FP32 wavefields: create the context with MSF_FP32");
    return MSF_ERR_UNSUPPORTED;
  }
  if (B_ <= 0 || !supported_length(nx_) || !supported_length(ny_)) {
    set_error("invalid lane shape");
    return MSF_ERR_ARG;
  }
  MSF_CUDA(cudaSetDevice(ctx_->device));
  MSF_CUDA(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, priority_));
  MSF_TRY(ctx_->alloc(&psi_, 8 * (size_t)plane_ * B_));
  // idle slots are still read by the column pass's tile copies
  MSF_CUDA(cudaMemsetAsync(psi_.p, 0, psi_.bytes, stream_));
  shift_off_ = round_up(sizeof(SlotPass) * B_ + sizeof(DetectTable) +
                            sizeof(DetectSlot) * B_, 256);
  table_bytes_ = round_up(shift_off_ + sizeof(int32_t) * 2 * B_, 256);
  MSF_TRY(ctx_->alloc(&table_, table_bytes_));
  MSF_CUDA(cudaMemsetAsync(table_.p, 0, table_bytes_, stream_));
  MSF_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&host_ring_), kRing * table_bytes_,
                         cudaHostAllocDefault));
  for (auto& e : ring_ev_) MSF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  MSF_TRY(ctx_->alloc(&err_, sizeof(int)));
  MSF_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_));
  pipe_col_ = (ctx_->pipe & MSF_PIPE_COL) && pipe_supported(nx_, ny_);
  // MSF_LANE_GROUPS=0: every step runs the slot passes (the two paths give
  // the same bits; the switch lets tests and benchmarks compare them)
  const char* u = std::getenv("MSF_LANE_GROUPS");
  groups_ok_ = !(u && u[0] == '0');
  if (pipe_col_) MSF_CUDA(encode_column_map(psi_.p, B_, nx_, ny_, col_map_));
  row_.psi = col_.psi = psi_.p;
  row_.batch_stride = col_.batch_stride = plane_;
  row_.nb = col_.nb = B_;
  row_.nx = col_.nx = nx_;
  row_.ny = col_.ny = ny_;
  MSF_TRY(ctx_->twiddles(ny_, false, &row_.tw));
  MSF_TRY(ctx_->twiddles(nx_, false, &col_.tw));
  row_.slots = col_.slots = static_cast<const SlotPass*>(table_.p);
  row_.prefetch_tables = (ctx_->pipe & MSF_ROW_PREFETCH) ? 1 : 0;
  slot_.assign(B_, Slot{});
  return MSF_OK;
}

msf_status Lane::grow_chunks(int n_chunks) {
  MSF_CUDA(cudaStreamSynchronize(stream_));
  if (graph_detect_) {  // it holds the old scratch pointer
    cudaGraphExecDestroy(graph_detect_);
    graph_detect_ = nullptr;
  }
  max_chunks_ = std::max(n_chunks, 1);
  MSF_TRY(ctx_->alloc(&partial_, sizeof(double) * 2 * (size_t)B_ * max_chunks_));
  return MSF_OK;
}

msf_status Lane::add(SlotJob* job) {
  const Grid& g = job->plan.spec->g;
  if (g.nx != nx_ || g.ny != ny_) {
    set_error("raster grid does not match the lane");
    return MSF_ERR_ARG;
  }
  if (job->plan.mtf) {
    set_error("rasters with a detector MTF run through msf_run, not slot lanes");
    return MSF_ERR_UNSUPPORTED;
  }
  if (job->plan.n_chunks > max_chunks_) MSF_TRY(grow_chunks(job->plan.n_chunks));
  row_.inv_s = col_.inv_s = 1.0 / g.s;
  const msf_specimen* spec = job->plan.spec;
  if (!skip_decided_) {
    skip_decided_ = true;
    if (pipe_col_ && spec->n_live_groups > 0) {
      MSF_TRY(ctx_->alloc(&dead_bits_, spec->dead_bits.bytes));
      MSF_TRY(ctx_->alloc(&live_groups_, spec->live_groups.bytes));
      MSF_CUDA(cudaMemcpyAsync(dead_bits_.p, spec->dead_bits.p, spec->dead_bits.bytes,
                               cudaMemcpyDeviceToDevice, stream_));
      MSF_CUDA(cudaMemcpyAsync(live_groups_.p, spec->live_groups.p, spec->live_groups.bytes,
                               cudaMemcpyDeviceToDevice, stream_));
      h_live_ = spec->h_live_groups;
      h_dead_cols_.assign(ny_, 0);
      const int T = row_line_threads(ny_, false);
      for (int t = 0; t < T; ++t)
        for (int m = 0; m < ny_ / T; ++m)
          if ((spec->h_dead_bits[t] >> m) & 1u) h_dead_cols_[t + T * m] = 1;
      row_.row_dead_bits = dead_bits_.as<uint32_t>();
      col_.live_groups = live_groups_.as<int32_t>();
      col_.n_live_groups = (int)h_live_.size();
      skip_ = true;
    }
  } else if (skip_ && (spec->n_live_groups == 0 || spec->h_live_groups != h_live_)) {
    // a raster whose band limit removes other columns: every pass from now
    // on moves all columns.  The slots in flight hold stale values in the
    // columns that were skipped, which are zero in the full computation:
    // write those zeros first.
    MSF_CUDA(cudaStreamSynchronize(stream_));
    if (graph_pass_) {
      cudaGraphExecDestroy(graph_pass_);
      graph_pass_ = nullptr;
    }
    for (int j0 = 0; j0 < ny_;) {
      if (!h_dead_cols_[j0]) { ++j0; continue; }
      int j1 = j0;
      while (j1 < ny_ && h_dead_cols_[j1]) ++j1;
      MSF_CUDA(cudaMemset2DAsync(static_cast<char*>(psi_.p) + 8 * (size_t)j0, 8 * (size_t)ny_,
                                 0, 8 * (size_t)(j1 - j0), (size_t)nx_ * B_, stream_));
      j0 = j1;
    }
    row_.row_dead_bits = nullptr;
    col_.live_groups = nullptr;
    col_.n_live_groups = 0;
    skip_ = false;
  }
  job->next_probe = 0;
  job->started = job->done = 0;
  job->complete = false;
  if (!job->finished) MSF_CUDA(cudaEventCreateWithFlags(&job->finished, cudaEventDisableTiming));
  queue_.push_back(job);
  return MSF_OK;
}

msf_status Lane::launch_passes() {
  MSF_CUDA(launch_row(false, ROW_SLOTS, row_, stream_));
  if (pipe_col_)
    MSF_CUDA(launch_col_slice_pipe(col_, false, col_map_, err_.as<int>(), stream_));
  else
    MSF_CUDA(launch_col(false, COL_SLOTS, col_, stream_));
  return MSF_OK;
}

msf_status Lane::launch_group(const SlotJob* job, int s, int base, int nb) {
  const RasterPlan& P = job->plan;
  const msf_specimen* spec = P.spec;
  const bool last = s + 1 == P.S;
  // the lane's pass arguments (twiddles, removed columns) for wavefields
  // base .. base + nb - 1, with this slice's tables, as msf_run sets them
  PassArgs row = row_, col = col_;
  row.slots = col.slots = nullptr;
  row.psi = col.psi = static_cast<char*>(psi_.p) + 8 * plane_ * base;
  row.nb = col.nb = nb;
  row.shifts = reinterpret_cast<const int32_t*>(static_cast<const char*>(table_.p) +
                                                shift_off_) + 2 * base;
  row.trans = static_cast<const char*>(spec->t.p) + 8 * plane_ * s;
  row.psi0 = static_cast<const char*>(P.psi0_tab.p) + 8 * plane_ * s;
  // removed columns: read as zero after the first slice, stored (as zeros)
  // only at the last
  row.row_dead_io = row.row_dead_bits ? ((s > 0 ? 1 : 0) | (last ? 0 : 2)) : 0;
  // the tuned row variants that round as the slot pass does (the default
  // FFT schedule): L1 table prefetch, L2 row prefetch, lines by probe, staged
  const int pipe = ctx_->pipe_for(nx_, ny_);
  const bool staged = staged_row_supported(nx_, ny_) && (pipe & MSF_ROW_STAGED);
  row.prefetch_tables = (pipe & MSF_ROW_PREFETCH) ? 1 : 0;
  row.l2_ahead = 0;
  if (!staged && (pipe & MSF_ROW_L2AHEAD)) set_row_ahead(ctx_, spec, &row);
  row.lines_by_probe = (!staged && (pipe & MSF_ROW_BYPROBE)) ? 1 : 0;
  if (s > 0 && staged)
    MSF_CUDA(launch_row_split_staged(row, err_.as<int>(), stream_, 0));
  else
    MSF_CUDA(launch_row(false, s == 0 ? ROW_SPLIT_FIRST : ROW_SPLIT, row, stream_));
  col.px = static_cast<const char*>(spec->prop.p) + 8 * (size_t)(nx_ + ny_) * s;
  col.py = static_cast<const char*>(col.px) + 8 * (size_t)nx_;
  col.mask_lo = spec->mask_lo.as<int32_t>();
  col.mask_hi = spec->mask_hi.as<int32_t>();
  if (pipe_col_) {
    // the lane's tensor map starts at wavefield 0; a group further in gets
    // its own (encoding is a host call that allocates nothing)
    alignas(64) unsigned char map[128];
    const void* m = col_map_;
    if (base != 0) {
      MSF_CUDA(encode_column_map(col.psi, nb, nx_, ny_, map));
      m = map;
    }
    MSF_CUDA(launch_col_slice_pipe(col, last, m, err_.as<int>(), stream_));
  } else {
    MSF_CUDA(launch_col(false, last ? COL_SLICE_LAST : COL_SLICE, col, stream_));
  }
  return MSF_OK;
}

msf_status Lane::launch_detect() {
  const char* det = static_cast<const char*>(table_.p) + sizeof(SlotPass) * B_;
  MSF_CUDA(launch_slot_detect(det, B_, max_chunks_, nx_, ny_, partial_.as<double>(), true,
                              stream_));
  return MSF_OK;
}

namespace {
template <typename F>
msf_status capture_graph(cudaStream_t stream, F&& enqueue, cudaGraphExec_t* out) {
  std::lock_guard<std::recursive_mutex> cap(capture_mutex());
  cudaGraph_t graph;
  MSF_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  msf_status st = enqueue();
  cudaError_t ce = cudaStreamEndCapture(stream, &graph);
  if (st != MSF_OK) return st;
  MSF_CUDA(ce);
  MSF_CUDA(cudaGraphInstantiate(out, graph, 0));
  cudaGraphDestroy(graph);
  return MSF_OK;
}
}  // namespace

msf_status Lane::capture_passes() {
  return capture_graph(stream_, [this] { return launch_passes(); }, &graph_pass_);
}

msf_status Lane::capture_detect() {
  return capture_graph(stream_, [this] { return launch_detect(); }, &graph_detect_);
}

msf_status Lane::step() {
  if (!busy()) return MSF_OK;
  // refill idle slots, in slot order, from the queue: oldest raster first,
  // or (fair) the raster with the fewest probes in flight, which takes a
  // contiguous share of the idle slots (ceil(idle left / rasters waiting),
  // at most its waiting probes; then the choice is made again), so that a
  // raster's probes sit in neighbouring slots and can run as one group
  std::vector<int> idle;
  for (int i = 0; i < B_; ++i)
    if (!slot_[i].job) idle.push_back(i);
  for (size_t k = 0; k < idle.size() && !queue_.empty();) {
    auto pick = queue_.begin();
    if (fair_)
      for (auto it = queue_.begin(); it != queue_.end(); ++it)
        if ((*it)->started - (*it)->done < (*pick)->started - (*pick)->done) pick = it;
    SlotJob* j = *pick;
    const size_t left = idle.size() - k;
    int64_t take = fair_ ? (int64_t)((left + queue_.size() - 1) / queue_.size()) : (int64_t)left;
    take = std::min<int64_t>(take, j->plan.n_probes - j->next_probe);
    for (int64_t q = 0; q < take; ++q) {
      Slot& sl = slot_[idle[k++]];
      sl.job = j;
      sl.probe = j->next_probe++;
      sl.s = 0;
      ++j->started;
      ++active_;
    }
    if (j->next_probe == j->plan.n_probes) queue_.erase(pick);
  }

  // this step's table, in the next free ring entry
  const int r = (int)(steps_ % kRing);
  MSF_CUDA(cudaEventSynchronize(ring_ev_[r]));
  unsigned char* h = host_ring_ + (size_t)r * table_bytes_;
  SlotPass* sp = reinterpret_cast<SlotPass*>(h);
  DetectTable* dt = reinterpret_cast<DetectTable*>(h + sizeof(SlotPass) * B_);
  DetectSlot* de = reinterpret_cast<DetectSlot*>(dt + 1);
  std::vector<int> done;
  int32_t* hshift = reinterpret_cast<int32_t*>(h + shift_off_);
  // groups: runs of neighbouring active slots at one slice of one raster
  struct Group {
    const SlotJob* job;
    int s, base, nb;
  };
  std::vector<Group> groups;
  for (int i = 0; i < B_; ++i) {
    const Slot& sl = slot_[i];
    SlotPass p;
    if (sl.job) {
      Group* g = groups.empty() ? nullptr : &groups.back();
      if (g && g->base + g->nb == i && g->job == sl.job && g->s == sl.s)
        ++g->nb;
      else
        groups.push_back(Group{sl.job, sl.s, i, 1});
      hshift[2 * i] = sl.job->plan.shifts[2 * sl.probe];
      hshift[2 * i + 1] = sl.job->plan.shifts[2 * sl.probe + 1];
      const RasterPlan& P = sl.job->plan;
      const msf_specimen* spec = P.spec;
      p.op = sl.s == 0 ? SLOT_FIRST : SLOT_NEXT;
      p.last = sl.s + 1 == P.S;
      p.trans = static_cast<const char*>(spec->t.p) + 8 * plane_ * sl.s;
      p.psi0 = static_cast<const char*>(P.psi0_tab.p) + 8 * plane_ * sl.s;
      p.px = static_cast<const char*>(spec->prop.p) + 8 * (size_t)(nx_ + ny_) * sl.s;
      p.py = static_cast<const char*>(p.px) + 8 * (size_t)nx_;
      p.mask_lo = spec->mask_lo.as<int32_t>();
      p.mask_hi = spec->mask_hi.as<int32_t>();
      p.sx = P.shifts[2 * sl.probe];
      p.sy = P.shifts[2 * sl.probe + 1];
      if (p.last) done.push_back(i);
    }
    sp[i] = p;
  }
  // detection entries in (raster, probe) order
  std::sort(done.begin(), done.end(), [&](int a, int b) {
    const Slot &x = slot_[a], &y = slot_[b];
    if (x.job->order != y.job->order) return x.job->order < y.job->order;
    return x.probe < y.probe;
  });
  DetectTable t;
  t.n_done = (int32_t)done.size();
  for (size_t k = 0; k < done.size(); ++k) {
    const Slot& sl = slot_[done[k]];
    const RasterPlan& P = sl.job->plan;
    DetectSlot e;
    e.psi = psi_.as<float2>() + plane_ * done[k];
    e.psi0k = P.psi0k.as<double>();
    e.idx = P.seg_idx.as<int32_t>();
    e.chunk_begin = P.chunk_begin.as<int32_t>();
    e.seg_chunk = P.seg_chunk.as<int32_t>();
    e.amp = P.amp.as<double>() + sl.probe * P.n_seg;
    e.inten = P.inten.as<double>() + sl.probe * P.n_seg;
    if (P.pix_modes) {
      e.acc_a = P.acc_a.as<double>();
      e.acc_i = P.acc_i.as<double>();
      t.any_pixel = 1;
    }
    e.n_chunks = P.n_chunks;
    e.ng = P.n_seg;
    e.sx = P.shifts[2 * sl.probe];
    e.sy = P.shifts[2 * sl.probe + 1];
    e.chunk_offset = t.total_chunks;
    t.total_chunks += P.n_chunks;
    de[k] = e;
  }
  *dt = t;
  // a step of at most kMaxGroups groups runs each group through the batched
  // passes; more fragmented steps run the slot passes
  const bool grouped = groups_ok_ && !groups.empty() && (int)groups.size() <= kMaxGroups;
  // the slot part always; the detection part when some slot finishes; the
  // shifts on grouped steps
  const size_t pass_bytes = sizeof(SlotPass) * B_;
  const size_t det_bytes = t.n_done ? sizeof(DetectTable) + sizeof(DetectSlot) * t.n_done : 0;
  const size_t copy_bytes = grouped ? shift_off_ + sizeof(int32_t) * 2 * B_
                                    : pass_bytes + det_bytes;
  MSF_CUDA(cudaMemcpyAsync(table_.p, h, copy_bytes, cudaMemcpyHostToDevice, stream_));
  MSF_CUDA(cudaEventRecord(ring_ev_[r], stream_));

  if (grouped) {
    for (const Group& g : groups) MSF_TRY(launch_group(g.job, g.s, g.base, g.nb));
    launches_ += 2 * ((int64_t)groups.size() - 1);
    ++grouped_steps_;
  } else {
    // the first slot step runs its launches directly (kernel attributes
    // are set on first use); later ones replay the captured graph
    if (ctx_->graphs && slot_steps_ >= 1 && !graph_pass_) MSF_TRY(capture_passes());
    if (graph_pass_) {
      MSF_CUDA(cudaGraphLaunch(graph_pass_, stream_));
    } else {
      MSF_TRY(launch_passes());
    }
    ++slot_steps_;
  }
  launches_ += 2;
  if (t.n_done) {
    if (ctx_->graphs && steps_ >= 1 && !graph_detect_) MSF_TRY(capture_detect());
    if (graph_detect_) {
      MSF_CUDA(cudaGraphLaunch(graph_detect_, stream_));
    } else {
      MSF_TRY(launch_detect());
    }
    launches_ += 3;
  }
  ++steps_;

  // advance every active slot by one slice
  for (int i = 0; i < B_; ++i) {
    Slot& sl = slot_[i];
    if (!sl.job) continue;
    if (sl.s + 1 == sl.job->plan.S) {
      SlotJob* j = sl.job;
      if (++j->done == j->plan.n_probes) {
        MSF_CUDA(cudaEventRecord(j->finished, stream_));
        j->complete = true;
      }
      sl = Slot{};
      --active_;
    } else {
      ++sl.s;
    }
  }
  return MSF_OK;
}

msf_status Lane::synchronize() {
  MSF_CUDA(cudaStreamSynchronize(stream_));
  return MSF_OK;
}

msf_status Lane::check_error() {
  int flag = 0;
  MSF_CUDA(cudaMemcpyAsync(&flag, err_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  MSF_CUDA(cudaStreamSynchronize(stream_));
  if (flag) {
    set_error("a pipelined slice pass gave up waiting for a tile copy (bounded wait)");
    return MSF_ERR_TIMEOUT;
  }
  return MSF_OK;
}

}  // namespace msf
