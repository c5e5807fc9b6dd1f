// Launch tiling autotuner.  The reference plans its FFTs with FFTW_MEASURE
// and keeps the plans as a wisdom file per grid (tem.cpp:583-616, exported
// at 1748-1765).  Here what is measured per grid is the tiling of the
// batched slice passes: probes per launch, whether the column pass runs as
// the persistent TMA-pipelined kernel, whether the split-wave row pass
// stages its slice tables in shared memory (or prefetches them into L1), and
// that row pass's FFT radix
// schedule (32 elements a thread in two or three stages, or 16 in three;
// 8 and 16 at 256 points).  The winner is kept per context
// and can be saved and reloaded as text, like wisdom.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "engine.hpp"
#include "trace.hpp"
#include "kernels.h"

namespace msf {

namespace {

std::string device_tag(int device) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return "unknown";
  std::string s(prop.name);
  for (char& c : s)
    if (c == ' ' || c == '\t') c = '_';
  return s;
}

}  // namespace

msf_status tune(msf_context* ctx, const msf_specimen* spec, msf_tuning* out) {
  TraceScope trace_scope("tune");
  const Grid& g = spec->g;
  const int64_t plane = (int64_t)g.nx * g.ny;
  const size_t cbytes = ctx->fp64 ? 16 : 8;
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    set_error("cudaSetDevice failed");
    return MSF_ERR_CUDA;
  }
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  std::vector<int> batches;
  for (int b : {8, 16, 32, 64, 128, 256})
    if ((double)cbytes * plane * b <= 0.5 * (double)free_b) batches.push_back(b);
  if (batches.empty()) batches.push_back(1);
  std::vector<int> pipes{ctx->pipe};
  if (!ctx->pipe_env) {
    const bool col = pipe_supported(g.nx, g.ny, ctx->fp64);
    const bool staged = !ctx->fp64 && staged_row_supported(g.nx, g.ny);
    // column pass plain or pipelined; FP32 row pass plain (with or without
    // its L1 table and L2 wavefield prefetches, lines by row or by probe)
    // or staged, each on either FFT radix schedule
    std::vector<int> rows{0};
    if (staged)
      rows = {0,
              MSF_ROW_PREFETCH,
              MSF_ROW_L2AHEAD,
              MSF_ROW_PREFETCH | MSF_ROW_L2AHEAD,
              MSF_ROW_PREFETCH | MSF_ROW_BYPROBE,
              MSF_ROW_PREFETCH | MSF_ROW_L2AHEAD | MSF_ROW_BYPROBE,
              MSF_ROW_ALT,
              MSF_ROW_PREFETCH | MSF_ROW_ALT,
              MSF_ROW_STAGED,
              MSF_ROW_STAGED | MSF_ROW_ALT};
    pipes.clear();
    for (int c : col ? std::vector<int>{0, MSF_PIPE_COL} : std::vector<int>{0})
      for (int r : rows) pipes.push_back(c | r);
  }
  const int saved_pipe = ctx->pipe;
  ctx->tuned.erase({g.nx, g.ny});  // time_passes then runs ctx->pipe
  msf_context::Tuned best;
  double best_ns = INFINITY;
  for (int pipe : pipes) {
    ctx->pipe = pipe;
    for (int b : batches) {
      // about 20 ms of passes per candidate, at least three repetitions
      const double bytes = 4.0 * cbytes * plane * b;
      const int reps = (int)std::max(3.0, std::min(50.0, 0.02 / (bytes / 5e12)));
      double ms_row = 0, ms_col = 0;
      const msf_status st = time_passes(ctx, spec, b, reps, &ms_row, &ms_col);
      if (st != MSF_OK) {
        ctx->pipe = saved_pipe;
        return st;
      }
      const double ns = 1e6 * (ms_row + ms_col) / b;
      // a larger tiling must win by 1 % to be taken
      if (ns < 0.99 * best_ns) {
        best_ns = ns;
        best.batch = b;
        best.pipe = pipe;
        best.ns_per_probe_slice = ns;
      }
    }
  }
  ctx->pipe = saved_pipe;
  ctx->tuned[{g.nx, g.ny}] = best;
  if (out) {
    out->nx = g.nx;
    out->ny = g.ny;
    out->batch = best.batch;
    out->pipe = best.pipe;
    out->ns_per_probe_slice = best.ns_per_probe_slice;
  }
  return MSF_OK;
}

}  // namespace msf

extern "C" {

int64_t msf_wisdom_export(const msf_context* ctx, char* buf, int64_t cap) {
  if (!ctx) return 0;
  std::ostringstream os;
  const std::string dev = msf::device_tag(ctx->device);
  for (const auto& kv : ctx->tuned) {
    char line[256];
    std::snprintf(line, sizeof line, "msf-wisdom 1 %s %s %d %d %d %d %.3f\n", dev.c_str(),
                  ctx->fp64 ? "fp64" : "fp32", kv.first.first, kv.first.second,
                  kv.second.batch, kv.second.pipe, kv.second.ns_per_probe_slice);
    os << line;
  }
  const std::string s = os.str();
  if (buf && cap > 0) {
    const size_t n = std::min<size_t>(s.size(), (size_t)cap - 1);
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
  }
  return (int64_t)s.size();
}

msf_status msf_wisdom_import(msf_context* ctx, const char* text, int32_t* n_imported) {
  if (!ctx || !text) return MSF_ERR_ARG;
  const std::string dev = msf::device_tag(ctx->device);
  std::istringstream in(text);
  std::string line;
  int32_t n = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string magic, d, prec;
    int version = 0, nx = 0, ny = 0, batch = 0, pipe = 0;
    double ns = 0;
    if (!(ls >> magic >> version >> d >> prec >> nx >> ny >> batch >> pipe >> ns)) continue;
    if (magic != "msf-wisdom" || version != 1 || d != dev) continue;
    if (prec != (ctx->fp64 ? "fp64" : "fp32") || nx <= 0 || ny <= 0 || batch <= 0) continue;
    msf_context::Tuned t;
    t.batch = batch;
    t.pipe = pipe & MSF_PIPE_ALL;
    t.ns_per_probe_slice = ns;
    ctx->tuned[{nx, ny}] = t;
    ++n;
  }
  if (n_imported) *n_imported = n;
  return MSF_OK;
}

}  // extern "C"
