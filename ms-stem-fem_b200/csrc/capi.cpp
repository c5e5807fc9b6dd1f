// extern "C" entry points of libmsf.so (declared in include/msf.h).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"
#include "kernels.h"
#include "msf.h"
#include "setup.hpp"

namespace msf {
const char* last_error();
}

using namespace msf;

namespace {
Grid grid_of(const msf_grid* g) {
  const int dx = g->dupe_x > 0 ? g->dupe_x : 1, dy = g->dupe_y > 0 ? g->dupe_y : 1,
            dz = g->dupe_z > 0 ? g->dupe_z : 1;
  return make_grid(g->nx, g->ny, g->voltage, g->xperiod * dx, g->yperiod * dy, g->zperiod * dz,
                   g->xmin, g->ymin, g->zmin, g->xperiod, g->yperiod, g->zperiod);
}
}  // namespace

extern "C" {

int32_t msf_abi_version(void) { return MSF_ABI_VERSION; }

const char* msf_last_error(void) { return msf::last_error(); }

const char* msf_status_string(msf_status s) {
  switch (s) {
    case MSF_OK: return "ok";
    case MSF_ERR_ARG: return "invalid argument";
    case MSF_ERR_UNSUPPORTED: return "unsupported";
    case MSF_ERR_CUDA: return "CUDA error";
    case MSF_ERR_NOMEM: return "out of memory";
    case MSF_ERR_IO: return "I/O error";
    case MSF_ERR_PARSE: return "parse error";
    case MSF_ERR_TIMEOUT: return "timeout";
    case MSF_ERR_BUSY: return "busy";
    case MSF_ERR_CANCELLED: return "cancelled";
  }
  return "unknown status";
}

msf_status msf_context_create(const msf_options* opt, msf_context** out) {
  if (!out) return MSF_ERR_ARG;
  *out = nullptr;
  msf_options o{};
  o.precision = MSF_FP64;
  o.use_graphs = 1;
  if (opt) o = *opt;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error(std::string("no CUDA device available: ") + cudaGetErrorString(e));
    return MSF_ERR_CUDA;
  }
  if (o.device < 0 || o.device >= ndev) {
    set_error("device ordinal out of range");
    return MSF_ERR_ARG;
  }
  if (o.precision != MSF_FP64 && o.precision != MSF_FP32) {
    set_error("precision must be MSF_FP64 or MSF_FP32");
    return MSF_ERR_ARG;
  }
  e = cudaSetDevice(o.device);
  if (e != cudaSuccess) {
    set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return MSF_ERR_CUDA;
  }
  msf_context* c = new msf_context;
  c->device = o.device;
  c->fp64 = o.precision == MSF_FP64;
  c->batch = o.batch;
  c->graphs = o.use_graphs != 0;
  if (const char* p = std::getenv("MSF_PIPE")) {
    c->pipe = std::atoi(p);
    c->pipe_env = true;
  }
  if (const char* p = std::getenv("MSF_ROW_AHEAD_PCT")) c->row_ahead_pct = std::max(1, std::atoi(p));
  if (const char* p = std::getenv("MSF_POTENTIAL"))
    c->potential = std::string(p) == "direct" ? 1 : std::string(p) == "fft" ? 2 : 0;
  c->budget = o.hbm_budget;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    set_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    return MSF_ERR_CUDA;
  }
  *out = c;
  return MSF_OK;
}

msf_status msf_context_destroy(msf_context* ctx) {
  if (!ctx) return MSF_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->tw64.clear();
  ctx->tw32.clear();
  {  // buffers released after this point free their memory directly
    std::lock_guard<std::mutex> lock(ctx->pool->m);
    ctx->pool->closed = true;
  }
  ctx->pool->trim();
  if (ctx->host_stage) {
    std::lock_guard<std::recursive_mutex> cap(msf::capture_mutex());
    cudaFreeHost(ctx->host_stage);
  }
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MSF_OK;
}

msf_status msf_context_synchronize(msf_context* ctx) {
  if (!ctx) return MSF_ERR_ARG;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    set_error(std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
    return MSF_ERR_CUDA;
  }
  return MSF_OK;
}

msf_status msf_context_transfer_bytes(msf_context* ctx, int64_t* h2d, int64_t* d2h,
                                      int32_t reset) {
  if (!ctx) return MSF_ERR_ARG;
  if (h2d) *h2d = ctx->h2d_bytes;
  if (d2h) *d2h = ctx->d2h_bytes;
  if (reset) ctx->h2d_bytes = ctx->d2h_bytes = 0;
  return MSF_OK;
}

msf_status msf_specimen_create(msf_context* ctx, const msf_grid* grid, const msf_atoms* atoms,
                               msf_specimen** out) {
  if (!ctx || !grid || !atoms || !out) return MSF_ERR_ARG;
  *out = nullptr;
  msf_specimen* s = new msf_specimen;
  msf_status st = build_specimen(ctx, grid, atoms, s);
  if (st != MSF_OK) {
    delete s;
    return st;
  }
  *out = s;
  return MSF_OK;
}

msf_status msf_specimen_destroy(msf_specimen* spec) {
  if (spec) {
    if (spec->ctx) cudaSetDevice(spec->ctx->device);
    delete spec;
  }
  return MSF_OK;
}

msf_status msf_specimen_slices(const msf_specimen* spec, int32_t* n_slices, double* lower,
                               double* thickness, int64_t* atoms_per_slice, int32_t cap) {
  if (!spec) return MSF_ERR_ARG;
  if (n_slices) *n_slices = spec->n_slices;
  const int n = std::min<int>(spec->n_slices, cap);
  for (int s = 0; s < n; ++s) {
    if (lower) lower[s] = spec->lower[s];
    if (thickness) thickness[s] = spec->thickness[s];
    if (atoms_per_slice) atoms_per_slice[s] = spec->counts[s];
  }
  return MSF_OK;
}

msf_status msf_specimen_transmission(const msf_specimen* spec, int32_t slice, double* out) {
  if (!spec || !out || slice < 0 || slice >= spec->n_slices) return MSF_ERR_ARG;
  const int64_t plane = (int64_t)spec->g.nx * spec->g.ny;
  msf_context* ctx = spec->ctx;
  cudaSetDevice(ctx->device);
  cudaError_t e;
  if (ctx->fp64) {
    e = cudaMemcpy(out, spec->t.as<double>() + 2 * plane * slice, 16 * plane,
                   cudaMemcpyDeviceToHost);
  } else {
    std::vector<float> tmp(2 * plane);
    e = cudaMemcpy(tmp.data(), spec->t.as<float>() + 2 * plane * slice, 8 * plane,
                   cudaMemcpyDeviceToHost);
    // FP32 contexts store tau = t - 1 (split-wave passes)
    for (int64_t k = 0; k < plane; ++k) {
      out[2 * k] = (double)tmp[2 * k] + 1.0;
      out[2 * k + 1] = tmp[2 * k + 1];
    }
  }
  if (e != cudaSuccess) {
    set_error(std::string("cudaMemcpy: ") + cudaGetErrorString(e));
    return MSF_ERR_CUDA;
  }
  return MSF_OK;
}

int64_t msf_specimen_device_bytes(const msf_specimen* spec) {
  return spec ? spec->device_bytes : 0;
}

int32_t msf_specimen_live_columns(const msf_specimen* spec) {
  return spec ? spec->n_live_columns : 0;
}

msf_status msf_run(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                   const msf_raster* raster, const msf_detect* detect, msf_results* results) {
  if (!ctx || !spec || spec->ctx != ctx) {
    set_error("specimen does not belong to this context");
    return MSF_ERR_ARG;
  }
  return run_raster(ctx, spec, optics, raster, detect, results);
}

msf_status msf_tune(msf_context* ctx, const msf_specimen* spec, msf_tuning* out) {
  if (!ctx || !spec || spec->ctx != ctx) {
    set_error("specimen does not belong to this context");
    return MSF_ERR_ARG;
  }
  return tune(ctx, spec, out);
}

msf_status msf_run_md(msf_context* ctx, int32_t n_snapshots,
                      const msf_specimen* const* snapshots, int32_t samples,
                      const msf_optics* optics, const msf_raster* raster,
                      const msf_detect* detect, msf_results* results) {
  if (!ctx) {
    set_error("null context");
    return MSF_ERR_ARG;
  }
  return run_md(ctx, n_snapshots, snapshots, samples, optics, raster, detect, results);
}

msf_status msf_run_plain(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                         const msf_raster* raster, const msf_detect* detect,
                         msf_results* results) {
  if (!ctx || !spec || spec->ctx != ctx) {
    set_error("specimen does not belong to this context");
    return MSF_ERR_ARG;
  }
  return run_raster_plain(ctx, spec, optics, raster, detect, results);
}

msf_status msf_context_keep_potentials(msf_context* ctx, int32_t on) {
  if (!ctx) return MSF_ERR_ARG;
  ctx->keep_potentials = on != 0;
  return MSF_OK;
}

msf_status msf_specimen_potential(const msf_specimen* spec, int32_t slice, double* out) {
  if (!spec || !out || slice < 0 || slice >= spec->n_slices) {
    set_error("msf_specimen_potential: no such slice");
    return MSF_ERR_ARG;
  }
  const size_t plane = (size_t)spec->g.nx * spec->g.ny;
  if (spec->h_potential.size() < 2 * plane * (size_t)(slice + 1)) {
    set_error("msf_specimen_potential: the specimen was built without "
              "msf_context_keep_potentials");
    return MSF_ERR_ARG;
  }
  std::memcpy(out, spec->h_potential.data() + 2 * plane * slice, 16 * plane);
  return MSF_OK;
}

int32_t msf_segment_count(const msf_grid* grid, const msf_detect* detect) {
  if (!grid || !detect) return -1;
  if (!(detect->outputs & MSF_OUT_FEM_MASK)) return 1;
  Grid g = grid_of(grid);
  const Rings r = make_rings(g, detect->dr);
  int32_t n = r.n_k + 1;
  if (detect->outputs & MSF_OUT_CORRELOGRAPH) n += r.n_k * make_cells(g, r).n_phi;
  return n;
}

msf_status msf_run_partial(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                           const msf_raster* raster, const msf_detect* detect, int64_t p_begin,
                           int64_t p_end, double* amp, double* inten, double* acc_a,
                           double* acc_i, msf_results* info) {
  if (!ctx || !spec || spec->ctx != ctx) {
    set_error("specimen does not belong to this context");
    return MSF_ERR_ARG;
  }
  return run_partial(ctx, spec, optics, raster, detect, p_begin, p_end, amp, inten, acc_a,
                     acc_i, info);
}

msf_status msf_finish(const msf_grid* grid, const msf_optics* optics, const msf_detect* detect,
                      int64_t n_probes, const double* amp, const double* inten,
                      const double* acc_a, const double* acc_i, msf_results* results) {
  if (!grid || !optics || !detect || !results || n_probes <= 0 || !inten ||
      ((detect->outputs & MSF_OUT_FEM_MASK) && !amp)) {
    set_error("msf_finish: null argument or empty raster");
    return MSF_ERR_ARG;
  }
  if (!supported_length(grid->nx) || !supported_length(grid->ny)) {
    set_error("unsupported grid");
    return MSF_ERR_UNSUPPORTED;
  }
  Grid g = grid_of(grid);
  Rings rings;
  if (detect->outputs & MSF_OUT_FEM_MASK) rings = make_rings(g, detect->dr);
  return finish_host(g, rings, *optics, *detect, n_probes, amp, inten, acc_a, acc_i, results);
}

msf_status msf_run_batch(msf_context* ctx, int32_t n, const msf_specimen* const* specs,
                         const msf_optics* optics, const msf_raster* rasters,
                         const msf_detect* detects, msf_results* results, int32_t slots) {
  if (!ctx) return MSF_ERR_ARG;
  return run_batch(ctx, n, specs, optics, rasters, detects, results, slots);
}

msf_status msf_probe(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                     double* out) {
  if (!ctx || !spec || !optics || !out) return MSF_ERR_ARG;
  cudaSetDevice(ctx->device);
  DevBuf p;
  msf_status st = build_probe(ctx, spec, optics, &p);
  if (st != MSF_OK) return st;
  const int64_t plane = (int64_t)spec->g.nx * spec->g.ny;
  cudaError_t e = cudaMemcpyAsync(out, p.p, 16 * plane, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMemcpy: ") + cudaGetErrorString(e));
    return MSF_ERR_CUDA;
  }
  return MSF_OK;
}

void msf_wavelength(double voltage, double* lambda, double* gamma) {
  double l = 0, g = 0;
  wavelength(voltage, &l, &g);
  if (lambda) *lambda = l;
  if (gamma) *gamma = g;
}

double msf_scherzer(int32_t which, double lambda, double aberration) {
  return scherzer(which, lambda, aberration);
}

int32_t msf_raster_points(double period, double origin, double spacing, double* out,
                          int32_t cap) {
  std::vector<double> p = raster_points(period, origin, spacing);
  for (int32_t k = 0; k < (int32_t)p.size() && k < cap; ++k) out[k] = p[k];
  return (int32_t)p.size();
}

msf_status msf_probe_shifts(const msf_grid* grid, const msf_raster* raster, int64_t* shifts) {
  if (!grid || !raster || !shifts) return MSF_ERR_ARG;
  Grid g = grid_of(grid);
  std::vector<double> xp(raster->x_p, raster->x_p + raster->n_x);
  std::vector<double> yp(raster->y_p, raster->y_p + raster->n_y);
  std::vector<int32_t> s;
  if (!probe_shifts(g, xp, yp, &s)) {
    set_error("a raster position lies half a pixel or more below the cell origin");
    return MSF_ERR_ARG;
  }
  for (size_t k = 0; k < s.size(); ++k) shifts[k] = s[k];
  return MSF_OK;
}

msf_status msf_slice_atoms(int64_t n_atoms, const double* q, double zmin, double zperiod,
                           double min_slice, int32_t* n_slices, double* lower,
                           double* thickness, int64_t* counts, int64_t* order, int32_t cap) {
  if (n_atoms < 0 || (n_atoms > 0 && !q)) return MSF_ERR_ARG;
  Slicing sl = slice_atoms(n_atoms, q, zmin, zperiod, min_slice);
  if (n_slices) *n_slices = (int32_t)sl.n();
  for (int64_t s = 0; s < sl.n() && s < cap; ++s) {
    if (lower) lower[s] = sl.lower[s];
    if (thickness) thickness[s] = sl.thickness[s];
    if (counts) counts[s] = sl.start[s + 1] - sl.start[s];
  }
  if (order)
    for (int64_t k = 0; k < (int64_t)sl.order.size(); ++k) order[k] = sl.order[k];
  return MSF_OK;
}

msf_status msf_time_passes(msf_context* ctx, const msf_specimen* spec, int32_t nb, int32_t reps,
                           double* ms_row, double* ms_col) {
  if (!ctx || !spec || nb <= 0 || reps <= 0) return MSF_ERR_ARG;
  return time_passes(ctx, spec, nb, reps, ms_row, ms_col);
}

msf_status msf_ring_bins(const msf_grid* grid, double dr, int32_t* bins, int32_t* n_k) {
  if (!grid) return MSF_ERR_ARG;
  Grid g = grid_of(grid);
  Rings r = make_rings(g, dr);
  if (bins) std::memcpy(bins, r.bin.data(), r.bin.size() * sizeof(int32_t));
  if (n_k) *n_k = r.n_k;
  return MSF_OK;
}

}  // extern "C"
