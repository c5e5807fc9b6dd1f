// Device engine: specimen build and the batched multislice raster.
//
// Set-up (FP64 on the device): per-species projected-potential LUT
// (scatterer_pap.hpp:45-230), per-slice transmission functions
// (slice.cpp:1451-1757) and the probe (adfstem.cpp:586-817).  Raster:
// probes in raster order are processed B at a time; each batch runs
// 2 x n_slices fused FFT passes (optionally replayed from a captured CUDA
// graph), then the detector / ring reductions.  Per-probe ring sums and ADF
// values stay on the device until the raster ends; the FEM statistics are
// then finished on the host in FP64 in the reference's order
// (adfstem.cpp:2489-3612).
#include "engine.hpp"
#include "trace.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "kernels.h"

namespace msf {

namespace {
thread_local std::string g_error;

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

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

template <typename T>
msf_status upload(msf_context* ctx, DevBuf* b, const std::vector<T>& h) {
  MSF_TRY(ctx->alloc(b, std::max<size_t>(1, h.size()) * sizeof(T)));
  if (!h.empty()) {
    MSF_CUDA(cudaMemcpyAsync(b->p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice,
                             ctx->stream));
    ctx->h2d_bytes += (int64_t)(h.size() * sizeof(T));
  }
  return MSF_OK;
}
}  // namespace

void set_error(const std::string& msg) { g_error = msg; }
const char* last_error() { return g_error.c_str(); }

void* Pool::take(size_t bytes, size_t* got) {
  std::lock_guard<std::mutex> lock(m);
  auto it = blocks.lower_bound(bytes);
  if (it == blocks.end() || it->first > 2 * bytes + (4u << 20)) return nullptr;
  void* p = it->second;
  *got = it->first;
  cached -= (int64_t)it->first;
  blocks.erase(it);
  return p;
}

std::recursive_mutex& capture_mutex() {
  static std::recursive_mutex m;
  return m;
}

void Pool::give(void* p, size_t bytes) {
  std::lock_guard<std::recursive_mutex> cap(capture_mutex());
  cudaDeviceSynchronize();
  std::lock_guard<std::mutex> lock(m);
  live -= (int64_t)bytes;
  if (closed) {
    cudaFree(p);
    return;
  }
  blocks.emplace(bytes, p);
  cached += (int64_t)bytes;
}

void Pool::trim() {
  std::lock_guard<std::recursive_mutex> cap(capture_mutex());
  std::lock_guard<std::mutex> lock(m);
  for (auto& kv : blocks) cudaFree(kv.second);
  blocks.clear();
  cached = 0;
}

void DevBuf::release() {
  if (p) {
    if (pool) {
      pool->give(p, bytes);
    } else {
      std::lock_guard<std::recursive_mutex> cap(capture_mutex());
      cudaFree(p);
    }
  }
  p = nullptr;
  bytes = 0;
  pool.reset();
}

}  // namespace msf

using namespace msf;

msf_status msf_context::alloc(DevBuf* b, size_t bytes) {
  b->release();
  if (budget > 0 && pool->live + (int64_t)bytes > budget) {
    set_error("device allocation of " + std::to_string(bytes) +
              " bytes exceeds the context's HBM budget");
    return MSF_ERR_NOMEM;
  }
  size_t got = 0;
  void* p = pool->take(bytes, &got);
  if (!p) {
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {  // hand the cached blocks back and try once more
      cudaGetLastError();
      pool->trim();
      e = cudaMalloc(&p, bytes);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
      return MSF_ERR_NOMEM;
    }
    got = bytes;
  }
  b->p = p;
  b->bytes = got;
  b->pool = pool;
  std::lock_guard<std::mutex> lock(pool->m);
  pool->live += (int64_t)got;
  return MSF_OK;
}

msf_status msf_context::twiddles(int n, bool want64, const void** out) {
  auto& m = want64 ? tw64 : tw32;
  auto it = m.find(n);
  if (it == m.end()) {
    std::vector<double> h(2 * (size_t)n);
    if (want64)
      fill_twiddles(n, h.data());
    else  // the FP32 passes also read each stage's factors as [r][k] copies
      fill_twiddles_f32_table(n, h);
    DevBuf b;
    if (want64) {
      MSF_TRY(upload(this, &b, h));
    } else {
      std::vector<float> f(h.begin(), h.end());
      MSF_TRY(upload(this, &b, f));
    }
    it = m.emplace(n, std::move(b)).first;
  }
  *out = it->second.p;
  return MSF_OK;
}

namespace msf {

namespace {

// Plain 2-D transforms of nb FP64 planes: forward (sign -1) or inverse with
// a scale, as row pass + column pass.
msf_status fft2d_f64(msf_context* ctx, const Grid& g, double* planes, int nb, bool inverse,
                     double scale) {
  PassArgs a;
  a.psi = planes;
  a.batch_stride = (int64_t)g.nx * g.ny;
  a.nb = nb;
  a.nx = g.nx;
  a.ny = g.ny;
  MSF_TRY(ctx->twiddles(g.ny, true, &a.tw));
  a.scale = 1.0;
  MSF_CUDA(launch_row(true, inverse ? ROW_INV : ROW_FWD, a, ctx->stream));
  MSF_TRY(ctx->twiddles(g.nx, true, &a.tw));
  a.scale = scale;
  if (inverse) {
    MSF_CUDA(launch_col(true, COL_INV, a, ctx->stream));
  } else {
    MSF_CUDA(launch_col(true, COL_FWD, a, ctx->stream));
    if (scale != 1.0)
      MSF_CUDA(launch_scale(planes, a.batch_stride * nb, scale, nullptr, ctx->stream));
  }
  return MSF_OK;
}

bool grid_ok(int n) { return supported_length(n); }

// slices with at least this many atoms take the FFT convolution for their
// potential (about the atom count at which it costs less than the direct sum)
constexpr int64_t kPotentialFftAtoms = 64;

}  // namespace

// Copies slice s's projected potential (before the exponential, as the
// reference's --paptif images show it, slice.cpp:1660-1690) to the
// specimen's host table.
msf_status keep_potential(msf_context* ctx, msf_specimen* spec, const double* t64, int64_t s) {
  const int64_t plane = (int64_t)spec->g.nx * spec->g.ny;
  if ((int64_t)spec->h_potential.size() < 2 * plane * (s + 1))
    spec->h_potential.resize((size_t)(2 * plane * (s + 1)));
  MSF_CUDA(cudaMemcpyAsync(spec->h_potential.data() + 2 * plane * s, t64, 16 * plane,
                           cudaMemcpyDeviceToHost, ctx->stream));
  MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MSF_OK;
}

msf_status build_specimen(msf_context* ctx, const msf_grid* gin, const msf_atoms* atoms,
                          msf_specimen* spec) {
  TraceScope trace_scope("specimen_build");
  const double t0 = now_s();
  if (!gin || !atoms) { set_error("null grid or atoms"); return MSF_ERR_ARG; }
  if (!grid_ok(gin->nx) || !grid_ok(gin->ny)) {
    set_error("grid " + std::to_string(gin->nx) + "x" + std::to_string(gin->ny) +
              " unsupported: each side must be a power of two in [64, 4096]");
    return MSF_ERR_UNSUPPORTED;
  }
  if (!(gin->xperiod > 0 && gin->yperiod > 0)) { set_error("periods must be positive"); return MSF_ERR_ARG; }
  const int dx = std::max(1, gin->dupe_x), dy = std::max(1, gin->dupe_y),
            dz = std::max(1, gin->dupe_z);
  // tem.cpp:1051-1143: replicate the cell when --dupe was given (FEM only;
  // the caller passes 1 1 1 otherwise).
  std::vector<double> q;
  std::vector<uint32_t> zz;
  const int64_t n0 = atoms->n_atoms;
  if (gin->replicate_atoms && dx * dy * dz > 1) {
    q.resize(3 * (size_t)n0 * dx * dy * dz);
    zz.resize((size_t)n0 * dx * dy * dz);
    for (int ii = 0; ii < dx; ++ii)
      for (int jj = 0; jj < dy; ++jj)
        for (int kk = 0; kk < dz; ++kk)
          for (int64_t i = 0; i < n0; ++i) {
            const size_t k = (size_t)(i + n0 * (kk + dz * (jj + dy * ii)));
            q[3 * k] = atoms->q[3 * i] + ii * gin->xperiod;
            q[3 * k + 1] = atoms->q[3 * i + 1] + jj * gin->yperiod;
            q[3 * k + 2] = atoms->q[3 * i + 2] + kk * gin->zperiod;
            zz[k] = atoms->z[i];
          }
  } else {
    q.assign(atoms->q, atoms->q + 3 * n0);
    zz.assign(atoms->z, atoms->z + n0);
  }
  const int64_t n = (int64_t)zz.size();
  spec->ctx = ctx;
  spec->g = make_grid(gin->nx, gin->ny, gin->voltage, gin->xperiod * dx, gin->yperiod * dy,
                      gin->zperiod * dz, gin->xmin, gin->ymin, gin->zmin, gin->xperiod,
                      gin->yperiod, gin->zperiod);
  const Grid& g = spec->g;
  const int64_t plane = (int64_t)g.nx * g.ny;

  // species in ascending Z (tem.cpp:944-972)
  std::vector<uint32_t> species(zz.begin(), zz.end());
  std::sort(species.begin(), species.end());
  species.erase(std::unique(species.begin(), species.end()), species.end());
  for (uint32_t z : species)
    if (!kirkland_params(z)) { set_error("atomic number out of range 1..103"); return MSF_ERR_ARG; }

  MSF_CUDA(cudaSetDevice(ctx->device));
  MSF_TRY(upload(ctx, &spec->kx, g.kx));
  MSF_TRY(upload(ctx, &spec->ky, g.ky));

  // per-species LUTs (scatterer_pap.hpp:109-190)
  DevBuf luts, luts_k, params;
  MSF_TRY(ctx->alloc(&luts, sizeof(double) * 2 * plane * std::max<size_t>(1, species.size())));
  std::vector<double> hp;
  for (uint32_t z : species) hp.insert(hp.end(), kirkland_params(z), kirkland_params(z) + 12);
  MSF_TRY(upload(ctx, &params, hp));
  const double ab_inv = 1 / (g.xpd * g.ypd);
  const double pref = g.lambda * g.gamma * ab_inv;
  for (size_t k = 0; k < species.size(); ++k) {
    MSF_CUDA(launch_lut_synth(luts.as<double>() + 2 * plane * k, spec->kx.as<double>(),
                              spec->ky.as<double>(), g.nx, g.ny, params.as<double>() + 12 * k,
                              pref, g.bw_pap * g.bw_pap, g.xmin, g.ymin, ctx->stream));
  }
  // slicing (slice.cpp:469-980) and per-atom pixel snaps (slice.cpp:1556-1572)
  auto host_prep = std::make_unique<TraceScope>("specimen_host_prep");
  Slicing sl = slice_atoms(n, q.data(), g.zmin, g.zpd, gin->min_slice);
  // which slices take the FFT convolution for their potential
  std::vector<uint8_t> by_fft(sl.n(), 0);
  for (int64_t s = 0; s < sl.n(); ++s) {
    const int64_t cnt = sl.start[s + 1] - sl.start[s];
    by_fft[s] = ctx->potential == 2 || (ctx->potential == 0 && cnt >= kPotentialFftAtoms);
  }
  const bool any_fft = std::find(by_fft.begin(), by_fft.end(), 1) != by_fft.end();
  if (any_fft && !species.empty()) {  // keep the k-space LUTs
    MSF_TRY(ctx->alloc(&luts_k, luts.bytes));
    MSF_CUDA(cudaMemcpyAsync(luts_k.p, luts.p, luts.bytes, cudaMemcpyDeviceToDevice,
                             ctx->stream));
  }
  if (!species.empty())
    MSF_TRY(fft2d_f64(ctx, g, luts.as<double>(), (int)species.size(), true,
                      1.0 / std::sqrt((double)(g.nx * (int64_t)g.ny))));
  spec->n_slices = (int)sl.n();
  spec->lower = sl.lower;
  spec->thickness = sl.thickness;
  spec->counts.resize(sl.n());
  for (int64_t s = 0; s < sl.n(); ++s) spec->counts[s] = sl.start[s + 1] - sl.start[s];
  std::vector<int32_t> asx(n), asy(n), asp(n);
  const double hx = 0.5 * (g.xx[1] - g.xx[0]), hy = 0.5 * (g.yy[1] - g.yy[0]);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t a = sl.order[k];
    const int64_t sx = snap(g.xx, q[3 * a], hx, 0), sy = snap(g.yy, q[3 * a + 1], hy, 0);
    if (sx < 0 || sy < 0) {
      set_error("atom " + std::to_string(a) + " lies half a pixel or more below the cell "
                "origin; the reference would index outside its arrays");
      return MSF_ERR_ARG;
    }
    asx[k] = (int32_t)sx;
    asy[k] = (int32_t)sy;
    asp[k] = (int32_t)(std::lower_bound(species.begin(), species.end(), zz[a]) - species.begin());
  }
  DevBuf dsx, dsy, dsp;
  MSF_TRY(upload(ctx, &dsx, asx));
  MSF_TRY(upload(ctx, &dsy, asy));
  MSF_TRY(upload(ctx, &dsp, asp));
  // pixel histograms of the FFT slices: (species, pixel, count) runs
  std::vector<int32_t> h_pix, h_sp;
  std::vector<double> h_cnt;
  std::vector<int64_t> h_start(sl.n() + 1, 0);
  for (int64_t s = 0; s < sl.n(); ++s) {
    if (by_fft[s]) {
      std::vector<int64_t> keys;
      for (int64_t k = sl.start[s]; k < sl.start[s + 1]; ++k)
        keys.push_back(((int64_t)asp[k] * g.nx + asx[k]) * g.ny + asy[k]);
      std::sort(keys.begin(), keys.end());
      for (size_t k = 0; k < keys.size();) {
        size_t e = k;
        while (e < keys.size() && keys[e] == keys[k]) ++e;
        h_sp.push_back((int32_t)(keys[k] / plane));
        h_pix.push_back((int32_t)(keys[k] % plane));
        h_cnt.push_back((double)(e - k));
        k = e;
      }
    }
    h_start[s + 1] = (int64_t)h_pix.size();
  }
  DevBuf d_hpix, d_hsp, d_hcnt, hist;
  if (any_fft) {
    MSF_TRY(upload(ctx, &d_hpix, h_pix));
    MSF_TRY(upload(ctx, &d_hsp, h_sp));
    MSF_TRY(upload(ctx, &d_hcnt, h_cnt));
    MSF_TRY(ctx->alloc(&hist, 16 * plane * std::max<size_t>(1, species.size())));
  }

  // band-limit mask (shared by the transmission build and the propagator)
  std::vector<int32_t> lo, hi;
  if (!bandlimit_mask(g, g.bw_t, &lo, &hi)) {
    set_error("band-limit mask is not an interval per column");
    return MSF_ERR_UNSUPPORTED;
  }
  MSF_TRY(upload(ctx, &spec->mask_lo, lo));
  MSF_TRY(upload(ctx, &spec->mask_hi, hi));
  {
    // a column keeps no kx at all when lo = 0 and hi = nx
    std::vector<uint8_t> dead(g.ny);
    for (int j = 0; j < g.ny; ++j) dead[j] = lo[j] == 0 && hi[j] == g.nx;
    spec->n_live_columns = (int)std::count(dead.begin(), dead.end(), 0);
    const bool fp = ctx->fp64;
    const int T = row_line_threads(g.ny, fp), cols = pipe_cols_for(g.nx, fp);
    if (T > 0 && g.ny / T <= 32 && cols > 0 && spec->n_live_columns < g.ny) {
      std::vector<uint32_t> bits(T, 0u);
      for (int t = 0; t < T; ++t)
        for (int m = 0; m < g.ny / T; ++m)
          if (dead[t + T * m]) bits[t] |= 1u << m;
      std::vector<int32_t> groups;
      for (int gi = 0; gi < g.ny / cols; ++gi) {
        bool live = false;
        for (int c = 0; c < cols; ++c) live = live || !dead[gi * cols + c];
        if (live) groups.push_back(gi);
      }
      MSF_TRY(upload(ctx, &spec->dead_bits, bits));
      MSF_TRY(upload(ctx, &spec->live_groups, groups));
      const int T1 = fp ? 0 : staged_row_threads(g.ny, 1);
      if (T1 > 0) {  // the same bits for the staged row pass's schedule 1
        std::vector<uint32_t> bits1(T1, 0u);
        for (int t = 0; t < T1; ++t)
          for (int m = 0; m < g.ny / T1; ++m)
            if (dead[t + T1 * m]) bits1[t] |= 1u << m;
        MSF_TRY(upload(ctx, &spec->dead_bits_alt, bits1));
      }
      spec->n_live_groups = (int)groups.size();
      spec->h_dead_bits = bits;
      spec->h_live_groups = groups;
    }
    // live element ranges of a row: [0, d0) and [d1, ny) around one run of
    // removed columns [d0, d1), widened to even bounds
    const int d0 = (int)(std::find(dead.begin(), dead.end(), 1) - dead.begin());
    int d1 = d0;
    while (d1 < g.ny && dead[d1]) ++d1;
    const bool one_run = d0 < g.ny && std::find(dead.begin() + d1, dead.end(), 1) == dead.end();
    const int a1 = one_run ? std::min(g.ny, (d0 + 1) & ~1) : g.ny;
    const int b0 = one_run ? (d1 & ~1) : g.ny;
    spec->row_live[0] = 0;
    spec->row_live[1] = a1;
    spec->row_live[2] = std::max(a1, b0);
    spec->row_live[3] = one_run ? g.ny : spec->row_live[2];
  }

  host_prep.reset();
  // transmission functions (slice.cpp:1544-1757)
  auto trans_scope = std::make_unique<TraceScope>("specimen_transmission");
  const size_t cbytes = ctx->fp64 ? 16 : 8;
  MSF_TRY(ctx->alloc(&spec->t, cbytes * plane * std::max<int64_t>(1, sl.n())));
  DevBuf scratch;
  if (!ctx->fp64) MSF_TRY(ctx->alloc(&scratch, 16 * plane));
  PassArgs a;
  a.batch_stride = plane;
  a.nb = 1;
  a.nx = g.nx;
  a.ny = g.ny;
  a.mask_lo = spec->mask_lo.as<int32_t>();
  a.mask_hi = spec->mask_hi.as<int32_t>();
  for (int64_t s = 0; s < sl.n(); ++s) {
    double* t64 = ctx->fp64 ? spec->t.as<double>() + 2 * plane * s : scratch.as<double>();
    const int64_t s0 = sl.start[s], cnt = sl.start[s + 1] - sl.start[s];
    if (by_fft[s] && !species.empty()) {
      // BACKWARD(lut_k * FORWARD(H)) / s, then the exponential
      MSF_CUDA(cudaMemsetAsync(hist.p, 0, hist.bytes, ctx->stream));
      MSF_CUDA(launch_histogram_scatter(hist.as<double>(), d_hpix.as<int32_t>() + h_start[s],
                                        d_hsp.as<int32_t>() + h_start[s],
                                        d_hcnt.as<double>() + h_start[s],
                                        (int)(h_start[s + 1] - h_start[s]), plane, ctx->stream));
      MSF_TRY(fft2d_f64(ctx, g, hist.as<double>(), (int)species.size(), false, 1.0));
      MSF_CUDA(launch_histogram_lut(t64, hist.as<double>(), luts_k.as<double>(),
                                    (int)species.size(), plane, ctx->stream));
      MSF_TRY(fft2d_f64(ctx, g, t64, 1, true, 1.0));
      const double sc = 1.0 / std::sqrt((double)(g.nx * (int64_t)g.ny));
      if (ctx->keep_potentials) {  // scale first, keep, exponentiate (same values)
        MSF_CUDA(launch_scale(t64, plane, sc, nullptr, ctx->stream));
        MSF_TRY(keep_potential(ctx, spec, t64, s));
        MSF_CUDA(launch_transmission_exp(t64, plane, 1.0, ctx->stream));
      } else {
        MSF_CUDA(launch_transmission_exp(t64, plane, sc, ctx->stream));
      }
    } else {
      MSF_CUDA(launch_potential(t64, luts.as<double>(), g.nx, g.ny, dsx.as<int32_t>() + s0,
                                dsy.as<int32_t>() + s0, dsp.as<int32_t>() + s0, (int)cnt,
                                ctx->stream, !ctx->keep_potentials));
      if (ctx->keep_potentials) {
        MSF_TRY(keep_potential(ctx, spec, t64, s));
        MSF_CUDA(launch_transmission_exp(t64, plane, 1.0, ctx->stream));
      }
    }
    a.psi = t64;
    MSF_TRY(ctx->twiddles(g.ny, true, &a.tw));
    MSF_CUDA(launch_row(true, ROW_FWD, a, ctx->stream));
    MSF_TRY(ctx->twiddles(g.nx, true, &a.tw));
    MSF_CUDA(launch_col(true, COL_FWD_MASK_INV, a, ctx->stream));
    MSF_TRY(ctx->twiddles(g.ny, true, &a.tw));
    a.scale = 1.0 / g.nxny;
    MSF_CUDA(launch_row(true, ROW_INV, a, ctx->stream));
    a.scale = 1.0;
    if (!ctx->fp64)
      MSF_CUDA(launch_to_f32_minus_one(t64, spec->t.as<float>() + 2 * plane * s, plane,
                                       ctx->stream));
  }

  if (trace_enabled()) MSF_CUDA(cudaStreamSynchronize(ctx->stream));  // device time in the record
  trans_scope.reset();
  // propagators (slice.cpp:1293-1363)
  spec->hprop.clear();
  for (int64_t s = 0; s < sl.n(); ++s) {
    std::vector<double> px, py;
    propagator(g, sl.thickness[s], &px, &py);
    spec->hprop.insert(spec->hprop.end(), px.begin(), px.end());
    spec->hprop.insert(spec->hprop.end(), py.begin(), py.end());
  }
  if (ctx->fp64) {
    MSF_TRY(upload(ctx, &spec->prop, spec->hprop));
  } else {
    std::vector<float> f(spec->hprop.begin(), spec->hprop.end());
    MSF_TRY(upload(ctx, &spec->prop, f));
  }
  MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  spec->device_bytes = (int64_t)(spec->t.bytes + spec->prop.bytes + spec->mask_lo.bytes +
                                 spec->mask_hi.bytes + spec->kx.bytes + spec->ky.bytes);
  spec->seconds_setup = now_s() - t0;
  return MSF_OK;
}

msf_status build_probe(msf_context* ctx, const msf_specimen* spec, const msf_optics* o,
                       DevBuf* probe64) {
  TraceScope trace_scope("probe_build");
  const Grid& g = spec->g;
  const int64_t plane = (int64_t)g.nx * g.ny;
  MSF_TRY(ctx->alloc(probe64, 16 * plane));
  const double lsq = g.lambda * g.lambda;
  const double amax_sq = o->alpha_max * o->alpha_max;
  // probe evaluated at (xx[0], yy[0]) (adfstem.cpp:586-645)
  MSF_CUDA(launch_probe_synth(probe64->as<double>(), spec->kx.as<double>(),
                              spec->ky.as<double>(), g.nx, g.ny, o->corrected, o->cs3, o->cs5,
                              o->defocus, g.lambda, lsq, amax_sq, g.xx[0], g.yy[0],
                              ctx->stream));
  // BACKWARD transform, / sqrtNxNy (adfstem.cpp:686-732)
  MSF_TRY(fft2d_f64(ctx, g, probe64->as<double>(), 1, true, 1.0 / g.s));
  // Ap = 1/sqrt(sum |psi|^2) (probe_wavefunction.cpp:287-315)
  DevBuf d_sum;
  MSF_TRY(ctx->alloc(&d_sum, sizeof(double)));
  MSF_CUDA(launch_norm2(probe64->as<double>(), plane, d_sum.as<double>(), ctx->stream));
  double sum = 0;
  MSF_CUDA(cudaMemcpyAsync(&sum, d_sum.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  const double ap = 1.0 / std::sqrt(sum);
  MSF_CUDA(launch_scale(probe64->as<double>(), plane, ap, nullptr, ctx->stream));
  return MSF_OK;
}

// The plain FP32 split-wave row pass's L2 prefetch ahead (MSF_ROW_L2AHEAD):
// the distance in CTAs and, when the removed columns are not stored, only
// the live element ranges of each row.
void set_row_ahead(const msf_context* ctx, const msf_specimen* spec, PassArgs* row) {
  const int resident = row_split_resident_ctas(spec->g.ny);
  row->l2_ahead = (int)((int64_t)resident * ctx->row_ahead_pct / 100);
  const int ny = spec->g.ny;
  const int whole[4] = {0, ny, ny, ny};
  const int* r = row->row_dead_bits ? spec->row_live : whole;
  for (int k = 0; k < 4; ++k) row->ahead_range[k] = r[k];
}

msf_status time_passes(msf_context* ctx, const msf_specimen* spec, int nb, int reps,
                       double* ms_row, double* ms_col) {
  TraceScope trace_scope("time_passes");
  const Grid& g = spec->g;
  const int64_t plane = (int64_t)g.nx * g.ny;
  const bool fp64 = ctx->fp64;
  const size_t cbytes = fp64 ? 16 : 8;
  MSF_CUDA(cudaSetDevice(ctx->device));
  DevBuf psi;
  MSF_TRY(ctx->alloc(&psi, cbytes * plane * nb));
  MSF_CUDA(cudaMemsetAsync(psi.p, 0, psi.bytes, ctx->stream));
  DevBuf psi0, zshift;
  if (!fp64) {  // split-wave row pass reads one vacuum plane and the shifts
    MSF_TRY(ctx->alloc(&psi0, 8 * plane));
    MSF_TRY(ctx->alloc(&zshift, sizeof(int32_t) * 2 * nb));
    MSF_CUDA(cudaMemsetAsync(psi0.p, 0, psi0.bytes, ctx->stream));
    MSF_CUDA(cudaMemsetAsync(zshift.p, 0, zshift.bytes, ctx->stream));
  }
  const RowOp rop = fp64 ? ROW_SLICE : ROW_SPLIT;
  PassArgs row, col;
  row.psi = col.psi = psi.p;
  row.batch_stride = col.batch_stride = plane;
  row.nb = col.nb = nb;
  row.nx = col.nx = g.nx;
  row.ny = col.ny = g.ny;
  MSF_TRY(ctx->twiddles(g.ny, fp64, &row.tw));
  MSF_TRY(ctx->twiddles(g.nx, fp64, &col.tw));
  row.inv_s = col.inv_s = 1.0 / g.s;
  row.trans = spec->t.p;
  row.psi0 = psi0.p;
  row.shifts = zshift.as<int32_t>();
  col.mask_lo = spec->mask_lo.as<int32_t>();
  col.mask_hi = spec->mask_hi.as<int32_t>();
  col.px = spec->prop.p;
  col.py = static_cast<const char*>(spec->prop.p) + cbytes * g.nx;
  // the same kernels run_raster launches for slices after the first
  const int pipe = ctx->pipe_for(g.nx, g.ny);
  const bool staged_row = !fp64 && staged_row_supported(g.nx, g.ny) && (pipe & MSF_ROW_STAGED);
  const int row_sched = !fp64 && staged_row_supported(g.nx, g.ny) && (pipe & MSF_ROW_ALT) ? 1 : 0;
  const bool pipe_row = !fp64 && !staged_row && !row_sched && pipe_supported(g.nx, g.ny) &&
                        (pipe & MSF_PIPE_ROW);
  const bool pipe_col = pipe_supported(g.nx, g.ny, fp64) && (pipe & MSF_PIPE_COL);
  alignas(64) unsigned char col_map[128];
  DevBuf d_err;
  MSF_TRY(ctx->alloc(&d_err, sizeof(int)));
  MSF_CUDA(cudaMemsetAsync(d_err.p, 0, sizeof(int), ctx->stream));
  if (pipe_col) MSF_CUDA(encode_column_map(psi.p, nb, g.nx, g.ny, col_map, fp64));
  if (pipe_col && !pipe_row && spec->n_live_groups > 0) {  // skip removed columns
    row.row_dead_bits = spec->dead_bits.as<uint32_t>();
    row.row_dead_io = 3;  // a slice between the first and the last
    col.live_groups = spec->live_groups.as<int32_t>();
    col.n_live_groups = spec->n_live_groups;
  }
  row.prefetch_tables = (pipe & MSF_ROW_PREFETCH) ? 1 : 0;
  if (!fp64 && !staged_row && row_sched == 0 && !pipe_row && (pipe & MSF_ROW_L2AHEAD))
    set_row_ahead(ctx, spec, &row);
  row.lines_by_probe = (!fp64 && !staged_row && row_sched == 0 && !pipe_row &&
                        (pipe & MSF_ROW_BYPROBE)) ? 1 : 0;
  PassArgs row_staged = row;  // schedule 1 reads the zero bits in its own layout
  if (row_sched == 1 && row.row_dead_bits) row_staged.row_dead_bits = spec->dead_bits_alt.as<uint32_t>();
  auto row_pass = [&]() {
    return staged_row       ? launch_row_split_staged(row_staged, d_err.as<int>(), ctx->stream,
                                                      row_sched)
           : row_sched == 1 ? launch_row_split_alt(row_staged, ctx->stream)
           : pipe_row       ? launch_row_split_pipe(row, d_err.as<int>(), ctx->stream)
                            : launch_row(fp64, rop, row, ctx->stream);
  };
  auto col_pass = [&]() {
    return pipe_col ? launch_col_slice_pipe(col, false, col_map, d_err.as<int>(), ctx->stream, fp64)
                    : launch_col(fp64, COL_SLICE, col, ctx->stream);
  };
  std::vector<cudaEvent_t> ev(2 * reps + 2);
  for (auto& e : ev) MSF_CUDA(cudaEventCreate(&e));
  // warm-up
  MSF_CUDA(row_pass());
  MSF_CUDA(col_pass());
  double tr = 0, tc = 0;
  for (int r = 0; r < reps; ++r) {
    MSF_CUDA(cudaEventRecord(ev[2 * r], ctx->stream));
    MSF_CUDA(row_pass());
    MSF_CUDA(cudaEventRecord(ev[2 * r + 1], ctx->stream));
    MSF_CUDA(col_pass());
    MSF_CUDA(cudaEventRecord(ev[2 * r + 2], ctx->stream));
  }
  MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  int err_flag = 0;
  MSF_CUDA(cudaMemcpy(&err_flag, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err_flag) {
    set_error("a pipelined slice pass gave up waiting for a tile copy (bounded wait)");
    return MSF_ERR_TIMEOUT;
  }
  for (int r = 0; r < reps; ++r) {
    float a = 0, b = 0;
    MSF_CUDA(cudaEventElapsedTime(&a, ev[2 * r], ev[2 * r + 1]));
    MSF_CUDA(cudaEventElapsedTime(&b, ev[2 * r + 1], ev[2 * r + 2]));
    tr += a;
    tc += b;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (ms_row) *ms_row = tr / reps;
  if (ms_col) *ms_col = tc / reps;
  return MSF_OK;
}

int64_t raster_plan_bytes(const msf_specimen* spec, bool fp64, int64_t n_probes,
                          bool pix_modes) {
  const int64_t plane = (int64_t)spec->g.nx * spec->g.ny;
  int64_t b = 16 * plane;                                    // probe
  if (!fp64) b += 8 * plane * spec->n_slices + 16 * plane;   // vacuum tables
  b += 8 * n_probes + 3 * 4 * plane;                         // shifts, segments
  b += 2 * 8 * n_probes * (int64_t)(spec->g.nx + 1);         // sums (n_seg <= nx + 1)
  if (pix_modes) b += 2 * 8 * plane;
  return b;
}

std::shared_ptr<const Rings> rings_for(msf_context* ctx, const Grid& g, double dr) {
  const msf_context::RingKey key{g.nx, g.ny, g.xpd, g.ypd, g.bw_t, dr};
  std::lock_guard<std::mutex> lock(ctx->ring_mu);
  auto it = ctx->ring_cache.find(key);
  if (it != ctx->ring_cache.end()) return it->second;
  auto r = std::make_shared<const Rings>(make_rings(g, dr));
  if (ctx->ring_cache.size() >= 16) ctx->ring_cache.clear();  // bound the host memory
  ctx->ring_cache.emplace(key, r);
  return r;
}

msf_status plan_raster(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                       const msf_raster* raster, const msf_detect* det, RasterPlan* P,
                       int64_t p_begin, int64_t p_end) {
  TraceScope trace_scope("raster_plan");
  if (!spec || !optics || !raster || !det || !P) { set_error("null argument"); return MSF_ERR_ARG; }
  const Grid& g = spec->g;
  const int64_t plane = (int64_t)g.nx * g.ny;
  const bool fp64 = ctx->fp64;
  const int S = spec->n_slices;
  if (S <= 0) { set_error("specimen has no slices"); return MSF_ERR_ARG; }
  std::vector<double> x_p(raster->x_p, raster->x_p + std::max(0, raster->n_x));
  std::vector<double> y_p(raster->y_p, raster->y_p + std::max(0, raster->n_y));
  const int64_t n_all = (int64_t)x_p.size() * (int64_t)y_p.size();
  if (n_all <= 0) { set_error("empty raster"); return MSF_ERR_ARG; }
  if (p_end < 0) p_end = n_all;
  if (p_begin < 0 || p_begin >= p_end || p_end > n_all) {
    set_error("probe range [" + std::to_string(p_begin) + ", " + std::to_string(p_end) +
              ") outside the raster's " + std::to_string(n_all) + " probes");
    return MSF_ERR_ARG;
  }
  const int64_t n_probes = p_end - p_begin;
  P->spec = spec;
  P->p_begin = p_begin;
  P->n_raster = n_all;
  P->optics = *optics;
  P->det = *det;
  P->n_probes = n_probes;
  P->S = S;
  P->plane = plane;
  P->want_adf = det->outputs & MSF_OUT_ADF_IMAGE;
  P->fem = det->outputs & MSF_OUT_FEM_MASK;
  P->pix_modes = det->outputs & (MSF_OUT_V_RE | MSF_OUT_OMEGA_VIMAGE | MSF_OUT_V_GT17 |
                                 MSF_OUT_V_RBAR);
  MSF_CUDA(cudaSetDevice(ctx->device));

  // probe
  MSF_TRY(build_probe(ctx, spec, optics, &P->probe64));
  P->setup_launches = 5;

  // FP32 runs carry only the scattered part of each wave; the vacuum part
  // psi0 (the probe propagated with t = 1) is the same for every probe up to
  // its integer shift, so it is built once here in FP64: psi0_tab[s] is the
  // real-space vacuum wave entering slice s (in the scale of the inverse-
  // transformed buffer) and psi0k the vacuum exit wave in k-space.
  if (!fp64) {
    DevBuf prop64;
    MSF_TRY(ctx->alloc(&P->psi0_tab, 8 * plane * (size_t)S));
    MSF_TRY(ctx->alloc(&P->psi0k, 16 * plane));
    MSF_TRY(upload(ctx, &prop64, spec->hprop));
    MSF_CUDA(cudaMemcpyAsync(P->psi0k.p, P->probe64.p, 16 * plane, cudaMemcpyDeviceToDevice,
                             ctx->stream));
    MSF_CUDA(launch_scale(P->psi0k.as<double>(), plane, g.nxny / g.s, nullptr, ctx->stream));
    PassArgs v;
    v.psi = P->psi0k.p;
    v.batch_stride = plane;
    v.nb = 1;
    v.nx = g.nx;
    v.ny = g.ny;
    v.mask_lo = spec->mask_lo.as<int32_t>();
    v.mask_hi = spec->mask_hi.as<int32_t>();
    v.inv_s = 1.0 / (g.s * g.s);  // Q(1, psi) = psi/s, then FFT2 and /s
    const void *tw_y = nullptr, *tw_x = nullptr;
    MSF_TRY(ctx->twiddles(g.ny, true, &tw_y));
    MSF_TRY(ctx->twiddles(g.nx, true, &tw_x));
    P->setup_launches += 1;
    for (int s = 0; s < S; ++s) {
      MSF_CUDA(launch_to_f32(P->psi0k.as<double>(), P->psi0_tab.as<float>() + 2 * plane * s,
                             2 * plane, ctx->stream));
      v.tw = tw_y;
      MSF_CUDA(launch_row(true, ROW_FWD, v, ctx->stream));
      v.tw = tw_x;
      v.px = prop64.as<double>() + 2 * (size_t)(g.nx + g.ny) * s;
      v.py = prop64.as<double>() + 2 * (size_t)(g.nx + g.ny) * s + 2 * g.nx;
      MSF_CUDA(launch_col(true, s + 1 == S ? COL_SLICE_LAST : COL_SLICE, v, ctx->stream));
      P->setup_launches += 3;
      if (s + 1 < S) {
        v.tw = tw_y;
        v.scale = 1.0;
        MSF_CUDA(launch_row(true, ROW_INV, v, ctx->stream));
        P->setup_launches += 1;
      }
    }
    // prop64 is released at the end of this scope: finish its readers first
    MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  }

  // per-probe pixel shifts: the reference's search carries its position
  // over from probe to probe, so they are found over the whole raster and
  // the range's slice is kept
  if (!probe_shifts(g, x_p, y_p, &P->shifts)) {
    set_error("a raster position lies half a pixel or more below the cell origin");
    return MSF_ERR_ARG;
  }
  P->shifts = std::vector<int32_t>(P->shifts.begin() + 2 * p_begin,
                                   P->shifts.begin() + 2 * p_end);
  MSF_TRY(upload(ctx, &P->d_shifts, P->shifts));

  // segments: ring bins (FEM) then the ADF detector annulus
  if (P->fem) P->rings = rings_for(ctx, g, det->dr);
  P->n_k = P->fem ? P->rings->n_k : 0;
  std::vector<int32_t> seg_idx, seg_start{0};
  if (P->fem) {
    seg_idx = P->rings->pix;
    for (int k = 0; k < P->n_k; ++k) seg_start.push_back(P->rings->start[k + 1]);
  }
  const std::vector<int32_t> adf_pix =
      detector_pixels(g, det->det_inner / g.lambda, det->det_outer / g.lambda);
  seg_idx.insert(seg_idx.end(), adf_pix.begin(), adf_pix.end());
  seg_start.push_back((int32_t)seg_idx.size());
  P->n_seg = P->n_k + 1;
  if (P->fem && (det->outputs & MSF_OUT_CORRELOGRAPH)) {
    // correlograph cells (k bin, phi bin) after the ADF annulus
    const Cells cells = make_cells(g, *P->rings);
    const size_t n_cells = (size_t)P->n_k * cells.n_phi;
    const int32_t base = (int32_t)seg_idx.size();
    seg_idx.insert(seg_idx.end(), cells.pix.begin(), cells.pix.end());
    for (size_t c = 0; c < n_cells; ++c) seg_start.push_back(base + cells.start[c + 1]);
    P->n_seg += (int)n_cells;
  }
  // chunks of at most kSegmentChunk pixels, never straddling two segments
  std::vector<int32_t> chunk_begin, seg_chunk;
  for (int gi = 0; gi < P->n_seg; ++gi) {
    seg_chunk.push_back((int32_t)chunk_begin.size());
    for (int32_t k = seg_start[gi]; k < seg_start[gi + 1]; k += kSegmentChunk)
      chunk_begin.push_back(k);
  }
  seg_chunk.push_back((int32_t)chunk_begin.size());
  P->n_chunks = (int)chunk_begin.size();
  chunk_begin.push_back(seg_start[P->n_seg]);
  MSF_TRY(upload(ctx, &P->seg_idx, seg_idx));
  MSF_TRY(upload(ctx, &P->chunk_begin, chunk_begin));
  MSF_TRY(upload(ctx, &P->seg_chunk, seg_chunk));
  MSF_TRY(ctx->alloc(&P->amp, sizeof(double) * n_probes * P->n_seg));
  MSF_TRY(ctx->alloc(&P->inten, sizeof(double) * n_probes * P->n_seg));
  if (P->pix_modes) {
    MSF_TRY(ctx->alloc(&P->acc_a, sizeof(double) * plane));
    MSF_TRY(ctx->alloc(&P->acc_i, sizeof(double) * plane));
    MSF_CUDA(cudaMemsetAsync(P->acc_a.p, 0, P->acc_a.bytes, ctx->stream));
    MSF_CUDA(cudaMemsetAsync(P->acc_i.p, 0, P->acc_i.bytes, ctx->stream));
  }
  // detector MTF (adfstem.cpp:298-414): table -> 2-D, BACKWARD transform,
  // band limit applied to that real-space array (kept as the reference does
  // it), FORWARD transform, / NxNy
  if (det->n_mtf > 0 && det->mtf_resolution != 0 && det->mtf && det->mtf_domain_sqr) {
    P->mtf = true;
    const std::vector<double> h =
        mtf_2d(g, det->mtf, det->mtf_domain_sqr, det->n_mtf, det->mtf_resolution);
    MSF_TRY(upload(ctx, &P->mtf2d, h));
    PassArgs a;
    a.psi = P->mtf2d.p;
    a.batch_stride = plane;
    a.nb = 1;
    a.nx = g.nx;
    a.ny = g.ny;
    a.scale = 1.0;
    MSF_TRY(ctx->twiddles(g.ny, true, &a.tw));
    MSF_CUDA(launch_row(true, ROW_INV, a, ctx->stream));
    MSF_TRY(ctx->twiddles(g.nx, true, &a.tw));
    MSF_CUDA(launch_col(true, COL_INV, a, ctx->stream));
    MSF_CUDA(launch_bw_limit(P->mtf2d.as<double>(), spec->mask_lo.as<int32_t>(),
                             spec->mask_hi.as<int32_t>(), g.nx, g.ny, ctx->stream));
    MSF_TRY(ctx->twiddles(g.ny, true, &a.tw));
    MSF_CUDA(launch_row(true, ROW_FWD, a, ctx->stream));
    MSF_TRY(ctx->twiddles(g.nx, true, &a.tw));
    MSF_CUDA(launch_col(true, COL_FWD, a, ctx->stream));
    MSF_CUDA(launch_scale(P->mtf2d.as<double>(), plane, 1.0 / g.nxny, nullptr, ctx->stream));
    P->setup_launches += 6;
  }
  // the host vectors above are staged by pageable copies: complete them
  MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MSF_OK;
}

// The detector MTF of nb exit waves (adfstem.cpp:2272-2385) into FP64 planes
// `out`: |psi(k)| with the direct beam blocked, BACKWARD transform, times the
// MTF / s (reference update order), FORWARD transform, / s, band limit.
msf_status mtf_stage(msf_context* ctx, const RasterPlan& P, bool fp64, const void* psi, int nb,
                     const SplitK& sk, double* out, cudaStream_t st) {
  const msf_specimen* spec = P.spec;
  const Grid& g = spec->g;
  const int64_t plane = P.plane;
  SplitK k = sk;
  k.nx = g.nx;
  k.ny = g.ny;
  MSF_CUDA(launch_mtf_magnitude(fp64, psi, plane, nb, spec->kx.as<double>(), spec->ky.as<double>(),
                                g.lambda * g.lambda, P.optics.alpha_max * P.optics.alpha_max, k,
                                out, st));
  PassArgs a;
  a.psi = out;
  a.batch_stride = plane;
  a.nb = nb;
  a.nx = g.nx;
  a.ny = g.ny;
  a.scale = 1.0;
  const void *tw_y = nullptr, *tw_x = nullptr;
  MSF_TRY(ctx->twiddles(g.ny, true, &tw_y));
  MSF_TRY(ctx->twiddles(g.nx, true, &tw_x));
  a.tw = tw_y;
  MSF_CUDA(launch_row(true, ROW_INV, a, st));
  a.tw = tw_x;
  MSF_CUDA(launch_col(true, COL_INV, a, st));
  MSF_CUDA(launch_mtf_multiply(out, P.mtf2d.as<double>(), plane, nb, 1.0 / g.s, st));
  a.tw = tw_y;
  MSF_CUDA(launch_row(true, ROW_FWD, a, st));
  a.tw = tw_x;
  MSF_CUDA(launch_col(true, COL_FWD, a, st));
  MSF_CUDA(launch_scale(out, plane * nb, 1.0 / g.s, nullptr, st));
  MSF_CUDA(launch_bw_limit(out, spec->mask_lo.as<int32_t>(), spec->mask_hi.as<int32_t>(), g.nx,
                           g.ny, st, nb));
  return MSF_OK;
}

// Ring (and correlograph cell) sums of the MTF-filtered waves replace those
// columns of the batch's rows; the ADF column (index n_k) keeps the
// unfiltered sums (adfstem.cpp:2245).
msf_status mtf_ring_sums(const RasterPlan& P, const SegmentPlan& seg, const double* mtf_psi,
                         int nb, double* scratch_amp, double* scratch_int, double* amp_out,
                         double* int_out, cudaStream_t st) {
  if (P.n_k <= 0) return MSF_OK;
  SplitK none;
  MSF_CUDA(launch_segment_sums(true, mtf_psi, P.plane, nb, seg, scratch_amp, scratch_int, none,
                               st));
  const size_t pitch = sizeof(double) * P.n_seg;
  const size_t spans[2][2] = {{0, (size_t)P.n_k}, {(size_t)P.n_k + 1, (size_t)P.n_seg}};
  for (const auto& sp : spans) {
    if (sp[1] <= sp[0]) continue;
    const size_t off = sp[0], width = sizeof(double) * (sp[1] - sp[0]);
    MSF_CUDA(cudaMemcpy2DAsync(amp_out + off, pitch, scratch_amp + off, pitch, width, nb,
                               cudaMemcpyDeviceToDevice, st));
    MSF_CUDA(cudaMemcpy2DAsync(int_out + off, pitch, scratch_int + off, pitch, width, nb,
                               cudaMemcpyDeviceToDevice, st));
  }
  return MSF_OK;
}

msf_status download_sums(msf_context* ctx, const RasterPlan& P, cudaStream_t stream,
                         double* amp, double* inten, double* acc_a, double* acc_i) {
  const size_t rows = (size_t)P.n_probes * P.n_seg;
  if (amp)
    MSF_CUDA(cudaMemcpyAsync(amp, P.amp.p, rows * sizeof(double), cudaMemcpyDeviceToHost,
                             stream));
  if (inten)
    MSF_CUDA(cudaMemcpyAsync(inten, P.inten.p, rows * sizeof(double), cudaMemcpyDeviceToHost,
                             stream));
  if (P.pix_modes && acc_a)
    MSF_CUDA(cudaMemcpyAsync(acc_a, P.acc_a.p, P.plane * sizeof(double),
                             cudaMemcpyDeviceToHost, stream));
  if (P.pix_modes && acc_i)
    MSF_CUDA(cudaMemcpyAsync(acc_i, P.acc_i.p, P.plane * sizeof(double),
                             cudaMemcpyDeviceToHost, stream));
  MSF_CUDA(cudaStreamSynchronize(stream));
  ctx->d2h_bytes += (int64_t)(((amp ? 1 : 0) + (inten ? 1 : 0)) * rows * sizeof(double)) +
                    (P.pix_modes ? ((acc_a ? 8 : 0) + (acc_i ? 8 : 0)) * P.plane : 0);
  return MSF_OK;
}

msf_status finish_raster(msf_context* ctx, const RasterPlan& P, cudaStream_t stream,
                         msf_results* res) {
  TraceScope trace_scope("raster_finish");
  // the sums land in the context's pinned staging buffer (no page faults on
  // fresh host memory, copies at the pinned rate)
  const size_t rows = (size_t)P.n_probes * P.n_seg;
  const size_t pix = P.pix_modes ? (size_t)P.plane : 0;
  const size_t need = sizeof(double) * (2 * rows + 2 * pix);
  std::lock_guard<std::mutex> lock(ctx->stage_mu);
  if (ctx->host_stage_bytes < need) {
    // freeing pinned memory can wait on the device: not during a capture
    // on another thread
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    if (ctx->host_stage) cudaFreeHost(ctx->host_stage);
    ctx->host_stage = nullptr;
    ctx->host_stage_bytes = 0;
    MSF_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ctx->host_stage), need,
                           cudaHostAllocDefault));
    ctx->host_stage_bytes = need;
  }
  double* amp = ctx->host_stage;
  double* inten = amp + rows;
  double* acc_a = P.pix_modes ? inten + rows : nullptr;
  double* acc_i = P.pix_modes ? acc_a + pix : nullptr;
  MSF_TRY(download_sums(ctx, P, stream, amp, inten, acc_a, acc_i));
  static const Rings no_rings;
  return finish_host(P.spec->g, P.rings ? *P.rings : no_rings, P.optics, P.det, P.n_probes,
                     amp, inten, acc_a, acc_i, res);
}

msf_status finish_host(const Grid& g, const Rings& rings, const msf_optics& optics,
                       const msf_detect& detect, int64_t n_probes, const double* amp,
                       const double* inten, const double* acc_a, const double* acc_i,
                       msf_results* res) {
  const int64_t plane = (int64_t)g.nx * g.ny;
  const uint32_t fem = detect.outputs & MSF_OUT_FEM_MASK;
  const bool pix_modes = detect.outputs & (MSF_OUT_V_RE | MSF_OUT_OMEGA_VIMAGE |
                                           MSF_OUT_V_GT17 | MSF_OUT_V_RBAR);
  const bool corr = fem && (detect.outputs & MSF_OUT_CORRELOGRAPH);
  const int n_k = fem ? rings.n_k : 0;
  Cells cells;
  if (corr) cells = make_cells(g, rings);
  const int n_phi = corr ? cells.n_phi : 0;
  const int n_seg = n_k + 1 + n_k * n_phi;
  if (pix_modes && fem && (!acc_a || !acc_i)) {
    set_error("pixel FEM modes need the per-pixel sums");
    return MSF_ERR_ARG;
  }
  if ((detect.outputs & MSF_OUT_ADF_IMAGE) && res->adf_image)
    for (int64_t p = 0; p < n_probes; ++p) res->adf_image[p] = inten[p * n_seg + n_k];

  // ---- FEM statistics on the host, in the reference's order -----------
  res->n_k = n_k;
  if (!fem) return MSF_OK;
  if (n_k > res->cap_k) {
    set_error("results.cap_k is smaller than the number of k bins (" + std::to_string(n_k) + ")");
    return MSF_ERR_ARG;
  }
  const msf_detect* det = &detect;
  std::vector<uint8_t> inside(n_k);
  for (int k = 0; k < n_k; ++k)
    inside[k] = (g.lambda * rings.bounds[k + 1] <= optics.alpha_max);  // adfstem.cpp:2518
  const std::vector<int32_t>& cnt = rings.counts;
  for (int k = 0; k < n_k; ++k) {
    if (res->k_lower) res->k_lower[k] = rings.bounds[k];
    if (res->bin_counts) res->bin_counts[k] = cnt[k];
  }
  for (int64_t p = 0; p < n_probes; ++p)
    for (int k = 0; k < n_k; ++k) {
      if (res->ring_amplitude) res->ring_amplitude[p * res->cap_k + k] = amp[p * n_seg + k];
      if (res->ring_intensity) res->ring_intensity[p * res->cap_k + k] = inten[p * n_seg + k];
    }
  const double n_r = (double)(size_t)n_probes;
  if (corr) {  // adfstem.cpp:2603-2652, 3617-3633
    if (n_phi > res->cap_phi) {
      set_error("results.cap_phi is smaller than the number of azimuthal bins (" +
                std::to_string(n_phi) + ")");
      return MSF_ERR_ARG;
    }
    res->n_phi = n_phi;
    if (res->phi_lower)
      for (int jj = 0; jj <= n_phi && jj < (int)cells.phi_bounds.size(); ++jj)
        res->phi_lower[jj] = cells.phi_bounds[jj];
    const size_t nc = (size_t)n_k * n_phi;
    std::vector<double> sum(nc, 0.0), sqr(nc, 0.0), one(nc);
    for (int64_t p = 0; p < n_probes; ++p) {
      const double* row = &amp[p * n_seg];
      for (int ii = 0; ii < n_k; ++ii) {
        const double S = inside[ii] ? 0.0 : row[ii];  // direct beam zeroed
        for (int jj = 0; jj < n_phi; ++jj) {
          const double Cv = inside[ii] ? 0.0 : row[n_k + 1 + (size_t)ii * n_phi + jj];
          const size_t c = ii + (size_t)jj * n_k;
          const double t = (cnt[ii] * Cv / S);
          one[c] = (t >= 1 && cnt[ii] != 0 && Cv != 0 && S != 0) ? (cnt[ii] * Cv / S) - 1 : 0.0;
          sum[c] += one[c];
          sqr[c] += one[c] * one[c];
        }
      }
      if (res->correlograph_probes)
        std::memcpy(res->correlograph_probes + p * nc, one.data(), nc * sizeof(double));
    }
    for (size_t c = 0; c < nc; ++c) sum[c] = sum[c] / n_r;
    if (res->correlograph) std::memcpy(res->correlograph, sum.data(), nc * sizeof(double));
    if (res->correlograph_sqr && (detect.outputs & MSF_OUT_CORRELOGRAPH_VAR))
      std::memcpy(res->correlograph_sqr, sqr.data(), nc * sizeof(double));
  }
  if (det->outputs & (MSF_OUT_V_OMEGA | MSF_OUT_VBAR_R)) {
    std::vector<double> sa2(n_k, 0.0), sa(n_k, 0.0), vs(n_k, 0.0);
    for (int64_t p = 0; p < n_probes; ++p) {
      const double* ring = &amp[p * n_seg];
      const double* ring2 = &inten[p * n_seg];
      for (int k = 0; k < n_k; ++k) {
        const double S1 = inside[k] ? 0.0 : ring[k];
        const double S2 = inside[k] ? 0.0 : ring2[k];
        sa2[k] += (S1 * S1) / (cnt[k] * cnt[k]);   // adfstem.cpp:2585-2601
        sa[k] += S1 / cnt[k];
        vs[k] += ((S2 / cnt[k]) / ((S1 * S1) / (cnt[k] * cnt[k]))) - 1.0;  // :2735-2748
      }
    }
    for (int k = 0; k < n_k; ++k) {
      if (res->v_omega && (det->outputs & MSF_OUT_V_OMEGA))
        res->v_omega[k] = (sa[k] == 0.0) ? 0.0 : (n_r * sa2[k] / (sa[k] * sa[k])) - 1.0;
      if (res->vbar_r && (det->outputs & MSF_OUT_VBAR_R)) res->vbar_r[k] = vs[k] / n_r;
    }
  }
  if (pix_modes) {  // adfstem.cpp:2926-3612
    std::vector<double> mean_a(plane), mean_sq(plane), mean_i(plane), var(plane);
    for (int64_t p = 0; p < plane; ++p) {
      mean_a[p] = acc_a[p] / n_r;
      mean_sq[p] = mean_a[p] * mean_a[p];
      mean_i[p] = acc_i[p] / n_r;
    }
    if (res->mean_amplitude) std::memcpy(res->mean_amplitude, mean_a.data(), plane * 8);
    if (res->mean_intensity) std::memcpy(res->mean_intensity, mean_i.data(), plane * 8);
    auto ring_sum = [&](const std::vector<double>& v, std::vector<double>* out) {
      out->assign(n_k, 0.0);
      for (int k = 0; k < n_k; ++k) {
        double s = 0.0;
        for (int32_t q = rings.start[k]; q < rings.start[k + 1]; ++q) s += v[rings.pix[q]];
        (*out)[k] = inside[k] ? 0.0 : s;
      }
    };
    std::vector<double> r1, r2, r3;
    ring_sum(mean_i, &r1);
    ring_sum(mean_sq, &r2);
    ring_sum(mean_a, &r3);
    for (int k = 0; k < n_k; ++k) {
      const double c = (double)cnt[k];
      const double cc = (double)(cnt[k] * cnt[k]);
      if (res->v_gt17 && (det->outputs & MSF_OUT_V_GT17)) res->v_gt17[k] = (r1[k] / c) / (r2[k] / c);
      if (res->v_re && (det->outputs & MSF_OUT_V_RE))
        res->v_re[k] = ((r1[k] / c) / (r3[k] * r3[k] / cc)) - 1.0;
      if (res->v_rbar && (det->outputs & MSF_OUT_V_RBAR))
        res->v_rbar[k] = ((r2[k] / c) / (r3[k] * r3[k] / cc)) - 1.0;
    }
    if (res->omega_vimage && (det->outputs & MSF_OUT_OMEGA_VIMAGE)) {
      const double lsq = g.lambda * g.lambda;
      const double amax_sq = optics.alpha_max * optics.alpha_max;
      for (int i = 0; i < g.nx; ++i)
        for (int j = 0; j < g.ny; ++j) {
          const int64_t p = j + (int64_t)g.ny * i;
          var[p] = (mean_i[p] / (mean_a[p] * mean_a[p])) - 1.0;
          const double ksqr = std::pow(g.kx[i], 2) + std::pow(g.ky[j], 2);
          if (lsq * ksqr <= amax_sq) var[p] = 0.0;
        }
      std::vector<double> r4;
      ring_sum(var, &r4);
      for (int k = 0; k < n_k; ++k) res->omega_vimage[k] = r4[k] / cnt[k];
    }
  }
  return MSF_OK;
}

// The batched passes and detection over the plan's probes; the sums stay on
// the device.  Fills the timing / count fields of `res` and, when asked,
// final_psi (the plan's last probe).
msf_status raster_sums(msf_context* ctx, const RasterPlan& P, msf_results* res) {
  TraceScope trace_scope("raster_passes");
  const msf_specimen* spec = P.spec;
  const Grid& g = spec->g;
  const int64_t plane = P.plane, n_probes = P.n_probes;
  const bool fp64 = ctx->fp64;
  const size_t cbytes = fp64 ? 16 : 8;
  const int S = P.S, n_seg = P.n_seg;

  // batch of wavefields: the context's, the tuned one for this grid, or
  // what half the free memory holds, at most 64
  int B = ctx->batch_for(g.nx, g.ny);
  if (B <= 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const int64_t cap = (int64_t)(0.5 * (double)free_b) / (int64_t)(cbytes * plane);
    B = (int)std::max<int64_t>(1, std::min<int64_t>(cap, 64));
  }
  B = (int)std::min<int64_t>(B, n_probes);
  DevBuf psi, d_partial, mtf_psi, mtf_amp, mtf_int;
  MSF_TRY(ctx->alloc(&psi, cbytes * plane * B));
  MSF_TRY(ctx->alloc(&d_partial, sizeof(double) * 2 * B * std::max(P.n_chunks, 1)));
  if (P.mtf) {
    MSF_TRY(ctx->alloc(&mtf_psi, 16 * plane * B));
    MSF_TRY(ctx->alloc(&mtf_amp, sizeof(double) * B * n_seg));
    MSF_TRY(ctx->alloc(&mtf_int, sizeof(double) * B * n_seg));
  }
  SegmentPlan seg;
  seg.idx = P.seg_idx.as<int32_t>();
  seg.chunk_begin = P.chunk_begin.as<int32_t>();
  seg.seg_chunk = P.seg_chunk.as<int32_t>();
  seg.n_chunks = P.n_chunks;
  seg.ng = n_seg;
  seg.partial = d_partial.as<double>();

  // persistent TMA-pipelined passes for FP32 grids they support
  const int pipe = ctx->pipe_for(g.nx, g.ny);
  const bool staged_row = !fp64 && staged_row_supported(g.nx, g.ny) && (pipe & MSF_ROW_STAGED);
  const int row_sched = !fp64 && staged_row_supported(g.nx, g.ny) && (pipe & MSF_ROW_ALT) ? 1 : 0;
  const bool pipe_row = !fp64 && !staged_row && !row_sched && pipe_supported(g.nx, g.ny) &&
                        (pipe & MSF_PIPE_ROW);
  const bool pipe_col = pipe_supported(g.nx, g.ny, fp64) && (pipe & MSF_PIPE_COL);
  alignas(64) unsigned char col_map[128];
  DevBuf d_err;
  MSF_TRY(ctx->alloc(&d_err, sizeof(int)));
  MSF_CUDA(cudaMemsetAsync(d_err.p, 0, sizeof(int), ctx->stream));
  if (pipe_col) MSF_CUDA(encode_column_map(psi.p, B, g.nx, g.ny, col_map, fp64));

  PassArgs row, col;
  if (pipe_col && !pipe_row && spec->n_live_groups > 0) {  // skip removed columns
    row.row_dead_bits = spec->dead_bits.as<uint32_t>();
    col.live_groups = spec->live_groups.as<int32_t>();
    col.n_live_groups = spec->n_live_groups;
  }
  row.psi = col.psi = psi.p;
  row.batch_stride = col.batch_stride = plane;
  row.nx = col.nx = g.nx;
  row.ny = col.ny = g.ny;
  MSF_TRY(ctx->twiddles(g.ny, fp64, &row.tw));
  MSF_TRY(ctx->twiddles(g.nx, fp64, &col.tw));
  row.inv_s = col.inv_s = 1.0 / g.s;
  row.prefetch_tables = (!fp64 && (pipe & MSF_ROW_PREFETCH)) ? 1 : 0;
  if (!fp64 && !staged_row && row_sched == 0 && !pipe_row && (pipe & MSF_ROW_L2AHEAD))
    set_row_ahead(ctx, spec, &row);
  row.lines_by_probe = (!fp64 && !staged_row && row_sched == 0 && !pipe_row &&
                        (pipe & MSF_ROW_BYPROBE)) ? 1 : 0;
  row.probe = P.probe64.p;
  row.first_scale = g.nxny / g.s;
  col.mask_lo = spec->mask_lo.as<int32_t>();
  col.mask_hi = spec->mask_hi.as<int32_t>();
  const char* tbase = static_cast<const char*>(spec->t.p);
  const char* pbase = static_cast<const char*>(spec->prop.p);
  const size_t prop_stride = cbytes * (g.nx + g.ny);

  // events around the passes of the first (eager) batch: the pass times
  // reported with the results are measured inside the run itself
  std::vector<cudaEvent_t> pass_ev;
  bool timing_passes = false;
  struct EventsGuard {
    std::vector<cudaEvent_t>* v;
    ~EventsGuard() {
      for (cudaEvent_t e : *v) cudaEventDestroy(e);
    }
  } pass_ev_guard{&pass_ev};

  // one batch: 2*S fused passes then the reductions
  auto enqueue_batch = [&](int nb, const int32_t* shifts_dev, double* amp_out,
                           double* int_out) -> msf_status {
    row.nb = col.nb = nb;
    row.shifts = shifts_dev;
    for (int s = 0; s < S; ++s) {
      // removed columns: not read after the first slice, not stored before
      // the last (which leaves zeros there for the detection)
      row.row_dead_io = (s > 0 ? 1 : 0) | (s + 1 < S ? 2 : 0);
      if (timing_passes) MSF_CUDA(cudaEventRecord(pass_ev[3 * s], ctx->stream));
      row.trans = tbase + cbytes * plane * s;
      RowOp op;
      if (fp64) {
        op = s == 0 ? ROW_SLICE_FIRST : ROW_SLICE;
      } else {
        op = s == 0 ? ROW_SPLIT_FIRST : ROW_SPLIT;
        row.psi0 = P.psi0_tab.as<float>() + 2 * plane * s;
      }
      if ((staged_row || row_sched == 1) && op == ROW_SPLIT) {
        PassArgs rs = row;  // schedule 1 reads the zero bits in its own layout
        if (row_sched == 1 && rs.row_dead_bits) rs.row_dead_bits = spec->dead_bits_alt.as<uint32_t>();
        if (staged_row)
          MSF_CUDA(launch_row_split_staged(rs, d_err.as<int>(), ctx->stream, row_sched));
        else
          MSF_CUDA(launch_row_split_alt(rs, ctx->stream));
      }
      else if (pipe_row && op == ROW_SPLIT)
        MSF_CUDA(launch_row_split_pipe(row, d_err.as<int>(), ctx->stream));
      else
        MSF_CUDA(launch_row(fp64, op, row, ctx->stream));
      if (timing_passes) MSF_CUDA(cudaEventRecord(pass_ev[3 * s + 1], ctx->stream));
      col.px = pbase + prop_stride * s;
      col.py = pbase + prop_stride * s + cbytes * g.nx;
      if (pipe_col)
        MSF_CUDA(launch_col_slice_pipe(col, s + 1 == S, col_map, d_err.as<int>(), ctx->stream,
                                       fp64));
      else
        MSF_CUDA(launch_col(fp64, s + 1 == S ? COL_SLICE_LAST : COL_SLICE, col, ctx->stream));
      if (timing_passes) MSF_CUDA(cudaEventRecord(pass_ev[3 * s + 2], ctx->stream));
    }
    SplitK sk;
    if (!fp64) {
      sk.psi0k = P.psi0k.as<double>();
      sk.shifts = shifts_dev;
      sk.nx = g.nx;
      sk.ny = g.ny;
    }
    MSF_CUDA(launch_segment_sums(fp64, psi.p, plane, nb, seg, amp_out, int_out, sk,
                                 ctx->stream));
    if (P.mtf) {
      MSF_TRY(mtf_stage(ctx, P, fp64, psi.p, nb, sk, mtf_psi.as<double>(), ctx->stream));
      MSF_TRY(mtf_ring_sums(P, seg, mtf_psi.as<double>(), nb, mtf_amp.as<double>(),
                            mtf_int.as<double>(), amp_out, int_out, ctx->stream));
      if (P.pix_modes)
        MSF_CUDA(launch_pixel_accum(true, mtf_psi.p, plane, nb, plane, P.acc_a.as<double>(),
                                    P.acc_i.as<double>(), SplitK{}, ctx->stream));
    } else if (P.pix_modes) {
      MSF_CUDA(launch_pixel_accum(fp64, psi.p, plane, nb, plane, P.acc_a.as<double>(),
                                  P.acc_i.as<double>(), sk, ctx->stream));
    }
    return MSF_OK;
  };

  cudaEvent_t ev0, ev1;
  MSF_CUDA(cudaEventCreate(&ev0));
  MSF_CUDA(cudaEventCreate(&ev1));
  MSF_CUDA(cudaEventRecord(ev0, ctx->stream));
  cudaGraphExec_t graph_exec = nullptr;
  DevBuf stage_shift, stage_amp, stage_int;
  const bool use_graph = ctx->graphs && n_probes / B >= 2;
  if (use_graph) {
    MSF_TRY(ctx->alloc(&stage_shift, sizeof(int32_t) * 2 * B));
    MSF_TRY(ctx->alloc(&stage_amp, sizeof(double) * B * n_seg));
    MSF_TRY(ctx->alloc(&stage_int, sizeof(double) * B * n_seg));
  }
  msf_status st = MSF_OK;
  DevBuf first;
  for (int64_t p0 = 0; p0 < n_probes && st == MSF_OK; p0 += B) {
    const int nb = (int)std::min<int64_t>(B, n_probes - p0);
    if (use_graph && nb == B && p0 > 0) {
      MSF_CUDA(cudaMemcpyAsync(stage_shift.p, P.d_shifts.as<int32_t>() + 2 * p0,
                               sizeof(int32_t) * 2 * nb, cudaMemcpyDeviceToDevice, ctx->stream));
      if (!graph_exec) {
        std::lock_guard<std::recursive_mutex> cap(capture_mutex());
        cudaGraph_t graph;
        MSF_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        st = enqueue_batch(nb, stage_shift.as<int32_t>(), stage_amp.as<double>(),
                           stage_int.as<double>());
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (st != MSF_OK) break;
        MSF_CUDA(ce);
        MSF_CUDA(cudaGraphInstantiate(&graph_exec, graph, 0));
        cudaGraphDestroy(graph);
      }
      MSF_CUDA(cudaGraphLaunch(graph_exec, ctx->stream));
      MSF_CUDA(cudaMemcpyAsync(P.amp.as<double>() + p0 * n_seg, stage_amp.p,
                               sizeof(double) * nb * n_seg, cudaMemcpyDeviceToDevice,
                               ctx->stream));
      MSF_CUDA(cudaMemcpyAsync(P.inten.as<double>() + p0 * n_seg, stage_int.p,
                               sizeof(double) * nb * n_seg, cudaMemcpyDeviceToDevice,
                               ctx->stream));
    } else {
      timing_passes = p0 == 0 && S >= 3;
      if (timing_passes) {
        pass_ev.assign(3 * (size_t)S, nullptr);
        for (auto& e : pass_ev) MSF_CUDA(cudaEventCreate(&e));
        res->pass_batch = nb;
      }
      st = enqueue_batch(nb, P.d_shifts.as<int32_t>() + 2 * p0, P.amp.as<double>() + p0 * n_seg,
                         P.inten.as<double>() + p0 * n_seg);
      timing_passes = false;
    }
    if (st == MSF_OK && p0 == 0 && res->first_psi) {
      // the first probe's exit wave (adfstem.cpp:2139-2221), before the
      // next batch reuses its buffer
      MSF_TRY(ctx->alloc(&first, 16 * plane));
      if (fp64)
        MSF_CUDA(cudaMemcpyAsync(first.p, psi.p, 16 * plane, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
      else
        MSF_CUDA(launch_assemble_split(psi.as<float>(), P.psi0k.as<double>(), g.nx, g.ny,
                                       P.shifts[0], P.shifts[1], first.as<double>(),
                                       ctx->stream));
    }
  }
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (st != MSF_OK) return st;
  MSF_CUDA(cudaEventRecord(ev1, ctx->stream));

  if (res->first_psi && first.p) {
    MSF_CUDA(cudaMemcpyAsync(res->first_psi, first.p, 16 * plane, cudaMemcpyDeviceToHost,
                             ctx->stream));
    MSF_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += 16 * plane;
  }
  if (res->final_psi && P.mtf) {
    // the reference's wave after its detector MTF stage (adfstem.cpp:2272-2385)
    const int last = (int)((n_probes - 1) % B);
    MSF_CUDA(cudaMemcpyAsync(res->final_psi, mtf_psi.as<double>() + 2 * plane * last, 16 * plane,
                             cudaMemcpyDeviceToHost, ctx->stream));
    MSF_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += 16 * plane;
  } else if (res->final_psi) {
    const int last = (int)((n_probes - 1) % B);
    if (fp64) {
      MSF_CUDA(cudaMemcpyAsync(res->final_psi, psi.as<double>() + 2 * plane * last,
                               16 * plane, cudaMemcpyDeviceToHost, ctx->stream));
    } else {
      // exit wave = scattered part + the vacuum part at this probe's shift
      DevBuf full;
      MSF_TRY(ctx->alloc(&full, 16 * plane));
      const int64_t pl = n_probes - 1;
      MSF_CUDA(launch_assemble_split(psi.as<float>() + 2 * plane * last, P.psi0k.as<double>(),
                                     g.nx, g.ny, P.shifts[2 * pl], P.shifts[2 * pl + 1],
                                     full.as<double>(), ctx->stream));
      MSF_CUDA(cudaMemcpyAsync(res->final_psi, full.p, 16 * plane, cudaMemcpyDeviceToHost,
                               ctx->stream));
      MSF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    ctx->d2h_bytes += (int64_t)cbytes * plane;
  }
  MSF_CUDA(cudaStreamSynchronize(ctx->stream));
  int err_flag = 0;
  MSF_CUDA(cudaMemcpy(&err_flag, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  ctx->d2h_bytes += 8;
  if (err_flag) {
    set_error("a pipelined slice pass gave up waiting for a tile copy (bounded wait)");
    return MSF_ERR_TIMEOUT;
  }
  float ms = 0;
  MSF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  res->seconds_raster = 1e-3 * ms;
  res->seconds_setup = 0;
  res->probe_slices = n_probes * S;
  res->ms_row_pass = res->ms_col_pass = 0;
  if (!pass_ev.empty()) {
    // row passes of slices 1..S-1 (after the probe-placing first), column
    // passes of slices 0..S-2 (before the last, which stops in k-space)
    double row_ms = 0, col_ms = 0;
    for (int s = 0; s < S; ++s) {
      float a = 0, b = 0;
      MSF_CUDA(cudaEventElapsedTime(&a, pass_ev[3 * s], pass_ev[3 * s + 1]));
      MSF_CUDA(cudaEventElapsedTime(&b, pass_ev[3 * s + 1], pass_ev[3 * s + 2]));
      if (s >= 1) row_ms += a;
      if (s + 1 < S) col_ms += b;
    }
    res->ms_row_pass = row_ms / (S - 1);
    res->ms_col_pass = col_ms / (S - 1);
  } else {
    res->pass_batch = 0;
  }
  {
    const int64_t n_batches = (n_probes + B - 1) / B;
    // probe: synth, 2 transform passes, norm, scale (+ FP32 copy); per batch:
    // 2*S slice passes, the segment sums (chunks, totals) and (pixel modes)
    // the accumulation
    // (MTF: magnitude, 4 transform passes, multiply, scale, band limit and
    // the ring sums of the filtered waves)
    res->kernel_launches =
        P.setup_launches +
        n_batches * (2 * S + 2 + (P.pix_modes ? 1 : 0) + (P.mtf ? 8 + (P.n_k > 0 ? 2 : 0) : 0));
  }
  return MSF_OK;
}

msf_status run_raster(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                      const msf_raster* raster, const msf_detect* det, msf_results* res) {
  if (!spec || !optics || !raster || !det || !res) { set_error("null argument"); return MSF_ERR_ARG; }
  RasterPlan P;
  MSF_TRY(plan_raster(ctx, spec, optics, raster, det, &P));
  MSF_TRY(raster_sums(ctx, P, res));
  return finish_raster(ctx, P, ctx->stream, res);
}

msf_status run_raster_plain(msf_context* ctx, const msf_specimen* spec,
                            const msf_optics* optics, const msf_raster* raster,
                            const msf_detect* det, msf_results* res) {
  TraceScope trace_scope("raster_plain");
  if (!spec || !optics || !raster || !det || !res) { set_error("null argument"); return MSF_ERR_ARG; }
  if (!ctx->fp64) {
    set_error("the plain per-pass path runs FP64 wavefields: use an MSF_FP64 context");
    return MSF_ERR_UNSUPPORTED;
  }
  RasterPlan P;
  MSF_TRY(plan_raster(ctx, spec, optics, raster, det, &P));
  const Grid& g = spec->g;
  const int64_t plane = P.plane;
  const int S = P.S;
  cudaStream_t st = ctx->stream;
  DevBuf psi, d_partial, mtf_psi, mtf_amp, mtf_int;
  MSF_TRY(ctx->alloc(&psi, 16 * plane));
  MSF_TRY(ctx->alloc(&d_partial, sizeof(double) * 2 * std::max(P.n_chunks, 1)));
  if (P.mtf) {
    MSF_TRY(ctx->alloc(&mtf_psi, 16 * plane));
    MSF_TRY(ctx->alloc(&mtf_amp, sizeof(double) * P.n_seg));
    MSF_TRY(ctx->alloc(&mtf_int, sizeof(double) * P.n_seg));
  }
  SegmentPlan seg;
  seg.idx = P.seg_idx.as<int32_t>();
  seg.chunk_begin = P.chunk_begin.as<int32_t>();
  seg.seg_chunk = P.seg_chunk.as<int32_t>();
  seg.n_chunks = P.n_chunks;
  seg.ng = P.n_seg;
  seg.partial = d_partial.as<double>();
  PassArgs a;
  a.psi = psi.p;
  a.batch_stride = plane;
  a.nb = 1;
  a.nx = g.nx;
  a.ny = g.ny;
  a.scale = 1.0;
  const void *tw_y = nullptr, *tw_x = nullptr;
  MSF_TRY(ctx->twiddles(g.ny, true, &tw_y));
  MSF_TRY(ctx->twiddles(g.nx, true, &tw_x));
  auto fft2 = [&](bool inverse) -> msf_status {
    a.tw = tw_y;
    MSF_CUDA(launch_row(true, inverse ? ROW_INV : ROW_FWD, a, st));
    a.tw = tw_x;
    MSF_CUDA(launch_col(true, inverse ? COL_INV : COL_FWD, a, st));
    return MSF_OK;
  };
  const double* t0 = spec->t.as<double>();
  const double* prop = spec->prop.as<double>();
  const int32_t* lo = spec->mask_lo.as<int32_t>();
  const int32_t* hi = spec->mask_hi.as<int32_t>();
  double* d = psi.as<double>();
  cudaEvent_t ev0, ev1;
  MSF_CUDA(cudaEventCreate(&ev0));
  MSF_CUDA(cudaEventCreate(&ev1));
  MSF_CUDA(cudaEventRecord(ev0, st));
  int64_t launches = 0;
  for (int64_t p = 0; p < P.n_probes; ++p) {
    // a15-a16: shifted probe, FORWARD transform, / sqrt(NxNy)
    MSF_CUDA(launch_place_probe(d, P.probe64.as<double>(), g.nx, g.ny, P.shifts[2 * p],
                                P.shifts[2 * p + 1], st));
    MSF_TRY(fft2(false));
    MSF_CUDA(launch_scale(d, plane, 1.0 / g.s, nullptr, st));
    launches += 4;
    for (int s = 0; s < S; ++s) {  // a17, one reference step per launch
      MSF_TRY(fft2(true));
      MSF_CUDA(launch_transmit(d, t0 + 2 * plane * s, plane, 1.0 / g.s, st));
      MSF_TRY(fft2(false));
      MSF_CUDA(launch_scale(d, plane, 1.0 / g.s, nullptr, st));
      MSF_CUDA(launch_bw_limit(d, lo, hi, g.nx, g.ny, st));
      const double* px = prop + 2 * (size_t)(g.nx + g.ny) * s;
      MSF_CUDA(launch_propagate(d, px, px + 2 * g.nx, lo, hi, g.nx, g.ny, st));
      launches += 8;
    }
    if (p == 0 && res->first_psi) {
      MSF_CUDA(cudaMemcpy(res->first_psi, d, 16 * plane, cudaMemcpyDeviceToHost));
      ctx->d2h_bytes += 16 * plane;
    }
    SplitK none;
    double* amp_p = P.amp.as<double>() + p * P.n_seg;
    double* int_p = P.inten.as<double>() + p * P.n_seg;
    MSF_CUDA(launch_segment_sums(true, d, plane, 1, seg, amp_p, int_p, none, st));
    launches += 2;
    const double* fem_src = d;
    if (P.mtf) {
      MSF_TRY(mtf_stage(ctx, P, true, d, 1, none, mtf_psi.as<double>(), st));
      MSF_TRY(mtf_ring_sums(P, seg, mtf_psi.as<double>(), 1, mtf_amp.as<double>(),
                            mtf_int.as<double>(), amp_p, int_p, st));
      fem_src = mtf_psi.as<double>();
      launches += 8 + (P.n_k > 0 ? 2 : 0);
    }
    if (P.pix_modes) {
      MSF_CUDA(launch_pixel_accum(true, fem_src, plane, 1, plane, P.acc_a.as<double>(),
                                  P.acc_i.as<double>(), none, st));
      launches += 1;
    }
  }
  MSF_CUDA(cudaEventRecord(ev1, st));
  MSF_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  MSF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  res->seconds_raster = 1e-3 * ms;
  res->seconds_setup = 0;
  res->probe_slices = P.n_probes * S;
  res->kernel_launches = P.setup_launches + launches;
  if (res->final_psi) {
    MSF_CUDA(cudaMemcpy(res->final_psi, P.mtf ? mtf_psi.as<double>() : d, 16 * plane,
                        cudaMemcpyDeviceToHost));
    ctx->d2h_bytes += 16 * plane;
  }
  return finish_raster(ctx, P, st, res);
}

msf_status run_partial(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                       const msf_raster* raster, const msf_detect* det, int64_t p_begin,
                       int64_t p_end, double* amp, double* inten, double* acc_a,
                       double* acc_i, msf_results* info) {
  TraceScope trace_scope("raster_partial");
  if (!spec || !optics || !raster || !det) { set_error("null argument"); return MSF_ERR_ARG; }
  RasterPlan P;
  MSF_TRY(plan_raster(ctx, spec, optics, raster, det, &P, p_begin, p_end));
  msf_results local{};
  msf_results* r = info ? info : &local;
  r->final_psi = nullptr;
  MSF_TRY(raster_sums(ctx, P, r));
  r->n_k = P.n_k;
  return download_sums(ctx, P, ctx->stream, amp, inten, acc_a, acc_i);
}

}  // namespace msf
