// Device-side engine behind the C ABI: contexts, specimens, raster runs.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "msf.h"
#include "setup.hpp"

namespace msf {

void set_error(const std::string& msg);

// Held while a thread captures a CUDA graph and while a thread waits for the
// whole device (cudaDeviceSynchronize, cudaFree): a device-wide wait from
// one thread would invalidate another thread's capture (the serving loop's
// builder and worker threads).
std::recursive_mutex& capture_mutex();

// Device memory of one context.  `live` bytes count against the context's
// budget; released blocks are kept for reuse by later allocations of about
// their size (a new specimen, raster or request then maps no new memory),
// and handed back to the driver when an allocation fails or the context
// goes away.  Shared by the context and its buffers, so a buffer released
// after its context frees its memory directly.
struct Pool {
  int64_t live = 0, cached = 0;
  bool closed = false;
  std::multimap<size_t, void*> blocks;
  std::mutex m;
  // A cached block of at least `bytes` and at most twice that (+4 MiB), or
  // nullptr; *got receives its size.
  void* take(size_t bytes, size_t* got);
  // Keeps a released block.  Waits for the device first, as cudaFree does,
  // so that no kernel still in flight on any stream can see it reused.
  void give(void* p, size_t bytes);
  void trim();  // cudaFree of every cached block
  ~Pool() { trim(); }
};

// Owning device allocation that counts against its context's budget.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  std::shared_ptr<Pool> pool;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    release();
    p = o.p; bytes = o.bytes; pool = std::move(o.pool);
    o.p = nullptr; o.bytes = 0; o.pool.reset();
    return *this;
  }
  ~DevBuf() { release(); }
  void release();
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace msf

// Slice-pass variants (bit mask): the persistent TMA-pipelined column pass,
// the persistent pipelined split-wave row pass, and the split-wave row pass
// with its transmission and vacuum rows staged in shared memory by bulk
// copies (which takes precedence over MSF_PIPE_ROW).
constexpr int MSF_PIPE_COL = 1, MSF_PIPE_ROW = 2, MSF_ROW_STAGED = 4;
// the split-wave row pass's alternative FFT radix schedule (16 elements a
// thread; staged or plain)
constexpr int MSF_ROW_ALT = 8;
// the plain split-wave row pass prefetches its transmission and vacuum rows
// into L1 (PassArgs::prefetch_tables)
constexpr int MSF_ROW_PREFETCH = 16;
// the plain split-wave row pass (default schedule) prefetches the wavefield
// rows of the CTAs one resident wave ahead into L2 (PassArgs::l2_ahead)
constexpr int MSF_ROW_L2AHEAD = 32;
// the plain split-wave row pass (default schedule) gives each CTA one row
// of consecutive probes (PassArgs::lines_by_probe)
constexpr int MSF_ROW_BYPROBE = 64;
constexpr int MSF_PIPE_ALL = MSF_PIPE_COL | MSF_PIPE_ROW | MSF_ROW_STAGED | MSF_ROW_ALT |
                             MSF_ROW_PREFETCH | MSF_ROW_L2AHEAD | MSF_ROW_BYPROBE;

struct msf_context {
  int device = 0;
  bool fp64 = true;
  int batch = 0;
  bool graphs = true;
  // slice-pass variants (MSF_PIPE_* / MSF_ROW_* bits) for grids the tuner
  // has not measured, overridden by the MSF_PIPE environment variable: the
  // pipelined column pass and the row pass that prefetches its tables
  // (measured 4 % faster for msf_run at 512^2-2048^2; bit-identical)
  int pipe = MSF_PIPE_COL | MSF_ROW_PREFETCH;
  // slice potentials: 0 FFT convolution for slices of at least 64 atoms,
  // direct sum otherwise; 1 always direct; 2 always FFT (MSF_POTENTIAL =
  // direct / fft)
  int potential = 0;
  int64_t budget = 0;
  std::shared_ptr<msf::Pool> pool = std::make_shared<msf::Pool>();
  int64_t allocated() const { return pool->live; }
  int64_t h2d_bytes = 0, d2h_bytes = 0;
  cudaStream_t stream = nullptr;
  std::map<int, msf::DevBuf> tw64, tw32;  // twiddle tables per length
  // autotuned launch tiling per grid (nx, ny): probes per launch and the
  // pipelined-pass mask (msf_tune, or imported wisdom)
  struct Tuned {
    int batch = 0;
    int pipe = 0;
    double ns_per_probe_slice = 0;
  };
  std::map<std::pair<int, int>, Tuned> tuned;
  int batch_for(int nx, int ny) const {
    auto it = tuned.find({nx, ny});
    return batch > 0 ? batch : it != tuned.end() ? it->second.batch : 0;
  }
  int pipe_for(int nx, int ny) const {
    auto it = tuned.find({nx, ny});
    return (pipe_env || it == tuned.end()) ? pipe : it->second.pipe;
  }
  bool pipe_env = false;  // MSF_PIPE given: it wins over tuning
  // distance of the row pass's L2 prefetch (MSF_ROW_L2AHEAD) in percent of
  // one resident wave of CTAs (MSF_ROW_AHEAD_PCT)
  int row_ahead_pct = 100;
  // FEM ring bins per grid and dr (host sort of every pixel by k^2: 34 ms at
  // 1024^2, 180 ms at 2048^2), reused by every raster planned on that grid
  struct RingKey {
    int nx, ny;
    double xpd, ypd, bw_t, dr;
    bool operator<(const RingKey& o) const {
      return std::tie(nx, ny, xpd, ypd, bw_t, dr) <
             std::tie(o.nx, o.ny, o.xpd, o.ypd, o.bw_t, o.dr);
    }
  };
  std::map<RingKey, std::shared_ptr<const msf::Rings>> ring_cache;
  std::mutex ring_mu;
  // pinned host buffer the per-probe and per-pixel sums of a raster are
  // copied into before the host finish (grown on demand, reused by every
  // raster; freed with the context)
  double* host_stage = nullptr;
  size_t host_stage_bytes = 0;
  std::mutex stage_mu;
  // specimens built by this context keep a host copy of every slice's
  // projected potential before the exponential (msf_specimen_potential)
  bool keep_potentials = false;
  msf_status alloc(msf::DevBuf* b, size_t bytes);
  msf_status twiddles(int n, bool fp64, const void** out);
};

struct msf_specimen {
  msf_context* ctx = nullptr;
  msf::Grid g;
  std::vector<double> lower, thickness;
  std::vector<int64_t> counts;
  int n_slices = 0;
  msf::DevBuf t;              // [slice][nx][ny] complex, context precision
  msf::DevBuf prop;           // [slice] {px[nx], py[ny]} complex, context precision
  msf::DevBuf mask_lo, mask_hi;
  // columns the band limit removes entirely: row-pass zero bits, and the
  // column groups of the pipelined column pass that keep any column
  msf::DevBuf dead_bits, live_groups;
  // the row-pass zero bits in the layout of the alternative FFT schedule of
  // the staged row pass (FP32 contexts; empty when it does not apply)
  msf::DevBuf dead_bits_alt;
  std::vector<uint32_t> h_dead_bits;  // host copies (slot lanes compare them)
  std::vector<int32_t> h_live_groups;
  int n_live_groups = 0, n_live_columns = 0;
  // element ranges of a row that hold live columns (two half-open ranges,
  // even bounds; the whole row when no column is removed or the removed
  // ones are not one run): what the row pass prefetches ahead into L2
  int row_live[4] = {0, 0, 0, 0};
  msf::DevBuf kx, ky;         // FP64 domains for device set-up kernels
  std::vector<double> hprop;  // FP64 propagators, host copy
  std::vector<double> h_potential;  // [slice][nx][ny] complex, when kept
  double seconds_setup = 0;
  int64_t device_bytes = 0;
};

namespace msf {

// Device state of one raster over one specimen: the probe, the vacuum-wave
// tables of split-wave FP32 runs, per-probe pixel shifts, the detector /
// ring pixel segments and the per-probe sums they fill.  Shared by the
// batched raster (run_raster) and the slot lanes that mix probes of several
// rasters (lanes.cpp).
struct RasterPlan {
  const msf_specimen* spec = nullptr;
  msf_optics optics{};
  msf_detect det{};
  int64_t p_begin = 0, n_raster = 0;  // this plan's probes: [p_begin, p_begin + n_probes)
  int64_t n_probes = 0;
  int S = 0;
  int64_t plane = 0;
  bool want_adf = false, pix_modes = false;
  uint32_t fem = 0;
  std::vector<int32_t> shifts;  // [n_probes][2] (sx, sy)
  DevBuf d_shifts;
  DevBuf probe64;               // normalised probe, real space, FP64
  DevBuf psi0_tab;              // FP32 runs: [S] vacuum wave entering slice s
  DevBuf psi0k;                 // FP32 runs: vacuum exit wave, k-space, FP64
  std::shared_ptr<const Rings> rings;  // FEM ring bins (shared, cached per grid)
  int n_k = 0, n_seg = 0, n_chunks = 0;
  DevBuf seg_idx, chunk_begin, seg_chunk;  // segments cut into chunks
  DevBuf amp, inten;            // [n_probes][n_seg] sums of |psi| and |psi|^2
  DevBuf acc_a, acc_i;          // [plane] sums over probes (pixel modes)
  bool mtf = false;             // detector MTF applied before the FEM sums
  DevBuf mtf2d;                 // [plane] complex FP64, band-limited as the reference does
  int64_t setup_launches = 0;
  int64_t device_bytes() const {
    return (int64_t)(d_shifts.bytes + probe64.bytes + psi0_tab.bytes + psi0k.bytes +
                     seg_idx.bytes + chunk_begin.bytes + seg_chunk.bytes + amp.bytes +
                     inten.bytes + acc_a.bytes + acc_i.bytes + mtf2d.bytes);
  }
};
// Device bytes plan_raster will allocate (for admission by an HBM budget).
int64_t raster_plan_bytes(const msf_specimen* spec, bool fp64, int64_t n_probes,
                          bool pix_modes);
// Plans probes [p_begin, p_end) of the raster (p_end < 0: to its end).
// The ring bins of grid g at bin-width factor dr, from the context's cache
// (computed on first use).
std::shared_ptr<const Rings> rings_for(msf_context* ctx, const Grid& g, double dr);
msf_status plan_raster(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                       const msf_raster* raster, const msf_detect* det, RasterPlan* plan,
                       int64_t p_begin = 0, int64_t p_end = -1);
// Copies the plan's per-probe sums ([n_probes][n_seg] each) and pixel sums
// to host arrays (any may be null), synchronising `stream`.
msf_status download_sums(msf_context* ctx, const RasterPlan& P, cudaStream_t stream,
                         double* amp, double* inten, double* acc_a, double* acc_i);
// Copies the plan's sums to the host (synchronising `stream`) and finishes
// the ADF image and FEM statistics in FP64 in the reference's order.
msf_status finish_raster(msf_context* ctx, const RasterPlan& plan, cudaStream_t stream,
                         msf_results* res);
// The ADF image and FEM statistics from per-probe sums of a whole raster
// (host only): amp / inten [n_probes][n_k + 1] (ring sums, then the ADF
// annulus), acc_a / acc_i the per-pixel sums over all probes (pixel modes).
msf_status finish_host(const Grid& g, const Rings& rings, const msf_optics& optics,
                       const msf_detect& detect, int64_t n_probes, const double* amp,
                       const double* inten, const double* acc_a, const double* acc_i,
                       msf_results* res);
// The raster one probe at a time, one launch per reference step (FP64).
msf_status run_raster_plain(msf_context* ctx, const msf_specimen* spec,
                            const msf_optics* optics, const msf_raster* raster,
                            const msf_detect* det, msf_results* res);
// Per-probe sums of probes [p_begin, p_end) of a raster (one shard).
msf_status run_partial(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                       const msf_raster* raster, const msf_detect* det, int64_t p_begin,
                       int64_t p_end, double* amp, double* inten, double* acc_a,
                       double* acc_i, msf_results* info);

msf_status build_specimen(msf_context* ctx, const msf_grid* grid, const msf_atoms* atoms,
                          msf_specimen* spec);
msf_status run_raster(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                      const msf_raster* raster, const msf_detect* detect, msf_results* res);
msf_status build_probe(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                       DevBuf* probe64);
msf_status time_passes(msf_context* ctx, const msf_specimen* spec, int nb, int reps,
                       double* ms_row, double* ms_col);
msf_status run_batch(msf_context* ctx, int n, const msf_specimen* const* specs,
                     const msf_optics* optics, const msf_raster* rasters,
                     const msf_detect* detects, msf_results* results, int slots);
int lane_slots(int want, int64_t plane, int lanes, int64_t probes);
struct PassArgs;
// The plain FP32 split-wave row pass's L2 prefetch ahead (MSF_ROW_L2AHEAD)
// for rows of `spec`'s grid: distance and live element ranges.
void set_row_ahead(const msf_context* ctx, const msf_specimen* spec, PassArgs* row);
struct SplitK;
// The detector MTF stage of nb exit waves into FP64 planes `out` (the plan
// supplies the grid, aperture and the 2-D MTF).
msf_status mtf_stage(msf_context* ctx, const RasterPlan& P, bool fp64, const void* psi, int nb,
                     const SplitK& sk, double* out, cudaStream_t st);
// MD-coupled FEM: every probe through `samples` snapshot specimens (sample s
// uses snapshot s mod n_snap), exit waves averaged coherently (md.cpp).
msf_status run_md(msf_context* ctx, int n_snap, const msf_specimen* const* snaps, int samples,
                  const msf_optics* optics, const msf_raster* raster, const msf_detect* det,
                  msf_results* res);
// Times the slice passes of `spec`'s grid at candidate tilings and records
// the fastest in ctx->tuned (tune.cpp).
msf_status tune(msf_context* ctx, const msf_specimen* spec, msf_tuning* out);
}  // namespace msf
