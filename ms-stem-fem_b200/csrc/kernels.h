// Host-callable launchers for the sm_100a kernels in kernels.cu.
// No CUDA types beyond cudaStream_t cross this header; all device pointers
// are passed as void* / typed raw pointers owned by the caller.
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace msf {

// Launch set-up that is per device (cudaFuncSetAttribute, occupancy):
// each launcher keeps one bit per device ordinal, so a process that uses
// several devices configures every one of them, and threads that race on
// the first launch of a device both do the (idempotent) set-up.  Ordinals
// past 63 redo the set-up on every launch.
struct PerDevice {
  std::atomic<uint64_t> bits{0};
  bool needed(int dev) const {
    return dev < 0 || dev >= 64 || !((bits.load(std::memory_order_acquire) >> dev) & 1u);
  }
  void mark(int dev) {
    if (dev >= 0 && dev < 64) bits.fetch_or(uint64_t(1) << dev, std::memory_order_release);
  }
};
inline int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) return -1;
  return d;
}
// SMs of the current device (cached per device ordinal).
int sm_count();
// Raise `func`'s dynamic shared-memory limit to `bytes` on the current
// device, once per device.
inline cudaError_t smem_limit_once(const void* func, int bytes, PerDevice& once) {
  const int dev = current_device();
  if (!once.needed(dev)) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) once.mark(dev);
  return e;
}

// Which fused operation a row pass (transform along y, contiguous) does.
enum RowOp : int {
  ROW_FWD = 0,          // forward DFT along y
  ROW_INV = 1,          // inverse DFT along y, then * scale
  ROW_SLICE = 2,        // inverse DFT, transmission multiply, forward DFT
  ROW_SLICE_FIRST = 3,  // place shifted probe, transmission multiply, fwd DFT
  // Split-wave slice passes (FP32): the buffer holds only the scattered part
  // delta = psi - psi0 of each probe's wave, where psi0 is the probe's
  // vacuum evolution (precomputed in FP64, shared by all probes up to an
  // integer shift) and the transmission is stored as tau = t - 1.
  ROW_SPLIT = 4,        // iDFT, delta' = Q(t, psi0 + delta) - psi0/s, DFT
  ROW_SPLIT_FIRST = 5,  // delta = 0 on entry: delta' = Q(t, psi0) - psi0/s
  // Split-wave pass of a slot batch (FP32): every probe reads its own slice
  // tables and step from PassArgs::slots (ROW_SPLIT_FIRST or ROW_SPLIT).
  ROW_SLOTS = 6,
};
// Which fused operation a column pass (transform along x, strided) does.
enum ColOp : int {
  COL_FWD = 0,           // forward DFT along x
  COL_INV = 1,           // inverse DFT along x, then * scale
  COL_FWD_MASK_INV = 2,  // forward DFT, band-limit mask, inverse DFT
  COL_SLICE = 3,         // fwd DFT, /s, mask, propagator, inverse DFT
  COL_SLICE_LAST = 4,    // fwd DFT, /s, mask, propagator (stay in k-space)
  COL_SLOTS = 5,         // COL_SLICE or COL_SLICE_LAST per slot (FP32)
};

// One probe slot's step in a slot batch: probes of different specimens (of
// one grid size) share a launch, each at its own slice.
enum SlotOp : int32_t {
  SLOT_IDLE = 0,   // empty slot: both passes skip it
  SLOT_FIRST = 1,  // first slice of a probe (scattered part zero on entry)
  SLOT_NEXT = 2,   // a later slice
};
struct SlotPass {
  const void* trans = nullptr;       // tau of this slice, [nx][ny] float2
  const void* psi0 = nullptr;        // vacuum wave entering this slice
  const void* px = nullptr;          // propagator of this slice along x
  const void* py = nullptr;          // ... along y
  const int32_t* mask_lo = nullptr;  // the specimen's band-limit mask
  const int32_t* mask_hi = nullptr;
  int32_t op = SLOT_IDLE;
  int32_t last = 0;                  // 1: last slice, stay in k-space
  int32_t sx = 0, sy = 0;            // the probe's pixel shift
};

struct PassArgs {
  void* psi = nullptr;            // [nb][nx][ny] complex (float2 or double2)
  int64_t batch_stride = 0;       // elements between arrays
  int nb = 1;                     // arrays in the batch
  int nx = 0, ny = 0;
  const void* tw = nullptr;       // twiddle table for the transformed length
  // row slice ops
  const void* trans = nullptr;    // [nx][ny] complex, this slice
  double inv_s = 1.0;             // 1/sqrt(nx*ny)
  const void* probe = nullptr;    // [nx][ny] complex, normalised real space
  const int32_t* shifts = nullptr;// [nb][2] (sx, sy)
  double first_scale = 1.0;       // nx*ny/s
  double scale = 1.0;             // ROW_INV / COL_INV
  // column mask and propagator
  const int32_t* mask_lo = nullptr;  // [ny]: keep i < lo[j] || i >= hi[j]
  const int32_t* mask_hi = nullptr;
  const void* px = nullptr;       // [nx] complex propagator along x (Real2)
  const void* py = nullptr;       // [ny] complex propagator along y (Real2)
  // split-wave row passes: vacuum wave entering this slice, [nx][ny]
  // complex, in the same scale as the inverse-transformed buffer
  const void* psi0 = nullptr;
  // slot batches (ROW_SLOTS, COL_SLOTS, pipelined column pass): [nb]
  const SlotPass* slots = nullptr;
  // Columns the band limit removes entirely (lo = 0, hi = nx: no kx kept):
  // the slice row passes store zeros there (bit m of word t: column
  // t + T*m, T the row transform's threads per line) ...
  const uint32_t* row_dead_bits = nullptr;
  // with row_dead_bits: bit 0, this pass's input was not stored in those
  // columns (read them as zero); bit 1, its output there need not be stored
  // (the next pass reads none of it)
  int row_dead_io = 0;
  // ... so the pipelined column pass skips the column groups that hold only
  // such columns: it walks live_groups[n_live_groups] (nullptr: all groups)
  const int32_t* live_groups = nullptr;
  int n_live_groups = 0;
  // split-wave row passes (ROW_SPLIT, ROW_SLOTS): prefetch the line's
  // transmission and vacuum rows into L1 at the start, and load the
  // wavefield past L1, so the update after the inverse transform finds its
  // tables in L1
  int prefetch_tables = 0;
  // split-wave row pass (ROW_SPLIT, plain launch): each CTA bulk-prefetches
  // into L2 the wavefield rows of the CTA l2_ahead places later in launch
  // order (0: off).  CTAs start in increasing linear order, so with
  // l2_ahead about one resident wave that CTA starts as this one ends and
  // finds its rows in L2 instead of waiting on HBM.  Only the element
  // ranges [ahead_range[0], ahead_range[1]) and [ahead_range[2],
  // ahead_range[3]) of a row are fetched (the live columns; even bounds).
  int l2_ahead = 0;
  int ahead_range[4] = {0, 0, 0, 0};
  // split-wave row pass (ROW_SPLIT, plain launch): the lines of a CTA are
  // one row of consecutive probes (grid (nb / lines, nx)) instead of
  // consecutive rows of one probe, so they share the row's transmission
  // and, for probes of one raster line, its vacuum row in L1.  Ignored when
  // nb is not a multiple of the lines per CTA.
  int lines_by_probe = 0;
};

// Vacuum part of the exit wave for split-wave detection: k-space values of
// the unshifted probe's vacuum exit wave (FP64, zero outside the aperture)
// and per-probe pixel shifts; each probe adds psi0k[m] * e^{-2 pi i
// (mx sx / nx + my sy / ny)} to its scattered part before |psi| is taken.
struct SplitK {
  const double* psi0k = nullptr;   // [nx][ny] complex; nullptr: not split
  const int32_t* shifts = nullptr; // [nb][2]
  int nx = 0, ny = 0;
};

// Returns false if the length is not supported.
bool supported_length(int n);
// Threads per line of the row transform of length n (its T); 0 if unsupported.
int row_line_threads(int n, bool fp64);
// Columns per tile of the pipelined column pass (0 if unsupported).
int pipe_cols_for(int nx, bool fp64);
cudaError_t launch_row(bool fp64, RowOp op, const PassArgs& a, cudaStream_t s);
// CTAs of the FP32 split-wave row pass (ROW_SPLIT, default schedule) that
// the current device holds at once for rows of length ny (0 if
// unsupported): the natural PassArgs::l2_ahead.
int row_split_resident_ctas(int ny);
// The FP32 split-wave row pass (ROW_SPLIT) on the alternative FFT radix
// schedule (16 elements a thread from 512 points, 8 at 256; row_dead_bits
// in that schedule's layout, staged_row_threads(ny, 1)); row lengths
// 256..2048.
cudaError_t launch_row_split_alt(const PassArgs& a, cudaStream_t s);
cudaError_t launch_col(bool fp64, ColOp op, const PassArgs& a, cudaStream_t s);

// ---- persistent TMA-pipelined slice passes (kernels_pipe.cu) ----
// The column pass: FP32 grids with sides 256..2048, FP64 grids with sides
// 256..1024; the split-wave row pass: FP32 only.
bool pipe_supported(int nx, int ny, bool fp64 = false);
// Split-wave row pass for slices after the first; *err set to 1 if a copy
// never arrived (bounded wait).
cudaError_t launch_row_split_pipe(const PassArgs& a, int* err, cudaStream_t s);
// Split-wave row pass for slices after the first with the slice tables
// staged: each CTA transforms one row of several probes and bulk-copies
// the shared transmission row and the probes' vacuum rows into shared
// memory during the inverse transform (FP32, row lengths 256..2048).
// Honours row_dead_bits / row_dead_io like launch_row (with the bit layout
// of the schedule's threads per line); *err set to 1 if a copy never
// arrived (bounded wait).  `schedule` picks the FFT radix schedule: 0 the
// default (32 elements a thread from 512 points), 1 half the elements and
// twice the threads per line.  Bit-identical to launch_row's ROW_SPLIT
// with schedule 0; schedule 1 rounds differently (another factorisation).
bool staged_row_supported(int nx, int ny);
// Threads per line of the staged row pass's transform (0 if unsupported).
int staged_row_threads(int ny, int schedule);
cudaError_t launch_row_split_staged(const PassArgs& a, int* err, cudaStream_t s,
                                    int schedule = 0);
// Column slice pass (COL_SLICE, or COL_SLICE_LAST when `last`; per slot
// when a.slots is set); `tensor_map` from encode_column_map over the same
// batch buffer.
cudaError_t launch_col_slice_pipe(const PassArgs& a, bool last, const void* tensor_map,
                                  int* err, cudaStream_t s, bool fp64 = false);
// Encode the 2-D tensor map (128 bytes) the column pass loads tiles with.
cudaError_t encode_column_map(void* psi, int nb, int nx, int ny, void* map_out,
                              bool fp64 = false);

// Twiddle table e^{-2 pi i m / n}, m < n, computed in FP64 on the host.
void fill_twiddles(int n, double* host_interleaved /* 2n */);
// The FP32 passes' table: fill_twiddles' n entries followed by each stage's
// factors again as [r][k] (copies of table entries, in the order the FP32
// schedules of length n read them: the main one, then the alternative).
void fill_twiddles_f32_table(int n, std::vector<double>& host_interleaved);

// ---- set-up kernels (FP64) ----
// sigma*V_z(k) of one species in k-space (scatterer_pap.hpp:109-151).
cudaError_t launch_lut_synth(double* out, const double* kx, const double* ky,
                             int nx, int ny, const double* params12,
                             double prefactor, double cutoff_sq, double xmin,
                             double ymin, cudaStream_t s);
// t(x,y) = sum of shifted LUTs over the slice's atoms, then
// e^{-Im} (cos Re, sin Re) (slice.cpp:1544-1725).  Atoms in slice order.
// exponentiate = false: stop at the sum (the projected potential).
cudaError_t launch_potential(double* t, const double* luts, int nx, int ny,
                             const int32_t* atom_sx, const int32_t* atom_sy,
                             const int32_t* atom_species, int n_atoms,
                             cudaStream_t s, bool exponentiate = true);
// Potential by FFT convolution (the direct sum's exact equivalent):
// H[sp[k]][pix[k]] = count[k] on zeroed planes; out = sum_s H_s * lut_s in
// k-space; t = e^{-Im v} (cos Re v, sin Re v) with v = t * scale.
cudaError_t launch_histogram_scatter(double* h, const int32_t* pix, const int32_t* sp,
                                     const double* count, int n, int64_t plane, cudaStream_t s);
cudaError_t launch_histogram_lut(double* out, const double* h, const double* lut_k,
                                 int n_species, int64_t plane, cudaStream_t s);
cudaError_t launch_transmission_exp(double* t, int64_t n, double scale, cudaStream_t s);
// Probe in k-space before the inverse transform (probe_wavefunction.cpp).
cudaError_t launch_probe_synth(double* out, const double* kx, const double* ky,
                               int nx, int ny, int corrected, double cs3,
                               double cs5, double defocus, double lambda,
                               double lambda_sq, double alpha_max_sq, double x0,
                               double y0, cudaStream_t s);
// out[0] = sum |a|^2 over n complex doubles (deterministic, one block).
cudaError_t launch_norm2(const double* a, int64_t n, double* out, cudaStream_t s);
// a *= s (n complex doubles); s read from device memory when dev_scale.
cudaError_t launch_scale(double* a, int64_t n, double s, const double* dev_rsqrt_of,
                         cudaStream_t st);
cudaError_t launch_to_f32(const double* in, float* out, int64_t n_real,
                          cudaStream_t s);

// ---- detection / FEM reductions on a batch of k-space waves ----
// Pixel segments (FEM ring bins, then the ADF annulus), each cut into chunks
// of at most kSegmentChunk pixels so that a large segment is summed by many
// CTAs; the chunk sums are then added in chunk order (deterministic).
constexpr int kSegmentChunk = 2048;
struct SegmentPlan {
  const int32_t* idx = nullptr;          // pixel lists of all segments, concatenated
  const int32_t* chunk_begin = nullptr;  // [n_chunks + 1] offsets into idx
  const int32_t* seg_chunk = nullptr;    // [ng + 1] first chunk of each segment
  int n_chunks = 0, ng = 0;
  double* partial = nullptr;             // scratch, 2 * nb * n_chunks doubles
};
// For every (probe b, segment g): amp[b*ng+g] = sum |psi|, inten[...] =
// sum |psi|^2 over the segment's pixels, FP64 (two launches).
cudaError_t launch_segment_sums(bool fp64, const void* psi, int64_t batch_stride,
                                int nb, const SegmentPlan& sp, double* amp, double* inten,
                                const SplitK& sk, cudaStream_t s);
// Detection of the slots that finished their last slice in a slot batch.
struct DetectSlot {
  const float2* psi = nullptr;         // the slot's exit wave (scattered, k-space)
  const double* psi0k = nullptr;       // the raster's vacuum exit wave
  const int32_t* idx = nullptr;        // the raster's segment plan
  const int32_t* chunk_begin = nullptr;
  const int32_t* seg_chunk = nullptr;
  double* amp = nullptr;               // this probe's row of the raster's sums
  double* inten = nullptr;
  double* acc_a = nullptr;             // the raster's pixel sums, or nullptr
  double* acc_i = nullptr;
  int32_t n_chunks = 0, ng = 0;
  int32_t sx = 0, sy = 0;
  int32_t chunk_offset = 0;            // sum of n_chunks over earlier entries
  int32_t pad = 0;
};
// Table the host writes per slot-batch step: `n_done` entries of `done`, in
// (raster, probe) order so pixel sums add probes in raster order.
struct DetectTable {
  int32_t n_done = 0;
  int32_t total_chunks = 0;
  int32_t any_pixel = 0;               // some entry has pixel sums
  int32_t pad = 0;
};
// Segment sums and pixel accumulation of the finished slots; `table` points
// at a DetectTable followed by its DetectSlot entries (device memory), and
// `partial` holds 2 * max_done * max_chunks doubles.  Fixed grids: the
// launches can be captured once and replayed with new table contents.
cudaError_t launch_slot_detect(const void* table, int max_done, int max_chunks, int nx, int ny,
                               double* partial, bool pixel_sums, cudaStream_t s);

// ---- plain per-pass path (FP64, one probe, one kernel per reference step)
cudaError_t launch_place_probe(double* psi, const double* probe, int nx, int ny, int sx, int sy,
                               cudaStream_t s);
cudaError_t launch_transmit(double* psi, const double* t, int64_t n, double inv_s,
                            cudaStream_t s);
cudaError_t launch_bw_limit(double* psi, const int32_t* lo, const int32_t* hi, int nx, int ny,
                            cudaStream_t s, int nb = 1);
cudaError_t launch_propagate(double* psi, const double* px, const double* py, const int32_t* lo,
                             const int32_t* hi, int nx, int ny, cudaStream_t s);

// ---- detector MTF (adfstem.cpp:2272-2385), FP64 planes ------------------
// out[b] = |psi_b(k)| (exit wave incl. the vacuum part of split-wave runs)
// where lambda^2 k^2 > alpha_max^2, else 0; imaginary parts 0.
cudaError_t launch_mtf_magnitude(bool fp64, const void* psi, int64_t stride, int nb,
                                 const double* kx, const double* ky, double lambda_sq,
                                 double amax_sq, const SplitK& sk, double* out, cudaStream_t s);
// psi_b <- psi_b * mtf / s (reference update order), nb planes.
cudaError_t launch_mtf_multiply(double* psi, const double* mtf, int64_t plane, int nb,
                                double inv_s, cudaStream_t s);

// out[p] = sum over r < world of in[r * n + p], added in rank order (FP64):
// the pixel sums of a sharded raster, the same bits on every rank.
cudaError_t launch_rank_sum(const double* in, int world, int64_t n, double* out,
                            cudaStream_t s);
// acc_a[p] += sum_b |psi_b[p]|, acc_i[p] += sum_b |psi_b[p]|^2 (FP64).
cudaError_t launch_pixel_accum(bool fp64, const void* psi, int64_t batch_stride,
                               int nb, int64_t npix, double* acc_a, double* acc_i,
                               const SplitK& sk, cudaStream_t s);
// out = (float)(in - 1) for the real parts, (float)in for the imaginary
// parts of n complex doubles: tau = t - 1 for split-wave passes.
cudaError_t launch_to_f32_minus_one(const double* in, float* out, int64_t n_complex,
                                    cudaStream_t s);
// MD-coupled FEM: acc_b += psi_b / divisor for nb planes [b][plane] (FP64
// acc), psi the exit wave in k-space incl. the vacuum part of split-wave
// runs (sk), batch stride `stride` elements.
cudaError_t launch_wave_accumulate(bool fp64, const void* psi, int64_t stride, int nb,
                                   int64_t plane, const SplitK& sk, double divisor, double* acc,
                                   cudaStream_t s);
// dst[i * dst_stride] += src[i * src_stride] / divisor, i < n.
cudaError_t launch_strided_accumulate(double* dst, int64_t dst_stride, const double* src,
                                      int64_t src_stride, int n, double divisor, cudaStream_t s);
// psi (complex) = delta (FP32, k-space) + shifted vacuum part (FP64), for
// one probe: used to return the exit wave of a split-wave run.
cudaError_t launch_assemble_split(const float* delta, const double* psi0k, int nx, int ny,
                                  int sx, int sy, double* out, cudaStream_t s);

}  // namespace msf
