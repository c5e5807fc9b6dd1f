// sm_100a kernels of the multislice path.
//
// Wavefield layout in HBM: [probe][x][y] complex (float2 / double2), y
// fastest, as the reference's fftw_complex psi[j + i*Ny] (adfstem.cpp:1665)
// with one contiguous nx*ny plane per probe of the batch.
//
// Per slice the two fused passes are
//   row pass    (contiguous, along y):  iDFT_y, t * psi / s (quirk kept),
//                                       DFT_y                  [ROW_SLICE]
//   column pass (strided,   along x):   DFT_x, / s, band-limit mask,
//                                       propagator, iDFT_x     [COL_SLICE]
// which together equal the reference's iFFT2 -> *t -> FFT2 -> bw_limit ->
// propagate (adfstem.cpp:1891-2048).  The first slice's row pass reads the
// shifted probe directly (ROW_SLICE_FIRST, adfstem.cpp:1632-1837) and the
// last slice's column pass stops in k-space for detection (COL_SLICE_LAST).
#include "kernels.h"
#include "fft_core.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace msf {

namespace {

constexpr double kRefPi = 3.14159265369;  // the reference's PI (adfstem.hpp:55)
constexpr int kSmemBudget = 220 * 1024;

// FP64 row passes: CTAs of 64 threads, four to an SM at up to 255
// registers, so their load and transform phases run out of step (measured
// 17 % faster at 1024^2 and 9 % at 2048^2 than one 256-thread CTA per SM).
#ifndef MSF_ROW_THREADS
#define MSF_ROW_THREADS 64
#endif
// FP32 row passes hold 32 complex values per thread (one CTA of 256 threads
// fills the register file): CTAs of 64 threads let four of them share an SM
// with their load and transform phases out of step.
#ifndef MSF_ROW_THREADS_F32
#define MSF_ROW_THREADS_F32 64
#endif
#ifndef MSF_COL_THREADS
#define MSF_COL_THREADS 256
#endif

// Threads of an FP32 pass that share an SM: 384 (at most 168 registers a
// thread, no spills) up to 1024-point lines, measured 3.6 % faster for the
// 1024^2 row pass than 256; 256 for 2048-point lines, whose transforms
// spill below 255 registers.
#ifndef MSF_THREADS_PER_SM
#define MSF_THREADS_PER_SM 384
#endif
#ifndef MSF_THREADS_PER_SM_LONG
#define MSF_THREADS_PER_SM_LONG 256
#endif
// Resident CTAs per SM the register allocator must allow, so that at least
// that many threads of a pass share an SM.
// FP64 passes: at least this many threads per SM (256: up to 255
// registers a thread, which their transforms need without spills).
#ifndef MSF_THREADS_PER_SM_F64
#define MSF_THREADS_PER_SM_F64 256
#endif
// FP32 row passes on the alternative FFT schedule (16 or 8 elements a
// thread): 512 threads per SM (at most 128 registers; 640 spilled heavily).
#ifndef MSF_THREADS_PER_SM_ALT
#define MSF_THREADS_PER_SM_ALT 512
#endif
constexpr int min_blocks(int real_bytes, int threads, int n, int schedule = 0) {
  if (real_bytes == 8)
    return MSF_THREADS_PER_SM_F64 > threads ? MSF_THREADS_PER_SM_F64 / threads : 1;
  const int want = schedule == 1 ? MSF_THREADS_PER_SM_ALT
                   : n >= 2048   ? MSF_THREADS_PER_SM_LONG
                                 : MSF_THREADS_PER_SM;
  return threads >= want ? 1 : want / threads;
}

// Lines (rows) per CTA of a row pass: about MSF_ROW_THREADS (FP64) or
// MSF_ROW_THREADS_F32 threads, small CTAs so that several reside per SM and
// their load / FFT / store phases overlap.
template <typename Real, int N, int V = 0>
constexpr int row_lines() {
  using Sh = Shape<N, Real, V>;
  constexpr int bytes = (Sh::N + (Sh::N >> ilog2(Sh::R0)) + 16) * (int)sizeof(Cx<Real>);
  int l = (sizeof(Real) == 4 ? MSF_ROW_THREADS_F32 : MSF_ROW_THREADS) / Sh::T;
  if (l < 1) l = 1;
  while (l > 1 && l * bytes > kSmemBudget) l >>= 1;
  return l;
}

// Columns per CTA of a column pass: as many as fit MSF_COL_THREADS threads
// (16 FP32 / 8 FP64 columns give 128-byte row segments).
template <typename Real, int N>
constexpr int col_cols() {
  using Sh = Shape<N, Real>;
  constexpr int bytes = (Sh::N + (Sh::N >> ilog2(Sh::R0)) + 16) * (int)sizeof(Cx<Real>);
  int c = sizeof(Real) == 4 ? 16 : 8;
  while (c > 1 && (c * bytes > kSmemBudget || c * Sh::T > MSF_COL_THREADS)) c >>= 1;
  return c;
}

// ------------------------------------------------------------ row pass ---
// A load that does not allocate in L1 (the wavefield is read once a pass),
// and a prefetch of one 128-byte line into L1.
template <typename C>
__device__ __forceinline__ C ld_stream(const C* p) {
  if constexpr (sizeof(C) == 8) {
    float2 v;
    asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
  } else {
    return *p;
  }
}
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// PassArgs::l2_ahead: the first LINES threads of the CTA each issue bulk L2
// prefetches of one wavefield row of the CTA a.l2_ahead places later in
// launch order (grid (nb, nx / LINES), or (nb / LINES, nx) with the lines
// by probe; x fastest).  Addresses and
// sizes are multiples of 16 bytes: rows start at multiples of N complex
// values and the ranges have even bounds.
template <typename C, int N, int LINES>
__device__ __forceinline__ void prefetch_rows_ahead(const PassArgs& a, bool by_probe) {
  if (threadIdx.x >= LINES) return;
  const int64_t lin = (int64_t)blockIdx.y * gridDim.x + blockIdx.x + a.l2_ahead;
  if (lin >= (int64_t)gridDim.x * gridDim.y) return;
  const int bx = (int)(lin % gridDim.x), by = (int)(lin / gridDim.x);
  const int b = by_probe ? bx * LINES + (int)threadIdx.x : bx;
  const int i = by_probe ? by : by * LINES + (int)threadIdx.x;
  const C* row = static_cast<const C*>(a.psi) + (int64_t)b * a.batch_stride + (int64_t)i * N;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int lo = a.ahead_range[2 * r], hi = a.ahead_range[2 * r + 1];
    if (hi > lo)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                   ::"l"(row + lo), "r"((hi - lo) * (int)sizeof(C))
                   : "memory");
  }
}

// Split-wave transmission step (split_elem) on one row held in registers
// (element t + T*m of row i); psi0 is the probe's vacuum wave, shifted like
// the probe.
template <typename Sh, typename C, typename Real>
__device__ __forceinline__ void split_update(C (&v)[Sh::E], const C* __restrict__ psi0,
                                             const C* __restrict__ trans, int nx, int i,
                                             int t, int sx, int sy, Real is) {
  constexpr int N = Sh::N, E = Sh::E, T = Sh::T;
  const int ix = (i < sx) ? i + nx - sx : i - sx;
  const C* prow = psi0 + (int64_t)ix * N;
  const C* trow = trans + (int64_t)i * N;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    if (m % kLoadChunk == 0) load_fence();
    const int y = t + T * m;
    const int iy = (y < sy) ? y + N - sy : y - sy;
    const C p0 = __ldg(prow + iy);
    const C tau = __ldg(trow + y);
    v[m] = split_elem(p0, tau, v[m], is);
  }
}

template <typename Real, int N, int LINES, int OP, int V = 0>
__global__ void __launch_bounds__(LINES * Shape<N, Real, V>::T,
                                  min_blocks((int)sizeof(Real), LINES * Shape<N, Real, V>::T, N,
                                             V))
row_kernel(const PassArgs a) {
  using C = Cx<Real>;
  using Sh = Shape<N, Real, V>;
  using SM = Smem<Sh, (int)sizeof(Cx<Real>), LINES, false>;
  constexpr int E = Sh::E, T = Sh::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* smem = reinterpret_cast<C*>(smem_raw);
  const int line = threadIdx.x / T;
  const int t = threadIdx.x % T;
  // lines of a CTA: consecutive rows of probe blockIdx.x, or row blockIdx.y
  // of consecutive probes (PassArgs::lines_by_probe)
  const bool by_probe = OP == ROW_SPLIT && a.lines_by_probe;
  const int b = by_probe ? (int)blockIdx.x * LINES + line : (int)blockIdx.x;
  const int i = by_probe ? (int)blockIdx.y : (int)blockIdx.y * LINES + line;
  C* sm = smem + line * SM::stride;
  C* row = static_cast<C*>(a.psi) + (int64_t)b * a.batch_stride + (int64_t)i * N;
  const C* tw = static_cast<const C*>(a.tw);
  auto sync = [] {
    if constexpr (T <= 32) __syncwarp();
    else __syncthreads();
  };
  C v[E];
  if constexpr (OP == ROW_SLOTS) {
    // slot batch: this CTA's probe reads its own slice tables.  The row
    // loads wait for the slot entry, so a CTA takes nx / (LINES * gridDim.y)
    // consecutive row groups of its slot and pays that wait once.
    // The entry is staged in shared memory and its fields re-read where
    // they are used (volatile), instead of living in registers across the
    // transforms, where they pushed the 512- and 1024-point passes into
    // spills (the plain passes read the same values from kernel parameters).
    __shared__ SlotPass sp_smem;
    if (threadIdx.x == 0) sp_smem = a.slots[b];
    __syncthreads();
    const volatile SlotPass& sp = sp_smem;
    if (sp.op == SLOT_IDLE) return;
    // columns the band limit removes entirely (when the lane skips them):
    // never loaded, stored (as zeros) only at the slot's last slice
    const uint32_t dead = a.row_dead_bits ? __ldg(a.row_dead_bits + t) : 0u;
    const int groups = a.nx / (LINES * (int)gridDim.y);
    for (int r = 0; r < groups; ++r) {
      const int ir = ((int)blockIdx.y * groups + r) * LINES + line;
      C* rrow = static_cast<C*>(a.psi) + (int64_t)b * a.batch_stride + (int64_t)ir * N;
      if (sp.op == SLOT_FIRST) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = C{(Real)0, (Real)0};
      } else {
#pragma unroll
        for (int m = 0; m < E; ++m)
          v[m] = ((dead >> m) & 1u) ? C{(Real)0, (Real)0}
                 : a.prefetch_tables ? ld_stream(rrow + t + T * m)
                                     : rrow[t + T * m];
      }
      if (a.prefetch_tables) {  // this row's tables into L1 during the inverse FFT
        constexpr int kLines = N * (int)sizeof(C) / 128;
        const int ix = (ir < sp.sx) ? ir + a.nx - sp.sx : ir - sp.sx;
        const char* trow = static_cast<const char*>(sp.trans) + (int64_t)ir * N * sizeof(C);
        const char* prow = static_cast<const char*>(sp.psi0) + (int64_t)ix * N * sizeof(C);
        for (int l = t; l < kLines; l += T) {
          prefetch_l1(trow + 128 * l);
          prefetch_l1(prow + 128 * l);
        }
      }
      if (sp.op != SLOT_FIRST) fft_line<Sh, true>(v, sm, t, tw, sync);
      split_update<Sh>(v, static_cast<const C*>(sp.psi0), static_cast<const C*>(sp.trans),
                       a.nx, ir, t, sp.sx, sp.sy, (Real)a.inv_s);
      fft_line<Sh, false>(v, sm, t, tw, sync);
      const bool last = sp.last != 0;
      // the removed-column bits again (an L1 hit) rather than a register
      // held across both transforms
      const uint32_t dead_st = a.row_dead_bits ? __ldg(a.row_dead_bits + t) : 0u;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        if (!((dead_st >> m) & 1u))
          rrow[t + T * m] = v[m];
        else if (last)
          rrow[t + T * m] = C{(Real)0, (Real)0};
      }
    }
    return;
  }
  if constexpr (OP == ROW_SLICE_FIRST) {
    const int sx = a.shifts[2 * b], sy = a.shifts[2 * b + 1];
    const int ix = (i < sx) ? i + a.nx - sx : i - sx;
    const C* prow = static_cast<const C*>(a.probe) + (int64_t)ix * N;
    const Real fs = (Real)a.first_scale;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int y = t + T * m;
      const int iy = (y < sy) ? y + N - sy : y - sy;
      v[m] = cscale(__ldg(prow + iy), fs);
    }
  } else if constexpr (OP == ROW_SPLIT_FIRST) {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = C{(Real)0, (Real)0};
  } else if constexpr (OP == ROW_SPLIT || OP == ROW_SLICE) {
    // columns removed by the band limit were not stored: they are zero
    const uint32_t skip = (a.row_dead_bits && (a.row_dead_io & 1)) ? __ldg(a.row_dead_bits + t)
                                                                  : 0u;
    if (OP == ROW_SPLIT && a.l2_ahead > 0)
      prefetch_rows_ahead<C, N, LINES>(a, by_probe);
    if (OP == ROW_SPLIT && a.prefetch_tables) {
#pragma unroll
      for (int m = 0; m < E; ++m)
        v[m] = ((skip >> m) & 1u) ? C{(Real)0, (Real)0} : ld_stream(row + t + T * m);
      // the line's tau row and (shifted) vacuum row: 128-byte lines spread
      // over the line's threads, issued after the wavefield loads
      constexpr int kLines = N * (int)sizeof(C) / 128;
      const int sx = a.shifts[2 * b];
      const int ix = (i < sx) ? i + a.nx - sx : i - sx;
      const char* trow = static_cast<const char*>(a.trans) + (int64_t)i * N * sizeof(C);
      const char* prow = static_cast<const char*>(a.psi0) + (int64_t)ix * N * sizeof(C);
      for (int l = t; l < kLines; l += T) {
        prefetch_l1(trow + 128 * l);
        prefetch_l1(prow + 128 * l);
      }
    } else {
#pragma unroll
      for (int m = 0; m < E; ++m)
        v[m] = ((skip >> m) & 1u) ? C{(Real)0, (Real)0} : row[t + T * m];
    }
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = row[t + T * m];
  }
  if constexpr (OP == ROW_SPLIT || OP == ROW_SPLIT_FIRST) {
    if constexpr (OP == ROW_SPLIT) fft_line<Sh, true>(v, sm, t, tw, sync);
    split_update<Sh>(v, static_cast<const C*>(a.psi0), static_cast<const C*>(a.trans), a.nx, i,
                     t, a.shifts[2 * b], a.shifts[2 * b + 1], (Real)a.inv_s);
    fft_line<Sh, false>(v, sm, t, tw, sync);
  } else if constexpr (OP == ROW_FWD) {
    fft_line<Sh, false>(v, sm, t, tw, sync);
  } else if constexpr (OP == ROW_INV) {
    fft_line<Sh, true>(v, sm, t, tw, sync);
    const Real s = (Real)a.scale;
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = cscale(v[m], s);
  } else {
    if constexpr (OP == ROW_SLICE) fft_line<Sh, true>(v, sm, t, tw, sync);
    // transmission multiply with the reference's in-place update order
    // (adfstem.cpp:1929-1949): the new real part feeds the imaginary part.
    const C* trow = static_cast<const C*>(a.trans) + (int64_t)i * N;
    const Real is = (Real)a.inv_s;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      if (m % kLoadChunk == 0) load_fence();
      const C tv = __ldg(trow + t + T * m);
      const Real re = (tv.x * v[m].x - tv.y * v[m].y) * is;
      const Real im = (tv.x * v[m].y + tv.y * re) * is;
      v[m] = C{re, im};
    }
    fft_line<Sh, false>(v, sm, t, tw, sync);
  }
  if constexpr (OP == ROW_SLICE || OP == ROW_SLICE_FIRST || OP == ROW_SPLIT ||
                OP == ROW_SPLIT_FIRST) {
    if (a.row_dead_bits) {  // columns the next band limit removes entirely
      const uint32_t dead = __ldg(a.row_dead_bits + t);
      if (a.row_dead_io & 2) {  // nobody reads them: leave them unstored
#pragma unroll
        for (int m = 0; m < E; ++m)
          if (!((dead >> m) & 1u)) row[t + T * m] = v[m];
        return;
      }
#pragma unroll
      for (int m = 0; m < E; ++m)
        if ((dead >> m) & 1u) v[m] = C{(Real)0, (Real)0};
    }
  }
#pragma unroll
  for (int m = 0; m < E; ++m) row[t + T * m] = v[m];
}

// --------------------------------------------------------- column pass ---
template <typename Real, int N, int COLS, int OP>
__global__ void __launch_bounds__(COLS * Shape<N, Real>::T,
                                  min_blocks((int)sizeof(Real), COLS * Shape<N, Real>::T, N))
col_kernel(const PassArgs a) {
  using C = Cx<Real>;
  using Sh = Shape<N, Real>;
  using SM = Smem<Sh, (int)sizeof(Cx<Real>), COLS, true>;
  constexpr int E = Sh::E, T = Sh::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* smem = reinterpret_cast<C*>(smem_raw);
  const int c = threadIdx.x % COLS;
  const int t = threadIdx.x / COLS;
  const int b = blockIdx.x;
  const int j = blockIdx.y * COLS + c;
  const int64_t ny = a.ny;
  C* col = static_cast<C*>(a.psi) + (int64_t)b * a.batch_stride + j;
  C* sm = smem + c * SM::stride;
  const C* tw = static_cast<const C*>(a.tw);
  auto sync = [] { __syncthreads(); };
  // slot batch: this CTA's probe brings its own mask, propagator and step
  const int32_t* mask_lo = a.mask_lo;
  const int32_t* mask_hi = a.mask_hi;
  const void* px_v = a.px;
  const void* py_v = a.py;
  [[maybe_unused]] bool stop_in_k = OP == COL_SLICE_LAST;
  if constexpr (OP == COL_SLOTS) {
    const SlotPass& sp = a.slots[b];
    if (sp.op == SLOT_IDLE) return;
    mask_lo = sp.mask_lo;
    mask_hi = sp.mask_hi;
    px_v = sp.px;
    py_v = sp.py;
    stop_in_k = sp.last != 0;
  }
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = col[(int64_t)(t + T * m) * ny];
  if constexpr (OP == COL_INV) {
    fft_line<Sh, true>(v, sm, t, tw, sync);
    const Real s = (Real)a.scale;
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = cscale(v[m], s);
  } else {
    fft_line<Sh, false>(v, sm, t, tw, sync);
    if constexpr (OP != COL_FWD) {
      const int lo = __ldg(mask_lo + j), hi = __ldg(mask_hi + j);
      if constexpr (OP == COL_FWD_MASK_INV) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
          const int i = t + T * m;
          if (!(i < lo || i >= hi)) v[m] = C{(Real)0, (Real)0};
        }
      } else {
        const Real is = (Real)a.inv_s;
        const C pyj = __ldg(static_cast<const C*>(py_v) + j);
        const C* px = static_cast<const C*>(px_v);
#pragma unroll
        for (int m = 0; m < E; ++m) {
          if (m % kLoadChunk == 0) load_fence();
          const int i = t + T * m;
          if (i < lo || i >= hi) {
            const C p = cmul(__ldg(px + i), pyj);  // slice.cpp:1396-1412
            v[m] = cmul(p, cscale(v[m], is));
          } else {
            v[m] = C{(Real)0, (Real)0};
          }
        }
      }
      if constexpr (OP == COL_FWD_MASK_INV || OP == COL_SLICE)
        fft_line<Sh, true>(v, sm, t, tw, sync);
      if constexpr (OP == COL_SLOTS)
        if (!stop_in_k) fft_line<Sh, true>(v, sm, t, tw, sync);
    }
  }
#pragma unroll
  for (int m = 0; m < E; ++m) col[(int64_t)(t + T * m) * ny] = v[m];
}

template <typename Real, int N, int OP, int V = 0>
cudaError_t row_launch(const PassArgs& a, cudaStream_t s) {
  constexpr int L = row_lines<Real, N, V>();
  using Sh = Shape<N, Real, V>;
  constexpr int smem = L * Smem<Sh, (int)sizeof(Cx<Real>), L, false>::stride * (int)sizeof(Cx<Real>);
  static PerDevice configured;
  auto k = row_kernel<Real, N, L, OP, V>;
  if (cudaError_t e = smem_limit_once((const void*)k, smem, configured); e != cudaSuccess)
    return e;
  if (a.nx % L != 0) return cudaErrorInvalidValue;
  int groups = a.nx / L;
  if constexpr (OP == ROW_SLOTS) {
    // up to 4 row groups per CTA while a slot keeps 256 CTAs
    int per = 1;
    while (per < 4 && groups % (2 * per) == 0 && groups / (2 * per) >= 256) per *= 2;
    groups /= per;
  }
  if (OP == ROW_SPLIT && a.lines_by_probe) {
    if (a.nb % L == 0) {
      k<<<dim3(a.nb / L, a.nx), L * Sh::T, smem, s>>>(a);
      return cudaGetLastError();
    }
    PassArgs rows = a;  // a batch the lines do not divide: rows of one probe
    rows.lines_by_probe = 0;
    k<<<dim3(a.nb, groups), L * Sh::T, smem, s>>>(rows);
    return cudaGetLastError();
  }
  dim3 grid(a.nb, groups);
  k<<<grid, L * Sh::T, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename Real, int N, int OP>
cudaError_t col_launch(const PassArgs& a, cudaStream_t s) {
  constexpr int CC = col_cols<Real, N>();
  using Sh = Shape<N, Real>;
  constexpr int smem = CC * Smem<Sh, (int)sizeof(Cx<Real>), CC, true>::stride * (int)sizeof(Cx<Real>);
  static PerDevice configured;
  auto k = col_kernel<Real, N, CC, OP>;
  if (cudaError_t e = smem_limit_once((const void*)k, smem, configured); e != cudaSuccess)
    return e;
  if (a.ny % CC != 0) return cudaErrorInvalidValue;
  dim3 grid(a.nb, a.ny / CC);
  k<<<grid, CC * Sh::T, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename Real, int OP>
cudaError_t row_dispatch(const PassArgs& a, cudaStream_t s) {
  switch (a.ny) {
    case 64: return row_launch<Real, 64, OP>(a, s);
    case 128: return row_launch<Real, 128, OP>(a, s);
    case 256: return row_launch<Real, 256, OP>(a, s);
    case 512: return row_launch<Real, 512, OP>(a, s);
    case 1024: return row_launch<Real, 1024, OP>(a, s);
    case 2048: return row_launch<Real, 2048, OP>(a, s);
    case 4096: return row_launch<Real, 4096, OP>(a, s);
  }
  return cudaErrorInvalidValue;
}

template <typename Real, int OP>
cudaError_t col_dispatch(const PassArgs& a, cudaStream_t s) {
  switch (a.nx) {
    case 64: return col_launch<Real, 64, OP>(a, s);
    case 128: return col_launch<Real, 128, OP>(a, s);
    case 256: return col_launch<Real, 256, OP>(a, s);
    case 512: return col_launch<Real, 512, OP>(a, s);
    case 1024: return col_launch<Real, 1024, OP>(a, s);
    case 2048: return col_launch<Real, 2048, OP>(a, s);
    case 4096: return col_launch<Real, 4096, OP>(a, s);
  }
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------ set-up kernels ---
__device__ __forceinline__ double ksq_exact(double kx, double ky) {
  // pow(kx,2) + pow(ky,2) / kx*kx + ky*ky without contraction
  return __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
}

__global__ void lut_synth_kernel(double2* out, const double* __restrict__ kx,
                                 const double* __restrict__ ky, int nx, int ny,
                                 const double* __restrict__ p, double pref,
                                 double cutoff_sq, double xmin, double ymin) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nx * ny) return;
  const int i = (int)(idx / ny), j = (int)(idx % ny);
  const double kxi = kx[i], kyj = ky[j];
  const double ksq = ksq_exact(kxi, kyj);
  double2 r = make_double2(0.0, 0.0);
  if (ksq < cutoff_sq) {
    // f_ej_single_scatterer (projected_atomic_potential.cpp:209-220)
    const double f = p[0] / (ksq + p[3]) + p[1] / (ksq + p[4]) + p[2] / (ksq + p[5]) +
                     p[6] * exp(-p[9] * ksq) + p[7] * exp(-p[10] * ksq) +
                     p[8] * exp(-p[11] * ksq);
    const double trig = 2 * kRefPi * (kxi * xmin + kyj * ymin);
    double sn, cs;
    sincos(trig, &sn, &cs);
    r.x = pref * f * cs;
    r.y = pref * f * sn;
  }
  out[idx] = r;
}

constexpr int kPotRows = 4;
constexpr int kPotChunk = 512;

// Each CTA owns a kPotRows x blockDim.x tile of the slice's potential and
// accumulates it in registers over the slice's atoms (staged in shared
// memory in chunks), in the reference's atom order so the FP64 sums equal
// slice.cpp:1594-1649 term for term.  The LUT spans the whole cell, so every
// atom contributes to every tile; no global atomics are used.
template <bool EXP>
__global__ void potential_kernel(double2* __restrict__ t, const double2* __restrict__ luts,
                                 int nx, int ny, const int32_t* __restrict__ asx,
                                 const int32_t* __restrict__ asy,
                                 const int32_t* __restrict__ asp, int n_atoms) {
  __shared__ int3 atoms[kPotChunk];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * kPotRows;
  const int64_t plane = (int64_t)nx * ny;
  double2 acc[kPotRows];
#pragma unroll
  for (int r = 0; r < kPotRows; ++r) acc[r] = make_double2(0.0, 0.0);
  for (int c0 = 0; c0 < n_atoms; c0 += kPotChunk) {
    const int cn = min(kPotChunk, n_atoms - c0);
    __syncthreads();
    for (int k = threadIdx.x; k < cn; k += blockDim.x)
      atoms[k] = make_int3(asx[c0 + k], asy[c0 + k], asp[c0 + k]);
    __syncthreads();
    if (j < ny) {
      for (int k = 0; k < cn; ++k) {
        const int3 a = atoms[k];
        const double2* lut = luts + (int64_t)a.z * plane;
        const int jy = (j < a.y) ? j + ny - a.y : j - a.y;
#pragma unroll
        for (int r = 0; r < kPotRows; ++r) {
          const int i = i0 + r;
          const int ix = (i < a.x) ? i + nx - a.x : i - a.x;
          const double2 l = __ldg(lut + (int64_t)ix * ny + jy);
          acc[r].x = __dadd_rn(acc[r].x, l.x);
          acc[r].y = __dadd_rn(acc[r].y, l.y);
        }
      }
    }
  }
  if (j < ny) {
#pragma unroll
    for (int r = 0; r < kPotRows; ++r) {
      if constexpr (EXP) {  // slice.cpp:1700-1725
        const double e = exp(-(acc[r].y));
        double sn, cs;
        sincos(acc[r].x, &sn, &cs);
        t[(int64_t)(i0 + r) * ny + j] = make_double2(e * cs, e * sn);
      } else {  // the projected potential itself (what --paptif shows)
        t[(int64_t)(i0 + r) * ny + j] = acc[r];
      }
    }
  }
}

// ---- potential by FFT convolution -------------------------------------
// The slice's sum over atoms of the LUT shifted to each atom's pixel is the
// circular convolution of the pixel histogram H with the LUT; with the LUT
// defined as BACKWARD(lut_k) / s (scatterer_pap.hpp:86-190) it equals
// BACKWARD(lut_k * FORWARD(H)) / s.
// H[sp][pix] = count for the slice's (species, pixel) pairs (unique pixels).
__global__ void histogram_scatter_kernel(double2* __restrict__ h, const int32_t* __restrict__ pix,
                                         const int32_t* __restrict__ sp,
                                         const double* __restrict__ count, int n,
                                         int64_t plane) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) h[(int64_t)sp[k] * plane + pix[k]] = make_double2(count[k], 0.0);
}

// out = sum over species of H_s * lut_s (k-space, FP64)
__global__ void histogram_lut_kernel(double2* __restrict__ out, const double2* __restrict__ h,
                                     const double2* __restrict__ lut_k, int n_species,
                                     int64_t plane) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= plane) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int s = 0; s < n_species; ++s) {
    const double2 a = h[(int64_t)s * plane + p], b = lut_k[(int64_t)s * plane + p];
    acc.x += a.x * b.x - a.y * b.y;
    acc.y += a.x * b.y + a.y * b.x;
  }
  out[p] = acc;
}

// t = e^{-Im v} (cos Re v, sin Re v) with v = t * scale (slice.cpp:1700-1725)
__global__ void transmission_exp_kernel(double2* __restrict__ t, int64_t n, double scale) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double re = t[k].x * scale, im = t[k].y * scale;
  const double e = exp(-(im));
  double sn, cs;
  sincos(re, &sn, &cs);
  t[k] = make_double2(e * cs, e * sn);
}

__global__ void probe_synth_kernel(double2* out, const double* __restrict__ kx,
                                   const double* __restrict__ ky, int nx, int ny,
                                   int corrected, double cs3, double cs5,
                                   double defocus, double lambda, double lsq,
                                   double amax_sq, double x0, double y0) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nx * ny) return;
  const int i = (int)(idx / ny), j = (int)(idx % ny);
  const double kxi = kx[i], kyj = ky[j];
  const double ksqr = ksq_exact(kxi, kyj);
  double2 r = make_double2(0.0, 0.0);
  if (__dmul_rn(lsq, ksqr) < amax_sq) {  // probe_wavefunction.cpp:100
    double chi;
    if (corrected) {  // lenses.cpp:263-290
      const double kl = ksqr * lsq;
      chi = kRefPi * lambda * ksqr * (-defocus + 0.5 * cs3 * kl + (1.0 / 3.0) * cs5 * (kl * kl));
    } else {  // lenses.cpp:249-261
      chi = kRefPi * lambda * ksqr * (0.5 * cs3 * lsq * ksqr - defocus);
    }
    const double trig = chi + 2 * kRefPi * ((kxi * x0) + (kyj * y0));
    double sn, cs;
    sincos(trig, &sn, &cs);
    r = make_double2(cs, -1.0 * sn);
  }
  out[idx] = r;
}

__global__ void norm2_kernel(const double2* __restrict__ a, int64_t n, double* out) {
  __shared__ double red[1024];
  double s = 0.0;
  for (int64_t k = threadIdx.x; k < n; k += blockDim.x) {
    const double2 v = a[k];
    s += v.x * v.x + v.y * v.y;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

__global__ void scale_kernel(double2* a, int64_t n, double s) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) a[k] = make_double2(a[k].x * s, a[k].y * s);
}

__global__ void to_f32_kernel(const double* __restrict__ in, float* __restrict__ out,
                              int64_t n) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = (float)in[k];
}

// ------------------------------------------------------- detection -------
// Value of one probe's exit wave at k-space pixel `pix`: the buffer value,
// plus (split-wave runs) the vacuum part shifted to the probe's position.
template <typename Real>
__device__ __forceinline__ double2 exit_value(const Cx<Real>* __restrict__ p, int pix,
                                              const SplitK& sk, int sx, int sy) {
  const Cx<Real> v = p[pix];
  double x = (double)v.x, y = (double)v.y;
  if (sk.psi0k) {
    const double2 z = __ldg(reinterpret_cast<const double2*>(sk.psi0k) + pix);
    if (z.x != 0.0 || z.y != 0.0) {
      const int mx = pix / sk.ny, my = pix - mx * sk.ny;
      // e^{-2 pi i (mx sx / nx + my sy / ny)} from exact integer phases
      const double f = (double)(((int64_t)mx * sx) % sk.nx) / sk.nx +
                       (double)(((int64_t)my * sy) % sk.ny) / sk.ny;
      double sn, cs;
      sincospi(-2.0 * f, &sn, &cs);
      x += z.x * cs - z.y * sn;
      y += z.x * sn + z.y * cs;
    }
  }
  return make_double2(x, y);
}

// Sum of a block's values into lane 0 of warp 0 (fixed order).
__device__ __forceinline__ void block_sum2(double& sa, double& si, double* ra, double* ri) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_down_sync(0xffffffffu, sa, o);
    si += __shfl_down_sync(0xffffffffu, si, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { ra[w] = sa; ri[w] = si; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    sa = l < nw ? ra[l] : 0.0;
    si = l < nw ? ri[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sa += __shfl_down_sync(0xffffffffu, sa, o);
      si += __shfl_down_sync(0xffffffffu, si, o);
    }
  }
}

// One chunk of one probe's segment pixels: partial_a/i[b * n_chunks + c].
template <typename Real>
__global__ void __launch_bounds__(256)
segment_chunk_kernel(const Cx<Real>* __restrict__ psi, int64_t stride,
                     const int32_t* __restrict__ idx, const int32_t* __restrict__ chunk_begin,
                     int n_chunks, double* partial_a, double* partial_i, const SplitK sk) {
  __shared__ double ra[32], ri[32];
  const int c = blockIdx.x, b = blockIdx.y;
  const Cx<Real>* p = psi + (int64_t)b * stride;
  const int sx = sk.psi0k ? sk.shifts[2 * b] : 0, sy = sk.psi0k ? sk.shifts[2 * b + 1] : 0;
  double sa = 0.0, si = 0.0;
  const int s0 = chunk_begin[c], s1 = chunk_begin[c + 1];
  for (int k = s0 + threadIdx.x; k < s1; k += blockDim.x) {
    const double2 v = exit_value<Real>(p, __ldg(idx + k), sk, sx, sy);
    const double i2 = v.x * v.x + v.y * v.y;
    si += i2;
    sa += sqrt(i2);
  }
  block_sum2(sa, si, ra, ri);
  if (threadIdx.x == 0) {
    partial_a[(int64_t)b * n_chunks + c] = sa;
    partial_i[(int64_t)b * n_chunks + c] = si;
  }
}

// Segment totals from the chunk sums, in chunk order: one CTA per probe.
__global__ void segment_reduce_kernel(const double* __restrict__ partial_a,
                                      const double* __restrict__ partial_i,
                                      const int32_t* __restrict__ seg_chunk, int ng,
                                      int n_chunks, double* amp, double* inten) {
  const int b = blockIdx.x;
  for (int g = threadIdx.x; g < ng; g += blockDim.x) {
    double sa = 0.0, si = 0.0;
    for (int c = seg_chunk[g]; c < seg_chunk[g + 1]; ++c) {
      sa += partial_a[(int64_t)b * n_chunks + c];
      si += partial_i[(int64_t)b * n_chunks + c];
    }
    if (amp) amp[(int64_t)b * ng + g] = sa;
    if (inten) inten[(int64_t)b * ng + g] = si;
  }
}

// ---- detector MTF (adfstem.cpp:2272-2385) ------------------------------
// out = |psi(k)| where lambda^2 k^2 > alpha_max^2 (the direct beam blocked),
// else 0, as a real FP64 plane per probe.
template <typename Real>
__global__ void mtf_magnitude_kernel(const Cx<Real>* __restrict__ psi, int64_t stride, int nb,
                                     const double* __restrict__ kx,
                                     const double* __restrict__ ky, double lambda_sq,
                                     double amax_sq, const SplitK sk, double2* out) {
  const int64_t plane = (int64_t)sk.nx * sk.ny;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= plane * nb) return;
  const int b = (int)(k / plane);
  const int p = (int)(k - (int64_t)b * plane);
  const int i = p / sk.ny, j = p - (p / sk.ny) * sk.ny;
  double m = 0.0;
  if (__dmul_rn(lambda_sq, ksq_exact(kx[i], ky[j])) > amax_sq) {
    const int sx = sk.psi0k ? sk.shifts[2 * b] : 0, sy = sk.psi0k ? sk.shifts[2 * b + 1] : 0;
    const double2 v = exit_value<Real>(psi + (int64_t)b * stride, p, sk, sx, sy);
    m = sqrt(v.x * v.x + v.y * v.y);
  }
  out[k] = make_double2(m, 0.0);
}

// psi <- psi * mtf / s with the reference's in-place update order (the new
// real part feeds the imaginary part), nb planes
__global__ void mtf_multiply_kernel(double2* __restrict__ psi, const double2* __restrict__ mtf,
                                    int64_t plane, int nb, double inv_s) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= plane * nb) return;
  const double2 v = psi[k], m = mtf[k % plane];
  const double re = (v.x * m.x - v.y * m.y) * inv_s;
  const double im = (re * m.y + v.y * m.x) * inv_s;
  psi[k] = make_double2(re, im);
}

// ---- slot batches: detection of the slots that finished -------------
__device__ __forceinline__ const DetectSlot* detect_entries(const void* table) {
  return reinterpret_cast<const DetectSlot*>(static_cast<const char*>(table) +
                                             sizeof(DetectTable));
}

// Work item w = one chunk of one finished slot: the entry is the last one
// whose chunk_offset <= w (entries without chunks share the next offset).
__global__ void __launch_bounds__(256)
slot_chunk_kernel(const void* table, int max_chunks, int nx, int ny, double* partial_a,
                  double* partial_i) {
  __shared__ double ra[32], ri[32];
  const DetectTable* h = static_cast<const DetectTable*>(table);
  const DetectSlot* e = detect_entries(table);
  const int n_done = h->n_done, total = h->total_chunks;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int lo = 0, hi = n_done - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (e[mid].chunk_offset <= w) lo = mid;
      else hi = mid - 1;
    }
    const DetectSlot& d = e[lo];
    const int c = w - d.chunk_offset;
    SplitK sk;
    sk.psi0k = d.psi0k;
    sk.nx = nx;
    sk.ny = ny;
    double sa = 0.0, si = 0.0;
    const int s0 = d.chunk_begin[c], s1 = d.chunk_begin[c + 1];
    for (int k = s0 + threadIdx.x; k < s1; k += blockDim.x) {
      const double2 v = exit_value<float>(d.psi, __ldg(d.idx + k), sk, d.sx, d.sy);
      const double i2 = v.x * v.x + v.y * v.y;
      si += i2;
      sa += sqrt(i2);
    }
    block_sum2(sa, si, ra, ri);
    if (threadIdx.x == 0) {
      partial_a[(int64_t)lo * max_chunks + c] = sa;
      partial_i[(int64_t)lo * max_chunks + c] = si;
    }
    __syncthreads();  // ra / ri are reused by the next work item
  }
}

// Segment totals of each finished slot, chunk sums added in chunk order.
__global__ void slot_reduce_kernel(const void* table, int max_chunks,
                                   const double* __restrict__ partial_a,
                                   const double* __restrict__ partial_i) {
  const DetectTable* h = static_cast<const DetectTable*>(table);
  const DetectSlot* e = detect_entries(table);
  for (int d = blockIdx.x; d < h->n_done; d += gridDim.x) {
    const DetectSlot& x = e[d];
    for (int g = threadIdx.x; g < x.ng; g += blockDim.x) {
      double sa = 0.0, si = 0.0;
      for (int c = x.seg_chunk[g]; c < x.seg_chunk[g + 1]; ++c) {
        sa += partial_a[(int64_t)d * max_chunks + c];
        si += partial_i[(int64_t)d * max_chunks + c];
      }
      x.amp[g] = sa;
      x.inten[g] = si;
    }
  }
}

// Pixel sums over the finished slots, entries in table order (probes of a
// raster in raster order), each pixel owned by one thread.
__global__ void slot_pixel_kernel(const void* table, int nx, int ny) {
  const DetectTable* h = static_cast<const DetectTable*>(table);
  const DetectSlot* e = detect_entries(table);
  const int n_done = h->any_pixel ? h->n_done : 0;
  const int64_t npix = (int64_t)nx * ny;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix && n_done > 0;
       p += (int64_t)gridDim.x * blockDim.x) {
    for (int d = 0; d < n_done; ++d) {
      const DetectSlot& x = e[d];
      if (!x.acc_a) continue;
      SplitK sk;
      sk.psi0k = x.psi0k;
      sk.nx = nx;
      sk.ny = ny;
      const double2 v = exit_value<float>(x.psi, (int)p, sk, x.sx, x.sy);
      const double i2 = v.x * v.x + v.y * v.y;
      x.acc_a[p] += sqrt(i2);
      x.acc_i[p] += i2;
    }
  }
}

template <typename Real>
__global__ void pixel_accum_kernel(const Cx<Real>* __restrict__ psi, int64_t stride,
                                   int nb, int64_t npix, double* acc_a, double* acc_i,
                                   const SplitK sk) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  double sa = acc_a[p], si = acc_i[p];
  for (int b = 0; b < nb; ++b) {
    const int sx = sk.psi0k ? sk.shifts[2 * b] : 0, sy = sk.psi0k ? sk.shifts[2 * b + 1] : 0;
    const double2 v = exit_value<Real>(psi + (int64_t)b * stride, (int)p, sk, sx, sy);
    const double x = v.x, y = v.y;
    const double i2 = x * x + y * y;
    sa += sqrt(i2);
    si += i2;
  }
  acc_a[p] = sa;
  acc_i[p] = si;
}

__global__ void to_f32_minus_one_kernel(const double2* __restrict__ in, float2* __restrict__ out,
                                        int64_t n) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = make_float2((float)(in[k].x - 1.0), (float)in[k].y);
}

// ---- MD-coupled FEM (ftem_lammps.cpp:3601-3610): the coherent average of
// each probe's exit wave over the specimen samples.  acc_b[p] += psi_b[p] /
// samples for nb planes, psi the exit wave in k-space including the vacuum
// part of split-wave runs; FP64.
template <typename Real>
__global__ void wave_accumulate_kernel(const Cx<Real>* __restrict__ psi, int64_t stride, int nb,
                                       int64_t plane, const SplitK sk, double divisor,
                                       double2* __restrict__ acc) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= plane * nb) return;
  const int b = (int)(k / plane);
  const int p = (int)(k - (int64_t)b * plane);
  const int sx = sk.psi0k ? sk.shifts[2 * b] : 0, sy = sk.psi0k ? sk.shifts[2 * b + 1] : 0;
  const double2 v = exit_value<Real>(psi + (int64_t)b * stride, p, sk, sx, sy);
  double2 a = acc[k];
  a.x += v.x / divisor;
  a.y += v.y / divisor;
  acc[k] = a;
}

// dst[i * dst_stride] += src[i * src_stride] / divisor, i < n
__global__ void strided_accumulate_kernel(double* __restrict__ dst, int64_t dst_stride,
                                          const double* __restrict__ src, int64_t src_stride,
                                          int n, double divisor) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[(int64_t)i * dst_stride] += src[(int64_t)i * src_stride] / divisor;
}

__global__ void assemble_split_kernel(const float2* __restrict__ delta, SplitK sk,
                                      int32_t sx, int32_t sy, double2* out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (int64_t)sk.nx * sk.ny) return;
  out[p] = exit_value<float>(delta, (int)p, sk, sx, sy);
}

// ---- plain per-pass path (FP64, one probe): one kernel per reference step
// psi[i][j] = probe[(i - sx) mod nx][(j - sy) mod ny] (adfstem.cpp:1632-1671)
__global__ void place_probe_kernel(double2* __restrict__ psi, const double2* __restrict__ probe,
                                   int nx, int ny, int sx, int sy) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)nx * ny) return;
  const int i = (int)(k / ny), j = (int)(k - (int64_t)i * ny);
  const int ii = i < sx ? i + nx - sx : i - sx;
  const int jj = j < sy ? j + ny - sy : j - sy;
  psi[k] = probe[(int64_t)ii * ny + jj];
}

// psi <- t * psi / s with the reference's in-place update order: the new
// real part feeds the imaginary part (adfstem.cpp:1929-1949)
__global__ void transmit_kernel(double2* __restrict__ psi, const double2* __restrict__ t,
                                int64_t n, double inv_s) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double2 v = psi[k], tv = t[k];
  const double re = (tv.x * v.x - tv.y * v.y) * inv_s;
  const double im = (tv.x * v.y + tv.y * re) * inv_s;
  psi[k] = make_double2(re, im);
}

// zero outside the band limit (bw_limit.cpp:30-47): column j keeps rows
// i < lo[j] and i >= hi[j]
__global__ void bw_limit_kernel(double2* __restrict__ psi, const int32_t* __restrict__ lo,
                                const int32_t* __restrict__ hi, int nx, int ny, int nb) {
  const int64_t plane = (int64_t)nx * ny;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= plane * nb) return;
  const int64_t p = k % plane;
  const int i = (int)(p / ny), j = (int)(p - (int64_t)i * ny);
  if (!(i < lo[j] || i >= hi[j])) psi[k] = make_double2(0.0, 0.0);
}

// psi(k) <- P_x(kx) P_y(ky) psi(k) inside the band limit, else 0
// (slice.cpp:1366-1421)
__global__ void propagate_kernel(double2* __restrict__ psi, const double2* __restrict__ px,
                                 const double2* __restrict__ py, const int32_t* __restrict__ lo,
                                 const int32_t* __restrict__ hi, int nx, int ny) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)nx * ny) return;
  const int i = (int)(k / ny), j = (int)(k - (int64_t)i * ny);
  if (i < lo[j] || i >= hi[j]) {
    psi[k] = cmul(cmul(px[i], py[j]), psi[k]);
  } else {
    psi[k] = make_double2(0.0, 0.0);
  }
}

inline unsigned blocks_for(int64_t n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace

// SMs of the current device (cached per device ordinal)
int sm_count() {
  static std::atomic<int> cached[64];
  const int dev = current_device();
  int n = (dev >= 0 && dev < 64) ? cached[dev].load() : 0;
  if (n <= 0) {
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev < 0 ? 0 : dev);
    if (n <= 0) n = 1;
    if (dev >= 0 && dev < 64) cached[dev].store(n);
  }
  return n;
}

namespace {
template <int N>
int row_split_resident(int dev) {
  // per device: the occupancy query does not change within a process
  static std::atomic<int> cached[64];
  int n = (dev >= 0 && dev < 64) ? cached[dev].load() : 0;
  if (n > 0) return n;
  constexpr int L = row_lines<float, N, 0>();
  using Sh = Shape<N, float, 0>;
  constexpr int smem = L * Smem<Sh, 8, L, false>::stride * 8;
  static PerDevice configured;
  auto k = row_kernel<float, N, L, ROW_SPLIT, 0>;
  int per_sm = 0;
  if (smem_limit_once((const void*)k, smem, configured) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, L * Sh::T, smem) != cudaSuccess)
    return 0;
  n = per_sm * sm_count();
  if (n > 0 && dev >= 0 && dev < 64) cached[dev].store(n);
  return n;
}
}  // namespace

int row_split_resident_ctas(int ny) {
  const int dev = current_device();
  switch (ny) {
    case 64: return row_split_resident<64>(dev);
    case 128: return row_split_resident<128>(dev);
    case 256: return row_split_resident<256>(dev);
    case 512: return row_split_resident<512>(dev);
    case 1024: return row_split_resident<1024>(dev);
    case 2048: return row_split_resident<2048>(dev);
    case 4096: return row_split_resident<4096>(dev);
  }
  return 0;
}

bool supported_length(int n) {
  return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024 || n == 2048 || n == 4096;
}

int row_line_threads(int n, bool fp64) {
  switch (n) {
    case 64: return fp64 ? Shape<64, double>::T : Shape<64, float>::T;
    case 128: return fp64 ? Shape<128, double>::T : Shape<128, float>::T;
    case 256: return fp64 ? Shape<256, double>::T : Shape<256, float>::T;
    case 512: return fp64 ? Shape<512, double>::T : Shape<512, float>::T;
    case 1024: return fp64 ? Shape<1024, double>::T : Shape<1024, float>::T;
    case 2048: return fp64 ? Shape<2048, double>::T : Shape<2048, float>::T;
    case 4096: return fp64 ? Shape<4096, double>::T : Shape<4096, float>::T;
  }
  return 0;
}

cudaError_t launch_row(bool fp64, RowOp op, const PassArgs& a, cudaStream_t s) {
  if (fp64) {
    switch (op) {
      case ROW_FWD: return row_dispatch<double, ROW_FWD>(a, s);
      case ROW_INV: return row_dispatch<double, ROW_INV>(a, s);
      case ROW_SLICE: return row_dispatch<double, ROW_SLICE>(a, s);
      case ROW_SLICE_FIRST: return row_dispatch<double, ROW_SLICE_FIRST>(a, s);
    }
  } else {
    switch (op) {
      case ROW_SLICE: return row_dispatch<float, ROW_SLICE>(a, s);
      case ROW_SLICE_FIRST: return row_dispatch<float, ROW_SLICE_FIRST>(a, s);
      case ROW_SPLIT: return row_dispatch<float, ROW_SPLIT>(a, s);
      case ROW_SPLIT_FIRST: return row_dispatch<float, ROW_SPLIT_FIRST>(a, s);
      case ROW_SLOTS: return row_dispatch<float, ROW_SLOTS>(a, s);
      default: return cudaErrorInvalidValue;  // set-up transforms run in FP64
    }
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_row_split_alt(const PassArgs& a, cudaStream_t s) {
  switch (a.ny) {
    case 256: return row_launch<float, 256, ROW_SPLIT, 1>(a, s);
    case 512: return row_launch<float, 512, ROW_SPLIT, 1>(a, s);
    case 1024: return row_launch<float, 1024, ROW_SPLIT, 1>(a, s);
    case 2048: return row_launch<float, 2048, ROW_SPLIT, 1>(a, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_col(bool fp64, ColOp op, const PassArgs& a, cudaStream_t s) {
  if (fp64) {
    switch (op) {
      case COL_FWD: return col_dispatch<double, COL_FWD>(a, s);
      case COL_INV: return col_dispatch<double, COL_INV>(a, s);
      case COL_FWD_MASK_INV: return col_dispatch<double, COL_FWD_MASK_INV>(a, s);
      case COL_SLICE: return col_dispatch<double, COL_SLICE>(a, s);
      case COL_SLICE_LAST: return col_dispatch<double, COL_SLICE_LAST>(a, s);
    }
  } else {
    switch (op) {
      case COL_SLICE: return col_dispatch<float, COL_SLICE>(a, s);
      case COL_SLICE_LAST: return col_dispatch<float, COL_SLICE_LAST>(a, s);
      case COL_SLOTS: return col_dispatch<float, COL_SLOTS>(a, s);
      default: return cudaErrorInvalidValue;
    }
  }
  return cudaErrorInvalidValue;
}

void fill_twiddles(int n, double* h) {
  const double two_pi = 6.283185307179586476925286766559;
  for (int m = 0; m < n; ++m) {
    const double a = two_pi * (double)m / (double)n;
    h[2 * m] = std::cos(a);
    h[2 * m + 1] = -std::sin(a);
  }
}

namespace {
template <int N, int V = 0>
void append_stage_twiddles(const double* base, std::vector<double>& out) {
  using Sh = Shape<N, float, V>;
  static_assert(Sh::TT, "stage copies are laid out for the FP32 schedules");
  for (int s = 1; s < Sh::S; ++s) {
    const int R = Sh::radix(s), NS = Sh::ns(s);
    if ((int)out.size() != 2 * (tt_base<Sh>() + Sh::tt_off(s))) std::abort();  // layout drift
    for (int r = 1; r < R; ++r)
      for (int k = 0; k < NS; ++k) {
        const int m = r * k * (N / (NS * R));
        out.push_back(base[2 * m]);
        out.push_back(base[2 * m + 1]);
      }
  }
}
}  // namespace

void fill_twiddles_f32_table(int n, std::vector<double>& h) {
  h.assign(2 * (size_t)n, 0.0);
  fill_twiddles(n, h.data());
  const std::vector<double> base = h;
  switch (n) {
    case 64: append_stage_twiddles<64>(base.data(), h); break;
    case 128: append_stage_twiddles<128>(base.data(), h); break;
    case 256:
      append_stage_twiddles<256>(base.data(), h);
      append_stage_twiddles<256, 1>(base.data(), h);
      break;
    case 512:
      append_stage_twiddles<512>(base.data(), h);
      append_stage_twiddles<512, 1>(base.data(), h);
      break;
    case 1024:
      append_stage_twiddles<1024>(base.data(), h);
      append_stage_twiddles<1024, 1>(base.data(), h);
      break;
    case 2048:
      append_stage_twiddles<2048>(base.data(), h);
      append_stage_twiddles<2048, 1>(base.data(), h);
      break;
    case 4096: append_stage_twiddles<4096>(base.data(), h); break;
    default: break;  // no FP32 pass of this length
  }
}

cudaError_t launch_lut_synth(double* out, const double* kx, const double* ky, int nx,
                             int ny, const double* params12, double prefactor,
                             double cutoff_sq, double xmin, double ymin, cudaStream_t s) {
  const int64_t n = (int64_t)nx * ny;
  lut_synth_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(out), kx, ky, nx, ny, params12, prefactor, cutoff_sq,
      xmin, ymin);
  return cudaGetLastError();
}

cudaError_t launch_potential(double* t, const double* luts, int nx, int ny,
                             const int32_t* asx, const int32_t* asy, const int32_t* asp,
                             int n_atoms, cudaStream_t s, bool exponentiate) {
  if (nx % kPotRows) return cudaErrorInvalidValue;
  const int tpb = ny < 256 ? ny : 256;
  dim3 grid((ny + tpb - 1) / tpb, nx / kPotRows);
  if (exponentiate)
    potential_kernel<true><<<grid, tpb, 0, s>>>(reinterpret_cast<double2*>(t),
                                                reinterpret_cast<const double2*>(luts), nx, ny,
                                                asx, asy, asp, n_atoms);
  else
    potential_kernel<false><<<grid, tpb, 0, s>>>(reinterpret_cast<double2*>(t),
                                                 reinterpret_cast<const double2*>(luts), nx,
                                                 ny, asx, asy, asp, n_atoms);
  return cudaGetLastError();
}

cudaError_t launch_probe_synth(double* out, const double* kx, const double* ky, int nx,
                               int ny, int corrected, double cs3, double cs5, double defocus,
                               double lambda, double lambda_sq, double alpha_max_sq,
                               double x0, double y0, cudaStream_t s) {
  const int64_t n = (int64_t)nx * ny;
  probe_synth_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(out), kx, ky, nx, ny, corrected, cs3, cs5, defocus, lambda,
      lambda_sq, alpha_max_sq, x0, y0);
  return cudaGetLastError();
}

cudaError_t launch_norm2(const double* a, int64_t n, double* out, cudaStream_t s) {
  norm2_kernel<<<1, 1024, 0, s>>>(reinterpret_cast<const double2*>(a), n, out);
  return cudaGetLastError();
}

cudaError_t launch_scale(double* a, int64_t n, double sc, const double*, cudaStream_t s) {
  scale_kernel<<<blocks_for(n, 256), 256, 0, s>>>(reinterpret_cast<double2*>(a), n, sc);
  return cudaGetLastError();
}

cudaError_t launch_to_f32(const double* in, float* out, int64_t n, cudaStream_t s) {
  to_f32_kernel<<<blocks_for(n, 256), 256, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

cudaError_t launch_segment_sums(bool fp64, const void* psi, int64_t stride, int nb,
                                const SegmentPlan& sp, double* amp, double* inten,
                                const SplitK& sk, cudaStream_t s) {
  if (sp.ng <= 0 || nb <= 0) return cudaSuccess;
  double* pa = sp.partial;
  double* pi = sp.partial + (int64_t)nb * sp.n_chunks;
  if (sp.n_chunks > 0) {
    dim3 grid(sp.n_chunks, nb);
    if (fp64)
      segment_chunk_kernel<double><<<grid, 256, 0, s>>>(
          static_cast<const double2*>(psi), stride, sp.idx, sp.chunk_begin, sp.n_chunks, pa, pi,
          sk);
    else
      segment_chunk_kernel<float><<<grid, 256, 0, s>>>(
          static_cast<const float2*>(psi), stride, sp.idx, sp.chunk_begin, sp.n_chunks, pa, pi,
          sk);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  segment_reduce_kernel<<<nb, 128, 0, s>>>(pa, pi, sp.seg_chunk, sp.ng, sp.n_chunks, amp, inten);
  return cudaGetLastError();
}

cudaError_t launch_histogram_scatter(double* h, const int32_t* pix, const int32_t* sp,
                                     const double* count, int n, int64_t plane, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  histogram_scatter_kernel<<<blocks_for(n, 256), 256, 0, s>>>(reinterpret_cast<double2*>(h), pix,
                                                              sp, count, n, plane);
  return cudaGetLastError();
}

cudaError_t launch_histogram_lut(double* out, const double* h, const double* lut_k,
                                 int n_species, int64_t plane, cudaStream_t s) {
  histogram_lut_kernel<<<blocks_for(plane, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(out), reinterpret_cast<const double2*>(h),
      reinterpret_cast<const double2*>(lut_k), n_species, plane);
  return cudaGetLastError();
}

cudaError_t launch_transmission_exp(double* t, int64_t n, double scale, cudaStream_t s) {
  transmission_exp_kernel<<<blocks_for(n, 256), 256, 0, s>>>(reinterpret_cast<double2*>(t), n,
                                                             scale);
  return cudaGetLastError();
}

cudaError_t launch_place_probe(double* psi, const double* probe, int nx, int ny, int sx, int sy,
                               cudaStream_t s) {
  place_probe_kernel<<<blocks_for((int64_t)nx * ny, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(psi), reinterpret_cast<const double2*>(probe), nx, ny, sx, sy);
  return cudaGetLastError();
}

cudaError_t launch_transmit(double* psi, const double* t, int64_t n, double inv_s,
                            cudaStream_t s) {
  transmit_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(psi), reinterpret_cast<const double2*>(t), n, inv_s);
  return cudaGetLastError();
}

cudaError_t launch_bw_limit(double* psi, const int32_t* lo, const int32_t* hi, int nx, int ny,
                            cudaStream_t s, int nb) {
  bw_limit_kernel<<<blocks_for((int64_t)nx * ny * nb, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(psi), lo, hi, nx, ny, nb);
  return cudaGetLastError();
}

cudaError_t launch_mtf_magnitude(bool fp64, const void* psi, int64_t stride, int nb,
                                 const double* kx, const double* ky, double lambda_sq,
                                 double amax_sq, const SplitK& sk, double* out, cudaStream_t s) {
  const int64_t n = (int64_t)sk.nx * sk.ny * nb;
  if (fp64)
    mtf_magnitude_kernel<double><<<blocks_for(n, 256), 256, 0, s>>>(
        static_cast<const double2*>(psi), stride, nb, kx, ky, lambda_sq, amax_sq, sk,
        reinterpret_cast<double2*>(out));
  else
    mtf_magnitude_kernel<float><<<blocks_for(n, 256), 256, 0, s>>>(
        static_cast<const float2*>(psi), stride, nb, kx, ky, lambda_sq, amax_sq, sk,
        reinterpret_cast<double2*>(out));
  return cudaGetLastError();
}

cudaError_t launch_mtf_multiply(double* psi, const double* mtf, int64_t plane, int nb,
                                double inv_s, cudaStream_t s) {
  mtf_multiply_kernel<<<blocks_for(plane * nb, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(psi), reinterpret_cast<const double2*>(mtf), plane, nb, inv_s);
  return cudaGetLastError();
}

cudaError_t launch_propagate(double* psi, const double* px, const double* py, const int32_t* lo,
                             const int32_t* hi, int nx, int ny, cudaStream_t s) {
  propagate_kernel<<<blocks_for((int64_t)nx * ny, 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(psi), reinterpret_cast<const double2*>(px),
      reinterpret_cast<const double2*>(py), lo, hi, nx, ny);
  return cudaGetLastError();
}

// out[p] = in[0][p] + in[1][p] + ... in rank order (FP64, no contraction)
__global__ void rank_sum_kernel(const double* __restrict__ in, int world, int64_t n,
                                double* __restrict__ out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int r = 0; r < world; ++r) acc = __dadd_rn(acc, in[(int64_t)r * n + p]);
    out[p] = acc;
  }
}

cudaError_t launch_rank_sum(const double* in, int world, int64_t n, double* out,
                            cudaStream_t s) {
  if (world <= 0 || n <= 0) return cudaErrorInvalidValue;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 8 * (int64_t)sm_count());
  rank_sum_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, world, n, out);
  return cudaGetLastError();
}

cudaError_t launch_slot_detect(const void* table, int max_done, int max_chunks, int nx, int ny,
                               double* partial, bool pixel_sums, cudaStream_t s) {
  if (max_done <= 0 || max_chunks <= 0) return cudaErrorInvalidValue;
  const int sms = sm_count();
  double* pa = partial;
  double* pi = partial + (int64_t)max_done * max_chunks;
  slot_chunk_kernel<<<4 * sms, 256, 0, s>>>(table, max_chunks, nx, ny, pa, pi);
  slot_reduce_kernel<<<max_done < sms ? max_done : sms, 128, 0, s>>>(table, max_chunks, pa, pi);
  if (pixel_sums) slot_pixel_kernel<<<2 * sms, 256, 0, s>>>(table, nx, ny);
  return cudaGetLastError();
}

cudaError_t launch_pixel_accum(bool fp64, const void* psi, int64_t stride, int nb,
                               int64_t npix, double* acc_a, double* acc_i, const SplitK& sk,
                               cudaStream_t s) {
  if (fp64)
    pixel_accum_kernel<double><<<blocks_for(npix, 256), 256, 0, s>>>(
        static_cast<const double2*>(psi), stride, nb, npix, acc_a, acc_i, sk);
  else
    pixel_accum_kernel<float><<<blocks_for(npix, 256), 256, 0, s>>>(
        static_cast<const float2*>(psi), stride, nb, npix, acc_a, acc_i, sk);
  return cudaGetLastError();
}

cudaError_t launch_to_f32_minus_one(const double* in, float* out, int64_t n, cudaStream_t s) {
  to_f32_minus_one_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      reinterpret_cast<const double2*>(in), reinterpret_cast<float2*>(out), n);
  return cudaGetLastError();
}

cudaError_t launch_wave_accumulate(bool fp64, const void* psi, int64_t stride, int nb,
                                   int64_t plane, const SplitK& sk, double divisor, double* acc,
                                   cudaStream_t s) {
  const int64_t n = plane * nb;
  if (fp64)
    wave_accumulate_kernel<double><<<blocks_for(n, 256), 256, 0, s>>>(
        static_cast<const double2*>(psi), stride, nb, plane, sk, divisor,
        reinterpret_cast<double2*>(acc));
  else
    wave_accumulate_kernel<float><<<blocks_for(n, 256), 256, 0, s>>>(
        static_cast<const float2*>(psi), stride, nb, plane, sk, divisor,
        reinterpret_cast<double2*>(acc));
  return cudaGetLastError();
}

cudaError_t launch_strided_accumulate(double* dst, int64_t dst_stride, const double* src,
                                      int64_t src_stride, int n, double divisor, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  strided_accumulate_kernel<<<blocks_for(n, 128), 128, 0, s>>>(dst, dst_stride, src, src_stride,
                                                                 n, divisor);
  return cudaGetLastError();
}

cudaError_t launch_assemble_split(const float* delta, const double* psi0k, int nx, int ny,
                                  int sx, int sy, double* out, cudaStream_t s) {
  SplitK sk;
  sk.psi0k = psi0k;
  sk.nx = nx;
  sk.ny = ny;
  const int64_t n = (int64_t)nx * ny;
  assemble_split_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      reinterpret_cast<const float2*>(delta), sk, sx, sy, reinterpret_cast<double2*>(out));
  return cudaGetLastError();
}

}  // namespace msf
