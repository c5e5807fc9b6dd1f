// Persistent, TMA-pipelined versions of the two FP32 slice passes.
//
// One CTA per SM walks a list of work items (a group of rows, or a group of
// columns, of one probe).  While it transforms item k out of one shared
// buffer, the tensor-memory accelerator already copies item k+1 into the
// other: rows arrive as 1-D bulk copies (cp.async.bulk), column tiles as
// 2-D tiled copies through a tensor map (cp.async.bulk.tensor), both
// completing on an mbarrier.  The transform itself is the same register
// Stockham FFT as kernels.cu; the buffer that just delivered the item also
// serves as the exchange buffer.
//
// Every wait is bounded: if an mbarrier phase does not complete within
// kSpinLimit polls the CTA records an error in *err and leaves its loop,
// first waiting (bounded again) for any copy it still has in flight.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "fft_core.cuh"
#include "kernels.h"

namespace msf {

namespace {

constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tile_g2s(void* dst, const CUtensorMap* map, int x, int y,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// A wavefield element loaded once per pass: not allocated in L1, which
// then keeps the twiddle table (read by every stage of every line).
__device__ __forceinline__ float2 ld_once(const float2* p) {
  float2 v;
  asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Thread 0 waits (bounded) for the buffer's phase, the CTA learns the
// outcome through shared memory, then every thread observes the completed
// phase itself (acquiring the copied data).
__device__ __forceinline__ bool cta_wait(uint64_t* bar, uint32_t parity, int* flag_smem) {
  if (threadIdx.x == 0) *flag_smem = mbar_wait_bounded(bar, parity) ? 1 : 0;
  __syncthreads();
  const bool ok = *flag_smem != 0;
  if (ok) mbar_wait_bounded(bar, parity);
  return ok;
}

// ------------------------------------------------------- row pass (split) --
template <int N, int LINES>
__global__ void __launch_bounds__(LINES * Shape<N, float>::T, 1)
row_split_pipe_kernel(const PassArgs a, int* err) {
  using C = float2;
  using Sh = Shape<N, float>;
  using SM = Smem<Sh, 8, LINES, false>;
  constexpr int E = Sh::E, T = Sh::T;
  static_assert(SM::stride % 2 == 0, "line starts must be 16-byte aligned for bulk copies");
  constexpr int BUF = LINES * SM::stride;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufs = reinterpret_cast<C*>(smem_raw);
  __shared__ uint64_t bars[2];
  __shared__ int flag;
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const int items = a.nb * (a.nx / LINES);
  auto sync = [] {
    if constexpr (T <= 32) __syncwarp();
    else __syncthreads();
  };
  auto issue = [&](int item, int which) {
    const int g = item / a.nb, b = item - (item / a.nb) * a.nb;
    const C* src = static_cast<const C*>(a.psi) + (int64_t)b * a.batch_stride +
                   (int64_t)g * LINES * N;
    C* dst = bufs + which * BUF;
    mbar_expect_tx(&bars[which], LINES * N * 8);
    for (int l = 0; l < LINES; ++l)
      bulk_g2s(dst + l * SM::stride, src + (int64_t)l * N, N * 8, &bars[which]);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int item = blockIdx.x;
  if (threadIdx.x == 0) {
    if (item < items) issue(item, 0);
    if (item + (int)gridDim.x < items) issue(item + gridDim.x, 1);
  }
  uint32_t parity[2] = {0, 0};
  const C* tw = static_cast<const C*>(a.tw);
  const float is = (float)a.inv_s;
  int k = 0;
  for (; item < items; ++k, item += gridDim.x) {
    const int w = k & 1;
    if (!cta_wait(&bars[w], parity[w], &flag)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        // the other buffer may still be receiving a copy: wait for it
        if (item + (int)gridDim.x < items) mbar_wait_bounded(&bars[w ^ 1], parity[w ^ 1]);
      }
      return;
    }
    parity[w] ^= 1;
    const int g = item / a.nb, b = item - (item / a.nb) * a.nb;
    const int i = g * LINES + line;
    C* sm = bufs + w * BUF + line * SM::stride;
    C v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[t + T * m];
    sync();
    fft_line<Sh, true>(v, sm, t, tw, sync);
    // split-wave transmission update, as ROW_SPLIT in kernels.cu
    const int sx = a.shifts[2 * b], sy = a.shifts[2 * b + 1];
    const int ix = (i < sx) ? i + a.nx - sx : i - sx;
    const C* prow = static_cast<const C*>(a.psi0) + (int64_t)ix * N;
    const C* trow = static_cast<const C*>(a.trans) + (int64_t)i * N;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      if (m % kLoadChunk == 0) load_fence();
      const int y = t + T * m;
      const int iy = (y < sy) ? y + N - sy : y - sy;
      const C p0 = __ldg(prow + iy);
      const C tau = __ldg(trow + y);
      v[m] = split_elem(p0, tau, v[m], is);
    }
    fft_line<Sh, false>(v, sm, t, tw, sync);
    C* row = static_cast<C*>(a.psi) + (int64_t)b * a.batch_stride + (int64_t)i * N;
#pragma unroll
    for (int m = 0; m < E; ++m) row[t + T * m] = v[m];
    __syncthreads();
    if (threadIdx.x == 0 && item + 2 * (int)gridDim.x < items) {
      fence_proxy_async();
      issue(item + 2 * gridDim.x, w);
    }
  }
}

// -------------------------------------------- row pass (split, staged) --
// The split-wave row pass with its slice tables staged in shared memory.
// One CTA transforms row i of P probes of the batch (one line each).  On
// entry bulk copies of the transmission row tau[i], which the P lines
// share, and of each probe's vacuum row psi0[(i - sx) mod nx] start (each
// line issues its own); meanwhile every line loads its scattered row from
// global memory and runs
// the inverse transform, so the update then reads tau and psi0 from shared
// memory with no L2 round trip left on its path.  Arithmetic is that of
// ROW_SPLIT (split_elem) element for element, so the results are
// bit-identical.  A probe index past the batch leaves its line idle (it
// still takes part in the barriers of a line that spans two warps).  V is
// the FFT radix schedule (Shape<N, float, V>).
template <int N, int V>
constexpr int staged_lines() {
  constexpr int T = Shape<N, float, V>::T;
  return T >= 128 ? 1 : 128 / T;
}
template <int N, int V>
constexpr int staged_min_ctas() {
  // schedule 0 (32 elements a thread): 384 threads per SM (168 registers)
  // up to 1024-point lines, 256 for 2048-point lines, whose transforms need
  // 255 registers; schedule 1 (16 or 8 elements): 512 (128 registers)
  constexpr int per_sm = V == 1 ? 512 : (N >= 2048 ? 256 : 384);
  return per_sm / (staged_lines<N, V>() * Shape<N, float, V>::T);
}
template <int N, int V>
constexpr int staged_smem() {
  using SM = Smem<Shape<N, float, V>, 8, staged_lines<N, V>(), false>;
  return (N + staged_lines<N, V>() * N + staged_lines<N, V>() * SM::stride) * 8;
}

template <int N, int P, int V>
__global__ void __launch_bounds__(P * Shape<N, float, V>::T, staged_min_ctas<N, V>())
row_split_staged_kernel(const PassArgs a, int* err) {
  using C = float2;
  using Sh = Shape<N, float, V>;
  using SM = Smem<Sh, 8, P, false>;
  constexpr int E = Sh::E, T = Sh::T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* tau_s = reinterpret_cast<C*>(smem_raw);  // [N]
  C* psi0_s = tau_s + N;                      // [P][N]
  C* exch = psi0_s + P * N;                   // [P][SM::stride]
  __shared__ uint64_t bar;
  __shared__ int flag;
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const int i = blockIdx.y;
  const int b0 = blockIdx.x * P;
  const int b = b0 + line;
  const int nvalid = a.nb - b0 < P ? a.nb - b0 : P;
  const bool valid = line < nvalid;
  if (threadIdx.x == 0) {  // the barrier expects every byte before any copy starts
    mbar_init(&bar, 1);
    mbar_fence_init();
    mbar_expect_tx(&bar, (uint32_t)((1 + nvalid) * N * 8));
  }
  __syncthreads();
  // each line's first thread fetches its own probe's shift and vacuum row,
  // so no thread waits on another's loads
  if (threadIdx.x == 0)
    bulk_g2s(tau_s, static_cast<const C*>(a.trans) + (int64_t)i * N, N * 8, &bar);
  if (t == 0 && valid) {
    const int sx = a.shifts[2 * b];
    const int ix = (i < sx) ? i + a.nx - sx : i - sx;
    bulk_g2s(psi0_s + line * N, static_cast<const C*>(a.psi0) + (int64_t)ix * N, N * 8, &bar);
  }
  auto sync = [] {
    if constexpr (T <= 32) __syncwarp();
    else __syncthreads();
  };
  C* row = static_cast<C*>(a.psi) + (int64_t)(valid ? b : 0) * a.batch_stride + (int64_t)i * N;
  const C* tw = static_cast<const C*>(a.tw);
  // columns removed by the band limit were not stored: they are zero
  const uint32_t dead = a.row_dead_bits ? __ldg(a.row_dead_bits + t) : 0u;
  const uint32_t skip = (a.row_dead_io & 1) ? dead : 0u;
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m)
    v[m] = (!valid || ((skip >> m) & 1u)) ? C{0.f, 0.f} : ld_once(row + t + T * m);
  C* sm = exch + line * SM::stride;
  fft_line<Sh, true>(v, sm, t, tw, sync);
  // wait (bounded) for the staged rows: warp-uniform for lines within a
  // warp, CTA-uniform for lines that span warps (they share barriers)
  bool ok;
  if constexpr (T <= 32) {
    int r = 0;
    if ((threadIdx.x & 31) == 0) r = mbar_wait_bounded(&bar, 0) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, r, 0) != 0;
    if (ok) mbar_wait_bounded(&bar, 0);  // every thread observes the phase
  } else {
    ok = cta_wait(&bar, 0, &flag);
  }
  if (!ok) {
    if (threadIdx.x == 0) {
      atomicExch(err, 1);
      mbar_wait_bounded(&bar, 0);  // the copies may still be landing
    }
    return;
  }
  if (valid) {
    const int sy = a.shifts[2 * b + 1];
    const C* p0 = psi0_s + line * N;
    const float is = (float)a.inv_s;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int y = t + T * m;
      const int iy = (y < sy) ? y + N - sy : y - sy;
      v[m] = split_elem(p0[iy], tau_s[y], v[m], is);
    }
  }
  fft_line<Sh, false>(v, sm, t, tw, sync);
  if (!valid) return;
  if (a.row_dead_bits) {  // columns the next band limit removes entirely
    if (a.row_dead_io & 2) {  // nobody reads them: leave them unstored
#pragma unroll
      for (int m = 0; m < E; ++m)
        if (!((dead >> m) & 1u)) row[t + T * m] = v[m];
      return;
    }
#pragma unroll
    for (int m = 0; m < E; ++m)
      if ((dead >> m) & 1u) v[m] = C{0.f, 0.f};
  }
#pragma unroll
  for (int m = 0; m < E; ++m) row[t + T * m] = v[m];
}

// ----------------------------------------------------- column slice pass --
// Resident CTAs per SM the register allocator must allow: at least
// MSF_COL_PIPE_THREADS_PER_SM threads of the pass per SM.
#ifndef MSF_COL_PIPE_THREADS_PER_SM
#define MSF_COL_PIPE_THREADS_PER_SM 256
#endif
constexpr int col_pipe_min_ctas(int threads) {
  return threads >= MSF_COL_PIPE_THREADS_PER_SM ? 1 : MSF_COL_PIPE_THREADS_PER_SM / threads;
}

// Real: float (the split-wave passes) or double (FP64 runs; a complex value
// is then two 8-byte tensor-map elements).  SLOTS (FP32 only): every probe
// of the batch brings its own mask, propagator and step (PassArgs::slots);
// LAST is then taken per probe from its slot.
template <typename Real, int N, int COLS, bool LAST, bool SLOTS>
__global__ void __launch_bounds__(COLS * Shape<N, Real>::T,
                                  col_pipe_min_ctas(COLS * Shape<N, Real>::T))
col_slice_pipe_kernel(const PassArgs a, const __grid_constant__ CUtensorMap tmap, int* err) {
  using C = Cx<Real>;
  using Sh = Shape<N, Real>;
  using SM = Smem<Sh, (int)sizeof(C), COLS, true>;
  constexpr int E = Sh::E, T = Sh::T;
  constexpr int EPC = (int)sizeof(C) / 8;  // tensor-map elements per complex value
  constexpr int BOX = N < 256 ? N : 256;
  constexpr int RAW = (N * COLS > COLS * SM::stride ? N * COLS : COLS * SM::stride);
  constexpr int BUF = (RAW + 15) / 16 * 16;  // 128-byte multiple
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufs = reinterpret_cast<C*>(smem_raw);
  __shared__ uint64_t bars[2];
  __shared__ int flag;
  const int c = threadIdx.x % COLS, t = threadIdx.x / COLS;
  // column groups to walk: all, or those with any column the band limit
  // keeps (the row pass stored zeros in the others)
  const int groups = a.live_groups ? a.n_live_groups : a.ny / COLS;
  const int items = a.nb * groups;
  auto group_of = [&](int gi) { return a.live_groups ? __ldg(a.live_groups + gi) : gi; };
  auto sync = [] { __syncthreads(); };
  auto issue = [&](int item, int which) {
    const int gi = item / a.nb, b = item - gi * a.nb;
    const int g = group_of(gi);
    C* dst = bufs + which * BUF;
    mbar_expect_tx(&bars[which], N * COLS * (int)sizeof(C));
#pragma unroll
    for (int q = 0; q < N / BOX; ++q)
      tile_g2s(dst + q * BOX * COLS, &tmap, g * COLS * EPC, b * a.nx + q * BOX, &bars[which]);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int item = blockIdx.x;
  if (threadIdx.x == 0) {
    if (item < items) issue(item, 0);
    if (item + (int)gridDim.x < items) issue(item + gridDim.x, 1);
  }
  uint32_t parity[2] = {0, 0};
  const C* tw = static_cast<const C*>(a.tw);
  const Real is = (Real)a.inv_s;
  const C* px = static_cast<const C*>(a.px);
  int k = 0;
  for (; item < items; ++k, item += gridDim.x) {
    const int w = k & 1;
    // a slot batch reads its slot entry before the tile wait, so that the
    // load overlaps the copy instead of following it
    SlotPass sp{};
    if constexpr (SLOTS) sp = a.slots[item % a.nb];
    if (!cta_wait(&bars[w], parity[w], &flag)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        if (item + (int)gridDim.x < items) mbar_wait_bounded(&bars[w ^ 1], parity[w ^ 1]);
      }
      return;
    }
    parity[w] ^= 1;
    const int gi = item / a.nb, b = item - gi * a.nb;
    const int g = group_of(gi);
    const int j = g * COLS + c;
    const int32_t* mask_lo = a.mask_lo;
    const int32_t* mask_hi = a.mask_hi;
    const C* pxb = px;
    const C* pyb = static_cast<const C*>(a.py);
    bool idle = false, stop_in_k = LAST;
    if constexpr (SLOTS) {
      idle = sp.op == SLOT_IDLE;
      mask_lo = sp.mask_lo;
      mask_hi = sp.mask_hi;
      pxb = static_cast<const C*>(sp.px);
      pyb = static_cast<const C*>(sp.py);
      stop_in_k = sp.last != 0;
    }
    if (!idle) {
      C* base = bufs + w * BUF;
      C v[E];
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = base[(t + T * m) * COLS + c];
      // the transform's first exchange opens with a barrier, which also
      // orders these tile reads before its writes into the same buffer
      if constexpr (Sh::S == 1) __syncthreads();
      C* sm = base + c * SM::stride;
      fft_line<Sh, false>(v, sm, t, tw, sync);
      const int lo = __ldg(mask_lo + j), hi = __ldg(mask_hi + j);
      const C pyj = __ldg(pyb + j);
#pragma unroll
      for (int m = 0; m < E; ++m) {
        if (m % kLoadChunk == 0) load_fence();
        const int i = t + T * m;
        if (i < lo || i >= hi) {
          const C p = cmul(__ldg(pxb + i), pyj);
          v[m] = cmul(p, cscale(v[m], is));
        } else {
          v[m] = C{Real(0), Real(0)};
        }
      }
      if (!stop_in_k) fft_line<Sh, true>(v, sm, t, tw, sync);
      C* col = static_cast<C*>(a.psi) + (int64_t)b * a.batch_stride + j;
#pragma unroll
      for (int m = 0; m < E; ++m) col[(int64_t)(t + T * m) * a.ny] = v[m];
    }
    __syncthreads();
    if (threadIdx.x == 0 && item + 2 * (int)gridDim.x < items) {
      fence_proxy_async();
      issue(item + 2 * gridDim.x, w);
    }
  }
}


template <int N>
constexpr int pipe_lines() { return 256 / Shape<N, float>::T; }
// Threads per CTA of the pipelined column pass; the grid holds as many
// persistent CTAs as fit on the SMs.
#ifndef MSF_COL_PIPE_THREADS
#define MSF_COL_PIPE_THREADS 256
#endif
template <typename Real, int N>
constexpr int pipe_cols() {
  int c = 16;
  while (c > 2 && c * Shape<N, Real>::T > MSF_COL_PIPE_THREADS) c >>= 1;
  return c;
}

template <int N>
cudaError_t row_pipe_launch(const PassArgs& a, int* err, cudaStream_t s) {
  constexpr int L = pipe_lines<N>();
  using SM = Smem<Shape<N, float>, 8, L, false>;
  constexpr int smem = 2 * L * SM::stride * 8;
  static PerDevice configured;
  auto k = row_split_pipe_kernel<N, L>;
  if (cudaError_t e = smem_limit_once((const void*)k, smem, configured); e != cudaSuccess)
    return e;
  const int items = a.nb * (a.nx / L);
  const int grid = items < sm_count() ? items : sm_count();
  k<<<grid, L * Shape<N, float>::T, smem, s>>>(a, err);
  return cudaGetLastError();
}

template <int N, int V>
cudaError_t row_staged_launch(const PassArgs& a, int* err, cudaStream_t s) {
  constexpr int P = staged_lines<N, V>();
  constexpr int smem = staged_smem<N, V>();
  static_assert(smem * staged_min_ctas<N, V>() <= 227 * 1024,
                "staged row pass: its CTAs per SM exceed shared memory");
  static PerDevice configured;
  auto k = row_split_staged_kernel<N, P, V>;
  const int dev = current_device();
  if (configured.needed(dev)) {
    // several CTAs per SM need the largest shared-memory carveout
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    configured.mark(dev);
  }
  if (a.nb <= 0) return cudaSuccess;
  dim3 grid((a.nb + P - 1) / P, a.nx);
  k<<<grid, P * Shape<N, float, V>::T, smem, s>>>(a, err);
  return cudaGetLastError();
}

template <typename Real, int N, bool LAST, bool SLOTS = false>
cudaError_t col_pipe_launch(const PassArgs& a, const CUtensorMap& map, int* err,
                            cudaStream_t s) {
  constexpr int CC = pipe_cols<Real, N>();
  constexpr int CB = (int)sizeof(Cx<Real>);
  using SM = Smem<Shape<N, Real>, CB, CC, true>;
  constexpr int RAW = (N * CC > CC * SM::stride ? N * CC : CC * SM::stride);
  constexpr int smem = 2 * ((RAW + 15) / 16 * 16) * CB;
  // resident CTAs per SM, found once per device after raising the limit
  static PerDevice configured;
  static std::atomic<int> per_sm_dev[64];
  auto k = col_slice_pipe_kernel<Real, N, CC, LAST, SLOTS>;
  const int dev = current_device();
  int per_sm = (dev >= 0 && dev < 64) ? per_sm_dev[dev].load() : 0;
  if (configured.needed(dev) || per_sm < 1) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, CC * Shape<N, Real>::T, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    if (dev >= 0 && dev < 64) per_sm_dev[dev].store(per_sm);
    configured.mark(dev);
  }
  const int items = a.nb * (a.live_groups ? a.n_live_groups : a.ny / CC);
  if (items <= 0) return cudaSuccess;
  const int grid = items < per_sm * sm_count() ? items : per_sm * sm_count();
  k<<<grid, CC * Shape<N, Real>::T, smem, s>>>(a, map, err);
  return cudaGetLastError();
}

}  // namespace

bool pipe_supported(int nx, int ny, bool fp64) {
  // FP64 tiles of 2048-point columns would be 2 columns (32-byte rows) wide
  auto ok = [fp64](int n) {
    return n == 256 || n == 512 || n == 1024 || (!fp64 && n == 2048);
  };
  return ok(nx) && ok(ny);
}

int pipe_cols_for(int nx, bool fp64) {
  if (fp64) {
    switch (nx) {
      case 256: return pipe_cols<double, 256>();
      case 512: return pipe_cols<double, 512>();
      case 1024: return pipe_cols<double, 1024>();
    }
    return 0;
  }
  switch (nx) {
    case 256: return pipe_cols<float, 256>();
    case 512: return pipe_cols<float, 512>();
    case 1024: return pipe_cols<float, 1024>();
    case 2048: return pipe_cols<float, 2048>();
  }
  return 0;
}

cudaError_t launch_row_split_pipe(const PassArgs& a, int* err, cudaStream_t s) {
  switch (a.ny) {
    case 256: return row_pipe_launch<256>(a, err, s);
    case 512: return row_pipe_launch<512>(a, err, s);
    case 1024: return row_pipe_launch<1024>(a, err, s);
    case 2048: return row_pipe_launch<2048>(a, err, s);
  }
  return cudaErrorInvalidValue;
}

bool staged_row_supported(int nx, int ny) {
  (void)nx;
  return ny == 256 || ny == 512 || ny == 1024 || ny == 2048;
}

int staged_row_threads(int ny, int schedule) {
  switch (ny) {
    case 256: return schedule ? Shape<256, float, 1>::T : Shape<256, float>::T;
    case 512: return schedule ? Shape<512, float, 1>::T : Shape<512, float>::T;
    case 1024: return schedule ? Shape<1024, float, 1>::T : Shape<1024, float>::T;
    case 2048: return schedule ? Shape<2048, float, 1>::T : Shape<2048, float>::T;
  }
  return 0;
}

cudaError_t launch_row_split_staged(const PassArgs& a, int* err, cudaStream_t s, int schedule) {
  if (schedule == 1) {
    switch (a.ny) {
      case 256: return row_staged_launch<256, 1>(a, err, s);
      case 512: return row_staged_launch<512, 1>(a, err, s);
      case 1024: return row_staged_launch<1024, 1>(a, err, s);
      case 2048: return row_staged_launch<2048, 1>(a, err, s);
    }
    return cudaErrorInvalidValue;
  }
  switch (a.ny) {
    case 256: return row_staged_launch<256, 0>(a, err, s);
    case 512: return row_staged_launch<512, 0>(a, err, s);
    case 1024: return row_staged_launch<1024, 0>(a, err, s);
    case 2048: return row_staged_launch<2048, 0>(a, err, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_col_slice_pipe(const PassArgs& a, bool last, const void* tensor_map,
                                  int* err, cudaStream_t s, bool fp64) {
  const CUtensorMap& m = *static_cast<const CUtensorMap*>(tensor_map);
  if (fp64) {
    if (a.slots) return cudaErrorInvalidValue;
    switch (a.nx) {
      case 256: return last ? col_pipe_launch<double, 256, true>(a, m, err, s) : col_pipe_launch<double, 256, false>(a, m, err, s);
      case 512: return last ? col_pipe_launch<double, 512, true>(a, m, err, s) : col_pipe_launch<double, 512, false>(a, m, err, s);
      case 1024: return last ? col_pipe_launch<double, 1024, true>(a, m, err, s) : col_pipe_launch<double, 1024, false>(a, m, err, s);
    }
    return cudaErrorInvalidValue;
  }
  if (a.slots) {
    switch (a.nx) {
      case 256: return col_pipe_launch<float, 256, false, true>(a, m, err, s);
      case 512: return col_pipe_launch<float, 512, false, true>(a, m, err, s);
      case 1024: return col_pipe_launch<float, 1024, false, true>(a, m, err, s);
      case 2048: return col_pipe_launch<float, 2048, false, true>(a, m, err, s);
    }
    return cudaErrorInvalidValue;
  }
  switch (a.nx) {
    case 256: return last ? col_pipe_launch<float, 256, true>(a, m, err, s) : col_pipe_launch<float, 256, false>(a, m, err, s);
    case 512: return last ? col_pipe_launch<float, 512, true>(a, m, err, s) : col_pipe_launch<float, 512, false>(a, m, err, s);
    case 1024: return last ? col_pipe_launch<float, 1024, true>(a, m, err, s) : col_pipe_launch<float, 1024, false>(a, m, err, s);
    case 2048: return last ? col_pipe_launch<float, 2048, true>(a, m, err, s) : col_pipe_launch<float, 2048, false>(a, m, err, s);
  }
  return cudaErrorInvalidValue;
}

// Tensor map over a batch of complex planes [nb*nx rows][ny columns] of
// 8-byte elements (one per FP32 complex value, two per FP64 one), box
// {cols, min(256, nx)} rows; no multicast, no swizzle.
cudaError_t encode_column_map(void* psi, int nb, int nx, int ny, void* map_out, bool fp64) {
  // looked up once per process (a thread-safe static: lanes of the request
  // loop encode maps from their worker thread)
  static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    return (e == cudaSuccess && q == cudaDriverEntryPointSuccess)
               ? reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn)
               : nullptr;
  }();
  if (!encode) return cudaErrorNotSupported;
  const int cols = pipe_cols_for(nx, fp64);
  if (!cols) return cudaErrorInvalidValue;
  const int epc = fp64 ? 2 : 1;  // 8-byte elements per complex value
  cuuint64_t dims[2] = {(cuuint64_t)ny * epc, (cuuint64_t)nx * (cuuint64_t)nb};
  cuuint64_t strides[1] = {(cuuint64_t)ny * 8 * epc};
  cuuint32_t box[2] = {(cuuint32_t)(cols * epc), (cuuint32_t)(nx < 256 ? nx : 256)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(static_cast<CUtensorMap*>(map_out), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, psi,
                      dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace msf
