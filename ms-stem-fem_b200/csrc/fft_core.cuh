// Register-resident Stockham FFT building blocks for sm_100a.
//
// A "line" is one 1-D transform of length N (a row along y, or a column
// along x, of the [x][y] wavefield).  It is held by T = N/E threads, each
// owning E elements in registers: thread t holds element t + T*m in slot m,
// on entry and on exit, for every shape below.  Between radix stages the
// line is exchanged through a padded shared-memory buffer; inside a stage
// each thread runs E/R radix-R butterflies fully in registers, with
// compile-time constant twiddles inside the butterfly and table twiddles
// (from an FP64-computed table) between stages.
//
// Because entry and exit layouts coincide, an inverse transform, a
// point-wise product and a forward transform chain with no data movement
// between them; this is what lets one kernel pass fuse "inverse FFT along y,
// multiply by the transmission function, forward FFT along y".
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

namespace msf {

#include "unit_roots.inc"

template <typename R> struct CxT;
template <> struct CxT<float> { using type = float2; };
template <> struct CxT<double> { using type = double2; };
template <typename R> using Cx = typename CxT<R>::type;

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return C{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) {
  return C{a.x * s, a.y * s};
}

// FP32 complex adds and scales on the paired FP32 pipe of sm_100 (one
// FADD2 / FMUL2 per complex operation), with the same per-component
// round-to-nearest results as the scalar operations.
#ifndef MSF_FP32X2
#define MSF_FP32X2 1
#endif
#if MSF_FP32X2 && defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
  return __fadd2_rn(a, b);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
template <> __device__ __forceinline__ float2 cscale<float2, float>(float2 a, float s) {
  return __fmul2_rn(a, make_float2(s, s));
}
#endif

// Split-wave transmission update of one element.  psi = psi0 + d with
// psi0 the vacuum wave and t = 1 + tau; the reference's in-place update
// (adfstem.cpp:1929-1949)
//   re' = (tr*re - ti*im)/s,  im' = (tr*im + ti*re')/s
// is linear over the reals, so the scattered part evolves as
//   dre' = (tau_r*p0r - ti*p0i + (1+tau_r)*dre - ti*dim)/s
//   dim' = (tau_r*p0i + (1+tau_r)*dim + ti*(p0r/s + dre'))/s
// with every term formed at the scale of d, not of psi0.  Every split-wave
// row pass calls this one function, so they agree bit for bit.
template <typename C, typename Real>
__device__ __forceinline__ C split_elem(C p0, C tau, C d, Real is) {
  const Real dre = (tau.x * p0.x - tau.y * p0.y + d.x + tau.x * d.x - tau.y * d.y) * is;
  const Real re_total = p0.x * is + dre;
  const Real dim = (tau.x * p0.y + d.y + tau.x * d.y + tau.y * re_total) * is;
  return C{dre, dim};
}

template <int I> using ic = std::integral_constant<int, I>;

// Loads issued between two fences may be scheduled together; a fence keeps
// later loads from being hoisted above it (register pressure control).
#ifndef MSF_LOAD_CHUNK
#define MSF_LOAD_CHUNK 8
#endif
constexpr int kLoadChunk = MSF_LOAD_CHUNK;
__device__ __forceinline__ void load_fence() { asm volatile("" ::: "memory"); }

// Compile-time loop: f(ic<B>), f(ic<B+S>), ... while < E.
template <int B, int E, int S = 1, typename F>
__device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) {
    f(ic<B>{});
    sfor<B + S, E, S>(f);
  }
}

// a * W_M^K, W_M = e^{-2 pi i / M} (forward) or its conjugate (inverse).
template <int K, int M, bool INV, typename C>
__device__ __forceinline__ C twc(C a) {
  static_assert(M <= 64 && 64 % M == 0, "butterfly radix must divide 64");
  using R = decltype(a.x);
  constexpr int k = (K * (64 / M)) & 63;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (k == 16) {  // forward -i, inverse +i
    return INV ? C{-a.y, a.x} : C{a.y, -a.x};
  } else if constexpr (k == 32) {
    return C{-a.x, -a.y};
  } else if constexpr (k == 48) {  // forward +i, inverse -i
    return INV ? C{a.y, -a.x} : C{-a.y, a.x};
  } else {
    constexpr R c = (R)cos64(k);
    constexpr R s = (R)sin64(k);
    if constexpr (INV) return C{a.x * c - a.y * s, a.x * s + a.y * c};
    else return C{a.x * c + a.y * s, a.y * c - a.x * s};
  }
}

__host__ __device__ constexpr int bitrev(int x, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((x >> b) & 1) << (bits - 1 - b);
  return r;
}
__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

// One radix-2 decimation-in-frequency layer over u[0..R) with span SPAN,
// then the remaining layers.
template <int R, int SPAN, bool INV, typename C>
__device__ __forceinline__ void dif_layers(C (&u)[R]) {
  sfor<0, R, 2 * SPAN>([&](auto base) {
    sfor<0, SPAN>([&](auto k) {
      constexpr int a = decltype(base)::value + decltype(k)::value;
      C x = u[a], y = u[a + SPAN];
      u[a] = cadd(x, y);
      u[a + SPAN] = twc<decltype(k)::value, 2 * SPAN, INV>(csub(x, y));
    });
  });
  if constexpr (SPAN > 1) dif_layers<R, SPAN / 2, INV>(u);
}

// In-place length-R DFT of v[OFF + r*STR], r < R, natural order in and out,
// by radix-2 decimation-in-frequency layers.
template <int R, bool INV, int OFF, int STR, typename C, int E>
__device__ __forceinline__ void dft_radix2(C (&v)[E]) {
  if constexpr (R > 1) {
    C u[R];
    sfor<0, R>([&](auto r) { u[decltype(r)::value] = v[OFF + decltype(r)::value * STR]; });
    dif_layers<R, R / 2, INV>(u);
    constexpr int bits = ilog2(R);
    sfor<0, R>([&](auto p) {
      constexpr int q = decltype(p)::value;
      v[OFF + bitrev(q, bits) * STR] = u[q];
    });
  }
}

// The same DFT as R = R1 * R2 (Cooley-Tukey, index maps n = R2 n1 + n2 and
// k = k1 + R1 k2): R2 DFTs of length R1 over n1, the twiddles W_R^(n2 k1),
// then R1 DFTs of length R2 over n2.  With R1 = 4 the first DFTs and all
// their internal twiddles are trivial (+-1, +-i), so a 32-point DFT as 4 x 8
// needs 28 general complex multiplies instead of the 34 of five radix-2
// layers, and a 16-point one as 4 x 4 needs 8 instead of 10.
template <int R1, int R2, bool INV, int OFF, int STR, typename C, int E>
__device__ __forceinline__ void dft_mixed(C (&v)[E]) {
  constexpr int R = R1 * R2;
  C u[R];  // u[R2 * n1 + n2] = x[R2 * n1 + n2]
  sfor<0, R>([&](auto r) { u[decltype(r)::value] = v[OFF + decltype(r)::value * STR]; });
  // over n1 for each n2: u[R2 * k1 + n2] = y[k1][n2]
  sfor<0, R2>([&](auto n2I) { dft_radix2<R1, INV, decltype(n2I)::value, R2>(u); });
  sfor<1, R1>([&](auto k1I) {
    constexpr int k1 = decltype(k1I)::value;
    sfor<1, R2>([&](auto n2I) {
      constexpr int n2 = decltype(n2I)::value;
      u[R2 * k1 + n2] = twc<(n2 * k1) % R, R, INV>(u[R2 * k1 + n2]);
    });
  });
  // over n2 for each k1: u[R2 * k1 + k2] = X[k1 + R1 * k2]
  sfor<0, R1>([&](auto k1I) { dft_radix2<R2, INV, R2 * decltype(k1I)::value, 1>(u); });
  sfor<0, R1>([&](auto k1I) {
    constexpr int k1 = decltype(k1I)::value;
    sfor<0, R2>([&](auto k2I) {
      constexpr int k2 = decltype(k2I)::value;
      v[OFF + (k1 + R1 * k2) * STR] = u[R2 * k1 + k2];
    });
  });
}

// In-place length-R DFT of v[OFF + r*STR], r < R, natural order in and out.
template <int R, bool INV, int OFF, int STR, typename C, int E>
__device__ __forceinline__ void dft(C (&v)[E]) {
#ifndef MSF_MIXED_RADIX
#define MSF_MIXED_RADIX 1
#endif
  if constexpr (MSF_MIXED_RADIX && R == 32) {
    dft_mixed<4, 8, INV, OFF, STR>(v);
  } else if constexpr (MSF_MIXED_RADIX && R == 16) {
    dft_mixed<4, 4, INV, OFF, STR>(v);
  } else {
    dft_radix2<R, INV, OFF, STR>(v);
  }
}

// ---------------------------------------------------------------- shapes --
// FFT length N: E elements per thread, S radix stages R0..R{S-1} (each R
// divides E).  FP64 keeps E <= 16 to bound register use.  V selects the
// radix schedule: V = 0 is the default of every kernel; V = 1 is the
// alternative schedule of the FP32 split-wave row pass at 256..2048 points
// (half the elements per thread, twice the threads per line, one more
// radix stage), which the launch autotuner times against V = 0 per grid.
template <int N, typename Real, int V = 0> struct Shape;
#define MSF_SHAPE(N_, REAL_, V_, E_, S_, R0_, R1_, R2_)                      \
  template <> struct Shape<N_, REAL_, V_> {                                   \
    static constexpr int N = N_, E = E_, S = S_, T = N_ / E_;                 \
    static constexpr int R0 = R0_, R1 = R1_, R2 = R2_;                        \
    __host__ __device__ static constexpr int radix(int s) { return s == 0 ? R0 : s == 1 ? R1 : R2; } \
    __host__ __device__ static constexpr int ns(int s) {                                          \
      return s == 0 ? 1 : s == 1 ? R0 : R0 * R1;                              \
    }                                                                         \
    using Real = REAL_;                                                       \
    static constexpr int V = V_;                                              \
    /* stage twiddles also stored as [r][k] after the N-entry table */        \
    static constexpr bool TT = sizeof(REAL_) == 4;                            \
    __host__ __device__ static constexpr int tt_off(int s) {                  \
      return s <= 1 ? 0 : tt_off(s - 1) + (radix(s - 1) - 1) * ns(s - 1);     \
    }                                                                         \
  };
MSF_SHAPE(64, float, 0, 8, 2, 8, 8, 1)
MSF_SHAPE(128, float, 0, 16, 2, 16, 8, 1)
MSF_SHAPE(256, float, 0, 16, 2, 16, 16, 1)
MSF_SHAPE(512, float, 0, 32, 2, 32, 16, 1)
MSF_SHAPE(1024, float, 0, 32, 2, 32, 32, 1)
MSF_SHAPE(2048, float, 0, 32, 3, 32, 8, 8)
MSF_SHAPE(4096, float, 0, 16, 3, 16, 16, 16)
MSF_SHAPE(256, float, 1, 8, 3, 8, 8, 4)
MSF_SHAPE(512, float, 1, 16, 3, 16, 16, 2)
MSF_SHAPE(1024, float, 1, 16, 3, 16, 16, 4)
MSF_SHAPE(2048, float, 1, 16, 3, 16, 16, 8)
MSF_SHAPE(64, double, 0, 8, 2, 8, 8, 1)
MSF_SHAPE(128, double, 0, 16, 2, 16, 8, 1)
MSF_SHAPE(256, double, 0, 16, 2, 16, 16, 1)
MSF_SHAPE(512, double, 0, 8, 3, 8, 8, 8)
MSF_SHAPE(1024, double, 0, 16, 3, 16, 16, 4)
MSF_SHAPE(2048, double, 0, 16, 3, 16, 16, 8)
MSF_SHAPE(4096, double, 0, 16, 3, 16, 16, 16)
#undef MSF_SHAPE

// Where a TT shape's stage copies start in the FP32 table: after the N plain
// entries for the main schedule (V = 0), after those and the main
// schedule's copies for the alternative one (V = 1).
template <class Sh>
__host__ __device__ constexpr int tt_base() {
  if constexpr (Sh::V == 0) {
    return Sh::N;
  } else {
    using S0 = Shape<Sh::N, typename Sh::Real, 0>;
    return S0::N + S0::tt_off(S0::S);
  }
}

// Worst bank multiplicity of one shared-memory access phase (128 bytes of
// lanes) over the exchanges of a line FFT, for lines `stride` elements
// apart.  Lanes are numbered lane = line_fast ? line + LINES*t : t + T*line;
// `line_fast` is the column pass's thread order (column index fastest).
template <class Sh, int ELEM_BYTES>
constexpr int bank_conflicts(int stride, int lines, bool line_fast) {
  const int P = 128 / ELEM_BYTES;           // lanes per conflict-free phase
  const int units = 128 / ELEM_BYTES;       // distinct bank slots per phase
  const int shift = ilog2(Sh::R0);
  int worst = 1;
  for (int s = 0; s + 1 < Sh::S; ++s) {     // exchange after stage s
    const int R = Sh::radix(s), NB = Sh::E / R, NS = Sh::ns(s);
    const int R2 = Sh::radix(s + 1), NB2 = Sh::E / R2;
    for (int pass = 0; pass < 2; ++pass) {  // 0: writes, 1: reads of next stage
      const int cnt_b = pass == 0 ? NB : NB2, cnt_r = pass == 0 ? R : R2;
      for (int b = 0; b < cnt_b; ++b)
        for (int r = 0; r < cnt_r; ++r) {
          int hits[32] = {};
          for (int lane = 0; lane < P; ++lane) {
            const int line = line_fast ? lane % lines : (Sh::T >= P ? 0 : lane / Sh::T);
            const int t = line_fast ? lane / lines : (Sh::T >= P ? lane : lane % Sh::T);
            const int j = t + Sh::T * b;
            const int a = pass == 0 ? (j / NS) * NS * R + (j % NS) + r * NS
                                    : j + r * (Sh::N / R2);
            const int addr = line * stride + a + (a >> shift);
            const int u = addr % units;
            hits[u] += 1;
            if (hits[u] > worst) worst = hits[u];
          }
        }
    }
  }
  return worst;
}

// Line stride (elements) with the fewest bank conflicts among the
// candidates base .. base + 16 (base = N plus one padding slot every R0).
template <class Sh, int ELEM_BYTES, int LINES, bool LINE_FAST>
constexpr int best_stride() {
  const int base = Sh::N + (Sh::N >> ilog2(Sh::R0));
  int best = base + 1, best_c = 1 << 30;
  for (int k = 0; k <= 16; ++k) {
    const int c = bank_conflicts<Sh, ELEM_BYTES>(base + k, LINES, LINE_FAST);
    if (c < best_c) { best_c = c; best = base + k; }
  }
  return best;
}

// Shared-memory line layout: one padding slot every R0 elements keeps the
// stride-R0 writes of the first exchange conflict-free; the line stride is
// chosen so lines sharing an access phase (columns of a column pass, short
// rows of a row pass) fall on different banks.
template <class Sh, int ELEM_BYTES = 8, int LINES = 1, bool LINE_FAST = false>
struct Smem {
  static constexpr int pad_shift = ilog2(Sh::R0);
  static constexpr int stride = best_stride<Sh, ELEM_BYTES, LINES, LINE_FAST>();
  __device__ __forceinline__ static int at(int a) { return a + (a >> pad_shift); }
};

// Transform one line in place.  v[m] holds element t + T*m on entry and
// X[t + T*m] on exit.  `sm` is this line's shared buffer (Smem<Sh>::stride
// elements), `tw` the table e^{-2 pi i m / N}, m < N (for Sh::TT shapes
// followed by each stage s >= 1's factors e^{-2 pi i r k / (NS R)} as
// [r - 1][k], r < R, k < NS, at tt_base<Sh>() + Sh::tt_off(s): copies of table entries,
// laid out so that a warp's lanes read consecutive addresses), and `sync` a
// barrier over all threads that share `sm` lines with this one.
template <class Sh, bool INV, typename C, class Sync>
__device__ __forceinline__ void fft_line(C (&v)[Sh::E], C* __restrict__ sm,
                                         int t, const C* __restrict__ tw,
                                         Sync&& sync) {
  constexpr int N = Sh::N, E = Sh::E, T = Sh::T;
  using SM = Smem<Sh>;
  sfor<0, Sh::S>([&](auto sI) {
    constexpr int s = decltype(sI)::value;
    constexpr int R = Sh::radix(s);
    constexpr int NB = E / R;
    constexpr int NS = Sh::ns(s);
    if constexpr (s > 0) {
      sfor<0, NB>([&](auto bI) {
        constexpr int b = decltype(bI)::value;
        const int j = t + T * b;
        sfor<0, R>([&](auto rI) {
          constexpr int r = decltype(rI)::value;
          v[b + r * NB] = sm[SM::at(j + r * (N / R))];
        });
      });
    }
    sfor<0, NB>([&](auto bI) {
      constexpr int b = decltype(bI)::value;
      if constexpr (NS > 1) {
        const int j = t + T * b;
        const int k = j & (NS - 1);
        sfor<1, R>([&](auto rI) {
          constexpr int r = decltype(rI)::value;
          // keep at most kLoadChunk table loads in flight: bounds the
          // registers the compiler spends on hoisted twiddles
          if constexpr (r % kLoadChunk == 0) load_fence();
          // Sh::TT: the same value from the stage's [r][k] copy, so that
          // the lanes of a warp (consecutive k) read consecutive entries
          const C w = Sh::TT ? __ldg(&tw[tt_base<Sh>() + Sh::tt_off(s) + (r - 1) * NS + k])
                             : __ldg(&tw[r * k * (N / (NS * R))]);
          v[b + r * NB] = INV ? cmulc(v[b + r * NB], w) : cmul(v[b + r * NB], w);
        });
      }
      dft<R, INV, b, NB>(v);
    });
    if constexpr (s + 1 < Sh::S) {
      sync();
      sfor<0, NB>([&](auto bI) {
        constexpr int b = decltype(bI)::value;
        const int j = t + T * b;
        const int base = (j / NS) * NS * R + (j & (NS - 1));
        sfor<0, R>([&](auto rI) {
          constexpr int r = decltype(rI)::value;
          sm[SM::at(base + r * NS)] = v[b + r * NB];
        });
      });
      sync();
    }
  });
}

}  // namespace msf
