// Shared-memory Stockham FFT core for sm_100a.
//
// A CTA transforms NC independent "columns" of length L that live in shared
// memory with layout [row][SROW] (column index fastest, SROW >= NC).  Every
// thread owns one column and E elements of it in registers; it processes
// E/R radix-R butterflies per stage.  Stages exchange data through shared
// memory (in place: read, sync, write, sync).  The first stage may take its
// inputs from anywhere (global memory with a padding map, a packing rule...)
// and the last stage hands its outputs back in registers, so the loads and
// stores of a pass fuse their index maps into the transform itself.
//
// Stockham autosort, for a stage of radix R whose predecessors span NS:
//   butterfly b reads rows b + r*(L/R), r in [0,R),
//   twiddles element r by W_L^{r * (b mod NS) * L/(NS*R)},
//   and writes rows (b/NS)*NS*R + (b mod NS) + r*NS.
// After the last stage row m holds output bin m in natural order.
//
// Both directions are unnormalised: forward uses exp(-2 pi i nk/L), inverse
// exp(+2 pi i nk/L), which is the convention of azeban's FFT<Dim>
// (include/azeban/operations/fft.hpp:80-107 in the reference).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace azb {

template <typename T> struct vec2;
template <> struct vec2<float> { using type = float2; };
template <> struct vec2<double> { using type = double2; };
template <typename T> using cvec = typename vec2<T>::type;

template <typename C> __device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) {
  C r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return cmk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmk<C>(a.x, -a.y); }
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { return cmk<C>(a.x * s, a.y * s); }
// multiply by (S * i): S=+1 -> i*z, S=-1 -> -i*z
template <int S, typename C> __device__ __forceinline__ C cmul_si(C a) {
  if constexpr (S > 0) return cmk<C>(-a.y, a.x);
  else return cmk<C>(a.y, -a.x);
}

// cos(2 pi m / 96) for m in [0, 24], the quarter table every radix in
// {2,3,4,6,8,12,16,24,32,48} needs.  Closed forms evaluated to 25 digits.
__host__ __device__ constexpr double cos96_q(int m) {
  constexpr double q[25] = {1.0,
                            0.9978589232386035067380698,
                            0.9914448613738104111445575,
                            0.9807852804032304491261822,
                            0.9659258262890682867497432,
                            0.9469301294951056642558043,
                            0.9238795325112867561281832,
                            0.8968727415326883038941039,
                            0.8660254037844386467637232,
                            0.8314696123025452370787884,
                            0.7933533402912351645797770,
                            0.7518398074789773964075194,
                            0.7071067811865475244008444,
                            0.6593458151000688684251246,
                            0.6087614290087206394160975,
                            0.5555702330196022247428308,
                            0.5,
                            0.4422886902190012819952390,
                            0.3826834323650897717284600,
                            0.3214394653031615807010576,
                            0.2588190451025207623488988,
                            0.1950903220161282678482849,
                            0.1305261922200515915484062,
                            0.0654031292301430668153156,
                            0.0};
  return q[m];
}
__host__ __device__ constexpr double cos96(int m) {
  m = ((m % 96) + 96) % 96;
  if (m <= 24) return cos96_q(m);
  if (m <= 48) return -cos96_q(48 - m);
  if (m <= 72) return -cos96_q(m - 48);
  return cos96_q(96 - m);
}
__host__ __device__ constexpr double sin96(int m) { return cos96(m - 24); }

// z * w_R^{S*m}, w_R = exp(2 pi i / R), with exact special cases.
template <int R, int S, int M, typename C> __device__ __forceinline__ C rot(C z) {
  constexpr int m = ((M % R) + R) % R;
  if constexpr (m == 0) {
    return z;
  } else if constexpr (2 * m == R) {
    return cmk<C>(-z.x, -z.y);
  } else if constexpr (4 * m == R) {
    return cmul_si<S>(z);
  } else if constexpr (4 * m == 3 * R) {
    return cmul_si<-S>(z);
  } else {
    using T = decltype(C::x);
    static_assert(96 % R == 0, "radix must divide 96");
    constexpr int m96 = m * (96 / R);
    const T c = T(cos96(m96));
    const T s = T(S * sin96(m96));
    return cmk<C>(z.x * c - z.y * s, z.x * s + z.y * c);
  }
}

// ---------------------------------------------------------------------------
// Small DFTs in registers, natural order in and out.  S = -1 forward, +1 inverse.
// ---------------------------------------------------------------------------
template <int R> struct Split;  // R = R1 * R2 for composite radices
template <> struct Split<6> { static constexpr int R1 = 2, R2 = 3; };
template <> struct Split<8> { static constexpr int R1 = 2, R2 = 4; };
template <> struct Split<12> { static constexpr int R1 = 4, R2 = 3; };
template <> struct Split<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Split<24> { static constexpr int R1 = 8, R2 = 3; };
template <> struct Split<32> { static constexpr int R1 = 4, R2 = 8; };
template <> struct Split<48> { static constexpr int R1 = 16, R2 = 3; };

template <int R, int S, typename C> struct DFT;

template <int S, typename C> struct DFT<1, S, C> {
  static __device__ __forceinline__ void run(C*) {}
};

template <int S, typename C> struct DFT<2, S, C> {
  static __device__ __forceinline__ void run(C* v) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int S, typename C> struct DFT<3, S, C> {
  static __device__ __forceinline__ void run(C* v) {
    using T = decltype(C::x);
    const T c = T(-0.5);
    const T s = T(S * 0.8660254037844386467637232);
    const C t1 = cadd(v[1], v[2]);
    const C t2 = cmk<C>(v[0].x + c * t1.x, v[0].y + c * t1.y);
    const C d = csub(v[1], v[2]);
    const C t3 = cmk<C>(-s * d.y, s * d.x);  // i * s * d
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

template <int S, typename C> struct DFT<4, S, C> {
  static __device__ __forceinline__ void run(C* v) {
    const C a = cadd(v[0], v[2]);
    const C b = csub(v[0], v[2]);
    const C c = cadd(v[1], v[3]);
    const C d = cmul_si<S>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  }
};

// FP32 butterflies on the paired FP32 pipe of sm_100 (one instruction adds or
// subtracts both components of a complex value).  a - b is fma(b, -1, a),
// which rounds exactly as the subtraction does, so results are bit-identical
// to the scalar forms above.  Multiplications by +-i stay scalar, where the
// component swap and sign cost nothing.
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}

template <int S> struct DFT<2, S, float2> {
  static __device__ __forceinline__ void run(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = padd(a, b);
    v[1] = psub(a, b);
  }
};

template <int S> struct DFT<3, S, float2> {
  static __device__ __forceinline__ void run(float2* v) {
    const float c = -0.5f;
    const float s = float(S * 0.8660254037844386467637232);
    const float2 t1 = padd(v[1], v[2]);
    const float2 t2 = __ffma2_rn(t1, make_float2(c, c), v[0]);
    const float2 d = psub(v[1], v[2]);
    const float2 t3 = make_float2(-s * d.y, s * d.x);  // i * s * d
    v[0] = padd(v[0], t1);
    v[1] = padd(t2, t3);
    v[2] = psub(t2, t3);
  }
};

template <int S> struct DFT<4, S, float2> {
  static __device__ __forceinline__ void run(float2* v) {
    const float2 a = padd(v[0], v[2]);
    const float2 b = psub(v[0], v[2]);
    const float2 c = padd(v[1], v[3]);
    const float2 t = psub(v[1], v[3]);
    v[0] = padd(a, c);
    v[2] = psub(a, c);
    // d = S i t:  b + d and b - d, componentwise
    if constexpr (S > 0) {
      v[1] = make_float2(b.x - t.y, b.y + t.x);
      v[3] = make_float2(b.x + t.y, b.y - t.x);
    } else {
      v[1] = make_float2(b.x + t.y, b.y - t.x);
      v[3] = make_float2(b.x - t.y, b.y + t.x);
    }
  }
};

// Composite radix R = R1 * R2:  n = R2*n1 + n2, k = k1 + R1*k2.
template <int R, int S, typename C> struct DFT {
  static constexpr int R1 = Split<R>::R1, R2 = Split<R>::R2;
  template <int N2> static __device__ __forceinline__ void inner(C* v, C (&y)[R]) {
    if constexpr (N2 < R2) {
      C t[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + N2];
      DFT<R1, S, C>::run(t);
      twiddle<N2, 0>(t);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) y[N2 * R1 + k1] = t[k1];
      inner<N2 + 1>(v, y);
    }
  }
  template <int N2, int K1> static __device__ __forceinline__ void twiddle(C (&t)[R1]) {
    if constexpr (K1 < R1) {
      t[K1] = rot<R, S, N2 * K1>(t[K1]);
      twiddle<N2, K1 + 1>(t);
    }
  }
  static __device__ __forceinline__ void run(C* v) {
    C y[R];
    inner<0>(v, y);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C t[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) t[n2] = y[n2 * R1 + k1];
      DFT<R2, S, C>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
  }
};

// ---------------------------------------------------------------------------
// Radix plans: product of radices = L, E = elements per thread (a multiple of
// every radix), TPL = L / E threads per column.
// ---------------------------------------------------------------------------
template <int... Rs> struct Radices {};

// Variant 0 ("std") keeps E <= 24; variant 1 ("wide") trades registers for
// fewer stages (one shared-memory exchange per transform where E <= 48 allows).
template <int L, int V = 0> struct Plan;
#define AZB_PLAN(Lv, Vv, Ev, ...)                        \
  template <> struct Plan<Lv, Vv> {                      \
    static constexpr int L = Lv;                         \
    static constexpr int E = Ev;                         \
    static constexpr int TPL = Lv / Ev;                  \
    using R = Radices<__VA_ARGS__>;                      \
  };
AZB_PLAN(4, 0, 4, 4)
AZB_PLAN(6, 0, 6, 6)
AZB_PLAN(8, 0, 8, 8)
AZB_PLAN(12, 0, 12, 12)
AZB_PLAN(16, 0, 16, 16)
AZB_PLAN(24, 0, 24, 8, 3)
AZB_PLAN(32, 0, 8, 8, 4)
AZB_PLAN(48, 0, 24, 8, 6)
AZB_PLAN(64, 0, 8, 8, 8)
AZB_PLAN(96, 0, 24, 8, 12)
AZB_PLAN(128, 0, 16, 8, 16)
AZB_PLAN(192, 0, 24, 8, 4, 6)
AZB_PLAN(256, 0, 16, 16, 16)
AZB_PLAN(384, 0, 24, 8, 8, 6)
AZB_PLAN(512, 0, 8, 8, 8, 8)
AZB_PLAN(768, 0, 24, 8, 8, 12)
AZB_PLAN(1024, 0, 16, 16, 4, 16)
AZB_PLAN(1536, 0, 24, 8, 8, 8, 3)
AZB_PLAN(4, 1, 4, 4)
AZB_PLAN(6, 1, 6, 6)
AZB_PLAN(8, 1, 8, 8)
AZB_PLAN(12, 1, 12, 12)
AZB_PLAN(16, 1, 16, 16)
AZB_PLAN(24, 1, 24, 24)
AZB_PLAN(32, 1, 32, 32)
AZB_PLAN(48, 1, 48, 48)
AZB_PLAN(64, 1, 16, 16, 4)
AZB_PLAN(96, 1, 24, 8, 12)
AZB_PLAN(128, 1, 16, 8, 16)
AZB_PLAN(192, 1, 24, 8, 24)
AZB_PLAN(256, 1, 16, 16, 16)
AZB_PLAN(384, 1, 48, 16, 24)
AZB_PLAN(512, 1, 32, 16, 32)
AZB_PLAN(768, 1, 48, 16, 48)
AZB_PLAN(1024, 1, 32, 32, 32)
AZB_PLAN(1536, 1, 48, 16, 4, 24)
#undef AZB_PLAN

template <typename RL> struct RadixInfo;
template <int... Rs> struct RadixInfo<Radices<Rs...>> {
  template <int A, int... B> static constexpr int first_() { return A; }
  template <int A, int... B> static constexpr int last_() {
    if constexpr (sizeof...(B) == 0) return A; else return last_<B...>();
  }
  static constexpr int first = first_<Rs...>();
  static constexpr int last = last_<Rs...>();
  static constexpr int count = sizeof...(Rs);
};

// ---------------------------------------------------------------------------
// The stage engine.
//   C      complex vector type (float2 / double2)
//   S      -1 forward, +1 inverse
//   L, E   length and elements per thread
//   SROW   shared-memory row stride in elements
// Thread (col, tl): tl in [0, L/E).  v[q*R + r] is element r of butterfly
// b = tl + q*(L/E) of the current stage.
// tw: table of W_L^m = exp(-2 pi i m / L), m in [0, L), in shared memory.
// ---------------------------------------------------------------------------
template <typename C, int S, int L, int E, int SROW>
struct Engine {
  static constexpr int TPL = L / E;

  // Row of element (q, r) of the FIRST stage's inputs (radix R0).
  template <int R0> static __device__ __forceinline__ int in_row(int tl, int q, int r) {
    return tl + q * TPL + r * (L / R0);
  }
  // Row of element (q, r) of the LAST stage's outputs (radix RL).
  template <int RL> static __device__ __forceinline__ int out_row(int tl, int q, int r) {
    return tl + q * TPL + r * (L / RL);
  }

  template <int NS, int R>
  static __device__ __forceinline__ void compute(C (&v)[E], int tl, const C* tw) {
#pragma unroll
    for (int q = 0; q < E / R; ++q) {
      if constexpr (NS > 1) {
        const int b = tl + q * TPL;
        const int j = b % NS;
        const int step = j * (L / (NS * R));
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C w = tw[r * step];
          v[q * R + r] = (S < 0) ? cmul(v[q * R + r], w) : cmulc(v[q * R + r], w);
        }
      }
      DFT<R, S, C>::run(&v[q * R]);
    }
  }

  template <int NS, int R>
  static __device__ __forceinline__ void store_smem(C* sm, const C (&v)[E], int col, int tl,
                                                    bool active) {
    if (!active) return;
#pragma unroll
    for (int q = 0; q < E / R; ++q) {
      const int b = tl + q * TPL;
      const int base = (b / NS) * NS * R + (b % NS);
#pragma unroll
      for (int r = 0; r < R; ++r) sm[(base + r * NS) * SROW + col] = v[q * R + r];
    }
  }

  template <int R>
  static __device__ __forceinline__ void load_smem(const C* sm, C (&v)[E], int col, int tl) {
#pragma unroll
    for (int q = 0; q < E / R; ++q) {
      const int b = tl + q * TPL;
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = sm[(b + r * (L / R)) * SROW + col];
    }
  }

  // Runs every stage.  On entry v holds the first stage's inputs (rows given
  // by in_row<R0>); on exit v holds the last stage's outputs (rows given by
  // out_row<RL>).  Every thread of the CTA must call it (it contains
  // barriers); threads with active == false take part in the barriers only
  // (no arithmetic, no shared-memory traffic).  Each exchange starts with a
  // barrier, so inputs may have come from sm.
  template <int NS, int R, int... Rest>
  static __device__ __forceinline__ void run(C* sm, C (&v)[E], int col, int tl, const C* tw,
                                             bool active, Radices<R, Rest...>) {
    if (active) compute<NS, R>(v, tl, tw);
    if constexpr (sizeof...(Rest) > 0) {
      __syncthreads();
      store_smem<NS, R>(sm, v, col, tl, active);
      __syncthreads();
      constexpr int RN = RadixInfo<Radices<Rest...>>::first;
      if (active) load_smem<RN>(sm, v, col, tl);
      run<NS * R, Rest...>(sm, v, col, tl, tw, active, Radices<Rest...>{});
    }
  }
};

// The first stage's inputs of a thread: v[q R0 + r] = load(in_row(q, r)).
// Split from the transform so a kernel can issue these loads before waiting
// for its twiddle table.
template <typename C, int L, typename P = Plan<L>, typename Load>
__device__ __forceinline__ void fft_load(C (&v)[P::E], int tl, Load&& load, bool active = true) {
  using Info = RadixInfo<typename P::R>;
  using Eng = Engine<C, -1, L, P::E, 1>;
  if (!active) return;
#pragma unroll
  for (int q = 0; q < P::E / Info::first; ++q) {
#pragma unroll
    for (int r = 0; r < Info::first; ++r) {
      v[q * Info::first + r] = load(Eng::template in_row<Info::first>(tl, q, r));
    }
  }
}

// Runs every stage on inputs already in v (from fft_load) and hands the
// outputs to store(row, value).  SYNC_STORE: put a barrier before the stores
// (needed when they go to sm).  Threads with active == false take part in
// the barriers only: they neither load, compute nor store.
template <typename C, int S, int L, int SROW, bool SYNC_STORE, typename P = Plan<L>, typename Store>
__device__ __forceinline__ void fft_run(C* sm, C (&v)[P::E], const C* tw, int col, int tl, Store&& store,
                                        bool active = true) {
  using Info = RadixInfo<typename P::R>;
  using Eng = Engine<C, S, L, P::E, SROW>;
  Eng::template run<1>(sm, v, col, tl, tw, active, typename P::R{});
  if constexpr (SYNC_STORE) __syncthreads();
  if (!active) return;
#pragma unroll
  for (int q = 0; q < P::E / Info::last; ++q) {
#pragma unroll
    for (int r = 0; r < Info::last; ++r) {
      store(Eng::template out_row<Info::last>(tl, q, r), v[q * Info::last + r]);
    }
  }
}

// Runs a full transform of the columns held by this CTA.
//   load(row) -> C     gives the first-stage input at `row`
//   store(row, C)      receives output bin `row`
template <typename C, int S, int L, int SROW, bool SYNC_STORE, typename P = Plan<L>, typename Load,
          typename Store>
__device__ __forceinline__ void fft_columns(C* sm, const C* tw, int col, int tl, Load&& load,
                                            Store&& store, bool active = true) {
  C v[P::E];
  fft_load<C, L, P>(v, tl, load, active);
  fft_run<C, S, L, SROW, SYNC_STORE, P>(sm, v, tw, col, tl, store, active);
}

// Copies the twiddle table W_L^m (m in [0,L)) from global into shared memory.
template <typename C, int L>
__device__ __forceinline__ void load_twiddles(C* tw_sm, const C* tw_g) {
  for (int m = threadIdx.x; m < L; m += blockDim.x) tw_sm[m] = tw_g[m];
}

}  // namespace azb
