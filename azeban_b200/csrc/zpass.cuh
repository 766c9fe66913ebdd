// Contiguous-axis pass of the right-hand side, fed by a TMA bulk copy.
//
// The work is the same as k_rows_product (c2r of the velocity lines, the CFL
// maximum, B = u (x) u in the reference's component order, r2c of the
// products, bins [0, nh) kept), but the input of a CTA's chunk of 2 NLP lines
// is one contiguous run of global memory, so a single elected thread moves it
// into shared memory with one cp.async.bulk, completing on an mbarrier: no
// thread issues a global load.  The inverse transform's first stage reads the
// half spectra there directly, the Hermitian extension folded into its loads.
// The mbarrier wait is bounded; a wait that runs out sets bit 1 of the
// member's error word, waits (bounded) for the copy to land, and the CTA
// returns.
//
// Reference: the inverse transform, max_norm and computeB of
// IncompressibleEuler::dudt (include/azeban/equations/incompressible_euler.hpp
// :103-120, :168-228) and the forward transform that follows
// (src/azeban/cuda/operations/cufft.cpp:133-149).
#pragma once

#include <type_traits>

#include "euler_kernels.cuh"

namespace azb {

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0u;
}
// Polls of a bounded mbarrier wait (the default of ZArgs::wait_polls, and the
// limit of the wait for an in-flight copy after a wait ran out).
constexpr int kWaitPolls = 1 << 22;
// Bounded wait on one phase of an mbarrier: at most `limit` polls; false if
// the phase did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// One bulk copy global -> shared of `bytes` (a multiple of 16, both addresses
// 16-byte aligned), completing as transaction bytes on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Two adjacent complex elements: one 16-byte store for FP32, else two.
template <typename C> __device__ __forceinline__ void store2(C* dst, C a, C b) {
  if constexpr (sizeof(C) == 8) {
    *reinterpret_cast<float4*>(dst) = make_float4(a.x, a.y, b.x, b.y);
  } else {
    dst[0] = a;
    dst[1] = b;
  }
}

// |x| as its IEEE bit pattern with the sign cleared.  For such patterns the
// unsigned order is the order of the values, and infinity and every NaN sort
// above all finite values, so one unsigned max gives max |x| and tells
// whether a non-finite value was met (the result is >= kInfBits).
template <typename T> struct AbsBits;
template <> struct AbsBits<float> {
  using U = unsigned int;
  static constexpr U kInfBits = 0x7f800000u;
  static __device__ __forceinline__ U of(float x) { return __float_as_uint(x) & 0x7fffffffu; }
  static __device__ __forceinline__ void to_ctrl(Ctrl* c, U b) { atomicMax(&c->umax32, b); }
};
template <> struct AbsBits<double> {
  using U = unsigned long long;
  static constexpr U kInfBits = 0x7ff0000000000000ull;
  static __device__ __forceinline__ U of(double x) {
    return static_cast<U>(__double_as_longlong(x)) & 0x7fffffffffffffffull;
  }
  static __device__ __forceinline__ void to_ctrl(Ctrl* c, U b) { atomicMax(&c->umax64, b); }
};

struct ZArgs {
  const void* in;   // lines of nh x DIM complex, component innermost, in_line apart
  void* out;        // lines of nh x NB complex, component innermost, out_line apart
  const void* tw;
  long long nlines;  // lines per member (even)
  int nh;            // spectral bins per line
  int nmem;          // members
  int in_line, out_line;  // line strides (elements; multiples of 2 lines' 16 bytes)
  long long in_mem, out_mem;  // member strides (elements)
  double norm;       // 1 / (N^{d/2} M^{d/2})
  Ctrl* ctrl;
  int wait_polls;    // limit of the wait for the chunk's bulk copy (kWaitPolls)
  int pstride;       // k_zfused: shared-memory elements between input line pairs
};

// Shared-memory layout of one CTA (bytes), shared by the kernel and its
// launcher: the mbarrier, the twiddle table, the product columns P and the
// velocity columns V.  Two layouts, by element size:
//  - FP32 (REGIONS): P [L][NFWD] and V [L][NINV] are separate regions whose
//    row strides equal their column counts (24 and 12 for 3-D pairs of
//    four).  With columns fastest in the transform's thread mapping a
//    half-warp then covers whole rows, or two rows whose banks do not
//    collide, and the row-wise phases map lanes across pairs as well as
//    rows.  The chunk's input is copied into P, dead until the products.
//  - FP64: one work area [L][NFWD + 1]; P is columns [0, NFWD), V the last
//    NINV of them (VOFF).  The product columns of pair p overlap only
//    velocity columns of pairs <= p, so a thread that owns a row and handles
//    its pairs in order writes the products in place.  The input has its
//    own buffer.  (Measured faster for 16-byte elements.)
template <typename T, int L, int NLP, int DIM, int V> struct ZShape {
  static constexpr int CB = int(sizeof(cvec<T>));
  static constexpr bool REGIONS = CB == 8;
  // FP32 with an even number of products: the products go to P as 16-byte
  // pairs (with rows of 24 elements a quarter-warp's stores then fall on
  // distinct bank groups)
  static constexpr bool PAIRED = REGIONS && (DIM * (DIM + 1) / 2) % 2 == 0;
  static constexpr int NB = DIM * (DIM + 1) / 2;
  static constexpr int NINV = DIM * NLP;
  static constexpr int NFWD = NB * NLP;
  static constexpr int SP = REGIONS ? NFWD : NFWD + 1;
  static constexpr int SV = REGIONS ? NINV : NFWD + 1;
  static constexpr int VOFF = REGIONS ? 0 : NFWD - NINV;
  static constexpr int TPL = Plan<L, V>::TPL;
  static constexpr int NT = NFWD * TPL;
  // FP32: ask for 16 (std plans) or 12 (wide plans) resident warps per SM, a
  // register cap the compiler meets without spills; FP64 plans need their
  // registers.
  static constexpr int MINB = CB != 8 ? 1 : V == 0 ? (512 + NT - 1) / NT : (384 + NT - 1) / NT;
  static constexpr int OFF_TW = 16;
  static constexpr int OFF_P = OFF_TW + L * CB;
  static constexpr int P_BYTES = ((L * SP * CB + 15) / 16) * 16;
  static constexpr int OFF_V = REGIONS ? OFF_P + P_BYTES : OFF_P + VOFF * CB;
  static constexpr int OFF_IN = REGIONS ? OFF_P : OFF_P + P_BYTES;
  static constexpr int BYTES = REGIONS ? OFF_V + L * SV * CB : OFF_IN;
  // complex elements of one chunk's input (2 NLP lines of in_line)
  static __host__ __device__ long long chunk_elems(int in_line) { return 2LL * NLP * in_line; }
  // -1 when the input does not fit in P (REGIONS), which holds it
  static __host__ __device__ long long smem_bytes(int in_line) {
    if (REGIONS) return chunk_elems(in_line) <= (long long)L * SP ? BYTES : -1;
    return BYTES + chunk_elems(in_line) * CB;
  }
};

// Plan of the inverse transforms: the velocity columns are DIM/NB of the
// product columns, so with the wide plan half (3-D) of the CTA would sit out
// the inverse phase.  The std plan runs more threads per column; take it when
// the CTA has the threads for it, so the inverse phase spreads over the CTA.
template <int L, int V, int NCOL, int NT> struct InvPlan {
  static constexpr bool kStd = V == 1 && NCOL * Plan<L, 0>::TPL <= NT && Plan<L, 0>::TPL > Plan<L, 1>::TPL;
  using type = typename std::conditional<kStd, Plan<L, 0>, Plan<L, V>>::type;
};

template <typename T, int L, int NLP, int DIM, int V>
__global__ void __launch_bounds__(ZShape<T, L, NLP, DIM, V>::NT, ZShape<T, L, NLP, DIM, V>::MINB)
    k_zpass(ZArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  using Z = ZShape<T, L, NLP, DIM, V>;
  constexpr int NB = Z::NB;
  constexpr int NINV = Z::NINV;
  constexpr int NFWD = Z::NFWD;
  constexpr int SP = Z::SP;
  constexpr int SV = Z::SV;
  constexpr int NT = Z::NT;
  extern __shared__ __align__(16) unsigned char az_smem[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(az_smem);
  C* tw = reinterpret_cast<C*>(az_smem + Z::OFF_TW);
  C* pw = reinterpret_cast<C*>(az_smem + Z::OFF_P);
  C* vw = reinterpret_cast<C*>(az_smem + Z::OFF_V);
  const C* cin = reinterpret_cast<const C*>(az_smem + Z::OFF_IN);
  const int member = blockIdx.y;
  Ctrl* ctrl = a.ctrl + member;
  if (ctrl->skip) return;
  const int tid = threadIdx.x;
  const int nh = a.nh;
  const int in_line = a.in_line;
  const int out_line = a.out_line;
  const long long line0 = (long long)blockIdx.x * 2 * NLP;
  // Line pairs of this chunk that exist (nlines is even, so a pair is whole).
  const int npairs = int((a.nlines - line0) / 2 < NLP ? (a.nlines - line0) / 2 : NLP);

  // Elected thread: one bulk copy of the chunk's lines into shared memory.
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_fence_init();
    const unsigned bytes = unsigned(2 * npairs * in_line * Z::CB);
    mbar_expect_tx(&bar[0], bytes);
    bulk_load(az_smem + Z::OFF_IN, reinterpret_cast<const C*>(a.in) + member * a.in_mem + line0 * in_line,
              bytes, &bar[0]);
  }
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar[0], 0u, a.wait_polls);
  if (__syncthreads_or(!ok)) {
    // The wait ran out: flag it (bit 1 of the member's error word), and let
    // one thread wait, bounded, for the copy to land before the CTA exits,
    // so no bulk copy is still writing into shared memory the SM may hand to
    // the next CTA.  The CTA's shared memory stays allocated until its last
    // thread exits.
    if (tid == 0) {
      atomicOr(&ctrl->err, 2);
      mbar_wait_bounded(&bar[0], 0u, kWaitPolls);
    }
    return;
  }
  using AB = AbsBits<T>;
  typename AB::U vbits = 0;  // running max |u| as bits (see AbsBits)

  // 1. Inverse transforms of the velocity columns into V.  Column (pair p,
  //    component q) holds component q of line 2p + i * component q of line
  //    2p+1.  Its first-stage inputs come straight from the chunk's half
  //    spectra: bin k < nh gives row k (X + iY) and row L - k (conj X + i
  //    conj Y); rows [nh, L - nh] are zero.  The imaginary parts of bin 0
  //    and bin L/2 are dropped, as a c2r does.
  {
    using PI = typename InvPlan<L, V, NINV, NT>::type;
    const bool active = tid < NINV * PI::TPL;
    const int col = active ? tid % NINV : 0;
    const int tl = active ? tid / NINV : 0;
    const int p = col / DIM;
    const C* la = cin + (2 * p) * in_line + (col - p * DIM);
    const C* lb = la + in_line;
    const bool live = p < npairs;
    auto load = [&](int m) {
      const bool lo = m < nh;
      const bool hi = m > L - nh;
      const int k = lo ? m : L - m;
      C x = cmk<C>(T(0), T(0)), y = x;
      if (live && (lo || hi)) {
        x = la[k * DIM];
        y = lb[k * DIM];
      }
      if (m == 0 || 2 * m == L) {
        x.y = T(0);
        y.y = T(0);
      }
      return lo ? cmk<C>(x.x - y.y, x.y + y.x) : cmk<C>(x.x + y.y, y.x - x.y);
    };
    fft_columns<C, +1, L, SV, true, PI>(
        vw, tw, col, tl, load, [&](int m, C v) { vw[m * SV + col] = v; }, active);
  }
  __syncthreads();

  // 2. CFL maximum and products B = u (x) u in the reference's component
  //    order (product c of line a in the real part, of line b in the
  //    imaginary part), from V into P.  REGIONS: lanes run over pairs
  //    fastest.  Else a thread owns a row and handles its pairs in order
  //    (each pair's products overwrite only velocity columns already read).
  const T norm = T(a.norm);
  auto product = [&](int m, int p) {
    const C* v = vw + m * SV + p * DIM;
    T u[2 * DIM];
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
      const C z = v[q];
      u[q] = z.x;        // line a
      u[DIM + q] = z.y;  // line b
    }
#pragma unroll
    for (int s = 0; s < 2 * DIM; ++s) {
      const typename AB::U b = AB::of(u[s]);
      vbits = b > vbits ? b : vbits;
      u[s] *= norm;
    }
    C* w = pw + m * SP + p * NB;
    if constexpr (DIM == 2) {
      w[0] = cmk<C>(u[0] * u[0], u[2] * u[2]);
      w[1] = cmk<C>(u[0] * u[1], u[2] * u[3]);
      w[2] = cmk<C>(u[1] * u[1], u[3] * u[3]);
    } else if constexpr (Z::PAIRED) {
      store2(w, cmk<C>(u[0] * u[0], u[3] * u[3]), cmk<C>(u[1] * u[0], u[4] * u[3]));
      store2(w + 2, cmk<C>(u[1] * u[1], u[4] * u[4]), cmk<C>(u[2] * u[0], u[5] * u[3]));
      store2(w + 4, cmk<C>(u[2] * u[1], u[5] * u[4]), cmk<C>(u[2] * u[2], u[5] * u[5]));
    } else {
      w[0] = cmk<C>(u[0] * u[0], u[3] * u[3]);
      w[1] = cmk<C>(u[1] * u[0], u[4] * u[3]);
      w[2] = cmk<C>(u[1] * u[1], u[4] * u[4]);
      w[3] = cmk<C>(u[2] * u[0], u[5] * u[3]);
      w[4] = cmk<C>(u[2] * u[1], u[5] * u[4]);
      w[5] = cmk<C>(u[2] * u[2], u[5] * u[5]);
    }
  };
  if constexpr (Z::REGIONS) {
    for (int idx = tid; idx < L * NLP; idx += NT) product(idx / NLP, idx % NLP);
  } else {
    for (int m = tid; m < L; m += NT) {
#pragma unroll
      for (int p = 0; p < NLP; ++p) product(m, p);
    }
  }
  __syncthreads();

  // 3. Forward transforms of the NFWD product columns, in place in P.
  {
    const int col = tid % NFWD;
    const int tl = tid / NFWD;
    fft_columns<C, -1, L, SP, true, P>(
        pw, tw, col, tl, [&](int m) { return pw[m * SP + col]; },
        [&](int m, C v) { pw[m * SP + col] = v; });
  }
  __syncthreads();

  // 4. Separate the two real spectra and write bins [0, nh), component
  //    fastest, so consecutive threads store consecutive elements of a line.
  C* out = reinterpret_cast<C*>(a.out) + member * a.out_mem + line0 * out_line;
  const int nb_nh = NB * nh;
#pragma unroll 1
  for (int p = 0; p < npairs; ++p) {
    C* oa = out + (2 * p) * out_line;
    C* ob = oa + out_line;
    for (int r = tid; r < nb_nh; r += NT) {
      const int kb = r / NB;
      const int cf = p * NB + (r - kb * NB);
      const C x = pw[kb * SP + cf];
      const C y = pw[(kb == 0 ? 0 : L - kb) * SP + cf];
      oa[r] = cmk<C>(T(0.5) * (x.x + y.x), T(0.5) * (x.y - y.y));
      ob[r] = cmk<C>(T(0.5) * (x.y + y.y), T(-0.5) * (x.x - y.x));
    }
  }

  // CFL reduction: warp, then block, then one atomic per CTA.  A non-finite
  // value sets the error bit; the maximum then records infinity.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const typename AB::U other = __shfl_xor_sync(0xffffffffu, vbits, o);
    vbits = other > vbits ? other : vbits;
  }
  __shared__ typename AB::U red[NT / 32];
  if ((tid & 31) == 0) red[tid >> 5] = vbits;
  __syncthreads();
  if (tid == 0) {
    typename AB::U m = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) m = red[w] > m ? red[w] : m;
    if (m >= AB::kInfBits) {
      atomicOr(&ctrl->err, 1);
      m = AB::kInfBits;
    }
    AB::to_ctrl(ctrl, m);
  }
}

}  // namespace azb
