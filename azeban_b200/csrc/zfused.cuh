// Contiguous-axis pass of the right-hand side with the products fused into
// the forward transform's loads.
//
// The same work as k_zpass (c2r of the velocity lines, the CFL maximum,
// B = u (x) u in the reference's component order, r2c of the products, bins
// [0, nh) kept), rearranged so the shared-memory traffic per line pair is
// smaller:
//  - the CFL maximum and the 1/(N^{d/2} M^{d/2}) scaling are applied to the
//    inverse transform's outputs in registers, as they are stored;
//  - there is no product phase: the forward transform's first stage reads the
//    two velocity factors of its product column and multiplies them;
//  - input, velocity and product columns share one region (each phase reads
//    its inputs into registers before the barrier that precedes its first
//    store), so a CTA needs one work area instead of two;
//  - each input line pair lands at a stride chosen on the host so that the
//    inverse transform's first-stage reads (the half spectra, Hermitian
//    extension folded in) fall on different banks, and the inverse
//    transform's threads take 16 column slots per row group when the CTA
//    has the threads, so a half-warp reads one row group.
// The mbarrier wait for the bulk copies is bounded as in k_zpass.
//
// Reference: the inverse transform, max_norm and computeB of
// IncompressibleEuler::dudt (include/azeban/equations/incompressible_euler.hpp
// :103-120, :168-228, incompressible_euler_functions.hpp:26-45) and the
// forward transform that follows (src/azeban/cuda/operations/cufft.cpp:133-149).
#pragma once

#include <type_traits>

#include "zpass.cuh"

namespace azb {

// Factors (i, j) of product c in the reference's component order:
// 2-D (11, 12, 22), 3-D (11, 21, 22, 31, 32, 33).
template <int DIM> __device__ __forceinline__ int prod_i(int c) {
  if constexpr (DIM == 2) return c == 2 ? 1 : 0;
  else return c == 0 ? 0 : (c < 3 ? 1 : 2);
}
template <int DIM> __device__ __forceinline__ int prod_j(int c) {
  if constexpr (DIM == 2) return c == 0 ? 0 : 1;
  else return (c == 0 || c == 1 || c == 3) ? 0 : ((c == 2 || c == 4) ? 1 : 2);
}

template <typename T, int L, int NLP, int DIM, int VF, int VI> struct ZFShape {
  static constexpr int CB = int(sizeof(cvec<T>));
  static constexpr int NB = DIM * (DIM + 1) / 2;
  static constexpr int NINV = DIM * NLP;
  static constexpr int NFWD = NB * NLP;
  using PF = Plan<L, VF>;
  static constexpr int NT = NFWD * PF::TPL;
  // The inverse plan asked for, if the CTA has the threads for its columns
  // (2-D has 2/3 as many velocity columns as product columns), else the
  // forward plan.
  using PI = typename std::conditional<NINV * Plan<L, VI>::TPL <= NT, Plan<L, VI>, Plan<L, VF>>::type;
  // Column slots per row group of the inverse transform: NINV rounded up to
  // 16 (or 8) when the CTA has the threads, so a half-warp covers one row
  // group (one tl) of the inverse.
  static constexpr int CS = (NINV <= 16 && 16 * PI::TPL <= NT) ? 16
                            : (NINV <= 8 && 8 * PI::TPL <= NT) ? 8 : NINV;
  static_assert(CS * PI::TPL <= NT, "the inverse transform needs CS * TPL threads");
  static constexpr long long V_ELEMS = (long long)L * NINV;
  static constexpr long long P_ELEMS = (long long)L * NFWD;
  // FP32: a register cap for 12 resident warps per SM; FP64 plans need theirs.
  static constexpr int MINB = CB == 8 ? (NT >= 384 ? 1 : 384 / NT) : 1;
  static constexpr int OFF_TW = 16;
  static constexpr int OFF_W = ((OFF_TW + L * CB + 15) / 16) * 16;
  // pstride: shared-memory elements from one input line pair to the next
  static __host__ __device__ long long smem_bytes(int pstride) {
    const long long in = (long long)NLP * pstride;
    const long long w = in > P_ELEMS ? in : P_ELEMS;
    return OFF_W + w * CB;
  }
};

// STD: nh == L/3 + 1 (the 3/2 rule), known at compile time, so the Hermitian
// read pattern of the inverse transform's first stage and the separation loop
// fold.
template <typename T, int L, int NLP, int DIM, int VF, int VI, bool STD = false>
__global__ void __launch_bounds__(ZFShape<T, L, NLP, DIM, VF, VI>::NT, ZFShape<T, L, NLP, DIM, VF, VI>::MINB)
    k_zfused(ZArgs a) {
  using C = cvec<T>;
  using Z = ZFShape<T, L, NLP, DIM, VF, VI>;
  using PI = typename Z::PI;
  using PF = typename Z::PF;
  constexpr int NB = Z::NB;
  constexpr int NINV = Z::NINV;
  constexpr int NFWD = Z::NFWD;
  constexpr int NT = Z::NT;
  extern __shared__ __align__(16) unsigned char az_smem[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(az_smem);
  C* tw = reinterpret_cast<C*>(az_smem + Z::OFF_TW);
  C* w = reinterpret_cast<C*>(az_smem + Z::OFF_W);
  const int member = blockIdx.y;
  Ctrl* ctrl = a.ctrl + member;
  if (ctrl->skip) return;
  const int tid = threadIdx.x;
  const int nh = STD ? L / 3 + 1 : a.nh;
  const int in_line = a.in_line;
  const int out_line = a.out_line;
  const int pstride = a.pstride;
  const long long line0 = (long long)blockIdx.x * 2 * NLP;
  const int npairs = int((a.nlines - line0) / 2 < NLP ? (a.nlines - line0) / 2 : NLP);

  // Elected thread: one bulk copy per line pair, pair p at w + p * pstride.
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_fence_init();
    const unsigned pair_bytes = unsigned(2 * in_line * Z::CB);
    mbar_expect_tx(&bar[0], unsigned(npairs) * pair_bytes);
    const C* src = reinterpret_cast<const C*>(a.in) + member * a.in_mem + line0 * in_line;
    for (int p = 0; p < npairs; ++p) bulk_load(w + p * pstride, src + 2LL * p * in_line, pair_bytes, &bar[0]);
  }
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar[0], 0u, a.wait_polls);
  if (__syncthreads_or(!ok)) {
    // as in k_zpass: flag, wait (bounded) for the copies to land, return
    if (tid == 0) {
      atomicOr(&ctrl->err, 2);
      mbar_wait_bounded(&bar[0], 0u, kWaitPolls);
    }
    return;
  }
  using AB = AbsBits<T>;
  typename AB::U vbits = 0;
  const T norm = T(a.norm);

  // 1. Inverse transforms of the velocity columns.  Column (pair p,
  //    component q) holds component q of line 2p + i * component q of line
  //    2p+1; its first stage reads the half spectra (bin k < nh gives row k
  //    as X + iY and row L - k as conj X + i conj Y; rows [nh, L - nh] are
  //    zero; the imaginary parts of bins 0 and L/2 are dropped, as a c2r
  //    does).  The outputs are checked into the CFL maximum unscaled, then
  //    scaled by 1/(N^{d/2} M^{d/2}) and stored as V.
  {
    const int col = tid % Z::CS;
    const int tl = tid / Z::CS;
    const bool active = col < NINV && tl < PI::TPL;
    const int p = active ? col / DIM : 0;
    const C* la = w + p * pstride + (active ? col - p * DIM : 0);
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
    C v[PI::E];
    fft_load<C, L, PI>(v, tl, load, active);
    fft_run<C, +1, L, NINV, true, PI>(
        w, v, tw, col, tl,
        [&](int m, C x) {
          const typename AB::U bx = AB::of(x.x), by = AB::of(x.y);
          vbits = bx > vbits ? bx : vbits;
          vbits = by > vbits ? by : vbits;
          w[m * NINV + col] = cmk<C>(x.x * norm, x.y * norm);
        },
        active);
  }
  __syncthreads();

  // 2. Forward transforms of the product columns (product c of line a in the
  //    real part, of line b in the imaginary part); the first stage forms
  //    the products from V.
  {
    const int col = tid % NFWD;
    const int tl = tid / NFWD;
    const int p = col / NB;
    const int c = col - p * NB;
    const int ci = p * DIM + prod_i<DIM>(c);
    const int cj = p * DIM + prod_j<DIM>(c);
    auto load = [&](int m) {
      const C x = w[m * NINV + ci];
      const C y = w[m * NINV + cj];
      return cmk<C>(x.x * y.x, x.y * y.y);
    };
    C v[PF::E];
    fft_load<C, L, PF>(v, tl, load);
    fft_run<C, -1, L, NFWD, true, PF>(w, v, tw, col, tl, [&](int m, C x) { w[m * NFWD + col] = x; });
  }
  __syncthreads();

  // 3. Separate the two real spectra and write bins [0, nh), component
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
      const C x = w[kb * NFWD + cf];
      const C y = w[(kb == 0 ? 0 : L - kb) * NFWD + cf];
      oa[r] = cmk<C>(T(0.5) * (x.x + y.x), T(0.5) * (x.y - y.y));
      ob[r] = cmk<C>(T(0.5) * (x.y + y.y), T(-0.5) * (x.x - y.x));
    }
  }

  // CFL reduction: warp, then block, then one atomic per CTA.
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
    for (int i = 0; i < NT / 32; ++i) m = red[i] > m ? red[i] : m;
    if (m >= AB::kInfBits) {
      atomicOr(&ctrl->err, 1);
      m = AB::kInfBits;
    }
    AB::to_ctrl(ctrl, m);
  }
}

// Shared-memory stride (elements) of one input line pair for k_zfused: at
// least the pair's 2 in_line elements, a multiple of 16 bytes, chosen among
// the next 16-byte steps to minimise the bank conflicts of the inverse
// transform's first-stage reads (a model of one warp's loads: lanes -> (row
// group tl, pair p, component q), word addresses p * pstride + q + DIM * k).
inline int zfused_pair_stride(int in_line, int cb, int nlp, int dim, int cs, int ninv) {
  const int step = 16 / cb;  // elements per 16 bytes
  const int base = ((2 * in_line + step - 1) / step) * step;
  const int group = 128 / cb;  // lanes served by one wavefront (8-byte: 16)
  const int wpe = cb / 4;      // 32-bit words per element
  int best = base, best_cost = 1 << 30;
  for (int k = 0; k < 16; ++k) {
    const int ps = base + k * step;
    int cost = 0;
    for (int dir = 0; dir < 3; ++dir) {      // rows k = m + tl, mirrored rows, line b
      for (int g0 = 0; g0 < 32; g0 += group) {
        int count[32] = {0};
        int seen[64];
        int ns = 0;
        for (int lane = g0; lane < g0 + group; ++lane) {
          const int col = lane % cs, tl = lane / cs;
          if (col >= ninv) continue;
          const int p = col / dim, q = col % dim;
          if (p >= nlp) continue;
          const int kk = dir == 1 ? 64 - tl : 64 + tl;
          const long long e = (long long)p * ps + q + (long long)dim * kk + (dir == 2 ? in_line : 0);
          for (int u = 0; u < wpe; ++u) {
            const int word = int((e * wpe + u) % 1024);
            bool dup = false;
            for (int i = 0; i < ns; ++i) dup = dup || seen[i] == word;
            if (!dup && ns < 64) {
              seen[ns++] = word;
              ++count[word % 32];
            }
          }
        }
        int mx = 0;
        for (int b = 0; b < 32; ++b) mx = count[b] > mx ? count[b] : mx;
        cost += mx;
      }
    }
    if (cost < best_cost) {
      best_cost = cost;
      best = ps;
    }
  }
  return best;
}

}  // namespace azb
