// Fused transform passes of the spectral-viscosity incompressible Euler
// right-hand side, and the plain real/complex transform passes of FFT<Dim>.
//
// One 3-D right-hand side (reference: IncompressibleEuler::dudt,
// include/azeban/equations/incompressible_euler.hpp:103-120) runs as five
// passes, each one HBM read and one HBM write of the live array.  The
// intermediates keep the component index innermost, so a tile of consecutive
// columns is one contiguous run per row in every pass:
//   1 k_cols<PAD,  inverse>  along x: u_hat [3][N][N][Nh] -> A1 [M][N][Nh][3]
//                            (copy_to_padded along x fused into the loads)
//   2 k_cols<PAD,  inverse>  along y: A1 -> A2 [M][M][Nh][3]
//   3 k_rows_product         along z: c2r, max|u|, B = u (x) u, r2c, keep
//                            k < Nh: A2 -> B1 [M][M][Nh][6]
//   4 k_cols<TRUNC, forward> along y, keep the N retained rows: B1 -> B2 [M][N][Nh][6]
//   5 k_fwd_epilogue         along x, keep retained rows, then computeDudt
//                            (Leray projection of i k.B, spectral viscosity)
//                            and the SSP-RK3 stage combination: B2 + u -> out
// 2-D uses passes 1 (along x), 3 (along y) and 5, with A1 [M][Nh][2] and
// B1 [M][Nh][3].
#pragma once

#include "az_types.h"
#include "fft_core.cuh"

namespace azb {

enum ColMode : int { COL_PLAIN = 0, COL_PAD = 1, COL_TRUNC = 2 };

// Padded row m -> source row of an axis of unpadded length n, or -1 for a
// zero (copy_to_padded_functions.hpp:36-51 in the reference; the Nyquist
// index n/2 stays on the positive side).
__device__ __forceinline__ int pad_src_row(int m, int n, int L) {
  if (m < n / 2 + 1) return m;
  if (m < n / 2 + 1 + L - n) return -1;
  return m - (L - n);
}

// Padded row m -> retained row of the unpadded axis, or -1 if dropped
// (inverse of i_B = i >= n/2+1 ? L - n + i : i, incompressible_euler.hpp:294-299).
__device__ __forceinline__ int retained_row(int m, int n, int L) {
  if (m <= n / 2) return m;
  if (m >= L - n / 2 + 1) return m - (L - n);
  return -1;
}

struct ColArgs {
  const void* in;
  void* out;
  const void* tw;
  long long ninner;  // contiguous columns per slab
  int ntile;         // ceil(ninner / NC)
  int n_short;       // unpadded length (input rows for PAD, output rows for TRUNC)
  long long in_row, out_row;
  long long in_outer, out_outer;
  long long in_comp, out_comp;
  long long in_mem, out_mem;
  Ctrl* ctrl;     // optional: per-member skip flags
  int clear_max;  // nonzero: also reset the member's CFL accumulator
  int in_ci;      // input component interleave: column p reads component p % in_ci
                  // at in_comp stride, position p / in_ci (1: plain columns)
  long long nouter_tiles;  // outer slabs (k_cols2: tile space = ntile * nouter_tiles)
  // Grouped columns (grp > 0): column p is entry q = p % grp of group
  // g = p / grp; entries q >= grp_valid are padding (not read, not written),
  // and the input of entry q sits at g * in_grp + (q / in_ci or q).
  int grp, grp_valid;
  long long in_grp;
};

// Batched column transforms along a strided axis.  grid = (ntile * nouter,
// ncomp, nmembers); block = NC * L/E threads.
// STD: the unpadded length is 2L/3 (the 3/2 rule, a.n_short == 2L/3), known at
// compile time, so the padding and truncation maps fold: rows whose fate does
// not depend on the thread's row offset are kept, zeroed or dropped without a
// test.
template <typename T, int L, int NC, int S, int MODE, int V, bool STD = false>
__global__ void __launch_bounds__(NC * Plan<L, V>::TPL) k_cols(ColArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  extern __shared__ __align__(16) unsigned char az_smem[];
  C* tw = reinterpret_cast<C*>(az_smem);
  C* sm = tw + L;
  const int member = blockIdx.z;
  if (a.ctrl != nullptr) {
    if (a.ctrl[member].skip) return;
    // The CFL accumulator is read only after the product pass of this
    // right-hand side, which runs after this kernel.
    if (a.clear_max && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
      a.ctrl[member].umax64 = 0ull;
      a.ctrl[member].umax32 = 0u;
    }
  }
  const int tile = blockIdx.x % a.ntile;
  const int outer = blockIdx.x / a.ntile;
  const int comp = blockIdx.y;
  const int col = threadIdx.x % NC;
  const int tl = threadIdx.x / NC;
  const long long p = (long long)tile * NC + col;
  bool valid = p < a.ninner;
  long long pin;
  if (a.grp > 0) {
    const long long g = p / a.grp;
    const int q = int(p - g * a.grp);
    valid = valid && q < a.grp_valid;
    pin = g * a.in_grp + (a.in_ci == 1 ? comp * a.in_comp + q : (q % a.in_ci) * a.in_comp + q / a.in_ci);
  } else {
    pin = a.in_ci == 1 ? comp * a.in_comp + p : (p % a.in_ci) * a.in_comp + p / a.in_ci;
  }
  const C* in = reinterpret_cast<const C*>(a.in) + member * a.in_mem + outer * a.in_outer + pin;
  C* out = reinterpret_cast<C*>(a.out) + member * a.out_mem + comp * a.out_comp +
           outer * a.out_outer + p;
  const int n = STD ? 2 * L / 3 : a.n_short;
  // Row offsets fit 32 bits (the launcher checks L * stride < 2^31).
  const int in_row = int(a.in_row);
  const int out_row = int(a.out_row);
  auto load = [&](int m) -> C {
    int src = m;
    if constexpr (MODE == COL_PAD) src = pad_src_row(m, n, L);
    if (!valid || src < 0) return cmk<C>(T(0), T(0));
    return in[src * in_row];
  };
  auto store = [&](int m, C v) {
    int dst = m;
    if constexpr (MODE == COL_TRUNC) dst = retained_row(m, n, L);
    if (valid && dst >= 0) out[dst * out_row] = v;
  };
  // The first-stage loads go out before the twiddle table is fetched, so the
  // two global round trips overlap.
  C v[P::E];
  fft_load<C, L, P>(v, tl, load);
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
  __syncthreads();
  fft_run<C, S, L, NC, false, P>(sm, v, tw, col, tl, store);
}

// Two-tile form of k_cols for plain (non-interleaved) inputs: a CTA takes
// tiles 2 bx and 2 bx + 1 of the (tile, outer) space, starts cp.async copies
// of both tiles' input rows into two shared buffers at once, transforms the
// first in place while the second's copies are in flight, then the second.
// Each thread copies its own column (col = tid % NC) on rows tid / NC + k L/E,
// so a copy costs a pointer step and one cp.async.
// grid = (ceil(ntile * nouter / 2), ncomp, nmembers); block = NC * L/E.
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* smem_dst, const void* gsrc, bool valid) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  const int n = valid ? BYTES : 0;
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(n) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(n) : "memory");
  }
}

template <typename T, int L, int NC, int S, int MODE, int V>
__global__ void __launch_bounds__(NC * Plan<L, V>::TPL) k_cols2(ColArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  constexpr int TPL = P::TPL;
  extern __shared__ __align__(16) unsigned char az_smem[];
  C* tw = reinterpret_cast<C*>(az_smem);
  C* buf0 = tw + L;
  const int member = blockIdx.z;
  if (a.ctrl != nullptr) {
    if (a.ctrl[member].skip) return;
    if (a.clear_max && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
      a.ctrl[member].umax64 = 0ull;
      a.ctrl[member].umax32 = 0u;
    }
  }
  const int col = threadIdx.x % NC;
  const int tl = threadIdx.x / NC;
  const int comp = blockIdx.y;
  const int n = a.n_short;
  const int in_rows = MODE == COL_PAD ? n : L;
  const int in_row = int(a.in_row);
  const int out_row = int(a.out_row);
  const long long t0 = 2LL * blockIdx.x;
  const long long tcount = (long long)a.ntile * a.nouter_tiles;
  const int ntiles_here = t0 + 1 < tcount ? 2 : 1;
  // Issue the copies of both tiles.
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (h < ntiles_here) {
      const long long t = t0 + h;
      const long long tile = t % a.ntile, outer = t / a.ntile;
      const long long p = tile * NC + col;
      const bool valid = p < a.ninner;
      const C* src = reinterpret_cast<const C*>(a.in) + member * a.in_mem + outer * a.in_outer +
                     comp * a.in_comp + (valid ? p : 0);
      C* dst = buf0 + h * (L * NC) + col;
      for (int r = tl; r < in_rows; r += TPL) cp_async_zfill<sizeof(C)>(dst + r * NC, src + r * in_row, valid);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (h == 0) {
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    if (h < ntiles_here) {
      const long long t = t0 + h;
      const long long tile = t % a.ntile, outer = t / a.ntile;
      const long long p = tile * NC + col;
      const bool valid = p < a.ninner;
      C* out = reinterpret_cast<C*>(a.out) + member * a.out_mem + comp * a.out_comp + outer * a.out_outer + p;
      C* sm = buf0 + h * (L * NC);
      fft_columns<C, S, L, NC, false, P>(
          sm, tw, col, tl,
          [&](int m) -> C {
            int src = m;
            if constexpr (MODE == COL_PAD) src = pad_src_row(m, n, L);
            return src >= 0 ? sm[src * NC + col] : cmk<C>(T(0), T(0));
          },
          [&](int m, C v) {
            int dst = m;
            if constexpr (MODE == COL_TRUNC) dst = retained_row(m, n, L);
            if (valid && dst >= 0) out[dst * out_row] = v;
          });
    }
  }
}

struct RowArgs {
  const void* in;   // lines of nh x DIM complex, component innermost
  void* out;        // lines of nh x NB complex, component innermost
  const void* tw;
  long long nlines;  // lines per member
  int nh;            // spectral bins per line (N/2+1)
  long long in_line, out_line;
  long long in_mem, out_mem;
  double norm;  // 1 / (N^{d/2} M^{d/2})
  Ctrl* ctrl;
};

template <typename T> __device__ __forceinline__ void atomic_max_abs(Ctrl* c, T v);
template <> __device__ __forceinline__ void atomic_max_abs<double>(Ctrl* c, double v) {
  atomicMax(&c->umax64, (unsigned long long)__double_as_longlong(v));
}
template <> __device__ __forceinline__ void atomic_max_abs<float>(Ctrl* c, float v) {
  atomicMax(&c->umax32, __float_as_uint(v));
}

// Hermitian extension of a half spectrum: bin m of the length-L spectrum of a
// real signal whose bins [0, nh) are stored at line[bin * stride] (nullptr:
// all zero).  The imaginary parts of bin 0 and of bin L/2 are dropped, as a
// c2r does.
template <typename C, int L>
__device__ __forceinline__ C herm_bin(const C* line, int nh, int m, int stride = 1) {
  using T = decltype(C::x);
  const bool mirror = m > L / 2;
  const int mm = mirror ? L - m : m;
  C v = cmk<C>(T(0), T(0));
  if (line != nullptr && mm < nh) v = line[mm * stride];
  if (mirror) v.y = -v.y;
  if (m == 0 || 2 * m == L) v.y = T(0);
  return v;
}

// Contiguous-axis pass of the right-hand side: for each pair of lines, the
// inverse real transform of the DIM velocity components (two real signals per
// complex transform, the first stage loaded straight from global memory with
// the Hermitian extension), the CFL maximum, the products B = u (x) u in the
// reference's component order, and the forward real transform of the
// products, of which only bins [0, nh) are written.
// grid = (ceil(nlines / (2 NLP)), nmembers); block = NB * NLP * L/E.
template <typename T, int L, int NLP, int DIM, int V>
__global__ void __launch_bounds__((DIM * (DIM + 1) / 2) * NLP * Plan<L, V>::TPL)
    k_rows_product(RowArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  constexpr int NB = DIM * (DIM + 1) / 2;
  constexpr int NINV = DIM * NLP;
  constexpr int NFWD = NB * NLP;
  constexpr int SROW = NFWD + 1;
  constexpr int TPL = P::TPL;
  constexpr int NT = NFWD * TPL;
  extern __shared__ __align__(16) unsigned char az_smem[];
  C* tw = reinterpret_cast<C*>(az_smem);
  C* sm = tw + L;
  const int member = blockIdx.y;
  Ctrl* ctrl = a.ctrl + member;
  if (ctrl->skip) return;
  const int tid = threadIdx.x;
  const long long line0 = (long long)blockIdx.x * 2 * NLP;
  const C* in = reinterpret_cast<const C*>(a.in) + member * a.in_mem;
  C* out = reinterpret_cast<C*>(a.out) + member * a.out_mem;
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
  __syncthreads();

  // 1. Inverse transforms.  Column col = (pair p, component q) holds
  //    component q of line 2p + i * component q of line 2p+1 (the same
  //    component of two neighbouring lines, so the two real signals sharing
  //    a transform have like magnitudes and neither inherits the other's
  //    rounding); its first stage reads global memory directly.
  {
    const bool active = tid < NINV * TPL;
    const int col = active ? tid % NINV : 0;
    const int tl = active ? tid / NINV : 0;
    const int p = col / DIM;
    const int q = col % DIM;
    const long long l0 = line0 + 2 * p;
    const long long l1 = l0 + 1;
    const C* src0 = (active && l0 < a.nlines) ? in + l0 * a.in_line + q : nullptr;
    const C* src1 = (active && l1 < a.nlines) ? in + l1 * a.in_line + q : nullptr;
    const int nh = a.nh;
    fft_columns<C, +1, L, SROW, true, P>(
        sm, tw, col, tl,
        [&](int m) {
          const C x = herm_bin<C, L>(src0, nh, m, DIM);
          const C y = herm_bin<C, L>(src1, nh, m, DIM);
          return cmk<C>(x.x - y.y, x.y + y.x);
        },
        [&](int m, C v) { sm[m * SROW + col] = v; }, active);
  }
  __syncthreads();

  // 2. CFL maximum and products.
  constexpr int MAXI = (NLP * L + NT - 1) / NT;
  T sv[MAXI][2 * DIM];
  T vmax = T(0);
  bool bad = false;
#pragma unroll
  for (int it = 0; it < MAXI; ++it) {
    const int idx = tid + it * NT;
    if (idx < NLP * L) {
      const int m = idx % L;
      const int p = idx / L;
      // sv[it][0, DIM): components of line a, [DIM, 2 DIM): of line b
#pragma unroll
      for (int q = 0; q < DIM; ++q) {
        const C z = sm[m * SROW + p * DIM + q];
        sv[it][q] = z.x;
        sv[it][DIM + q] = z.y;
      }
#pragma unroll
      for (int s = 0; s < 2 * DIM; ++s) {
        const T av = fabs(sv[it][s]);
        bad |= !isfinite(av);
        vmax = fmax(vmax, av);
      }
    }
  }
  __syncthreads();
  const T norm = T(a.norm);
#pragma unroll
  for (int it = 0; it < MAXI; ++it) {
    const int idx = tid + it * NT;
    if (idx < NLP * L) {
      const int m = idx % L;
      const int p = idx / L;
      T pa[NB], pb[NB];
      if constexpr (DIM == 2) {
        const T a1 = norm * sv[it][0], a2 = norm * sv[it][1];
        const T b1 = norm * sv[it][2], b2 = norm * sv[it][3];  // line b
        pa[0] = a1 * a1; pa[1] = a1 * a2; pa[2] = a2 * a2;
        pb[0] = b1 * b1; pb[1] = b1 * b2; pb[2] = b2 * b2;
      } else {
        const T a1 = norm * sv[it][0], a2 = norm * sv[it][1], a3 = norm * sv[it][2];
        const T b1 = norm * sv[it][3], b2 = norm * sv[it][4], b3 = norm * sv[it][5];
        pa[0] = a1 * a1; pa[1] = a2 * a1; pa[2] = a2 * a2;
        pa[3] = a3 * a1; pa[4] = a3 * a2; pa[5] = a3 * a3;
        pb[0] = b1 * b1; pb[1] = b2 * b1; pb[2] = b2 * b2;
        pb[3] = b3 * b1; pb[4] = b3 * b2; pb[5] = b3 * b3;
      }
#pragma unroll
      for (int c = 0; c < NB; ++c) sm[m * SROW + p * NB + c] = cmk<C>(pa[c], pb[c]);
    }
  }
  __syncthreads();

  // 3. Forward transforms of the NFWD product columns (product c of line a
  //    in the real part, of line b in the imaginary part).
  {
    const int col = tid % NFWD;
    const int tl = tid / NFWD;
    fft_columns<C, -1, L, SROW, true, P>(
        sm, tw, col, tl, [&](int m) { return sm[m * SROW + col]; },
        [&](int m, C v) { sm[m * SROW + col] = v; });
  }
  __syncthreads();

  // 4. Separate the two real spectra and write bins [0, nh), component
  //    fastest so the stores of a line are contiguous.
  const int nb_nh = NB * a.nh;
#pragma unroll 1
  for (int p = 0; p < NLP; ++p) {
    const long long la = line0 + 2 * p;
    C* oa = out + la * a.out_line;
    C* ob = oa + a.out_line;
    const bool va = la < a.nlines;
    const bool vb = la + 1 < a.nlines;
    for (int r = tid; r < nb_nh; r += NT) {
      const int k = r / NB;
      const int c = r - k * NB;
      const int cf = p * NB + c;
      const C fk = sm[k * SROW + cf];
      const C fm = sm[(k == 0 ? 0 : L - k) * SROW + cf];
      if (va) oa[r] = cmk<C>(T(0.5) * (fk.x + fm.x), T(0.5) * (fk.y - fm.y));
      if (vb) ob[r] = cmk<C>(T(0.5) * (fk.y + fm.y), T(-0.5) * (fk.x - fm.x));
    }
  }

  // CFL reduction: warp, then block, then one atomic per CTA.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  const unsigned anybad = __any_sync(0xffffffffu, bad);
  __shared__ T red[32];
  __shared__ int redbad;
  if (tid == 0) redbad = 0;
  __syncthreads();
  if ((tid & 31) == 0) {
    red[tid >> 5] = vmax;
    if (anybad) redbad = 1;
  }
  __syncthreads();
  if (tid == 0) {
    T m = T(0);
    for (int w = 0; w < (NT + 31) / 32; ++w) m = fmax(m, red[w]);
    atomic_max_abs<T>(ctrl, m);
    if (redbad) atomicOr(&ctrl->err, 1);
  }
}

// Layout of one member's state: element (component c, retained row i, mode
// p) at c * comp + i * row + p * ps.  Planar, the reference's [d][N]..[Nh]:
// comp = N^{d-1} Nh, row = N^{d-2} Nh, ps = 1.  Component innermost,
// [N]..[Nh][d] (the stepper's stage buffers): comp = 1, row = d N^{d-2} Nh,
// ps = d, so a tile's few modes are d times more contiguous bytes per row.
struct StateLayout {
  int comp, row, ps;
};

struct EpiArgs {
  const void* B;  // [M][modes][NB], component innermost
  const void* u;
  const void* u0;
  void* out;
  const void* tw;
  long long ninner;  // modes per retained row: N*Nh (3-D) or Nh (2-D)
  int ntile;
  int N, nh;
  long long B_row, B_mem;
  StateLayout lu, lu0, lout;  // layouts of u, u0 and out
  long long u_mem;
  int mode;
  Visc visc;
  const Ctrl* ctrl;
  // > 0: B's modes are grouped, nh per group with a group stride of b_grp
  // elements (the padded rows of B2 [M][N][b_grp]); 0: contiguous modes.
  long long b_grp;
};

// nu(|k|) of the reference's viscosity laws
// (include/azeban/equations/spectral_viscosity.hpp:27-123), evaluated from
// |k|^2: SmoothCutoff1D takes (|k|/k0)^2 = |k|^2 / k0^2 and Quadratic
// (|k|/2 pi)^2 = |k|^2 / (2 pi)^2, so neither needs the square root.  Step1D
// compares |k| > k0 as the reference does, on the square root.
template <typename T> __device__ __forceinline__ T visc_from_k2(const Visc& v, T absk2, T inv_k0sq) {
  switch (v.type) {
    case VISC_SMOOTH_CUTOFF: {
      const T k2 = absk2 * inv_k0sq;
      const T k4 = k2 * k2;
      const T k8 = k4 * k4;
      const T k16 = k8 * k8;
      const T k18 = k16 * k2;
      const T q = T(1) - exp(-k18);
      const T pk = (v.s == 1.0) ? absk2 : T(pow(absk2, T(v.s)));
      return -T(v.eps) * pk * q;
    }
    case VISC_STEP: {
      const T k = sqrt(absk2);
      const T q = k > T(v.k0) ? T(1) : T(0);
      const T pk = (v.s == 1.0) ? k * k : T(pow(k, T(2 * v.s)));
      return -T(v.eps) * pk * q;
    }
    case VISC_QUADRATIC: {
      const T kn2 = absk2 * T(1.0 / (4 * 3.14159265358979323846 * 3.14159265358979323846));
      return -T(v.eps) * fmax(T(0), kn2 - T(v.N));
    }
    default:
      return T(0);
  }
}

// Forward transform along x of the NB product components, kept at the N
// retained rows, then per mode: L = (I - k k^T/|k|^2)(i k.B_hat),
// dudt = |k| = 0 ? 0 : -L + nu(|k|) u_hat (incompressible_euler.hpp:230-347,
// incompressible_euler_functions.hpp:47-112), then the stage combination:
//   MODE_DUDT: out = dudt
//   MODE_RK1:  out = u + dt dudt                      (ssp_rk3.hpp:55)
//   MODE_RK2:  out = 3/4 u0 + 1/4 (u + dt dudt)       (ssp_rk3.hpp:57-58)
//   MODE_RK3:  out = 2/3 (u + dt dudt) + 1/3 u0       (ssp_rk3.hpp:60-61)
// grid = (ntile, nmembers); block = NB * NCM * L/E.
// FP32 std plans of up to 384 threads: two resident CTAs per SM.
template <typename T, int L, int NCM, int DIM, int V> struct EpiMinBlocks {
  static constexpr int value =
      (sizeof(T) == 4 && V == 0 && (DIM * (DIM + 1) / 2) * NCM * Plan<L, V>::TPL <= 384) ? 2 : 1;
};

// STD: N == 2L/3 (the 3/2 rule), known at compile time, so the retained-row
// map and the per-mode row loops fold.
template <typename T, int L, int NCM, int DIM, int V, bool STD = false>
__global__ void __launch_bounds__((DIM * (DIM + 1) / 2) * NCM * Plan<L, V>::TPL,
                                  EpiMinBlocks<T, L, NCM, DIM, V>::value)
    k_fwd_epilogue(EpiArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  constexpr int NB = DIM * (DIM + 1) / 2;
  constexpr int NC = NB * NCM;
  constexpr int SROW = NC;
  constexpr int TPL = P::TPL;
  constexpr int NT = NC * TPL;
  extern __shared__ __align__(16) unsigned char az_smem[];
  C* tw = reinterpret_cast<C*>(az_smem);
  C* sm = tw + L;
  const int member = blockIdx.y;
  if (a.ctrl != nullptr && a.ctrl[member].skip) return;
  const int tid = threadIdx.x;
  const int tile = blockIdx.x;
  const int N = STD ? 2 * L / 3 : a.N;
  {
    // column col = (mode pl, component c) with c fastest: one contiguous run
    const int col = tid % NC;
    const int tl = tid / NC;
    const int pl = col / NB;
    const long long p = (long long)tile * NCM + pl;
    const bool valid = p < a.ninner;
    long long bcol;
    if (a.b_grp > 0) {
      const long long g = p / a.nh;
      bcol = g * a.b_grp + (p - g * a.nh) * NB + (col - pl * NB);
    } else {
      bcol = (long long)tile * NC + col;
    }
    const C* Bp = reinterpret_cast<const C*>(a.B) + member * a.B_mem + bcol;
    const int B_row = int(a.B_row);  // L * B_row < 2^31, checked by the launcher
    // First-stage loads before the twiddle table, as in k_cols.
    C v[P::E];
    fft_load<C, L, P>(v, tl, [&](int m) -> C { return valid ? Bp[m * B_row] : cmk<C>(T(0), T(0)); });
    load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
    __syncthreads();
    fft_run<C, -1, L, SROW, true, P>(sm, v, tw, col, tl, [&](int m, C x) {
      const int i = retained_row(m, N, L);
      if (i >= 0) sm[i * SROW + col] = x;
    });
  }
  __syncthreads();

  const double dtd = (a.mode != MODE_DUDT && a.ctrl != nullptr) ? a.ctrl[member].dt : 0.0;
  const T dt = T(dtd);
  const T twopi = T(2 * 3.14159265358979323846);
  const C* u = reinterpret_cast<const C*>(a.u) + member * a.u_mem;
  const C* u0 = reinterpret_cast<const C*>(a.u0) + member * a.u_mem;
  C* out = reinterpret_cast<C*>(a.out) + member * a.u_mem;
  const StateLayout lu = a.lu, lu0 = a.lu0, lout = a.lout;  // offsets < 2^31, checked by the launcher
  const T inv_k0sq = T(1.0 / (a.visc.k0 * a.visc.k0));
  // The stage combination as a uniform coefficient instead of per-element
  // branches: t = u + dt d (d itself for MODE_DUDT), r = ct t + (1 - ct) u0,
  // evaluated as u0 + ct (t - u0) (u0 = 0 and ct = 1 for MODE_DUDT and
  // MODE_RK1).  The weights then sum to exactly one in either precision: with
  // the FP32 weights 2/3 and 1/3 the sum is 1 + 3e-8, which scales the state
  // by that factor at every step.  t - u0 is exact while t and u0 lie within a
  // factor of two (Sterbenz), so the form rounds once, in the fma.
  const bool use_u = a.mode != MODE_DUDT;
  const T dd = use_u ? dt : T(1);
  const T ct = a.mode == MODE_RK2 ? T(0.25) : a.mode == MODE_RK3 ? T(2.0 / 3.0) : T(1);
  // NT is a multiple of NCM, so a thread keeps one mode column pl (and its
  // second and third wavenumbers) and walks the retained rows i.
  const int pl = tid % NCM;
  const int p = tile * NCM + pl;
  if (p >= a.ninner) return;
  T k2, k3;
  if constexpr (DIM == 2) {
    k2 = twopi * T(p);
    k3 = T(0);
  } else {
    const int j = p / a.nh;
    const int kk = p - j * a.nh;
    k2 = twopi * T(j >= N / 2 + 1 ? j - N : j);
    k3 = twopi * T(kk);
  }
  // Rows of this thread: i = tid / NCM + it * ISTEP.  For the first MAXIT
  // rows (all of them when N <= 2L/3 + 1, the 3/2 padding) its state values
  // (u, and u0 for the RK2/RK3 combinations) are loaded first, so their
  // latencies overlap; further rows load as they go.
  constexpr int ISTEP = NT / NCM;
  constexpr int MAXIT = (2 * L / 3 + 1 + ISTEP - 1) / ISTEP;
  const int i0 = tid / NCM;
  const bool need_u0 = a.mode == MODE_RK2 || a.mode == MODE_RK3;
  C uv[MAXIT][DIM], wv[MAXIT][DIM];
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int i = i0 + it * ISTEP;
    if (i < N) {
      const int ou = i * lu.row + p * lu.ps, ow = i * lu0.row + p * lu0.ps;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        uv[it][c] = u[c * lu.comp + ou];
        wv[it][c] = need_u0 ? u0[c * lu0.comp + ow] : cmk<C>(T(0), T(0));
      }
    }
  }
  auto process = [&](int i, const C (&uc_)[DIM], const C (&wc_)[DIM]) {
    const int oo = i * lout.row + p * lout.ps;
    const int i_ = i >= N / 2 + 1 ? i - N : i;
    const T k1 = twopi * T(i_);
    C Bv[NB];
    if constexpr (sizeof(C) == 8 && NB % 2 == 0) {
      // 16-byte reads: with rows of NB * NCM elements a quarter-warp's reads
      // fall on distinct bank groups
      const float4* b4 = reinterpret_cast<const float4*>(sm + i * SROW + pl * NB);
#pragma unroll
      for (int c = 0; c < NB / 2; ++c) {
        const float4 q = b4[c];
        Bv[2 * c] = cmk<C>(q.x, q.y);
        Bv[2 * c + 1] = cmk<C>(q.z, q.w);
      }
    } else {
#pragma unroll
      for (int c = 0; c < NB; ++c) Bv[c] = sm[i * SROW + pl * NB + c];
    }
    // b = i k.B (force = 0), then L = b - k (k.b) / |k|^2
    C Lh[DIM];
    T absk2;
    if constexpr (DIM == 2) {
      absk2 = k1 * k1 + k2 * k2;
      const C b1 = cmk<C>(-k1 * Bv[0].y - k2 * Bv[1].y, k1 * Bv[0].x + k2 * Bv[1].x);
      const C b2 = cmk<C>(-k1 * Bv[1].y - k2 * Bv[2].y, k1 * Bv[1].x + k2 * Bv[2].x);
      const T inv = T(1) / absk2;
      const C sk = cmk<C>((k1 * b1.x + k2 * b2.x) * inv, (k1 * b1.y + k2 * b2.y) * inv);
      Lh[0] = cmk<C>(b1.x - k1 * sk.x, b1.y - k1 * sk.y);
      Lh[1] = cmk<C>(b2.x - k2 * sk.x, b2.y - k2 * sk.y);
    } else {
      absk2 = k1 * k1 + k2 * k2 + k3 * k3;
      // B order: 0 B11, 1 B21, 2 B22, 3 B31, 4 B32, 5 B33
      const C b1 = cmk<C>(-k1 * Bv[0].y - k2 * Bv[1].y - k3 * Bv[3].y,
                          k1 * Bv[0].x + k2 * Bv[1].x + k3 * Bv[3].x);
      const C b2 = cmk<C>(-k1 * Bv[1].y - k2 * Bv[2].y - k3 * Bv[4].y,
                          k1 * Bv[1].x + k2 * Bv[2].x + k3 * Bv[4].x);
      const C b3 = cmk<C>(-k1 * Bv[3].y - k2 * Bv[4].y - k3 * Bv[5].y,
                          k1 * Bv[3].x + k2 * Bv[4].x + k3 * Bv[5].x);
      const T inv = T(1) / absk2;
      const C sk = cmk<C>((k1 * b1.x + k2 * b2.x + k3 * b3.x) * inv, (k1 * b1.y + k2 * b2.y + k3 * b3.y) * inv);
      Lh[0] = cmk<C>(b1.x - k1 * sk.x, b1.y - k1 * sk.y);
      Lh[1] = cmk<C>(b2.x - k2 * sk.x, b2.y - k2 * sk.y);
      Lh[2] = cmk<C>(b3.x - k3 * sk.x, b3.y - k3 * sk.y);
    }
    const T nu = visc_from_k2<T>(a.visc, absk2, inv_k0sq);
    const bool zero = absk2 == T(0);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const C uc = uc_[c];
      const C d = zero ? cmk<C>(T(0), T(0)) : cmk<C>(-Lh[c].x + nu * uc.x, -Lh[c].y + nu * uc.y);
      const C t = use_u ? cmk<C>(uc.x + dd * d.x, uc.y + dd * d.y) : d;
      const C w = wc_[c];
      out[c * lout.comp + oo] = cmk<C>(fma(ct, t.x - w.x, w.x), fma(ct, t.y - w.y, w.y));
    }
  };
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int i = i0 + it * ISTEP;
    if (i < N) process(i, uv[it], wv[it]);
  }
  for (int i = i0 + MAXIT * ISTEP; i < N; i += ISTEP) {
    const int ou = i * lu.row + p * lu.ps, ow = i * lu0.row + p * lu0.ps;
    C uc[DIM], wc[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      uc[c] = u[c * lu.comp + ou];
      wc[c] = need_u0 ? u0[c * lu0.comp + ow] : cmk<C>(T(0), T(0));
    }
    process(i, uc, wc);
  }
}

// ---------------------------------------------------------------------------
// Plain real <-> complex transforms along the contiguous axis (FFT<Dim>).
// Two real lines share one complex transform.
// ---------------------------------------------------------------------------
struct RealRowArgs {
  const void* in;
  void* out;
  const void* tw;
  long long nlines;
  long long in_line, out_line;  // in elements of the respective type
};

// c2r: lines of L/2+1 complex -> L real.  grid = ceil(nlines / (2 NLP)).
template <typename T, int L, int NLP, int V>
__global__ void __launch_bounds__(NLP * Plan<L, V>::TPL) k_rows_c2r(RealRowArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  constexpr int SROW = NLP + 1;
  constexpr int NT = NLP * P::TPL;
  constexpr int LH = L / 2 + 1;
  extern __shared__ __align__(16) unsigned char az_smem[];
  C* tw = reinterpret_cast<C*>(az_smem);
  C* sm = tw + L;
  const int tid = threadIdx.x;
  const long long line0 = (long long)blockIdx.x * 2 * NLP;
  const C* in = reinterpret_cast<const C*>(a.in);
  T* out = reinterpret_cast<T*>(a.out);
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
  for (int idx = tid; idx < NLP * L; idx += NT) {
    const int m = idx % L;
    const int p = idx / L;
    const long long la = line0 + 2 * p;
    const C xa = herm_bin<C, L>(la < a.nlines ? in + la * a.in_line : nullptr, LH, m);
    const C xb = herm_bin<C, L>(la + 1 < a.nlines ? in + (la + 1) * a.in_line : nullptr, LH, m);
    sm[m * SROW + p] = cmk<C>(xa.x - xb.y, xa.y + xb.x);
  }
  __syncthreads();
  {
    const int col = tid % NLP;
    const int tl = tid / NLP;
    fft_columns<C, +1, L, SROW, true, P>(
        sm, tw, col, tl, [&](int m) { return sm[m * SROW + col]; },
        [&](int m, C v) { sm[m * SROW + col] = v; });
  }
  __syncthreads();
  for (int idx = tid; idx < 2 * NLP * L; idx += NT) {
    const int m = idx % L;
    const int ln = idx / L;
    const long long line = line0 + ln;
    if (line < a.nlines) {
      const C z = sm[m * SROW + ln / 2];
      out[line * a.out_line + m] = (ln & 1) ? z.y : z.x;
    }
  }
}

// r2c: lines of L real -> L/2+1 complex.  grid = ceil(nlines / (2 NLP)).
template <typename T, int L, int NLP, int V>
__global__ void __launch_bounds__(NLP * Plan<L, V>::TPL) k_rows_r2c(RealRowArgs a) {
  using C = cvec<T>;
  using P = Plan<L, V>;
  constexpr int SROW = NLP + 1;
  constexpr int NT = NLP * P::TPL;
  constexpr int LH = L / 2 + 1;
  extern __shared__ __align__(16) unsigned char az_smem[];
  C* tw = reinterpret_cast<C*>(az_smem);
  C* sm = tw + L;
  T* smr = reinterpret_cast<T*>(sm);
  const int tid = threadIdx.x;
  const long long line0 = (long long)blockIdx.x * 2 * NLP;
  const T* in = reinterpret_cast<const T*>(a.in);
  C* out = reinterpret_cast<C*>(a.out);
  load_twiddles<C, L>(tw, reinterpret_cast<const C*>(a.tw));
  for (int idx = tid; idx < 2 * NLP * L; idx += NT) {
    const int m = idx % L;
    const int ln = idx / L;
    const long long line = line0 + ln;
    const T x = line < a.nlines ? in[line * a.in_line + m] : T(0);
    smr[2 * (m * SROW + ln / 2) + (ln & 1)] = x;
  }
  __syncthreads();
  {
    const int col = tid % NLP;
    const int tl = tid / NLP;
    fft_columns<C, -1, L, SROW, true, P>(
        sm, tw, col, tl, [&](int m) { return sm[m * SROW + col]; },
        [&](int m, C v) { sm[m * SROW + col] = v; });
  }
  __syncthreads();
  for (int idx = tid; idx < NLP * LH; idx += NT) {
    const int k = idx % LH;
    const int p = idx / LH;
    const C fk = sm[k * SROW + p];
    const C fm = sm[((L - k) % L) * SROW + p];
    const long long la = line0 + 2 * p;
    if (la < a.nlines)
      out[la * a.out_line + k] = cmk<C>(T(0.5) * (fk.x + fm.x), T(0.5) * (fk.y - fm.y));
    if (la + 1 < a.nlines)
      out[(la + 1) * a.out_line + k] = cmk<C>(T(0.5) * (fk.y + fm.y), T(-0.5) * (fk.x - fm.x));
  }
}

// ---------------------------------------------------------------------------
// Control kernels: one thread per solve.
// ---------------------------------------------------------------------------
// Start of a step with a host-given max_dt (TimeIntegrator::integrate).
__global__ void k_ctrl_begin_host(Ctrl* c, int n, double max_dt);
// Start of a step inside simulate_until: max_dt = min(t_end - time, cap)
// (src/azeban/simulation.cpp:91-95); a finished solve is marked skip.
__global__ void k_ctrl_begin_sim(Ctrl* c, int n, double cap);
// Clears the CFL accumulator before a right-hand side.
__global__ void k_ctrl_clear_max(Ctrl* c, int n);
// dt = min(C / (N u_max), max_dt), u_max = max / M^d (incompressible_euler.hpp:116-124).
__global__ void k_ctrl_dt(Ctrl* c, int n, double C, double Nphys, double Md, int fp32);
// time += dt for every solve that stepped (simulation.cpp:100).
__global__ void k_ctrl_end(Ctrl* c, int n);

}  // namespace azb
