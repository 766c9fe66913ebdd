// Launchers for every pass kernel of one (precision, transform length L).
// Each instantiation unit (inst_<prec>_<L>.cu) compiles one KernelSet, so the
// build parallelises over lengths.
#pragma once

#include <cuda_runtime.h>

#include "euler_kernels.cuh"
#include "zfused.cuh"
#include "zpass.cuh"

namespace azb {

// COLK_PAD_INV_WIDE: the padding inverse pass that reads the state (the first
// pass of a 3-D right-hand side), on tiles of TileShape::ncx columns.
enum ColKind : int {
  COLK_PAD_INV = 0,
  COLK_PLAIN_INV = 1,
  COLK_TRUNC_FWD = 2,
  COLK_PLAIN_FWD = 3,
  COLK_PAD_INV_WIDE = 4
};

// Tile shapes of one (precision, L).  Threads per CTA and shared memory
// follow from them; they are the knobs a tuner turns.
struct TileShape {
  int nc;     // columns per CTA, column passes
  int ncx;    // columns per CTA, the first (state-reading) pass of a 3-D right-hand side
  int nlp2;   // line pairs per CTA, 2-D product pass
  int nlp3;   // line pairs per CTA, 3-D product pass
  int ncm2;   // modes per CTA, 2-D epilogue pass
  int ncm3;   // modes per CTA, 3-D epilogue pass
  int nlpr;   // line pairs per CTA, plain r2c / c2r
};

// Every launcher takes the plan variant v (0 std, 1 wide; see Plan<L, V>).
struct KernelSet {
  int L;
  int precision;  // 0 FP64, 1 FP32
  TileShape tiles[2];  // per plan variant (bit 0 of a variant number)
  cudaError_t (*cols)(int v, int kind, const ColArgs&, unsigned gx, unsigned gy, unsigned gz, cudaStream_t);
  cudaError_t (*rows_product)(int v, int dim, const RowArgs&, unsigned gx, unsigned gy, cudaStream_t);
  // Bulk-copy form of the product pass (plan variant v & 1).
  cudaError_t (*zpass)(int v, int dim, const ZArgs&, cudaStream_t);
  // Fused product pass (bit 0: forward plan, bit 1: inverse plan).
  cudaError_t (*zfused)(int v, int dim, const ZArgs&, cudaStream_t);
  cudaError_t (*epilogue)(int v, int dim, const EpiArgs&, unsigned gx, unsigned gy, cudaStream_t);
  cudaError_t (*c2r)(int v, const RealRowArgs&, unsigned gx, cudaStream_t);
  cudaError_t (*r2c)(int v, const RealRowArgs&, unsigned gx, cudaStream_t);
};

constexpr int kpow2floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}
constexpr int kclamp(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

template <typename T, int L, int V> struct Tiles {
  static constexpr int CB = int(sizeof(cvec<T>));
  static constexpr int NC = kclamp(kpow2floor(49152 / (L * CB)), 2, 32);
  // The first pass reads the state in runs of NCX elements per row, rows a
  // plane apart: at least 128 bytes per run where the shared-memory budget
  // of NC allows fewer (measured at L = 768 in FP32: 16 columns 1.48 ms
  // against 8 columns 1.96 ms at 512^3; the other column passes keep NC, for
  // which 16 columns were slower).
  static constexpr int NCX = (CB == 8 && NC * CB < 128 && L <= 768) ? 128 / CB : NC;
  static constexpr int NLP3 = kclamp(kpow2floor(81920 / (L * 6 * CB)), 1, 16);
  static constexpr int NLP2 = kclamp(kpow2floor(81920 / (L * 3 * CB)), 1, 16);
  // FP32 at L = 768: twice the budget, 4 modes per CTA (one CTA per SM;
  // measured 2.95 ms against 3.67 ms with 2 modes at 512^3).
  static constexpr int NCM3 = kclamp(kpow2floor(((CB == 8 && L == 768) ? 163840 : 81920) / (L * 6 * CB)), 1, 16);
  static constexpr int NCM2 = kclamp(kpow2floor(81920 / (L * 3 * CB)), 1, 16);
  static constexpr int NLPR = kclamp(kpow2floor(49152 / (L * CB)), 1, 64);
};

// Line pairs per chunk of k_zfused: a work area of about 80 KB, raised until
// the CTA's thread count is a whole number of warps.
template <typename T, int L, int DIM, int VF> struct ZFTile {
  static constexpr int CB = int(sizeof(cvec<T>));
  static constexpr int NB = DIM * (DIM + 1) / 2;
  static constexpr int TPL = Plan<L, VF>::TPL;
  static constexpr int BUDGET = kclamp(kpow2floor(81920 / (L * NB * CB)), 1, 16);
  static constexpr int G = (TPL % 32 == 0) ? 32 : (TPL % 16 == 0) ? 16 : (TPL % 8 == 0) ? 8
                         : (TPL % 4 == 0) ? 4 : (TPL % 2 == 0) ? 2 : 1;  // gcd(TPL, 32)
  static constexpr int MIN = DIM == 3 ? (G >= 16 ? 1 : 16 / G) : 32 / G;
  static constexpr int NLP = BUDGET > MIN ? BUDGET : MIN;
  static_assert((NB * NLP * TPL) % 32 == 0, "k_zfused needs whole warps");
};

// Line pairs per chunk of k_zpass: about 80 KB of work area, raised until the
// CTA's thread count is a whole number of warps.
template <typename T, int L, int DIM, int V> struct ZTile {
  static constexpr int CB = int(sizeof(cvec<T>));
  static constexpr int NB = DIM * (DIM + 1) / 2;
  static constexpr int TPL = Plan<L, V>::TPL;
  // About 80 KB of work area; 40 KB from L = 768 on, where the twiddle table
  // and the longer lines would otherwise leave room for one CTA per SM.
  static constexpr int BUDGET = kclamp(kpow2floor((L >= 768 ? 40960 : 81920) / (L * NB * CB)), 1, 16);
  static constexpr int G = (TPL % 32 == 0) ? 32 : (TPL % 16 == 0) ? 16 : (TPL % 8 == 0) ? 8
                         : (TPL % 4 == 0) ? 4 : (TPL % 2 == 0) ? 2 : 1;  // gcd(TPL, 32)
  static constexpr int MIN = DIM == 3 ? (G >= 16 ? 1 : 16 / G) : 32 / G;
  static constexpr int NLP = BUDGET > MIN ? BUDGET : MIN;
  static_assert((NB * NLP * TPL) % 32 == 0, "k_zpass needs whole warps");
};

template <typename K> inline cudaError_t set_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

template <typename T, int L, int V> struct LaunchV {
  using C = cvec<T>;
  using TS = Tiles<T, L, V>;
  static constexpr int TPL = Plan<L, V>::TPL;

  template <int S, int MODE, bool STD, int NC>
  static cudaError_t col_kernel_(const ColArgs& a, dim3 g, cudaStream_t st) {
    const size_t smem = size_t(L + L * NC) * sizeof(C);
    auto k = k_cols<T, L, NC, S, MODE, V, STD>;
    static const cudaError_t attr = set_smem(k, smem);
    if (attr != cudaSuccess) return attr;
    k<<<g, NC * TPL, smem, st>>>(a);
    return cudaGetLastError();
  }

  // The padding and truncating passes of the 3/2 rule (n == 2L/3) take the
  // form with the maps folded at compile time.
  template <int S, int MODE, int NC = TS::NC>
  static cudaError_t col_kernel(const ColArgs& a, dim3 g, cudaStream_t st) {
    if constexpr (MODE != COL_PLAIN && L % 3 == 0) {
      if (3LL * a.n_short == 2LL * L) return col_kernel_<S, MODE, true, NC>(a, g, st);
    }
    return col_kernel_<S, MODE, false, NC>(a, g, st);
  }

  // The column kernels index rows with 32-bit offsets.
  static bool rows_fit(const ColArgs& a) {
    const long long lim = 0x7fffffffLL;
    return (long long)L * a.in_row < lim && (long long)L * a.out_row < lim;
  }

  // Two-tile kernel: g.x is the (tile, outer) count; each CTA takes two.
  template <int S, int MODE>
  static cudaError_t col2_kernel(const ColArgs& a, dim3 g, cudaStream_t st) {
    constexpr int NC = TS::NC;
    const size_t smem = size_t(L + 2 * L * NC) * sizeof(C);
    auto k = k_cols2<T, L, NC, S, MODE, V>;
    static const cudaError_t attr = set_smem(k, smem);
    if (attr != cudaSuccess) return attr;
    ColArgs b = a;
    b.nouter_tiles = a.ntile > 0 ? (long long)g.x / a.ntile : 0;
    const dim3 g2((g.x + 1) / 2, g.y, g.z);
    k<<<g2, NC * TPL, smem, st>>>(b);
    return cudaGetLastError();
  }

  static cudaError_t cols2(int kind, const ColArgs& a, dim3 g, cudaStream_t st) {
    switch (kind) {
      case COLK_PAD_INV: return col2_kernel<+1, COL_PAD>(a, g, st);
      case COLK_PLAIN_INV: return col2_kernel<+1, COL_PLAIN>(a, g, st);
      case COLK_TRUNC_FWD: return col2_kernel<-1, COL_TRUNC>(a, g, st);
      case COLK_PLAIN_FWD: return col2_kernel<-1, COL_PLAIN>(a, g, st);
      default: return cudaErrorInvalidValue;
    }
  }

  static cudaError_t cols(int kind, const ColArgs& a, dim3 g, cudaStream_t st) {
    if (!rows_fit(a)) return cudaErrorInvalidValue;
    switch (kind) {
      case COLK_PAD_INV: return col_kernel<+1, COL_PAD>(a, g, st);
      case COLK_PLAIN_INV: return col_kernel<+1, COL_PLAIN>(a, g, st);
      case COLK_TRUNC_FWD: return col_kernel<-1, COL_TRUNC>(a, g, st);
      case COLK_PLAIN_FWD: return col_kernel<-1, COL_PLAIN>(a, g, st);
      case COLK_PAD_INV_WIDE: return col_kernel<+1, COL_PAD, TS::NCX>(a, g, st);
      default: return cudaErrorInvalidValue;
    }
  }

  template <int DIM, int NLP>
  static cudaError_t rows_kernel(const RowArgs& a, dim3 g, cudaStream_t st) {
    constexpr int NB = DIM * (DIM + 1) / 2;
    const size_t smem = size_t(L + L * (NB * NLP + 1)) * sizeof(C);
    auto k = k_rows_product<T, L, NLP, DIM, V>;
    static const cudaError_t attr = set_smem(k, smem);
    if (attr != cudaSuccess) return attr;
    k<<<g, NB * NLP * TPL, smem, st>>>(a);
    return cudaGetLastError();
  }

  static cudaError_t rows(int dim, const RowArgs& a, dim3 g, cudaStream_t st) {
    if (dim == 2) return rows_kernel<2, TS::NLP2>(a, g, st);
    if (dim == 3) return rows_kernel<3, TS::NLP3>(a, g, st);
    return cudaErrorInvalidValue;
  }

  template <int DIM>
  static cudaError_t zpass(const ZArgs& a, cudaStream_t st) {
    constexpr int NLP = ZTile<T, L, DIM, V>::NLP;
    using Z = ZShape<T, L, NLP, DIM, V>;
    auto k = k_zpass<T, L, NLP, DIM, V>;
    const long long smem = Z::smem_bytes(a.in_line);
    if (smem < 0 || smem > 227 * 1024) return cudaErrorInvalidValue;
    if (a.in_line < a.nh * DIM || a.out_line < a.nh * Z::NB) return cudaErrorInvalidValue;
    // The bulk copy needs a 16-byte aligned chunk of whole line pairs.
    const long long lb = (long long)a.in_line * Z::CB;
    if ((reinterpret_cast<uintptr_t>(a.in) & 15) != 0 || (2 * lb) % 16 != 0 ||
        (a.in_mem * Z::CB) % 16 != 0 || (a.nlines & 1) != 0)
      return cudaErrorInvalidValue;
    // Raise the kernel's dynamic shared-memory limit to what this launch needs
    // (the kernel also holds a little static shared memory).
    static long long granted = 48 * 1024;
    if (smem > granted) {
      const cudaError_t ce = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (ce != cudaSuccess) {
        cudaGetLastError();
        return ce;
      }
      granted = smem;
    }
    const long long chunks = (a.nlines + 2 * NLP - 1) / (2 * NLP);
    if (chunks == 0 || a.nmem == 0) return cudaSuccess;
    if (chunks > 0x7fffffffLL || a.nmem > 65535) return cudaErrorInvalidValue;
    k<<<dim3(unsigned(chunks), unsigned(a.nmem)), Z::NT, size_t(smem), st>>>(a);
    return cudaGetLastError();
  }

  static cudaError_t zpass(int dim, const ZArgs& a, cudaStream_t st) {
    if (dim == 2) return zpass<2>(a, st);
    if (dim == 3) return zpass<3>(a, st);
    return cudaErrorInvalidValue;
  }

  // k_zfused with forward plan V (this struct's) and inverse plan VI; the
  // form with nh folded at compile time for the 3/2 rule (nh == L/3 + 1).
  template <int DIM, int VI>
  static cudaError_t zfused(const ZArgs& a0, cudaStream_t st) {
    if constexpr (L % 3 == 0) {
      if (a0.nh == L / 3 + 1) return zfused_<DIM, VI, true>(a0, st);
    }
    return zfused_<DIM, VI, false>(a0, st);
  }

  template <int DIM, int VI, bool STD>
  static cudaError_t zfused_(const ZArgs& a0, cudaStream_t st) {
    constexpr int NLP = ZFTile<T, L, DIM, V>::NLP;
    using Z = ZFShape<T, L, NLP, DIM, V, VI>;
    auto k = k_zfused<T, L, NLP, DIM, V, VI, STD>;
    if (a0.in_line < a0.nh * DIM || a0.out_line < a0.nh * Z::NB) return cudaErrorInvalidValue;
    // Each pair's bulk copy needs 16-byte aligned source, destination and size.
    const long long pair_bytes = 2LL * a0.in_line * Z::CB;
    if ((reinterpret_cast<uintptr_t>(a0.in) & 15) != 0 || pair_bytes % 16 != 0 ||
        (a0.in_mem * Z::CB) % 16 != 0 || (a0.nlines & 1) != 0)
      return cudaErrorInvalidValue;
    ZArgs a = a0;
    a.pstride = zfused_pair_stride(a.in_line, Z::CB, NLP, DIM, Z::CS, Z::NINV);
    const long long smem = Z::smem_bytes(a.pstride);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    static long long granted = 48 * 1024;
    if (smem > granted) {
      const cudaError_t ce = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (ce != cudaSuccess) {
        cudaGetLastError();
        return ce;
      }
      granted = smem;
    }
    const long long chunks = (a.nlines + 2 * NLP - 1) / (2 * NLP);
    if (chunks == 0 || a.nmem == 0) return cudaSuccess;
    if (chunks > 0x7fffffffLL || a.nmem > 65535) return cudaErrorInvalidValue;
    k<<<dim3(unsigned(chunks), unsigned(a.nmem)), Z::NT, size_t(smem), st>>>(a);
    return cudaGetLastError();
  }

  static cudaError_t zfused(int vi, int dim, const ZArgs& a, cudaStream_t st) {
    if (dim == 2) return vi ? zfused<2, 1>(a, st) : zfused<2, 0>(a, st);
    if (dim == 3) return vi ? zfused<3, 1>(a, st) : zfused<3, 0>(a, st);
    return cudaErrorInvalidValue;
  }

  template <int DIM, int NCM, bool STD>
  static cudaError_t epi_kernel_(const EpiArgs& a, dim3 g, cudaStream_t st) {
    constexpr int NB = DIM * (DIM + 1) / 2;
    const size_t smem = size_t(L + L * NB * NCM) * sizeof(C);
    auto k = k_fwd_epilogue<T, L, NCM, DIM, V, STD>;
    static const cudaError_t attr = set_smem(k, smem);
    if (attr != cudaSuccess) return attr;
    k<<<g, NB * NCM * TPL, smem, st>>>(a);
    return cudaGetLastError();
  }

  template <int DIM, int NCM>
  static cudaError_t epi_kernel(const EpiArgs& a, dim3 g, cudaStream_t st) {
    if constexpr (L % 3 == 0) {
      if (3LL * a.N == 2LL * L) return epi_kernel_<DIM, NCM, true>(a, g, st);
    }
    return epi_kernel_<DIM, NCM, false>(a, g, st);
  }

  static cudaError_t epi(int dim, const EpiArgs& a, dim3 g, cudaStream_t st) {
    // 32-bit offsets: rows of B and one member's state.
    const long long lim = 0x7fffffffLL;
    if ((long long)L * a.B_row >= lim) return cudaErrorInvalidValue;
    for (const StateLayout& l : {a.lu, a.lu0, a.lout})
      if ((long long)(dim - 1) * l.comp + (long long)(a.N - 1) * l.row + (a.ninner - 1) * l.ps >= lim)
        return cudaErrorInvalidValue;
    if (dim == 2) return epi_kernel<2, TS::NCM2>(a, g, st);
    if (dim == 3) return epi_kernel<3, TS::NCM3>(a, g, st);
    return cudaErrorInvalidValue;
  }

  static cudaError_t c2r(const RealRowArgs& a, unsigned gx, cudaStream_t st) {
    constexpr int NLP = TS::NLPR;
    const size_t smem = size_t(L + L * (NLP + 1)) * sizeof(C);
    auto k = k_rows_c2r<T, L, NLP, V>;
    static const cudaError_t attr = set_smem(k, smem);
    if (attr != cudaSuccess) return attr;
    k<<<gx, NLP * TPL, smem, st>>>(a);
    return cudaGetLastError();
  }

  static cudaError_t r2c(const RealRowArgs& a, unsigned gx, cudaStream_t st) {
    constexpr int NLP = TS::NLPR;
    const size_t smem = size_t(L + L * (NLP + 1)) * sizeof(C);
    auto k = k_rows_r2c<T, L, NLP, V>;
    static const cudaError_t attr = set_smem(k, smem);
    if (attr != cudaSuccess) return attr;
    k<<<gx, NLP * TPL, smem, st>>>(a);
    return cudaGetLastError();
  }

  static TileShape tiles() { return {TS::NC, TS::NCX, TS::NLP2, TS::NLP3, TS::NCM2, TS::NCM3, TS::NLPR}; }
};

template <typename T, int L> struct Launch {
  static cudaError_t cols(int v, int kind, const ColArgs& a, unsigned gx, unsigned gy, unsigned gz,
                          cudaStream_t st) {
    const dim3 g(gx, gy, gz);
    // bit 1: the two-tile kernel, for plain (non-interleaved) inputs whose
    // tile count divides evenly into the grid
    if ((v & 2) && a.in_ci == 1 && a.grp == 0 && a.ntile > 0 && gx % unsigned(a.ntile) == 0 &&
        LaunchV<T, L, 0>::rows_fit(a))
      return (v & 1) ? LaunchV<T, L, 1>::cols2(kind, a, g, st) : LaunchV<T, L, 0>::cols2(kind, a, g, st);
    return (v & 1) ? LaunchV<T, L, 1>::cols(kind, a, g, st) : LaunchV<T, L, 0>::cols(kind, a, g, st);
  }
  static cudaError_t rows_product(int v, int dim, const RowArgs& a, unsigned gx, unsigned gy,
                                  cudaStream_t st) {
    const dim3 g(gx, gy, 1);
    return v ? LaunchV<T, L, 1>::rows(dim, a, g, st) : LaunchV<T, L, 0>::rows(dim, a, g, st);
  }
  static cudaError_t zpass(int v, int dim, const ZArgs& a, cudaStream_t st) {
    return (v & 1) ? LaunchV<T, L, 1>::zpass(dim, a, st) : LaunchV<T, L, 0>::zpass(dim, a, st);
  }
  // v bit 0: forward plan, bit 1: inverse plan
  static cudaError_t zfused(int v, int dim, const ZArgs& a, cudaStream_t st) {
    const int vi = (v >> 1) & 1;
    return (v & 1) ? LaunchV<T, L, 1>::zfused(vi, dim, a, st) : LaunchV<T, L, 0>::zfused(vi, dim, a, st);
  }
  static cudaError_t epilogue(int v, int dim, const EpiArgs& a, unsigned gx, unsigned gy,
                              cudaStream_t st) {
    const dim3 g(gx, gy, 1);
    return v ? LaunchV<T, L, 1>::epi(dim, a, g, st) : LaunchV<T, L, 0>::epi(dim, a, g, st);
  }
  static cudaError_t c2r(int v, const RealRowArgs& a, unsigned gx, cudaStream_t st) {
    return v ? LaunchV<T, L, 1>::c2r(a, gx, st) : LaunchV<T, L, 0>::c2r(a, gx, st);
  }
  static cudaError_t r2c(int v, const RealRowArgs& a, unsigned gx, cudaStream_t st) {
    return v ? LaunchV<T, L, 1>::r2c(a, gx, st) : LaunchV<T, L, 0>::r2c(a, gx, st);
  }
  static const KernelSet* get() {
    static const KernelSet ks = {L,
                                 sizeof(T) == 8 ? 0 : 1,
                                 {LaunchV<T, L, 0>::tiles(), LaunchV<T, L, 1>::tiles()},
                                 &cols,
                                 &rows_product,
                                 &zpass,
                                 &zfused,
                                 &epilogue,
                                 &c2r,
                                 &r2c};
    return &ks;
  }
};

}  // namespace azb

#define AZB_INSTANTIATE(TYPE, TAG, LEN)                              \
  namespace azb {                                                    \
  const KernelSet* kernel_set_##TAG##_##LEN() { return Launch<TYPE, LEN>::get(); } \
  }
