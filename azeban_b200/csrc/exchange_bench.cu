// A measurement of the exchange between the two stages of a transform, done
// two ways on the 384-point wide plan (radix 16, one exchange, radix 24; the
// plan of the FP32 product pass's forward transforms, 8 threads per column
// with 48 elements each):
//  - through shared memory, as every transform pass does: each thread stores
//    its 48 stage-1 outputs and loads the 48 stage-2 inputs it needs (the
//    pass engine itself, Engine::run);
//  - with warp shuffles: a column's 8 threads sit in consecutive lanes and
//    transpose their data in registers, an 8 x 8 block transpose in three
//    rounds (round i swaps, between lanes t and t ^ 2^i, the blocks whose
//    destination lane differs from the lane in bit i; 24 complex values per
//    lane and round, 144 32-bit shuffles per lane in all).
// Both compute the same transform; the butterflies and twiddles are the
// engine's.  It exists to decide whether warp-shuffle exchanges pay in these
// passes, which are bound by shared-memory traffic (product pass) or by
// instruction issue (the others).
//
// A CTA transforms 32 columns of 384 FP32 complex values held in registers
// `reps` times (each repetition feeds the outputs back in as inputs: the same
// work), so the time per transform follows from two repetition counts.  Both
// forms run two 256-thread CTAs per SM (at most 128 registers per thread; the
// shuffle form then spills 20 bytes per thread); the shuffle form also runs
// without that cap (204 registers, one CTA per SM).
#include <cuda_runtime.h>

#include <cmath>
#include <random>
#include <vector>

#include "runtime_internal.h"

namespace azb {

constexpr int kXbL = 384;
constexpr int kXbThreads = 256;
constexpr int kXbCols = kXbThreads / 8;  // 8 threads per column
using XbPlan = Plan<kXbL, 1>;            // E = 48: radices 16, 24
static_assert(XbPlan::E == 48 && XbPlan::TPL == 8, "wide plan of 384");
using XbEng = Engine<float2, -1, kXbL, 48, kXbCols>;

// Lane transpose among the 8 lanes of a column.  On entry v[16 q + r] is
// row 16 (tl + 8 q) + r of the stage-1 outputs (q < 3, r < 16); it goes to
// lane r mod 8.  On exit v[24 q' + r'] is row (tl + 8 q') + 16 r', the order
// the radix-24 stage reads (Engine::load_smem<24>).
__device__ __forceinline__ void lane_transpose8(float2 (&v)[48], int tl) {
  // S[d][q][h] = v[16 q + 8 h + d]: block d goes to lane d
  float2 S[8][3][2];
#pragma unroll
  for (int d = 0; d < 8; ++d)
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) S[d][q][h] = v[16 * q + 8 * h + d];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const bool bit = (tl >> i) & 1;
#pragma unroll
    for (int d0 = 0; d0 < 8; ++d0) {
      if (d0 & (1 << i)) continue;
      const int d1 = d0 | (1 << i);
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float2 send = bit ? S[d0][q][h] : S[d1][q][h];
          float2 recv;
          recv.x = __shfl_xor_sync(0xffffffffu, send.x, 1 << i);
          recv.y = __shfl_xor_sync(0xffffffffu, send.y, 1 << i);
          if (bit) S[d0][q][h] = recv;
          else S[d1][q][h] = recv;
        }
    }
  }
  // lane tl now holds, in S[s][q][h], row 16 (s + 8 q) + 8 h + tl
#pragma unroll
  for (int s = 0; s < 8; ++s)
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) v[24 * h + s + 8 * q] = S[s][q][h];
}

// METHOD 0: shared-memory exchange (column-fastest threads, as the passes);
// METHOD 1: lane transpose (a column's threads in consecutive lanes).
// MINB: resident CTAs per SM the register allocation is held to.
template <int METHOD, int MINB>
__global__ void __launch_bounds__(kXbThreads, MINB) k_exchange384(const float2* in, float2* out, const float2* twg,
                                                                  int reps) {
  extern __shared__ __align__(16) unsigned char az_smem[];
  float2* tw = reinterpret_cast<float2*>(az_smem);
  float2* sm = tw + kXbL;
  const int tid = threadIdx.x;
  const int col = METHOD == 0 ? tid % kXbCols : (tid / 32) * 4 + (tid % 32) / 8;
  const int tl = METHOD == 0 ? tid / kXbCols : tid % 8;
  const float2* src = in + ((size_t)blockIdx.x * kXbCols + col) * kXbL;
  float2 v[48];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int r = 0; r < 16; ++r) v[16 * q + r] = src[XbEng::in_row<16>(tl, q, r)];
  load_twiddles<float2, kXbL>(tw, twg);
  __syncthreads();
  for (int k = 0; k < reps; ++k) {
    if constexpr (METHOD == 0) {
      XbEng::run<1>(sm, v, col, tl, tw, true, Radices<16, 24>{});
    } else {
      XbEng::compute<1, 16>(v, tl, tw);
      lane_transpose8(v, tl);
      XbEng::compute<16, 24>(v, tl, tw);
    }
  }
  float2* dst = out + ((size_t)blockIdx.x * kXbCols + col) * kXbL;
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int r = 0; r < 24; ++r) dst[XbEng::out_row<24>(tl, q, r)] = v[24 * q + r];
}

}  // namespace azb

using namespace azb;

az_status az_bench_exchange384(int method, int ctas, double* ns_per_column, double* max_rel_err) {
  if (method < 0 || method > 2 || ctas < 1 || ctas > 65535 || !ns_per_column || !max_rel_err)
    return set_error(AZ_ERR_INVALID, "az_bench_exchange384: bad argument");
  const void* tw = nullptr;
  az_status st = device_twiddles(1, kXbL, &tw);
  if (st != AZ_OK) return st;
  const size_t n = size_t(ctas) * kXbCols * kXbL;
  std::vector<float2> h(n), outh(n);
  std::mt19937 rng(2024);
  std::uniform_real_distribution<float> dist(-1.f, 1.f);
  for (auto& v : h) v = make_float2(dist(rng), dist(rng));
  float2 *din = nullptr, *dout = nullptr;
  if (cudaMalloc(&din, n * sizeof(float2)) != cudaSuccess) return set_error(AZ_ERR_NOMEM, "az_bench_exchange384");
  if (cudaMalloc(&dout, n * sizeof(float2)) != cudaSuccess) {
    cudaFree(din);
    return set_error(AZ_ERR_NOMEM, "az_bench_exchange384");
  }
  const size_t smem = sizeof(float2) * (kXbL + (method == 0 ? size_t(kXbL) * kXbCols : 0));
  cudaError_t ce = cudaFuncSetAttribute(method == 0 ? k_exchange384<0, 2> : method == 1 ? k_exchange384<1, 2>
                                                                                       : k_exchange384<1, 1>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  auto launch = [&](int reps) {
    const float2* t = static_cast<const float2*>(tw);
    if (method == 0) k_exchange384<0, 2><<<ctas, kXbThreads, smem>>>(din, dout, t, reps);
    else if (method == 1) k_exchange384<1, 2><<<ctas, kXbThreads, smem>>>(din, dout, t, reps);
    else k_exchange384<1, 1><<<ctas, kXbThreads, smem>>>(din, dout, t, reps);
  };
  auto timed = [&](int reps, double* ms_out) {
    launch(reps);  // warm-up
    cudaEventRecord(e0);
    launch(reps);
    cudaEventRecord(e1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    *ms_out = double(ms);
    return e;
  };
  if (ce == cudaSuccess) ce = cudaMemcpy(din, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
  double t1 = 0, t2 = 0;
  const int r1 = 8, r2 = 40;
  if (ce == cudaSuccess) ce = timed(r1, &t1);
  if (ce == cudaSuccess) ce = timed(r2, &t2);
  if (ce == cudaSuccess) {
    launch(1);  // one transform, for the accuracy check
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpy(outh.data(), dout, n * sizeof(float2), cudaMemcpyDeviceToHost);
  cudaFree(din);
  cudaFree(dout);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  *ns_per_column = (t2 - t1) * 1e6 / (double(r2 - r1) * ctas * kXbCols);
  // accuracy of one transform against an FP64 DFT on a few columns
  double err = 0, ref_max = 0;
  const int check = 8;
  for (int c = 0; c < check; ++c) {
    const float2* x = h.data() + size_t(c) * kXbL;
    for (int k = 0; k < kXbL; ++k) {
      double re = 0, im = 0;
      for (int m = 0; m < kXbL; ++m) {
        const double a = -2.0 * 3.14159265358979323846 * double((long long)k * m % kXbL) / kXbL;
        re += x[m].x * std::cos(a) - x[m].y * std::sin(a);
        im += x[m].x * std::sin(a) + x[m].y * std::cos(a);
      }
      const float2 y = outh[size_t(c) * kXbL + k];
      err = std::fmax(err, std::hypot(y.x - re, y.y - im));
      ref_max = std::fmax(ref_max, std::hypot(re, im));
    }
  }
  *max_rel_err = err / ref_max;
  return AZ_OK;
}
