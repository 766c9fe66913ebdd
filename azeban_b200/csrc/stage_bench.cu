// A measurement of one radix-16 DFT stage on a shared-memory tile, done two
// ways: the FP32 butterflies the transform passes use (DFT<16>, paired-FP32
// adds), and a DFT-as-GEMM stage on the tensor pipe.  It exists to decide
// whether a DFT-as-GEMM radix stage is faster than the butterflies for the
// FP32 bulk form (the product pass is bound by shared-memory traffic and
// instruction issue, the work such a stage would move to the tensor pipe).
//
// The GEMM form: the 16-point DFT of a column x is y = F x with F the 16x16
// DFT matrix; in real arithmetic [Re y; Im y] = [[Re F, -Im F], [Im F, Re F]]
// [Re x; Im x], a 32x32 by 32xn product for n columns.  TF32 keeps 10
// mantissa bits, too few for FP32 accuracy, so each operand is split into a
// TF32 head and a TF32 tail and the product is head*head + head*tail +
// tail*head (the three-term split; the tail*tail term is below FP32
// rounding).  The MMA is mma.sync m16n8k8 with FP32 accumulation.
//
// A CTA holds 16 x 128 complex values in shared memory, applies the stage
// `reps` times (in place), and writes the tile back; the time per stage and
// column follows from two rep counts.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "runtime_internal.h"

namespace azb {

constexpr int kSbCols = 128;  // columns per CTA
constexpr int kSbStride = 132;  // tile row stride (elements): rows 4 bank pairs apart
constexpr int kSbThreads = 128;

// One radix-16 stage per column with the transform passes' butterflies.
__global__ void __launch_bounds__(kSbThreads) k_stage_butterfly(float2* data, int reps) {
  __shared__ float2 tile[16][kSbStride];
  float2* g = data + (size_t)blockIdx.x * 16 * kSbCols;
  for (int i = threadIdx.x; i < 16 * kSbCols; i += kSbThreads) tile[i / kSbCols][i % kSbCols] = g[i];
  __syncthreads();
  const int col = threadIdx.x;
  for (int r = 0; r < reps; ++r) {
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = tile[k][col];
    DFT<16, -1, float2>::run(v);
#pragma unroll
    for (int k = 0; k < 16; ++k) tile[k][col] = v[k];
    __syncthreads();
  }
  for (int i = threadIdx.x; i < 16 * kSbCols; i += kSbThreads) g[i] = tile[i / kSbCols][i % kSbCols];
}

__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Element (row, col) of the 32x32 real form of the 16-point forward DFT.
__device__ __forceinline__ float dft_real(int row, int col) {
  const int k = row & 15, n = col & 15;
  const double a = -2.0 * 3.14159265358979323846 * double((k * n) & 15) / 16.0;
  const double c = cos(a), s = sin(a);
  if (row < 16) return float(col < 16 ? c : -s);  // Re y = Re F Re x - Im F Im x
  return float(col < 16 ? s : c);                 // Im y = Im F Re x + Re F Im x
}

// The same stage as a 32x32 by 32x128 real product, three-term TF32 split.
// Four warps, each owning 32 columns (4 tiles of 8); the DFT matrix's
// fragments stay in registers across reps.
__global__ void __launch_bounds__(kSbThreads) k_stage_gemm(float2* data, int reps) {
  __shared__ float2 tile[16][kSbStride];
  float2* g = data + (size_t)blockIdx.x * 16 * kSbCols;
  for (int i = threadIdx.x; i < 16 * kSbCols; i += kSbThreads) tile[i / kSbCols][i % kSbCols] = g[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  // A fragments (m-tile mt, k-step ks): a0 (gq, tq), a1 (gq+8, tq), a2 (gq, tq+4), a3 (gq+8, tq+4)
  unsigned ah[2][4][4], al[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int rows[4] = {16 * mt + gq, 16 * mt + gq + 8, 16 * mt + gq, 16 * mt + gq + 8};
      const int cols[4] = {8 * ks + tq, 8 * ks + tq, 8 * ks + tq + 4, 8 * ks + tq + 4};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float f = dft_real(rows[e], cols[e]);
        const unsigned h = to_tf32(f);
        ah[mt][ks][e] = h;
        al[mt][ks][e] = to_tf32(f - __uint_as_float(h));
      }
    }
  __syncthreads();
  for (int rep = 0; rep < reps; ++rep) {
    float acc[4][2][4];  // [n-tile][m-tile][c regs]; m-tile 0 gives Re y, 1 gives Im y
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[nt][mt][e] = 0.f;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int col = 32 * warp + 8 * nt + gq;  // B fragment column n = gq
      // real rows 8 ks + tq (+4): k-steps 0, 1 read Re of complex rows 0-15,
      // k-steps 2, 3 Im of the same rows, so one 8-byte load serves two k-steps
      float2 xv[2][2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        xv[h][0] = tile[8 * h + tq][col];
        xv[h][1] = tile[8 * h + tq + 4][col];
      }
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const float x0 = ks < 2 ? xv[ks][0].x : xv[ks - 2][0].y;
        const float x1 = ks < 2 ? xv[ks][1].x : xv[ks - 2][1].y;
        const unsigned bh0 = to_tf32(x0), bh1 = to_tf32(x1);
        const unsigned bl0 = to_tf32(x0 - __uint_as_float(bh0)), bl1 = to_tf32(x1 - __uint_as_float(bh1));
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          mma_tf32(acc[nt][mt], al[mt][ks], bh0, bh1);
          mma_tf32(acc[nt][mt], ah[mt][ks], bl0, bl1);
          mma_tf32(acc[nt][mt], ah[mt][ks], bh0, bh1);
        }
      }
    }
    __syncthreads();
    // C fragment: c0 (gq, 2tq), c1 (gq, 2tq+1), c2 (gq+8, 2tq), c3 (gq+8, 2tq+1);
    // m-tiles 0 and 1 are Re and Im of complex row gq (+8): one 8-byte store
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = gq + (e >= 2 ? 8 : 0);
        const int c = 32 * warp + 8 * nt + 2 * tq + (e & 1);
        tile[r][c] = make_float2(acc[nt][0][e], acc[nt][1][e]);
      }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < 16 * kSbCols; i += kSbThreads) g[i] = tile[i / kSbCols][i % kSbCols];
}

}  // namespace azb

using namespace azb;

az_status az_bench_radix16_stage(int method, int ctas, double* ns_per_column_stage, double* max_rel_err) {
  if ((method != 0 && method != 1) || ctas < 1 || !ns_per_column_stage || !max_rel_err)
    return set_error(AZ_ERR_INVALID, "az_bench_radix16_stage: bad argument");
  const size_t n = size_t(ctas) * 16 * kSbCols;
  std::vector<float2> h(n), out(n);
  std::mt19937 rng(12345);
  std::uniform_real_distribution<float> dist(-1.f, 1.f);
  for (auto& v : h) v = make_float2(dist(rng), dist(rng));
  float2* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(float2)) != cudaSuccess) return set_error(AZ_ERR_NOMEM, "az_bench_radix16_stage");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  auto launch = [&](int reps) {
    if (method == 0) k_stage_butterfly<<<ctas, kSbThreads>>>(d, reps);
    else k_stage_gemm<<<ctas, kSbThreads>>>(d, reps);
  };
  auto timed = [&](int reps, double* ms_out) {
    cudaError_t e = cudaMemcpy(d, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    launch(reps);  // warm-up
    e = cudaMemcpy(d, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    cudaEventRecord(e0);
    launch(reps);
    cudaEventRecord(e1);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    *ms_out = double(ms);
    return e;
  };
  const int r1 = 16, r2 = 80;
  double t1 = 0, t2 = 0;
  if (ce == cudaSuccess) ce = timed(r1, &t1);
  if (ce == cudaSuccess) ce = timed(r2, &t2);
  // accuracy of one stage against an FP64 DFT
  if (ce == cudaSuccess) ce = cudaMemcpy(d, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) {
    launch(1);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpy(out.data(), d, n * sizeof(float2), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  *ns_per_column_stage = (t2 - t1) * 1e6 / (double(r2 - r1) * ctas * kSbCols);
  double err = 0, ref_max = 0;
  const int check = ctas < 8 ? ctas : 8;
  for (int b = 0; b < check; ++b)
    for (int c = 0; c < kSbCols; ++c)
      for (int k = 0; k < 16; ++k) {
        double re = 0, im = 0;
        for (int m = 0; m < 16; ++m) {
          const double a = -2.0 * 3.14159265358979323846 * double((k * m) & 15) / 16.0;
          const float2 x = h[(size_t(b) * 16 + m) * kSbCols + c];
          re += x.x * std::cos(a) - x.y * std::sin(a);
          im += x.x * std::sin(a) + x.y * std::cos(a);
        }
        const float2 y = out[(size_t(b) * 16 + k) * kSbCols + c];
        err = std::fmax(err, std::hypot(y.x - re, y.y - im));
        ref_max = std::fmax(ref_max, std::hypot(re, im));
      }
  *max_rel_err = err / ref_max;
  return AZ_OK;
}
