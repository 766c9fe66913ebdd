// Kinetic energy and enstrophy of spectral states, in FP64 with compensated
// (Neumaier) sums in a fixed order, so a member's value is the same whether
// it is reduced alone or inside a batch.
//
// For the unnormalised r2c spectrum u_hat of an N^d grid (Parseval):
//   E     = 1/2 <|u|^2>     = 1/(2 N^{2d}) sum_k w_k |u_hat_k|^2
//   Omega = 1/2 <|curl u|^2> = 1/(2 N^{2d}) sum_k w_k |k|^2 |u_hat_k|^2
// with k = 2 pi n and w_k = 1 on the planes k_last = 0 and k_last = N/2, 2
// elsewhere (the half spectrum stands for the full one); the enstrophy form
// holds for a divergence-free u_hat.  The reference computes spectra of these
// quantities in src/azeban/operations/energy_spectrum.cpp and
// enstrophy_spectrum.cpp.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "runtime_internal.h"

namespace azb {

struct Neu {
  double s = 0.0, c = 0.0;
  __host__ __device__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
  __host__ __device__ double value() const { return s + c; }
};

constexpr int kDiagThreads = 256;
constexpr int kDiagParts = 512;  // partial sums per member

// Partial sums over a fixed, contiguous range of modes per CTA.
template <typename T, int DIM>
__global__ void __launch_bounds__(kDiagThreads)
    k_diag_partials(const cvec<T>* u, long long N, long long nh, long long plane, long long member,
                    double* parts) {
  const int b = blockIdx.y;
  const long long per = (plane + kDiagParts - 1) / kDiagParts;
  const long long lo = blockIdx.x * per;
  const long long hi = lo + per < plane ? lo + per : plane;
  const cvec<T>* base = u + b * member;
  Neu e, w;
  const double twopi = 2 * 3.14159265358979323846;
  for (long long idx = lo + threadIdx.x; idx < hi; idx += kDiagThreads) {
    const long long k = idx % nh;
    const long long rest = idx / nh;
    long long i, j = 0;
    if (DIM == 2) {
      i = rest;
    } else {
      j = rest % N;
      i = rest / N;
    }
    const double i_ = double(i >= N / 2 + 1 ? i - N : i);
    const double j_ = double(j >= N / 2 + 1 ? j - N : j);
    double k2 = i_ * i_ + double(k) * double(k);
    if (DIM == 3) k2 += j_ * j_;
    k2 *= twopi * twopi;
    const double wk = (k == 0 || 2 * k == N) ? 1.0 : 2.0;
    double a2 = 0.0;
    for (int c = 0; c < DIM; ++c) {
      const cvec<T> v = base[c * plane + idx];
      a2 += double(v.x) * double(v.x) + double(v.y) * double(v.y);
    }
    e.add(wk * a2);
    w.add(wk * k2 * a2);
  }
  __shared__ double se[kDiagThreads], ce[kDiagThreads], sw[kDiagThreads], cw[kDiagThreads];
  se[threadIdx.x] = e.s;
  ce[threadIdx.x] = e.c;
  sw[threadIdx.x] = w.s;
  cw[threadIdx.x] = w.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    Neu E, W;
    for (int t = 0; t < kDiagThreads; ++t) {
      E.add(se[t]);
      E.add(ce[t]);
      W.add(sw[t]);
      W.add(cw[t]);
    }
    parts[(b * kDiagParts + blockIdx.x) * 2 + 0] = E.value();
    parts[(b * kDiagParts + blockIdx.x) * 2 + 1] = W.value();
  }
}

__global__ void k_diag_final(const double* parts, double scale, double* out) {
  const int b = blockIdx.x;
  if (threadIdx.x != 0) return;
  Neu E, W;
  for (int p = 0; p < kDiagParts; ++p) {
    E.add(parts[(b * kDiagParts + p) * 2 + 0]);
    W.add(parts[(b * kDiagParts + p) * 2 + 1]);
  }
  out[2 * b + 0] = 0.5 * scale * E.value();
  out[2 * b + 1] = 0.5 * scale * W.value();
}

// Partials and per-member (energy, enstrophy) of `batch` members of u_hat
// [batch][dim][N]([N])[N/2+1]; buf holds kDiagDoublesPerMember per member:
// the partial sums, then the results at buf + batch * kDiagParts * 2.
cudaError_t diag_launch(int dim, int precision, long long N, const void* u_hat, int batch, double* buf,
                        cudaStream_t st) {
  const long long nh = N / 2 + 1;
  const long long plane = (dim == 2 ? N : N * N) * nh;
  const long long member = dim * plane;
  double* parts = buf;
  double* res = parts + size_t(batch) * kDiagParts * 2;
  const dim3 grid(kDiagParts, unsigned(batch));
  if (precision == AZ_PREC_F64) {
    if (dim == 2) k_diag_partials<double, 2><<<grid, kDiagThreads, 0, st>>>((const double2*)u_hat, N, nh, plane, member, parts);
    else k_diag_partials<double, 3><<<grid, kDiagThreads, 0, st>>>((const double2*)u_hat, N, nh, plane, member, parts);
  } else {
    if (dim == 2) k_diag_partials<float, 2><<<grid, kDiagThreads, 0, st>>>((const float2*)u_hat, N, nh, plane, member, parts);
    else k_diag_partials<float, 3><<<grid, kDiagThreads, 0, st>>>((const float2*)u_hat, N, nh, plane, member, parts);
  }
  const double Nd = dim == 2 ? double(N) * N : double(N) * N * N;
  k_diag_final<<<unsigned(batch), 32, 0, st>>>(parts, 1.0 / (Nd * Nd), res);
  return cudaGetLastError();
}

}  // namespace azb

using namespace azb;

az_status az_euler_diagnostics(az_euler e, const void* u_hat, void* stream, double* energy, double* enstrophy) {
  if (!e || !u_hat) return set_error(AZ_ERR_INVALID, "az_euler_diagnostics: null argument");
  static_assert(kDiagParts * 2 + 2 == kDiagDoublesPerMember, "diagnostics buffer layout");
  double* res = e->diag + size_t(e->batch) * kDiagParts * 2;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t ce = diag_launch(e->dim, e->prec, e->N, u_hat, e->batch, e->diag, st);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  std::vector<double> h(size_t(e->batch) * 2);
  ce = cudaMemcpyAsync(h.data(), res, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  for (int b = 0; b < e->batch; ++b) {
    if (energy) energy[b] = h[2 * b];
    if (enstrophy) enstrophy[b] = h[2 * b + 1];
  }
  return AZ_OK;
}
