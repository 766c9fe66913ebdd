// Divergence-free projection of a spectral velocity field, used when initial
// data is built (reference: leray(), src/azeban/operations/leray.cpp:28-116,
// called from Initializer::initialize, include/azeban/init/initializer.hpp:68-75).
#include <cuda_runtime.h>

#include <string>

#include "../../include/azeban_b200.h"
#include "fft_core.cuh"

namespace azb {

// u_hat [batch][dim][N]([N])[nh]; one thread per mode.
template <typename T, int DIM>
__global__ void k_leray(cvec<T>* u, long long N, long long nh, long long plane, long long member) {
  using C = cvec<T>;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = blockIdx.y;
  if (idx >= plane) return;
  C* base = u + b * member;
  const long long k = idx % nh;
  const long long rest = idx / nh;
  long long i, j = 0;
  if (DIM == 2) {
    i = rest;
  } else {
    j = rest % N;
    i = rest / N;
  }
  const long long i_ = i >= N / 2 + 1 ? i - N : i;
  const long long j_ = j >= N / 2 + 1 ? j - N : j;
  const T twopi = T(2 * 3.14159265358979323846);
  T kv[3];
  kv[0] = twopi * T(i_);
  if (DIM == 2) {
    kv[1] = twopi * T(k);
  } else {
    kv[1] = twopi * T(j_);
    kv[2] = twopi * T(k);
  }
  T absk2 = kv[0] * kv[0];
  for (int a = 1; a < DIM; ++a) absk2 = absk2 + kv[a] * kv[a];
  C v[3];
  for (int a = 0; a < DIM; ++a) v[a] = base[a * plane + idx];
  for (int a = 0; a < DIM; ++a) {
    C acc = cmk<C>(T(0), T(0));
    if (absk2 != T(0)) {
      for (int c = 0; c < DIM; ++c) {
        const T coef = T(a == c ? 1 : 0) - (kv[a] * kv[c]) / absk2;
        acc = cmk<C>(acc.x + coef * v[c].x, acc.y + coef * v[c].y);
      }
    }
    base[a * plane + idx] = acc;
  }
}

}  // namespace azb

using namespace azb;

az_status az_leray(int dim, long long N, int precision, void* u_hat, int batch, void* stream) {
  if ((dim != 2 && dim != 3) || N < 2 || !u_hat || batch < 1 ||
      (precision != AZ_PREC_F64 && precision != AZ_PREC_F32))
    return AZ_ERR_INVALID;
  const long long nh = N / 2 + 1;
  const long long plane = (dim == 2 ? N : N * N) * nh;
  const long long member = dim * plane;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid(unsigned((plane + 255) / 256), unsigned(batch));
  if (precision == AZ_PREC_F64) {
    if (dim == 2) k_leray<double, 2><<<grid, 256, 0, st>>>((double2*)u_hat, N, nh, plane, member);
    else k_leray<double, 3><<<grid, 256, 0, st>>>((double2*)u_hat, N, nh, plane, member);
  } else {
    if (dim == 2) k_leray<float, 2><<<grid, 256, 0, st>>>((float2*)u_hat, N, nh, plane, member);
    else k_leray<float, 3><<<grid, 256, 0, st>>>((float2*)u_hat, N, nh, plane, member);
  }
  return cudaGetLastError() == cudaSuccess ? AZ_OK : AZ_ERR_CUDA;
}
