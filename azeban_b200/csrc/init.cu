// Initial data on the device: the pointwise sampling of the generators, a
// counter-based random stream, and the spectral envelope and energy
// normalisation of the random fields.
//
// Reference: Initializer::initialize (include/azeban/init/initializer.hpp
// :48-75) fills a physical field on the host, transforms it and projects it
// (src/azeban/init/taylor_green.cpp:29-76 and :146-206,
// src/azeban/init/double_shear_layer.cpp:25-66).  Here the physical field is
// sampled on the device, straight into the caller's array; the transform and
// the projection are az_fft_forward and az_leray.
//
// Random numbers come from Philox4x32-10 (J. K. Salmon, M. A. Moraes,
// R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011): a counter-based generator, so value c of stream (seed, member) is
// a pure function of (seed, member, c), the same on every GPU and whatever
// the launch shape.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "runtime_internal.h"

namespace azb {

// ---------------------------------------------------------------------------
// Philox4x32-10: ten rounds of two 32x32 -> 64-bit multiplications and a key
// schedule by the Weyl increments, as the paper specifies.
// ---------------------------------------------------------------------------
struct Philox4 {
  unsigned v[4];
};

__host__ __device__ inline Philox4 philox4x32_10(Philox4 c, unsigned k0, unsigned k1) {
  constexpr unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr unsigned W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    const unsigned long long p0 = (unsigned long long)M0 * c.v[0];
    const unsigned long long p1 = (unsigned long long)M1 * c.v[2];
    const unsigned hi0 = unsigned(p0 >> 32), lo0 = unsigned(p0);
    const unsigned hi1 = unsigned(p1 >> 32), lo1 = unsigned(p1);
    Philox4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Uniform double in (0, 1] from two 32-bit words (53 random bits).
__host__ __device__ inline double u01(unsigned a, unsigned b) {
  const unsigned long long x = ((unsigned long long)a << 32 | b) >> 11;
  return (double(x) + 1.0) * (1.0 / 9007199254740992.0);
}

// Stream (seed, member), block c: four words.
__host__ __device__ inline Philox4 stream_block(unsigned long long seed, unsigned long long member,
                                                unsigned long long c) {
  Philox4 ctr;
  ctr.v[0] = unsigned(c);
  ctr.v[1] = unsigned(c >> 32);
  ctr.v[2] = unsigned(member);
  ctr.v[3] = unsigned(member >> 32);
  return philox4x32_10(ctr, unsigned(seed), unsigned(seed >> 32));
}

// Per-member parameters of the pointwise generators (device memory).
struct InitParams {
  int kind, dim;
  long long N;
  double rho, delta;
  const double* deltas;  // Taylor-Green perturbations [batch][8 or 24], or null
  const double* phases;  // shear-layer phases [batch]
  unsigned long long seed, member0;
};

// One thread per grid point of one member (blockIdx.y); the field is
// [batch][dim][N]..[N] real.
template <typename T>
__global__ void k_init_physical(T* u, InitParams p) {
  const long long N = p.N;
  const long long npts = p.dim == 2 ? N * N : N * N * N;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = blockIdx.y;
  if (idx >= npts) return;
  T* base = u + b * p.dim * npts;
  const double twopi = 2 * 3.14159265358979323846;
  long long i, j, k = 0;
  if (p.dim == 2) {
    i = idx / N;
    j = idx % N;
  } else {
    i = idx / (N * N);
    j = (idx / N) % N;
    k = idx % N;
  }
  if (p.kind == AZ_INIT_TAYLOR_GREEN || p.kind == AZ_INIT_TAYLOR_GREEN_WORKLOAD) {
    // x = 2 pi i / N (taylor_green.cpp:40-41, :158-160)
    const double x = twopi / double(N) * double(i);
    const double y = twopi / double(N) * double(j);
    const double z = twopi / double(N) * double(k);
    if (p.kind == AZ_INIT_TAYLOR_GREEN_WORKLOAD) {
      // (sin x cos y, -cos x sin y) / (sin x cos y cos z, -cos x sin y cos z, 0)
      if (p.dim == 2) {
        base[idx] = T(sin(x) * cos(y));
        base[npts + idx] = T(-cos(x) * sin(y));
      } else {
        base[idx] = T(sin(x) * cos(y) * cos(z));
        base[npts + idx] = T(-cos(x) * sin(y) * cos(z));
        base[2 * npts + idx] = T(0);
      }
      return;
    }
    // the reference's field with its perturbation modes (taylor_green.cpp:29-46, :146-184)
    const double* dl = p.deltas ? p.deltas + b * (p.dim == 2 ? 8 : 24) : nullptr;
    if (p.dim == 2) {
      const double s2x = sin(2 * x), c2x = cos(2 * x), s2y = sin(2 * y), c2y = cos(2 * y);
      double v[2] = {1.0 * cos(x) * sin(y), -1.0 * sin(x) * cos(y)};
      for (int d = 0; d < 2; ++d) {
        if (!dl) break;
        v[d] += dl[0 + 4 * d] * s2x * s2y;
        v[d] += dl[1 + 4 * d] * s2x * c2y;
        v[d] += dl[2 + 4 * d] * c2x * s2y;
        v[d] += dl[3 + 4 * d] * c2x * c2y;
      }
      base[idx] = T(v[0]);
      base[npts + idx] = T(v[1]);
    } else {
      const double s2x = sin(2 * x), c2x = cos(2 * x), s2y = sin(2 * y), c2y = cos(2 * y);
      const double s2z = sin(2 * z), c2z = cos(2 * z);
      double v[3] = {1.0 * cos(x) * sin(y) * sin(z), -1.0 * sin(x) * cos(y) * sin(z),
                     0.0 * sin(x) * sin(y) * cos(z)};
      for (int d = 0; d < 3; ++d) {
        if (!dl) break;
        v[d] += dl[0 + 8 * d] * s2x * s2y * s2z;
        v[d] += dl[1 + 8 * d] * s2x * s2y * c2z;
        v[d] += dl[2 + 8 * d] * s2x * c2y * s2z;
        v[d] += dl[3 + 8 * d] * s2x * c2y * c2z;
        v[d] += dl[4 + 8 * d] * c2x * s2y * s2z;
        v[d] += dl[5 + 8 * d] * c2x * s2y * c2z;
        v[d] += dl[6 + 8 * d] * c2x * c2y * s2z;
        v[d] += dl[7 + 8 * d] * c2x * c2y * c2z;
      }
      base[idx] = T(v[0]);
      base[npts + idx] = T(v[1]);
      base[2 * npts + idx] = T(v[2]);
    }
    return;
  }
  if (p.kind == AZ_INIT_DOUBLE_SHEAR_LAYER) {
    // double_shear_layer.cpp:29-43, with a phase phi in v = delta sin(2 pi x + phi)
    const double x = double(i) / double(N);
    const double y = double(j) / double(N);
    double u0;
    if (p.rho == 0) {
      u0 = fabs(y - 0.5) < 0.25 ? 1.0 : -1.0;
    } else if (y < 0.5) {
      u0 = tanh(twopi * (y - 0.25) / p.rho);
    } else {
      u0 = tanh(twopi * (0.75 - y) / p.rho);
    }
    // phase: given, or U[0, 2 pi) from the first value of stream (seed, member0 + b)
    double phi;
    if (p.phases) {
      phi = p.phases[b];
    } else {
      const Philox4 r = stream_block(p.seed, p.member0 + b, 0);
      phi = twopi * (u01(r.v[0], r.v[1]) - 1.0 / 9007199254740992.0);
    }
    base[idx] = T(u0);
    base[npts + idx] = T(p.delta * sin(twopi * x + phi));
    return;
  }
  // AZ_INIT_GAUSSIAN_NOISE: independent standard normals, Box-Muller on the
  // stream (seed, member0 + b): block c gives the values of components
  // 2c, 2c + 1 of the flat [dim][points] member.
  for (int c = 0; c < p.dim; ++c) {
    const long long e = c * npts + idx;
    const Philox4 r = stream_block(p.seed, p.member0 + b, (unsigned long long)(e >> 1));
    const double u1 = u01(r.v[0], r.v[1]);
    const double u2 = u01(r.v[2], r.v[3]);
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    base[e] = T((e & 1) ? rad * s : rad * co);
  }
}

// u_hat *= |n|^exponent per mode (n the integer wavevector), 0 at n = 0:
// the amplitude envelope of the random fields.
template <typename T>
__global__ void k_init_envelope(cvec<T>* u, int dim, long long N, long long nh, long long plane, double exponent) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = blockIdx.y;
  if (idx >= plane) return;
  const long long kk = idx % nh;
  const long long rest = idx / nh;
  long long i, j = 0;
  if (dim == 2) {
    i = rest;
  } else {
    j = rest % N;
    i = rest / N;
  }
  const double i_ = double(i >= N / 2 + 1 ? i - N : i);
  const double j_ = double(j >= N / 2 + 1 ? j - N : j);
  const double n2 = i_ * i_ + j_ * j_ + double(kk) * double(kk);
  const double a = n2 > 0 ? pow(n2, 0.5 * exponent) : 0.0;
  for (int c = 0; c < dim; ++c) {
    cvec<T>& v = u[(b * dim + c) * plane + idx];
    v.x = T(double(v.x) * a);
    v.y = T(double(v.y) * a);
  }
}

// u_hat *= sqrt(target / e[b]) per member, e = (energy, enstrophy) pairs in
// device memory.
template <typename T>
__global__ void k_init_scale(cvec<T>* u, long long member_elems, const double* e, double target) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = blockIdx.y;
  if (idx >= member_elems) return;
  const double en = e[2 * b];
  const double s = en > 0 ? sqrt(target / en) : 0.0;
  cvec<T>& v = u[b * member_elems + idx];
  v.x = T(double(v.x) * s);
  v.y = T(double(v.y) * s);
}

}  // namespace azb

using namespace azb;

az_status az_init_physical(const az_init_desc* d, void* u, void* stream) {
  if (!d || !u) return set_error(AZ_ERR_INVALID, "az_init_physical: null argument");
  if (d->dim != 2 && d->dim != 3) return set_error(AZ_ERR_INVALID, "az_init_physical: dim must be 2 or 3");
  if (d->N < 2 || d->batch < 1) return set_error(AZ_ERR_INVALID, "az_init_physical: bad size or batch");
  if (d->precision != AZ_PREC_F64 && d->precision != AZ_PREC_F32)
    return set_error(AZ_ERR_INVALID, "az_init_physical: unknown precision");
  if (d->kind == AZ_INIT_DOUBLE_SHEAR_LAYER && d->dim != 2)
    return set_error(AZ_ERR_INVALID, "Double shear layer is only available in 2d");
  if (d->kind < AZ_INIT_TAYLOR_GREEN || d->kind > AZ_INIT_GAUSSIAN_NOISE)
    return set_error(AZ_ERR_INVALID, "az_init_physical: unknown generator");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Given perturbation amplitudes or phases travel to the device in a
  // stream-ordered buffer (the call then waits for its copy, so the caller's
  // host arrays may be freed on return).  Without them nothing is copied and
  // the call does not wait: shear-layer phases come from the random stream.
  const int nd = d->dim == 2 ? 8 : 24;
  const size_t nparam = (d->deltas ? size_t(d->batch) * nd : 0) + (d->phases ? size_t(d->batch) : 0);
  double* dev = nullptr;
  cudaError_t ce = cudaSuccess;
  if (nparam > 0) {
    ce = cudaMallocAsync(&dev, nparam * sizeof(double), st);
    if (ce != cudaSuccess) return set_error(AZ_ERR_NOMEM, "az_init_physical: parameter buffer");
    size_t off = 0;
    if (d->deltas) {
      ce = cudaMemcpyAsync(dev, d->deltas, size_t(d->batch) * nd * sizeof(double), cudaMemcpyHostToDevice, st);
      off = size_t(d->batch) * nd;
    }
    if (ce == cudaSuccess && d->phases)
      ce = cudaMemcpyAsync(dev + off, d->phases, size_t(d->batch) * sizeof(double), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      cudaFreeAsync(dev, st);
      return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
    }
  }
  InitParams p{};
  p.kind = d->kind;
  p.dim = d->dim;
  p.N = d->N;
  p.rho = d->rho;
  p.delta = d->delta;
  p.deltas = d->deltas ? dev : nullptr;
  p.phases = d->phases ? dev + (d->deltas ? size_t(d->batch) * nd : 0) : nullptr;
  p.seed = d->seed;
  p.member0 = (unsigned long long)d->member0;
  const long long npts = d->dim == 2 ? d->N * d->N : d->N * d->N * d->N;
  const dim3 grid(unsigned((npts + 255) / 256), unsigned(d->batch));
  if (d->precision == AZ_PREC_F64)
    k_init_physical<double><<<grid, 256, 0, st>>>(static_cast<double*>(u), p);
  else
    k_init_physical<float><<<grid, 256, 0, st>>>(static_cast<float*>(u), p);
  ce = cudaGetLastError();
  if (dev) cudaFreeAsync(dev, st);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  return AZ_OK;
}

az_status az_init_envelope(int dim, long long N, int precision, void* u_hat, int batch, double exponent,
                           void* stream) {
  if (!u_hat || (dim != 2 && dim != 3) || N < 2 || batch < 1)
    return set_error(AZ_ERR_INVALID, "az_init_envelope: bad argument");
  const long long nh = N / 2 + 1;
  const long long plane = (dim == 2 ? N : N * N) * nh;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid(unsigned((plane + 255) / 256), unsigned(batch));
  if (precision == AZ_PREC_F64)
    k_init_envelope<double><<<grid, 256, 0, st>>>(static_cast<double2*>(u_hat), dim, N, nh, plane, exponent);
  else
    k_init_envelope<float><<<grid, 256, 0, st>>>(static_cast<float2*>(u_hat), dim, N, nh, plane, exponent);
  const cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  return AZ_OK;
}

// Energy of every member, then u_hat *= sqrt(target / energy) per member on
// the device (the energies never leave it).
az_status az_init_normalize_energy(int dim, long long N, int precision, void* u_hat, int batch, double target,
                                   void* stream) {
  if (!u_hat || (dim != 2 && dim != 3) || N < 2 || batch < 1 || !(target > 0))
    return set_error(AZ_ERR_INVALID, "az_init_normalize_energy: bad argument");
  const long long nh = N / 2 + 1;
  const long long member = dim * (dim == 2 ? N : N * N) * nh;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* buf = nullptr;  // partial sums, then per-member (energy, enstrophy)
  cudaError_t ce = cudaMallocAsync(&buf, sizeof(double) * size_t(batch) * kDiagDoublesPerMember, st);
  if (ce != cudaSuccess) return set_error(AZ_ERR_NOMEM, "az_init_normalize_energy: reduction buffer");
  ce = diag_launch(dim, precision, N, u_hat, batch, buf, st);
  if (ce == cudaSuccess) {
    const double* res = buf + size_t(batch) * (kDiagDoublesPerMember - 2);
    const dim3 grid(unsigned((member + 255) / 256), unsigned(batch));
    if (precision == AZ_PREC_F64)
      k_init_scale<double><<<grid, 256, 0, st>>>(static_cast<double2*>(u_hat), member, res, target);
    else
      k_init_scale<float><<<grid, 256, 0, st>>>(static_cast<float2*>(u_hat), member, res, target);
    ce = cudaGetLastError();
  }
  cudaFreeAsync(buf, st);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  return AZ_OK;
}

az_status az_random_uniform(unsigned long long seed, unsigned long long member, unsigned long long index,
                            double* out) {
  if (!out) return set_error(AZ_ERR_INVALID, "az_random_uniform: null argument");
  const Philox4 r = stream_block(seed, member, index);
  *out = u01(r.v[0], r.v[1]) - 1.0 / 9007199254740992.0;
  return AZ_OK;
}

az_status az_philox4x32_10(const unsigned* counter, const unsigned* key, unsigned* out) {
  if (!counter || !key || !out) return set_error(AZ_ERR_INVALID, "az_philox4x32_10: null argument");
  Philox4 c;
  for (int i = 0; i < 4; ++i) c.v[i] = counter[i];
  const Philox4 r = philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
  return AZ_OK;
}
