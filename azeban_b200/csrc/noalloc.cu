// The right-hand side without any allocation by the library.
//
// Some callers cannot let a library allocate device memory: a host code that
// owns every device allocation through its own pool or arena (a cudaMalloc
// from inside the library bypasses its accounting, or fails under its memory
// cap), or a run whose device memory is fixed at start-up.  For them,
// az_euler_dudt_noalloc takes its scratch from one file-scope device array of
// AZ_NOALLOC_SCRATCH_BYTES instead of a workspace; the caller passes the
// input and output arrays as usual.
//
// The array is a static __device__ variable: every GPU that loads the library
// holds it until the process exits.  Host code cannot use its name as a device
// address, so every call looks the address up on the current device with
// cudaGetSymbolAddress (a lookup the runtime answers from its module table
// after the first call, which may load the module: make the first call on a
// device before any stream capture).  Looking it up each time keeps the
// address right after a cudaDeviceReset, which loads the module anew.  All
// calls share the one array and it keeps the last call's contents, so each
// call rewrites everything it reads (control block, twiddle table) before
// use.  Calls whose work overlaps on the GPU (other streams, other host
// threads) race on the array.  The kernels report device-side failures (a
// non-finite velocity, a bounded wait that ran out) in the control block at
// the start of the array; az_euler_noalloc_status reads it, allocating
// nothing either.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <string>

#include "runtime_internal.h"

namespace azb {

static __device__ __align__(256) unsigned char g_noalloc_scratch[AZ_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device.
static az_status noalloc_scratch(void** out) {
  void* p = nullptr;
  const cudaError_t ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (ce != cudaSuccess)
    return set_error(AZ_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce)).c_str());
  *out = p;
  return AZ_OK;
}

// W_L^m = exp(-2 pi i m / L) for m in [0, L), from sincospi in FP64.
template <typename T>
__global__ void k_noalloc_twiddles(cvec<T>* tw, int L) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < L) {
    double s, c;
    sincospi(-2.0 * double(m) / double(L), &s, &c);
    tw[m] = cmk<cvec<T>>(T(c), T(s));
  }
}

static size_t round256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace azb

using namespace azb;

az_status az_euler_dudt_noalloc(int dim, long long N_phys, long long N_phys_pad, int precision,
                                const az_visc* visc, void* dudt_hat, const void* u_hat, void* stream) {
  if (!visc || !dudt_hat || !u_hat) return set_error(AZ_ERR_INVALID, "az_euler_dudt_noalloc: null argument");
  if (dim != 2 && dim != 3)
    return set_error(AZ_ERR_INVALID, "Incompressible Euler is only implemented for 2D and 3D");
  if (N_phys < 2 || (N_phys % 2) != 0) return set_error(AZ_ERR_INVALID, "N_phys must be even and >= 2");
  if (N_phys_pad < N_phys) return set_error(AZ_ERR_INVALID, "N_phys_pad must be >= N_phys");
  if (precision != AZ_PREC_F64 && precision != AZ_PREC_F32) return set_error(AZ_ERR_INVALID, "unknown precision");
  if (visc->type < 0 || visc->type > 3) return set_error(AZ_ERR_INVALID, "unknown viscosity type");
  const KernelSet* ks = find_kernel_set(precision, int(N_phys_pad));
  if (!ks) return set_error(AZ_ERR_UNSUPPORTED, "N_phys_pad has no compiled transform length");

  az_euler_s e;
  e.dim = dim;
  e.prec = precision;
  e.batch = 1;
  e.N = N_phys;
  e.M = N_phys_pad;
  e.Nh = e.N / 2 + 1;
  e.visc.type = visc->type;
  e.visc.eps = visc->eps;
  e.visc.s = visc->s;
  e.visc.k0 = visc->k0;
  e.visc.N = visc->N;
  e.eps_visc = visc->type == AZ_VISC_NONE ? 0.0 : visc->eps;
  e.ks = ks;
  e.csize = precision == AZ_PREC_F64 ? 16 : 8;
  e.prof = false;
  const int kbase = dim == 2 ? 3 : 0;
  e.v_cols = tuned_variant(precision, int(N_phys_pad), kbase + 0);
  e.v_rows = tuned_variant(precision, int(N_phys_pad), kbase + 1);
  e.v_epi = tuned_variant(precision, int(N_phys_pad), kbase + 2);
  const long long M = e.M;
  euler_layout(&e);
  e.state_elems = e.state_mem;

  // Scratch layout: control block | twiddle table | buf0 | buf1 | buf2.
  const size_t ctrl_bytes = round256(sizeof(Ctrl));
  const size_t tw_bytes = round256(size_t(M) * e.csize);
  size_t need = ctrl_bytes + tw_bytes;
  size_t off[3];
  for (int b = 0; b < 3; ++b) {
    off[b] = need;
    need += round256(size_t(e.buf_mem[b]) * e.csize);
  }
  if (need > size_t(AZ_NOALLOC_SCRATCH_BYTES)) {
    const std::string msg = "az_euler_dudt_noalloc: this size needs " + std::to_string(need) +
                            " bytes of scratch, above the fixed " +
                            std::to_string((long long)AZ_NOALLOC_SCRATCH_BYTES) +
                            " bytes; use az_euler_create / az_euler_dudt";
    return set_error(AZ_ERR_UNSUPPORTED, msg.c_str());
  }
  void* base = nullptr;
  az_status st = noalloc_scratch(&base);
  if (st != AZ_OK) return st;
  char* b = static_cast<char*>(base);
  e.ctrl = reinterpret_cast<Ctrl*>(b);
  e.tw = b + ctrl_bytes;
  e.work = b;
  e.work_bytes = need;
  for (int i = 0; i < 3; ++i) e.buf[i] = b + off[i];

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The array keeps the previous call's contents: rewrite the control block
  // and the twiddle table of this call's length before the passes read them.
  cudaError_t ce = cudaMemsetAsync(e.ctrl, 0, sizeof(Ctrl), s);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  const unsigned g = unsigned((M + 255) / 256);
  if (precision == AZ_PREC_F64)
    k_noalloc_twiddles<double><<<g, 256, 0, s>>>(reinterpret_cast<double2*>(b + ctrl_bytes), int(M));
  else
    k_noalloc_twiddles<float><<<g, 256, 0, s>>>(reinterpret_cast<float2*>(b + ctrl_bytes), int(M));
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  return euler_dudt_launch(&e, dudt_hat, u_hat, s);
}

az_status az_euler_noalloc_status(void* stream) {
  void* base = nullptr;
  az_status st = noalloc_scratch(&base);
  if (st != AZ_OK) return st;
  // The control block sits at the start of the array; its error word is the
  // only part read.  The copy goes to a local (pageable) int: no allocation.
  int err = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t ce = cudaMemcpyAsync(&err, static_cast<const char*>(base) + offsetof(Ctrl, err), sizeof(int),
                                   cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) return set_error(AZ_ERR_CUDA, cudaGetErrorString(ce));
  return ctrl_status(err);
}
