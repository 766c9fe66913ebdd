// Internal to the library: the equation descriptor shared by the runtime
// units (runtime.cu, noalloc.cu).
#pragma once

#include <cstddef>

#include "../../include/azeban_b200.h"
#include "az_types.h"
#include "kernel_set.cuh"

struct az_euler_s {
  int dim, prec, batch;
  // Members the step kernels launch over (0: all of batch).  Set only while a
  // step is captured for a group's active prefix; members past it are not
  // touched.
  int nlaunch = 0;
  long long N, M, Nh;
  azb::Visc visc;
  double eps_visc;  // Equation::visc()
  const azb::KernelSet* ks;
  const void* tw;
  size_t csize;  // bytes per complex element
  // workspace: buf0 [6][M][N][Nh] (3-D) | [2][M][Nh] (2-D), buf1, buf2
  void* work = nullptr;
  size_t work_bytes = 0;
  char* buf[3] = {nullptr, nullptr, nullptr};
  long long buf_mem[3] = {0, 0, 0};  // member strides (elements)
  // Row strides (elements) of the intermediates; a padded one is a whole
  // number of 128-byte lines.  3-D: A1, A2 rows of 3 Nh, B1, B2 rows of
  // 6 Nh; 2-D: A1 rows of 2 Nh (ra1), B1 rows of 3 Nh (rb1).
  long long ra1 = 0, ra2 = 0, rb1 = 0, rb2 = 0;
  long long state_mem;               // member stride of a state array
  long long state_elems;             // batch * state_mem
  azb::Ctrl* ctrl = nullptr;              // [batch]
  double norm;
  double Md;
  bool prof = true;  // false: never record per-pass timing events
  int v_cols = 0, v_rows = 0, v_epi = 0;  // plan variants of the three pass kinds
  double* diag = nullptr;  // partial sums of the energy / enstrophy reduction
};

// Doubles of az_euler_s::diag per member.
constexpr int kDiagDoublesPerMember = 512 * 2 + 2;

namespace azb {
// Energy and enstrophy partial sums and results of `batch` members of u_hat
// [batch][dim][N]([N])[N/2+1] into buf (kDiagDoublesPerMember per member;
// the (energy, enstrophy) pairs at buf + batch * (kDiagDoublesPerMember - 2)).
cudaError_t diag_launch(int dim, int precision, long long N, const void* u_hat, int batch, double* buf,
                        cudaStream_t st);
}  // namespace azb


namespace azb {
// Sizes, member strides, padded row strides, normalisation and M^d of an
// equation whose dim, N, M, Nh and csize are set.
void euler_layout(az_euler_s* e);
// One right-hand side of every member of `e` (MODE_DUDT), the launch sequence
// of az_euler_dudt: resets the members' skip flags, then runs the passes.
az_status euler_dudt_launch(az_euler e, void* dudt_hat, const void* u_hat, cudaStream_t st);
// Sets the thread's last-error string and returns st.
az_status set_error(az_status st, const char* msg);
// AZ_OK for a zero Ctrl::err word, else the status (and message) it encodes:
// bit 1 AZ_ERR_TIMEOUT, bit 0 AZ_ERR_NONFINITE.
az_status ctrl_status(int err);
// The device twiddle table W_L^m (m in [0, L)) of the current device, built
// once per (device, precision, L) and kept until exit.
az_status device_twiddles(int precision, int L, const void** out);
// Compiled kernels of one (precision, transform length), or nullptr.
const KernelSet* find_kernel_set(int precision, int L);
// Plan variant (0 std, 1 wide) the tuning table holds for a pass kind
// (0 column passes, 1 product pass, 2 epilogue pass).
int tuned_variant(int precision, int L, int kind);
}  // namespace azb
