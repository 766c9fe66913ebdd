// Host runtime behind the C ABI: solve descriptors, workspaces, twiddle
// tables, and the launch sequences of one right-hand side, one SSP-RK3 step
// and one simulate_until.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/azeban_b200.h"
#include "az_types.h"
#include "kernel_set.cuh"
#include "runtime_internal.h"

namespace azb {

#define AZB_LENGTHS(X) \
  X(4) X(6) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024) X(1536)

#define AZB_DECL(LEN)                            \
  const KernelSet* kernel_set_f64_##LEN();       \
  const KernelSet* kernel_set_f32_##LEN();
AZB_LENGTHS(AZB_DECL)
#undef AZB_DECL

static const KernelSet* kernel_set(int precision, int L) {
#define AZB_CASE(LEN) \
  case LEN: return precision == 0 ? kernel_set_f64_##LEN() : kernel_set_f32_##LEN();
  switch (L) {
    AZB_LENGTHS(AZB_CASE)
    default: return nullptr;
  }
#undef AZB_CASE
}

static const int kLengths[] = {
#define AZB_LIST(LEN) LEN,
    AZB_LENGTHS(AZB_LIST)
#undef AZB_LIST
};

// ---------------------------------------------------------------------------
// Tuning table: plan variant per (precision, length, pass kind).  Defaults:
// FP32 uses the wide plans (fewer exchanges), FP64 the register-lean ones.
// AZ_PLAN_VARIANT="c,r,e" overrides every entry; az_tune_set overrides one.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mutex;
static std::map<std::tuple<int, int, int>, int> g_tune;

int tuned_variant(int precision, int L, int kind) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tune.find(std::make_tuple(precision, L, kind));
  if (it != g_tune.end()) return it->second;
  if (const char* env = std::getenv("AZ_PLAN_VARIANT")) {
    int v[3] = {0, 0, 0};
    if (std::sscanf(env, "%d,%d,%d", &v[0], &v[1], &v[2]) == 3 && kind >= 0 && kind < 6)
      return kind % 3 == 2 ? (v[2] & 1) : (v[kind % 3] & (kind % 3 == 1 ? 7 : 3));
  }
  return precision == 1 ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static az_status fail(az_status st, const std::string& msg) {
  g_err = msg;
  return st;
}

static az_status cuda_fail(cudaError_t e, const char* what) {
  return fail(AZ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Status of a nonzero Ctrl::err word: bit 0 a non-finite value met by the CFL
// reduction, bit 1 a bounded wait on a kernel's own bulk copy that ran out
// (the kernel then returned early and its output is incomplete).
static az_status ctrl_error(int err) {
  if (err & 2)
    return fail(AZ_ERR_TIMEOUT, "a bounded bulk-copy wait inside a transform pass ran out; the pass is incomplete");
  return fail(AZ_ERR_NONFINITE, "non-finite value in the CFL reduction");
}

// Polls of the product pass's bounded wait for its bulk copy (kWaitPolls
// unless az_debug_set_wait_limit changed it).
static int g_wait_polls = kWaitPolls;

#define AZB_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// ---------------------------------------------------------------------------
// Twiddle tables W_L^m = exp(-2 pi i m / L), one per (device, precision, L),
// evaluated in long double and rounded once.
// ---------------------------------------------------------------------------
static std::mutex g_tw_mutex;
static std::map<std::tuple<int, int, int>, void*> g_tw;

static az_status twiddles(int precision, int L, const void** out);
az_status device_twiddles(int precision, int L, const void** out) { return twiddles(precision, L, out); }

static az_status twiddles(int precision, int L, const void** out) {
  int dev = 0;
  AZB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  auto key = std::make_tuple(dev, precision, L);
  auto it = g_tw.find(key);
  if (it != g_tw.end()) {
    *out = it->second;
    return AZ_OK;
  }
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<double> h64(2 * L);
  std::vector<float> h32(2 * L);
  for (int m = 0; m < L; ++m) {
    const long double a = -2.0L * pi * (long double)m / (long double)L;
    long double c = cosl(a), s = sinl(a);
    // Exact values at the quarter points.
    if ((4 * m) % L == 0) {
      const int q = (4 * m) / L;
      c = (q == 0) ? 1.0L : (q == 2 ? -1.0L : 0.0L);
      s = (q == 1) ? -1.0L : (q == 3 ? 1.0L : 0.0L);
    }
    h64[2 * m] = (double)c;
    h64[2 * m + 1] = (double)s;
    h32[2 * m] = (float)c;
    h32[2 * m + 1] = (float)s;
  }
  void* d = nullptr;
  const size_t bytes = precision == 0 ? h64.size() * sizeof(double) : h32.size() * sizeof(float);
  AZB_CUDA(cudaMalloc(&d, bytes));
  AZB_CUDA(cudaMemcpy(d, precision == 0 ? (const void*)h64.data() : (const void*)h32.data(), bytes,
                      cudaMemcpyHostToDevice));
  g_tw[key] = d;
  *out = d;
  return AZ_OK;
}

static long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// Optional per-pass timing: each pass launch bracketed by two events on its
// own stream; durations and algorithmic bytes accumulate per pass id.
// ---------------------------------------------------------------------------
enum PassId : int { P_INV_X = 0, P_INV_Y = 1, P_PRODUCT = 2, P_FWD_Y = 3, P_EPILOGUE = 4, P_NPASS = 5 };
struct ProfRec {
  int pass;
  double bytes;
  cudaEvent_t a, b;
};
static bool g_prof = false;
static std::vector<ProfRec> g_prof_recs;
static std::vector<cudaEvent_t> g_prof_pool;

static cudaEvent_t prof_event() {
  if (!g_prof_pool.empty()) {
    cudaEvent_t e = g_prof_pool.back();
    g_prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

struct ProfScope {
  int pass;
  double bytes;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  ProfScope(int p, double by, cudaStream_t s, bool allowed = true) : pass(p), bytes(by), st(s) {
    if (g_prof && allowed) {
      a = prof_event();
      cudaEventRecord(a, st);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEvent_t b = prof_event();
      cudaEventRecord(b, st);
      g_prof_recs.push_back({pass, bytes, a, b});
    }
  }
};

}  // namespace azb

using namespace azb;

// ---------------------------------------------------------------------------
// Equation
// ---------------------------------------------------------------------------
const char* az_last_error_string(void) { return g_err.c_str(); }

az_status az_supported_lengths(int* out, int cap, int* n) {
  const int cnt = int(sizeof(kLengths) / sizeof(kLengths[0]));
  if (n) *n = cnt;
  if (out)
    for (int i = 0; i < cnt && i < cap; ++i) out[i] = kLengths[i];
  return AZ_OK;
}

namespace azb {
// Elements per 128-byte line of the equation's complex type.
static long long pad_line(long long elems, size_t csize) {
  const long long q = 128 / (long long)csize;
  return (elems + q - 1) / q * q;
}

void euler_layout(az_euler_s* e) {
  const long long N = e->N, M = e->M, Nh = e->Nh;
  // Which intermediates get padded rows (bits 0-3: A1, A2, B1, B2).  Padding
  // pays where a column pass reads the rows (forward y reads B1: 128-byte
  // aligned tiles) and costs where a pass streams whole lines or groups its
  // columns (the product pass reads A2, the epilogue B2, inverse x writes
  // A1), so only B1 is padded unless AZ_PAD_MASK says otherwise.
  int mask = 0x4;
  if (const char* env = std::getenv("AZ_PAD_MASK")) mask = std::atoi(env) & 0xf;
  auto row = [&](long long elems, int bit) { return (mask >> bit) & 1 ? pad_line(elems, e->csize) : elems; };
  if (e->dim == 3) {
    e->ra1 = row(3 * Nh, 0);
    e->ra2 = row(3 * Nh, 1);
    e->rb1 = row(6 * Nh, 2);
    e->rb2 = row(6 * Nh, 3);
    e->buf_mem[0] = std::max(M * N * e->ra1, M * N * e->rb2);  // A1 [M][N][ra1], later B2 [M][N][rb2]
    e->buf_mem[1] = M * M * e->ra2;                             // A2 [M][M][ra2]
    e->buf_mem[2] = M * M * e->rb1;                             // B1 [M][M][rb1]
    e->state_mem = 3 * N * N * Nh;
    // 1 / (N^{3/2} M^{3/2}) with the integer powers by repeated
    // multiplication, as computeB forms it (incompressible_euler.hpp:171-173)
    const double sn = std::sqrt((double)N), sm = std::sqrt((double)M);
    e->norm = 1.0 / ((sn * (sn * sn)) * (sm * (sm * sm)));
    e->Md = (double)(M * M * M);
  } else {
    e->ra1 = row(2 * Nh, 0);
    e->rb1 = row(3 * Nh, 2);
    e->ra2 = e->ra1;
    e->rb2 = e->rb1;
    e->buf_mem[0] = M * e->ra1;  // A1 [M][ra1]
    e->buf_mem[1] = M * e->rb1;  // B1 [M][rb1]
    e->buf_mem[2] = 0;
    e->state_mem = 2 * N * Nh;
    const double sn = std::sqrt((double)N), sm = std::sqrt((double)M);
    e->norm = 1.0 / ((sn * sn) * (sm * sm));
    e->Md = (double)(M * M);
  }
}
}  // namespace azb

az_status az_euler_create(const az_euler_desc* d, az_euler* out) {
  if (!d || !out) return fail(AZ_ERR_INVALID, "az_euler_create: null argument");
  *out = nullptr;
  if (d->dim != 2 && d->dim != 3) return fail(AZ_ERR_INVALID, "Incompressible Euler is only implemented for 2D and 3D");
  if (d->N_phys < 2 || (d->N_phys % 2) != 0) return fail(AZ_ERR_INVALID, "N_phys must be even and >= 2");
  if (d->N_phys_pad < d->N_phys) return fail(AZ_ERR_INVALID, "N_phys_pad must be >= N_phys");
  if (d->precision != AZ_PREC_F64 && d->precision != AZ_PREC_F32) return fail(AZ_ERR_INVALID, "unknown precision");
  if (d->batch < 1) return fail(AZ_ERR_INVALID, "batch must be >= 1");
  if (d->visc.type < 0 || d->visc.type > 3) return fail(AZ_ERR_INVALID, "unknown viscosity type");
  const KernelSet* ks = kernel_set(d->precision, int(d->N_phys_pad));
  if (!ks)
    return fail(AZ_ERR_UNSUPPORTED, "N_phys_pad = " + std::to_string(d->N_phys_pad) +
                                        " has no compiled transform length");
  auto* e = new az_euler_s();
  e->dim = d->dim;
  e->prec = d->precision;
  e->batch = d->batch;
  e->N = d->N_phys;
  e->M = d->N_phys_pad;
  e->Nh = e->N / 2 + 1;
  e->visc.type = d->visc.type;
  e->visc.eps = d->visc.eps;
  e->visc.s = d->visc.s;
  e->visc.k0 = d->visc.k0;
  e->visc.N = d->visc.N;
  e->eps_visc = d->visc.type == AZ_VISC_NONE ? 0.0 : d->visc.eps;
  e->ks = ks;
  e->csize = d->precision == 0 ? 16 : 8;
  const int kbase = e->dim == 2 ? 3 : 0;
  e->v_cols = tuned_variant(e->prec, int(e->M), kbase + 0);
  e->v_rows = tuned_variant(e->prec, int(e->M), kbase + 1);
  e->v_epi = tuned_variant(e->prec, int(e->M), kbase + 2);
  euler_layout(e);
  e->state_elems = e->state_mem * e->batch;
  size_t off[3];
  size_t total = 0;
  for (int b = 0; b < 3; ++b) {
    off[b] = total;
    const size_t bytes = size_t(e->buf_mem[b]) * e->batch * e->csize;
    total += (bytes + 255) / 256 * 256;
  }
  az_status st = twiddles(e->prec, int(e->M), &e->tw);
  if (st != AZ_OK) {
    delete e;
    return st;
  }
  cudaError_t ce = cudaMalloc(&e->work, total);
  if (ce != cudaSuccess) {
    delete e;
    cudaGetLastError();
    return fail(AZ_ERR_NOMEM, "az_euler_create: workspace of " + std::to_string(total) +
                                  " bytes: " + cudaGetErrorString(ce));
  }
  e->work_bytes = total;
  for (int b = 0; b < 3; ++b) e->buf[b] = static_cast<char*>(e->work) + off[b];
  ce = cudaMalloc(&e->ctrl, sizeof(Ctrl) * e->batch);
  if (ce != cudaSuccess) {
    cudaFree(e->work);
    delete e;
    cudaGetLastError();
    return fail(AZ_ERR_NOMEM, "az_euler_create: control block");
  }
  ce = cudaMalloc(&e->diag, sizeof(double) * kDiagDoublesPerMember * e->batch);
  if (ce != cudaSuccess) {
    cudaFree(e->work);
    cudaFree(e->ctrl);
    delete e;
    cudaGetLastError();
    return fail(AZ_ERR_NOMEM, "az_euler_create: diagnostics buffer");
  }
  ce = cudaMemset(e->ctrl, 0, sizeof(Ctrl) * e->batch);
  if (ce != cudaSuccess) {
    cudaFree(e->work);
    cudaFree(e->ctrl);
    delete e;
    return cuda_fail(ce, "cudaMemset");
  }
  *out = e;
  return AZ_OK;
}

az_status az_euler_destroy(az_euler e) {
  if (!e) return AZ_OK;
  cudaFree(e->work);
  cudaFree(e->ctrl);
  cudaFree(e->diag);
  delete e;
  return AZ_OK;
}

int az_euler_n_vars(az_euler e) { return e ? e->dim : 0; }
double az_euler_visc(az_euler e) { return e ? e->eps_visc : 0.0; }
size_t az_euler_workspace_size(az_euler e) { return e ? e->work_bytes : 0; }

namespace azb {

// Members the step kernels launch over: a prefix [0, n) of the batch.
static inline int launch_members(az_euler e) { return e->nlaunch > 0 ? e->nlaunch : e->batch; }

// The contiguous-axis product pass over every member.  Bits of the tuned
// variant: 0 the radix plan, 1 the bulk-copy kernel (k_zpass) instead of
// k_rows_product.
static cudaError_t product_pass(az_euler e, int dim, const RowArgs& r, cudaStream_t st) {
  const KernelSet* ks = e->ks;
  if (e->v_rows & 6) {
    ZArgs z{};
    z.in = r.in;
    z.out = r.out;
    z.tw = r.tw;
    z.nlines = r.nlines;
    z.nh = r.nh;
    z.nmem = launch_members(e);
    z.in_line = int(r.in_line);
    z.out_line = int(r.out_line);
    z.in_mem = r.in_mem;
    z.out_mem = r.out_mem;
    z.norm = r.norm;
    z.ctrl = r.ctrl;
    z.wait_polls = g_wait_polls;
    if (e->v_rows & 4) return ks->zfused(e->v_rows & 3, dim, z, st);
    return ks->zpass(e->v_rows & 1, dim, z, st);
  }
  const int nlp = dim == 3 ? ks->tiles[e->v_rows & 1].nlp3 : ks->tiles[e->v_rows & 1].nlp2;
  return ks->rows_product(e->v_rows & 1, dim, r, unsigned(cdiv(r.nlines, 2 * nlp)), unsigned(launch_members(e)),
                          st);
}

// A member's state layout: planar (the reference's [d][N]..[Nh], every array
// a caller passes) or component innermost ([N]..[Nh][d], the stepper's own
// stage buffers: the pass-1 reads and the epilogue's state accesses of a
// tile of a few modes are then d times wider per row).
static StateLayout state_layout(az_euler e, bool inner) {
  const long long N = e->N, Nh = e->Nh;
  const int d = e->dim;
  const long long plane = d == 3 ? N * Nh : Nh;  // modes of one retained row
  if (inner) return StateLayout{1, int(d * plane), d};
  return StateLayout{int(d == 3 ? N * N * Nh : N * Nh), int(plane), 1};
}

// One right-hand side of every member: out <- stage(mode, u, u0, RHS(u)).
// first_stage: compute dt = min(C/(N u_max), max_dt) after the product pass.
// u_inner / u0_inner / out_inner: the array is in the component-innermost
// layout (else planar).
static az_status rhs(az_euler e, const void* u, bool u_inner, const void* u0, bool u0_inner, void* out,
                     bool out_inner, int mode, bool first_stage, double C, cudaStream_t st) {
  const KernelSet* ks = e->ks;
  const long long N = e->N, M = e->M, Nh = e->Nh;
  const unsigned B = unsigned(launch_members(e));
  const int nc = ks->tiles[e->v_cols & 1].nc;
  cudaError_t ce;
  if (e->dim == 3) {
    // pass 1: inverse along x with padding, state [3][N][N][Nh] -> A1 [M][N][r3]
    // (column p: group y = p / r3, entry q = 3 z + component, q < 3 Nh)
    // (the single-tile kernel runs it on the wider tiles of the first pass)
    const bool wide = !(e->v_cols & 2);
    const int nc1 = wide ? ks->tiles[e->v_cols & 1].ncx : nc;
    ColArgs a1{};
    a1.in = u;
    a1.out = e->buf[0];
    a1.tw = e->tw;
    a1.ninner = N * e->ra1;
    a1.ntile = int(cdiv(a1.ninner, nc1));
    a1.n_short = int(N);
    a1.in_row = u_inner ? 3 * N * Nh : N * Nh;
    a1.out_row = N * e->ra1;
    if (e->ra1 != 3 * Nh) {
      a1.grp = int(e->ra1);
      a1.grp_valid = int(3 * Nh);
      a1.in_grp = u_inner ? 3 * Nh : Nh;
    }
    // component innermost: entry q = 3 z + component is already the input's
    // order, so the columns read straight runs
    a1.in_comp = u_inner ? 0 : N * N * Nh;
    a1.in_ci = u_inner ? 1 : 3;
    a1.in_mem = e->state_mem;
    a1.out_mem = e->buf_mem[0];
    a1.ctrl = e->ctrl;
    a1.clear_max = 1;
    {
      ProfScope ps(P_INV_X, double(B) * 3 * (N * N * Nh + M * N * Nh) * e->csize, st, e->prof);
      ce = ks->cols(e->v_cols, wide ? COLK_PAD_INV_WIDE : COLK_PAD_INV, a1, unsigned(a1.ntile), 1, B, st);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "rhs pass 1");
    // pass 2: inverse along y with padding, A1 -> A2 [M][M][r3]
    ColArgs a2{};
    a2.in = e->buf[0];
    a2.out = e->buf[1];
    a2.tw = e->tw;
    a2.ninner = 3 * Nh;
    a2.ntile = int(cdiv(a2.ninner, nc));
    a2.n_short = int(N);
    a2.in_row = e->ra1;
    a2.out_row = e->ra2;
    a2.in_outer = N * e->ra1;
    a2.out_outer = M * e->ra2;
    a2.in_ci = 1;
    a2.in_mem = e->buf_mem[0];
    a2.out_mem = e->buf_mem[1];
    a2.ctrl = e->ctrl;
    {
      ProfScope ps(P_INV_Y, double(B) * 3 * (M * N * Nh + M * M * Nh) * e->csize, st, e->prof);
      ce = ks->cols(e->v_cols, COLK_PAD_INV, a2, unsigned(a2.ntile * M), 1, B, st);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "rhs pass 2");
    // pass 3: z lines, product, CFL max: A2 -> B1 [M][M][r6]
    RowArgs r{};
    r.in = e->buf[1];
    r.out = e->buf[2];
    r.tw = e->tw;
    r.nlines = M * M;
    r.nh = int(Nh);
    r.in_line = e->ra2;
    r.out_line = e->rb1;
    r.in_mem = e->buf_mem[1];
    r.out_mem = e->buf_mem[2];
    r.norm = e->norm;
    r.ctrl = e->ctrl;
    {
      ProfScope ps(P_PRODUCT, double(B) * 9 * (M * M * Nh) * e->csize, st, e->prof);
      ce = product_pass(e, 3, r, st);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "rhs pass 3");
  } else {
    // pass 1: inverse along x with padding, state [2][N][Nh] -> A1 [M][r3]
    ColArgs a1{};
    a1.in = u;
    a1.out = e->buf[0];
    a1.tw = e->tw;
    a1.ninner = 2 * Nh;
    a1.ntile = int(cdiv(a1.ninner, nc));
    a1.n_short = int(N);
    a1.in_row = u_inner ? 2 * Nh : Nh;
    a1.out_row = e->ra1;
    a1.in_comp = u_inner ? 0 : N * Nh;
    a1.in_ci = u_inner ? 1 : 2;
    a1.in_mem = e->state_mem;
    a1.out_mem = e->buf_mem[0];
    a1.ctrl = e->ctrl;
    a1.clear_max = 1;
    {
      ProfScope ps(P_INV_X, double(B) * 2 * (N * Nh + M * Nh) * e->csize, st, e->prof);
      ce = ks->cols(e->v_cols, COLK_PAD_INV, a1, unsigned(a1.ntile), 1, B, st);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "rhs pass 1 (2-D)");
    // pass 2: y lines, product, CFL max: A1 -> B1 [M][r6]
    RowArgs r{};
    r.in = e->buf[0];
    r.out = e->buf[1];
    r.tw = e->tw;
    r.nlines = M;
    r.nh = int(Nh);
    r.in_line = e->ra1;
    r.out_line = e->rb1;
    r.in_mem = e->buf_mem[0];
    r.out_mem = e->buf_mem[1];
    r.norm = e->norm;
    r.ctrl = e->ctrl;
    {
      ProfScope ps(P_PRODUCT, double(B) * 5 * (M * Nh) * e->csize, st, e->prof);
      ce = product_pass(e, 2, r, st);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "rhs pass 2 (2-D)");
  }
  if (first_stage) {
    k_ctrl_dt<<<unsigned(cdiv(B, 128)), 128, 0, st>>>(e->ctrl, int(B), C, double(N), e->Md, e->prec);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return cuda_fail(ce, "k_ctrl_dt");
  }
  const char* bsrc;
  long long b_row, b_mem, ninner;
  if (e->dim == 3) {
    // pass 4: forward along y, keep retained rows: B1 -> B2 [M][N][r6]
    ColArgs a4{};
    a4.in = e->buf[2];
    a4.out = e->buf[0];
    a4.tw = e->tw;
    a4.ninner = 6 * Nh;
    a4.ntile = int(cdiv(a4.ninner, nc));
    a4.n_short = int(N);
    a4.in_row = e->rb1;
    a4.out_row = e->rb2;
    a4.in_outer = M * e->rb1;
    a4.out_outer = N * e->rb2;
    a4.in_ci = 1;
    a4.in_mem = e->buf_mem[2];
    a4.out_mem = e->buf_mem[0];
    a4.ctrl = e->ctrl;
    {
      ProfScope ps(P_FWD_Y, double(B) * 6 * (M * M * Nh + M * N * Nh) * e->csize, st, e->prof);
      ce = ks->cols(e->v_cols, COLK_TRUNC_FWD, a4, unsigned(a4.ntile * M), 1, B, st);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "rhs pass 4");
    bsrc = e->buf[0];
    b_row = N * e->rb2;
    b_mem = e->buf_mem[0];
    ninner = N * Nh;
  } else {
    bsrc = e->buf[1];
    b_row = e->rb1;
    b_mem = e->buf_mem[1];
    ninner = Nh;
  }
  EpiArgs ep{};
  ep.B = bsrc;
  ep.u = u;
  ep.u0 = u0 ? u0 : u;
  ep.out = out;
  ep.tw = e->tw;
  ep.ninner = ninner;
  const int ncm = e->dim == 3 ? ks->tiles[e->v_epi].ncm3 : ks->tiles[e->v_epi].ncm2;
  ep.ntile = int(cdiv(ninner, ncm));
  ep.N = int(N);
  ep.nh = int(Nh);
  ep.B_row = b_row;
  ep.B_mem = b_mem;
  ep.b_grp = (e->dim == 3 && e->rb2 != 6 * Nh) ? e->rb2 : 0;
  ep.lu = state_layout(e, u_inner);
  ep.lu0 = u0 ? state_layout(e, u0_inner) : ep.lu;
  ep.lout = state_layout(e, out_inner);
  ep.u_mem = e->state_mem;
  ep.mode = mode;
  ep.visc = e->visc;
  ep.ctrl = e->ctrl;
  {
    // B read + u read + out write (+ u0 read in stages 2 and 3)
    const long long nb = e->dim == 3 ? 6 : 3;
    const long long modes = e->dim == 3 ? N * N * Nh : N * Nh;
    const double elems = double(nb) * M * ninner + double(e->dim) * modes * ((mode >= MODE_RK2) ? 3 : 2);
    ProfScope ps(P_EPILOGUE, double(B) * elems * e->csize, st, e->prof);
    ce = ks->epilogue(e->v_epi, e->dim, ep, unsigned(ep.ntile), B, st);
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "rhs epilogue pass");
  return AZ_OK;
}

}  // namespace azb

az_status az_euler_dudt(az_euler e, void* dudt_hat, const void* u_hat, double t, double dt, double C,
                        void* stream) {
  (void)t;
  (void)dt;
  if (!e || !dudt_hat || !u_hat) return fail(AZ_ERR_INVALID, "az_euler_dudt: null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // A plain right-hand side: clear any skip flag left by a finished simulation.
  k_ctrl_begin_host<<<unsigned(cdiv(e->batch, 128)), 128, 0, st>>>(e->ctrl, e->batch, 0.0);
  AZB_CUDA(cudaGetLastError());
  return rhs(e, u_hat, false, nullptr, false, dudt_hat, false, MODE_DUDT, false, C, st);
}

namespace azb {
az_status euler_dudt_launch(az_euler e, void* dudt_hat, const void* u_hat, cudaStream_t st) {
  k_ctrl_begin_host<<<unsigned(cdiv(e->batch, 128)), 128, 0, st>>>(e->ctrl, e->batch, 0.0);
  AZB_CUDA(cudaGetLastError());
  return rhs(e, u_hat, false, nullptr, false, dudt_hat, false, MODE_DUDT, false, 0.0, st);
}
az_status set_error(az_status st, const char* msg) { return fail(st, msg); }
const KernelSet* find_kernel_set(int precision, int L) { return kernel_set(precision, L); }
az_status ctrl_status(int err) { return err ? ctrl_error(err) : AZ_OK; }
}  // namespace azb

az_status az_debug_set_wait_limit(int polls) {
  if (polls < 0) return fail(AZ_ERR_INVALID, "az_debug_set_wait_limit: polls must be >= 0");
  g_wait_polls = polls;
  return AZ_OK;
}

int az_debug_get_wait_limit(void) { return g_wait_polls; }

az_status az_euler_dt(az_euler e, double C, void* stream, double* out) {
  if (!e || !out) return fail(AZ_ERR_INVALID, "az_euler_dt: null argument");
  std::vector<Ctrl> h(e->batch);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AZB_CUDA(cudaMemcpyAsync(h.data(), e->ctrl, sizeof(Ctrl) * e->batch, cudaMemcpyDeviceToHost, st));
  AZB_CUDA(cudaStreamSynchronize(st));
  for (int b = 0; b < e->batch; ++b) {
    double umax;
    if (e->prec == 0) {
      std::memcpy(&umax, &h[b].umax64, sizeof(double));
    } else {
      float f;
      std::memcpy(&f, &h[b].umax32, sizeof(float));
      umax = f;
    }
    const double u_max_ = umax / e->Md;
    out[b] = C / ((double)e->N * u_max_);
  }
  for (int b = 0; b < e->batch; ++b)
    if (h[b].err) return ctrl_error(h[b].err);
  return AZ_OK;
}

az_status az_tune_set(int precision, int L, int kind, int variant) {
  const int vmax = kind % 3 == 2 ? 1 : kind % 3 == 1 ? 7 : 3;
  if ((precision != 0 && precision != 1) || kind < 0 || kind > 5 || variant < 0 || variant > vmax)
    return fail(AZ_ERR_INVALID, "az_tune_set: bad argument");
  if (!kernel_set(precision, L)) return fail(AZ_ERR_UNSUPPORTED, "az_tune_set: no compiled length");
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune[std::make_tuple(precision, L, kind)] = variant;
  return AZ_OK;
}

az_status az_tune_get(int precision, int L, int kind, int* variant) {
  if (!variant || kind < 0 || kind > 5) return fail(AZ_ERR_INVALID, "az_tune_get: bad argument");
  *variant = tuned_variant(precision, L, kind);
  return AZ_OK;
}

az_status az_profile_enable(int on) {
  g_prof = on != 0;
  return AZ_OK;
}

az_status az_profile_read(double* ms, double* bytes, long long* launches, int npass) {
  if (npass < P_NPASS) return fail(AZ_ERR_INVALID, "az_profile_read: need room for every pass");
  for (int p = 0; p < npass; ++p) {
    if (ms) ms[p] = 0;
    if (bytes) bytes[p] = 0;
    if (launches) launches[p] = 0;
  }
  for (auto& r : g_prof_recs) {
    cudaError_t ce = cudaEventSynchronize(r.b);
    if (ce != cudaSuccess) return cuda_fail(ce, "az_profile_read");
    float t = 0;
    cudaEventElapsedTime(&t, r.a, r.b);
    if (ms) ms[r.pass] += t;
    if (bytes) bytes[r.pass] += r.bytes;
    if (launches) launches[r.pass] += 1;
    g_prof_pool.push_back(r.a);
    g_prof_pool.push_back(r.b);
  }
  g_prof_recs.clear();
  return AZ_OK;
}

// ---------------------------------------------------------------------------
// SSP-RK3
// ---------------------------------------------------------------------------
struct az_rk3_s {
  az_euler eq;
  void* u1 = nullptr;
  void* u2 = nullptr;
};

az_status az_rk3_create(az_euler eq, az_rk3* out) {
  if (!eq || !out) return fail(AZ_ERR_INVALID, "az_rk3_create: null argument");
  auto* r = new az_rk3_s();
  r->eq = eq;
  const size_t bytes = size_t(eq->state_elems) * eq->csize;
  if (cudaMalloc(&r->u1, bytes) != cudaSuccess || cudaMalloc(&r->u2, bytes) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(r->u1);
    cudaFree(r->u2);
    delete r;
    return fail(AZ_ERR_NOMEM, "az_rk3_create: stage arrays");
  }
  *out = r;
  return AZ_OK;
}

az_status az_rk3_destroy(az_rk3 r) {
  if (!r) return AZ_OK;
  cudaFree(r->u1);
  cudaFree(r->u2);
  delete r;
  return AZ_OK;
}

namespace azb {
// The three stages of SSP_RK3::integrate (ssp_rk3.hpp:48-64); the control
// block must already hold max_dt and skip for this step.
static az_status rk3_stages(az_rk3 r, void* u, double C, cudaStream_t st) {
  az_euler e = r->eq;
  az_status s;
  // u (the caller's) is planar; the stage buffers u1 and u2 are component
  // innermost.
  s = rhs(e, u, false, nullptr, false, r->u1, true, MODE_RK1, true, C, st);
  if (s != AZ_OK) return s;
  s = rhs(e, r->u1, true, u, false, r->u2, true, MODE_RK2, false, C, st);
  if (s != AZ_OK) return s;
  return rhs(e, r->u2, true, u, false, u, false, MODE_RK3, false, C, st);
}
}  // namespace azb

az_status az_rk3_integrate(az_rk3 r, double t, double max_dt, double C, void* u_hat, void* stream,
                           double* dt_out) {
  (void)t;
  if (!r || !u_hat) return fail(AZ_ERR_INVALID, "az_rk3_integrate: null argument");
  az_euler e = r->eq;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_ctrl_begin_host<<<unsigned(cdiv(e->batch, 128)), 128, 0, st>>>(e->ctrl, e->batch, max_dt);
  AZB_CUDA(cudaGetLastError());
  az_status s = rk3_stages(r, u_hat, C, st);
  if (s != AZ_OK) return s;
  std::vector<Ctrl> h(e->batch);
  AZB_CUDA(cudaMemcpyAsync(h.data(), e->ctrl, sizeof(Ctrl) * e->batch, cudaMemcpyDeviceToHost, st));
  AZB_CUDA(cudaStreamSynchronize(st));
  for (int b = 0; b < e->batch; ++b) {
    if (dt_out) dt_out[b] = h[b].dt;
    if (h[b].err) return ctrl_error(h[b].err);
  }
  return AZ_OK;
}

// ---------------------------------------------------------------------------
// Simulation
// ---------------------------------------------------------------------------
struct az_sim_s {
  az_rk3 ts;
  double C;
  void* u = nullptr;
  Ctrl* host = nullptr;  // pinned mirror of the control blocks
  // One captured SSP-RK3 step.  Every value that changes from step to step
  // (dt, clock, skip flag, CFL maximum) lives in the device control block, so
  // the same graph replays every step.
  cudaGraphExec_t exec = nullptr;
  bool graph_failed = false;
  // The same step over a prefix [0, n) of the members, per n (groups'
  // active-prefix steps).
  std::map<int, cudaGraphExec_t> exec_prefix;
};

az_status az_sim_create(az_rk3 ts, double C, const void* u_init, void* stream, az_sim* out) {
  if (!ts || !u_init || !out) return fail(AZ_ERR_INVALID, "az_sim_create: null argument");
  az_euler e = ts->eq;
  auto* s = new az_sim_s();
  s->ts = ts;
  s->C = C;
  const size_t bytes = size_t(e->state_elems) * e->csize;
  if (cudaMalloc(&s->u, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return fail(AZ_ERR_NOMEM, "az_sim_create: state");
  }
  if (cudaMallocHost(&s->host, sizeof(Ctrl) * e->batch) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(s->u);
    delete s;
    return fail(AZ_ERR_NOMEM, "az_sim_create: pinned control mirror");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t ce = cudaMemcpyAsync(s->u, u_init, bytes, cudaMemcpyDeviceToDevice, st);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(e->ctrl, 0, sizeof(Ctrl) * e->batch, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) {
    cudaFree(s->u);
    cudaFreeHost(s->host);
    delete s;
    return cuda_fail(ce, "az_sim_create");
  }
  *out = s;
  return AZ_OK;
}

az_status az_sim_destroy(az_sim s) {
  if (!s) return AZ_OK;
  if (s->exec) cudaGraphExecDestroy(s->exec);
  for (auto& kv : s->exec_prefix) cudaGraphExecDestroy(kv.second);
  cudaFree(s->u);
  cudaFreeHost(s->host);
  delete s;
  return AZ_OK;
}

void* az_sim_u(az_sim s) { return s ? s->u : nullptr; }

namespace azb {
__global__ void k_ctrl_set_tend(Ctrl* c, int n, double t_end) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    c[i].t_end = t_end;
    c[i].skip = 0;
  }
}
__global__ void k_ctrl_finish(Ctrl* c, int n, double t_end) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    c[i].time = t_end;  // simulation.cpp:102
    c[i].skip = 0;
  }
}

static double visc_cap(az_euler e, double C) {
  const double eps = e->eps_visc;
  if (eps == 0.0) return INFINITY;
  const double piN = 3.14159265358979323846 * (double)e->N;
  return C * 2. / (eps * (piN * piN));  // simulation.cpp:92-93
}

static az_status sim_step(az_sim s, cudaStream_t st) {
  az_euler e = s->ts->eq;
  const int nb = launch_members(e);
  const unsigned g = unsigned(cdiv(nb, 128));
  k_ctrl_begin_sim<<<g, 128, 0, st>>>(e->ctrl, nb, visc_cap(e, s->C));
  AZB_CUDA(cudaGetLastError());
  az_status r = rk3_stages(s->ts, s->u, s->C, st);
  if (r != AZ_OK) return r;
  k_ctrl_end<<<g, 128, 0, st>>>(e->ctrl, nb);
  AZB_CUDA(cudaGetLastError());
  return AZ_OK;
}
// Captures one step into a graph (once).  Returns false if the graph is not
// usable (per-pass profiling is on, or capture failed), in which case the
// caller launches eagerly.
static bool sim_graph(az_sim s) {
  if (g_prof || s->graph_failed) return false;
  if (s->exec) return true;
  cudaStream_t cap = nullptr;
  if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    s->graph_failed = true;
    return false;
  }
  cudaGraph_t g = nullptr;
  bool ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    const az_status st = sim_step(s, cap);
    const cudaError_t ce = cudaStreamEndCapture(cap, &g);
    ok = st == AZ_OK && ce == cudaSuccess && g != nullptr;
  }
  if (ok) ok = cudaGraphInstantiate(&s->exec, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cap);
  if (!ok) {
    cudaGetLastError();
    s->exec = nullptr;
    s->graph_failed = true;
  }
  return ok;
}

static az_status sim_run_steps(az_sim s, int n, cudaStream_t st) {
  if (n <= 0) return AZ_OK;
  if (sim_graph(s)) {
    for (int i = 0; i < n; ++i) AZB_CUDA(cudaGraphLaunch(s->exec, st));
    return AZ_OK;
  }
  for (int i = 0; i < n; ++i) {
    az_status r = sim_step(s, st);
    if (r != AZ_OK) return r;
  }
  return AZ_OK;
}

// Captures one step over members [0, n) into a graph (once per n); nullptr
// when graphs are unusable (per-pass profiling, failed capture), and the
// caller then launches eagerly.
static cudaGraphExec_t sim_graph_prefix(az_sim s, int n) {
  if (g_prof || s->graph_failed) return nullptr;
  auto it = s->exec_prefix.find(n);
  if (it != s->exec_prefix.end()) return it->second;
  az_euler e = s->ts->eq;
  cudaStream_t cap = nullptr;
  if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  e->nlaunch = n;
  bool ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    const az_status st = sim_step(s, cap);
    const cudaError_t ce = cudaStreamEndCapture(cap, &g);
    ok = st == AZ_OK && ce == cudaSuccess && g != nullptr;
  }
  e->nlaunch = 0;
  if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cap);
  if (!ok) {
    cudaGetLastError();
    return nullptr;
  }
  s->exec_prefix[n] = ex;
  return ex;
}

static az_status sim_steps_prefix(az_sim s, int n, int nsteps, cudaStream_t st) {
  if (cudaGraphExec_t ex = sim_graph_prefix(s, n)) {
    for (int i = 0; i < nsteps; ++i) AZB_CUDA(cudaGraphLaunch(ex, st));
    return AZ_OK;
  }
  az_euler e = s->ts->eq;
  e->nlaunch = n;
  az_status r = AZ_OK;
  for (int i = 0; i < nsteps && r == AZ_OK; ++i) r = sim_step(s, st);
  e->nlaunch = 0;
  return r;
}
}  // namespace azb

az_status az_sim_simulate_until(az_sim s, double t, void* stream) {
  if (!s) return fail(AZ_ERR_INVALID, "az_sim_simulate_until: null argument");
  az_euler e = s->ts->eq;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned g = unsigned(cdiv(e->batch, 128));
  k_ctrl_set_tend<<<g, 128, 0, st>>>(e->ctrl, e->batch, t);
  AZB_CUDA(cudaGetLastError());
  int chunk = 1;
  for (;;) {
    az_status r = sim_run_steps(s, chunk, st);
    if (r != AZ_OK) return r;
    AZB_CUDA(cudaMemcpyAsync(s->host, e->ctrl, sizeof(Ctrl) * e->batch, cudaMemcpyDeviceToHost, st));
    AZB_CUDA(cudaStreamSynchronize(st));
    // A member is done once its clock reached t (simulation.cpp:90).
    double min_left = INFINITY;
    bool any = false;
    for (int b = 0; b < e->batch; ++b) {
      if (s->host[b].err) return ctrl_error(s->host[b].err);
      if (s->host[b].time < t) {
        any = true;
        const double dt = s->host[b].dt > 0 ? s->host[b].dt : 0.0;
        const double left = dt > 0 ? (t - s->host[b].time) / dt : 1.0;
        if (left < min_left) min_left = left;
      }
    }
    if (!any) break;
    // Steps that cannot overshoot any member's end (a finished member's
    // steps are skipped on the device anyway).
    chunk = int(std::floor(min_left * 0.9));
    if (chunk < 1) chunk = 1;
    if (chunk > 64) chunk = 64;
  }
  k_ctrl_finish<<<g, 128, 0, st>>>(e->ctrl, e->batch, t);
  AZB_CUDA(cudaGetLastError());
  return AZ_OK;
}

az_status az_sim_steps(az_sim s, int nsteps, void* stream) {
  if (!s || nsteps < 0) return fail(AZ_ERR_INVALID, "az_sim_steps: bad argument");
  az_euler e = s->ts->eq;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned g = unsigned(cdiv(e->batch, 128));
  k_ctrl_set_tend<<<g, 128, 0, st>>>(e->ctrl, e->batch, INFINITY);
  AZB_CUDA(cudaGetLastError());
  return sim_run_steps(s, nsteps, st);
}

namespace azb {
__global__ void k_ctrl_member(Ctrl* c, double time, double t_end, int clear_steps) {
  c->time = time;
  c->t_end = t_end;
  c->skip = 0;
  c->err = 0;
  c->dt = 0.0;
  if (clear_steps) c->nsteps = 0;
}
}  // namespace azb

az_status az_sim_member_start(az_sim s, int member, const void* u_hat_member, double t_end, void* stream) {
  if (!s || !u_hat_member) return fail(AZ_ERR_INVALID, "az_sim_member_start: null argument");
  az_euler e = s->ts->eq;
  if (member < 0 || member >= e->batch) return fail(AZ_ERR_INVALID, "az_sim_member_start: member out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t bytes = size_t(e->state_mem) * e->csize;
  AZB_CUDA(cudaMemcpyAsync(static_cast<char*>(s->u) + size_t(member) * bytes, u_hat_member, bytes,
                           cudaMemcpyDeviceToDevice, st));
  k_ctrl_member<<<1, 1, 0, st>>>(e->ctrl + member, 0.0, t_end, 1);
  AZB_CUDA(cudaGetLastError());
  return AZ_OK;
}

az_status az_sim_member_stop(az_sim s, int member, void* stream) {
  if (!s) return fail(AZ_ERR_INVALID, "az_sim_member_stop: null argument");
  az_euler e = s->ts->eq;
  if (member < 0 || member >= e->batch) return fail(AZ_ERR_INVALID, "az_sim_member_stop: member out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // A clock past its end makes every kernel of the next steps skip the slot.
  k_ctrl_member<<<1, 1, 0, st>>>(e->ctrl + member, 1.0, 0.0, 1);
  AZB_CUDA(cudaGetLastError());
  return AZ_OK;
}

// ---------------------------------------------------------------------------
// Groups: several simulations (any dimension, size or precision) advanced by
// one captured graph per step, each on its own branch of the graph.
// ---------------------------------------------------------------------------
struct az_group_s {
  std::vector<az_sim> sims;
  cudaGraphExec_t exec = nullptr;
  // Branch streams and events of the active-prefix steps.
  std::vector<cudaStream_t> br;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
};

static void group_free_branches(az_group g) {
  for (cudaStream_t b : g->br)
    if (b) cudaStreamDestroy(b);
  for (cudaEvent_t j : g->join)
    if (j) cudaEventDestroy(j);
  if (g->fork) cudaEventDestroy(g->fork);
  g->br.clear();
  g->join.clear();
  g->fork = nullptr;
}

az_status az_group_create(az_sim* sims, int n, az_group* out) {
  if (!sims || n < 1 || !out) return fail(AZ_ERR_INVALID, "az_group_create: bad argument");
  if (g_prof) return fail(AZ_ERR_INVALID, "az_group_create: per-pass profiling must be off while a graph is captured");
  auto* g = new az_group_s();
  g->sims.assign(sims, sims + n);
  for (az_sim s : g->sims)
    if (!s) {
      delete g;
      return fail(AZ_ERR_INVALID, "az_group_create: null simulation");
    }
  // Capture: fork one branch per simulation from a root stream, join back.
  std::vector<cudaStream_t> br(n, nullptr);
  cudaStream_t root = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join(n, nullptr);
  bool ok = cudaStreamCreateWithFlags(&root, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; ok && i < n; ++i)
    ok = cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming) == cudaSuccess;
  cudaGraph_t graph = nullptr;
  az_status step_status = AZ_OK;
  if (ok) ok = cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    cudaEventRecord(fork, root);
    for (int i = 0; i < n; ++i) {
      cudaStreamWaitEvent(br[i], fork, 0);
      if (step_status == AZ_OK) step_status = sim_step(g->sims[i], br[i]);
      cudaEventRecord(join[i], br[i]);
      cudaStreamWaitEvent(root, join[i], 0);
    }
    const cudaError_t ce = cudaStreamEndCapture(root, &graph);
    ok = ce == cudaSuccess && step_status == AZ_OK && graph != nullptr;
  }
  if (ok) ok = cudaGraphInstantiate(&g->exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  for (int i = 0; i < n; ++i) {
    if (br[i]) cudaStreamDestroy(br[i]);
    if (join[i]) cudaEventDestroy(join[i]);
  }
  if (fork) cudaEventDestroy(fork);
  if (root) cudaStreamDestroy(root);
  if (ok) {
    g->br.assign(n, nullptr);
    g->join.assign(n, nullptr);
    ok = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < n; ++i)
      ok = cudaStreamCreateWithFlags(&g->br[i], cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming) == cudaSuccess;
  }
  if (!ok) {
    const cudaError_t last = cudaGetLastError();
    if (g->exec) cudaGraphExecDestroy(g->exec);
    group_free_branches(g);
    delete g;
    if (step_status != AZ_OK) return step_status;
    return fail(AZ_ERR_CUDA, std::string("az_group_create: graph capture failed: ") + cudaGetErrorString(last));
  }
  *out = g;
  return AZ_OK;
}

az_status az_group_destroy(az_group g) {
  if (!g) return AZ_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  group_free_branches(g);
  delete g;
  return AZ_OK;
}

az_status az_group_steps(az_group g, int nsteps, void* stream) {
  if (!g || nsteps < 0) return fail(AZ_ERR_INVALID, "az_group_steps: bad argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int i = 0; i < nsteps; ++i) AZB_CUDA(cudaGraphLaunch(g->exec, st));
  return AZ_OK;
}

az_status az_group_steps_active(az_group g, int nsteps, const int* nactive, void* stream) {
  if (!g || nsteps < 0 || !nactive) return fail(AZ_ERR_INVALID, "az_group_steps_active: bad argument");
  const int n = int(g->sims.size());
  for (int i = 0; i < n; ++i)
    if (nactive[i] < 0 || nactive[i] > g->sims[i]->ts->eq->batch)
      return fail(AZ_ERR_INVALID, "az_group_steps_active: active count out of range");
  if (nsteps == 0) return AZ_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AZB_CUDA(cudaEventRecord(g->fork, st));
  for (int i = 0; i < n; ++i) {
    if (nactive[i] == 0) continue;
    // Prefixes are rounded up to powers of two, so few graphs are captured.
    const int batch = g->sims[i]->ts->eq->batch;
    int nb = 1;
    while (nb < nactive[i]) nb <<= 1;
    if (nb > batch) nb = batch;
    AZB_CUDA(cudaStreamWaitEvent(g->br[i], g->fork, 0));
    const az_status r = sim_steps_prefix(g->sims[i], nb, nsteps, g->br[i]);
    if (r != AZ_OK) return r;
    AZB_CUDA(cudaEventRecord(g->join[i], g->br[i]));
    AZB_CUDA(cudaStreamWaitEvent(st, g->join[i], 0));
  }
  return AZ_OK;
}

az_status az_group_set_end(az_group g, double t, void* stream) {
  if (!g) return fail(AZ_ERR_INVALID, "az_group_set_end: null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (az_sim s : g->sims) {
    az_euler e = s->ts->eq;
    k_ctrl_set_tend<<<unsigned(cdiv(e->batch, 128)), 128, 0, st>>>(e->ctrl, e->batch, t);
    AZB_CUDA(cudaGetLastError());
  }
  return AZ_OK;
}

az_status az_group_simulate_until(az_group g, double t, void* stream) {
  if (!g) return fail(AZ_ERR_INVALID, "az_group_simulate_until: null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  az_status r = az_group_set_end(g, t, stream);
  if (r != AZ_OK) return r;
  // Each chunk steps only the members up to each simulation's last unfinished
  // one (none once a simulation is done), so a simulation that finished
  // early costs nothing while the others run on.
  const int n = int(g->sims.size());
  std::vector<int> active(n);
  for (int i = 0; i < n; ++i) active[i] = g->sims[i]->ts->eq->batch;
  int chunk = 1;
  for (;;) {
    r = az_group_steps_active(g, chunk, active.data(), stream);
    if (r != AZ_OK) return r;
    double min_left = INFINITY;
    bool any = false;
    for (az_sim s : g->sims) {
      az_euler e = s->ts->eq;
      AZB_CUDA(cudaMemcpyAsync(s->host, e->ctrl, sizeof(Ctrl) * e->batch, cudaMemcpyDeviceToHost, st));
    }
    AZB_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
      az_sim s = g->sims[i];
      az_euler e = s->ts->eq;
      active[i] = 0;
      for (int b = 0; b < e->batch; ++b) {
        if (s->host[b].err) return ctrl_error(s->host[b].err);
        if (s->host[b].time < t) {
          any = true;
          active[i] = b + 1;
          const double dt = s->host[b].dt;
          const double left = dt > 0 ? (t - s->host[b].time) / dt : 1.0;
          if (left < min_left) min_left = left;
        }
      }
    }
    if (!any) break;
    chunk = int(std::floor(min_left * 0.9));
    if (chunk < 1) chunk = 1;
    if (chunk > 64) chunk = 64;
  }
  for (az_sim s : g->sims) {
    az_euler e = s->ts->eq;
    k_ctrl_finish<<<unsigned(cdiv(e->batch, 128)), 128, 0, st>>>(e->ctrl, e->batch, t);
    AZB_CUDA(cudaGetLastError());
  }
  return AZ_OK;
}

az_status az_sim_state(az_sim s, void* stream, double* time, long long* nsteps, double* dt) {
  if (!s) return fail(AZ_ERR_INVALID, "az_sim_state: null argument");
  az_euler e = s->ts->eq;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AZB_CUDA(cudaMemcpyAsync(s->host, e->ctrl, sizeof(Ctrl) * e->batch, cudaMemcpyDeviceToHost, st));
  AZB_CUDA(cudaStreamSynchronize(st));
  for (int b = 0; b < e->batch; ++b) {
    if (time) time[b] = s->host[b].time;
    if (nsteps) nsteps[b] = s->host[b].nsteps;
    if (dt) dt[b] = s->host[b].dt;
  }
  return AZ_OK;
}

// ---------------------------------------------------------------------------
// Control kernels
// ---------------------------------------------------------------------------
namespace azb {
__global__ void k_ctrl_begin_host(Ctrl* c, int n, double max_dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    c[i].skip = 0;
    c[i].max_dt = max_dt;
    c[i].err = 0;
  }
}
__global__ void k_ctrl_begin_sim(Ctrl* c, int n, double cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    if (!(c[i].time < c[i].t_end)) {
      c[i].skip = 1;
    } else {
      c[i].skip = 0;
      c[i].max_dt = fmin(c[i].t_end - c[i].time, cap);
    }
  }
}
__global__ void k_ctrl_clear_max(Ctrl* c, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    c[i].umax64 = 0ull;
    c[i].umax32 = 0u;
  }
}
__global__ void k_ctrl_dt(Ctrl* c, int n, double C, double Nphys, double Md, int fp32) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !c[i].skip) {
    const double m = fp32 ? (double)__uint_as_float(c[i].umax32) : __longlong_as_double((long long)c[i].umax64);
    const double u_max_ = m / Md;
    const double dtc = C / (Nphys * u_max_);
    c[i].dt = fmin(dtc, c[i].max_dt);
  }
}
__global__ void k_ctrl_end(Ctrl* c, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !c[i].skip) {
    c[i].time += c[i].dt;
    c[i].nsteps += 1;
  }
}
}  // namespace azb

// ---------------------------------------------------------------------------
// FFT<Dim>
// ---------------------------------------------------------------------------
struct az_fft_s {
  int dim, prec, direction, nt;
  long long n_vars;
  long long shape[3];
  long long nh;
  const KernelSet* ks[3] = {nullptr, nullptr, nullptr};
  const void* tw[3] = {nullptr, nullptr, nullptr};
  void* u_hat;
  void* u;
  void* work = nullptr;
  size_t work_bytes = 0;
  bool owns_work = false;  // allocated here (on the first backward transform)
  size_t csize;
};

az_status az_fft_create(const az_fft_desc* d, void* u_hat, void* u, az_fft* out) {
  if (!d || !out || !u_hat || !u) return fail(AZ_ERR_INVALID, "az_fft_create: null argument");
  *out = nullptr;
  if (d->dim < 1 || d->dim > 3) return fail(AZ_ERR_INVALID, "az_fft_create: dim must be 1, 2 or 3");
  if (d->transform_last < 1 || d->transform_last > d->dim)
    return fail(AZ_ERR_INVALID, "az_fft_create: transform_last must be in [1, dim]");
  if (d->n_vars < 1) return fail(AZ_ERR_INVALID, "az_fft_create: n_vars must be >= 1");
  if (d->precision != AZ_PREC_F64 && d->precision != AZ_PREC_F32)
    return fail(AZ_ERR_INVALID, "az_fft_create: unknown precision");
  auto* f = new az_fft_s();
  f->dim = d->dim;
  f->prec = d->precision;
  f->direction = d->direction;
  f->nt = d->transform_last;
  f->n_vars = d->n_vars;
  f->u_hat = u_hat;
  f->u = u;
  f->csize = d->precision == 0 ? 16 : 8;
  for (int a = 0; a < d->dim; ++a) {
    f->shape[a] = d->shape[a];
    const bool transformed = a >= d->dim - d->transform_last;
    if (!transformed) continue;
    const KernelSet* ks = kernel_set(d->precision, int(d->shape[a]));
    if (!ks || d->shape[a] < 4) {
      delete f;
      return fail(AZ_ERR_UNSUPPORTED,
                  "az_fft_create: length " + std::to_string(d->shape[a]) + " has no compiled transform");
    }
    f->ks[a] = ks;
    az_status s = twiddles(d->precision, int(d->shape[a]), &f->tw[a]);
    if (s != AZ_OK) {
      delete f;
      return s;
    }
  }
  f->nh = d->shape[d->dim - 1] / 2 + 1;
  long long celems = f->n_vars * f->nh;
  for (int a = 0; a < d->dim - 1; ++a) celems *= d->shape[a];
  // Only backward transforms over more than one axis use a work area; it is
  // allocated on the first of them unless az_fft_set_work_area gave one, so
  // a forward-only FFT never allocates (nor frees: cudaFree waits for the
  // whole device).
  if (f->nt > 1) f->work_bytes = size_t(celems) * f->csize;
  *out = f;
  return AZ_OK;
}

az_status az_fft_destroy(az_fft f) {
  if (!f) return AZ_OK;
  if (f->owns_work) cudaFree(f->work);
  delete f;
  return AZ_OK;
}

az_status az_fft_set_work_area(az_fft f, void* work) {
  if (!f || !work) return fail(AZ_ERR_INVALID, "az_fft_set_work_area: null argument");
  if (f->owns_work) cudaFree(f->work);
  f->work = work;
  f->owns_work = false;
  return AZ_OK;
}

size_t az_fft_work_area_size(az_fft f) { return f ? f->work_bytes : 0; }

namespace azb {
// Column transform of the complex array [n_vars][n0..][nh] along axis `ax`.
static az_status fft_axis(az_fft f, int ax, const void* in, void* out, int kind, cudaStream_t st) {
  const KernelSet* ks = f->ks[ax];
  const long long rows = f->shape[ax];
  long long inner = f->nh;
  for (int a = ax + 1; a < f->dim - 1; ++a) inner *= f->shape[a];
  long long outer = f->n_vars;
  for (int a = 0; a < ax; ++a) outer *= f->shape[a];
  ColArgs c{};
  c.in = in;
  c.out = out;
  c.tw = f->tw[ax];
  c.ninner = inner;
  const int v = tuned_variant(f->prec, int(rows), 0) & 1;  // plain FFT axes: plan bit only
  c.ntile = int(cdiv(inner, ks->tiles[v].nc));
  c.n_short = int(rows);
  c.in_row = inner;
  c.out_row = inner;
  c.in_outer = rows * inner;
  c.out_outer = rows * inner;
  c.ctrl = nullptr;
  c.in_ci = 1;
  // grid.y carries the outer index in slices of at most 65535
  long long done = 0;
  while (done < outer) {
    const long long chunk = outer - done > 65535 ? 65535 : outer - done;
    ColArgs cc = c;
    cc.in = static_cast<const char*>(in) + done * rows * inner * f->csize;
    cc.out = static_cast<char*>(out) + done * rows * inner * f->csize;
    cc.in_comp = rows * inner;
    cc.out_comp = rows * inner;
    cc.in_outer = 0;
    cc.out_outer = 0;
    cudaError_t ce = ks->cols(v, kind, cc, unsigned(cc.ntile), unsigned(chunk), 1, st);
    if (ce != cudaSuccess) return cuda_fail(ce, "fft column pass");
    done += chunk;
  }
  return AZ_OK;
}
}  // namespace azb

az_status az_fft_forward(az_fft f, void* stream) {
  if (!f) return fail(AZ_ERR_INVALID, "az_fft_forward: null argument");
  if (!(f->direction & AZ_FFT_FORWARD)) return fail(AZ_ERR_INVALID, "FFT was not planned for forward transforms");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int last = f->dim - 1;
  long long lines = f->n_vars;
  for (int a = 0; a < last; ++a) lines *= f->shape[a];
  RealRowArgs r{};
  r.in = f->u;
  r.out = f->u_hat;
  r.tw = f->tw[last];
  r.nlines = lines;
  r.in_line = f->shape[last];
  r.out_line = f->nh;
  const int v = tuned_variant(f->prec, int(f->shape[last]), 1) & 1;  // plan bit only
  cudaError_t ce = f->ks[last]->r2c(v, r, unsigned(cdiv(lines, 2 * f->ks[last]->tiles[v].nlpr)), st);
  if (ce != cudaSuccess) return cuda_fail(ce, "fft r2c pass");
  for (int ax = last - 1; ax >= f->dim - f->nt; --ax) {
    az_status s = fft_axis(f, ax, f->u_hat, f->u_hat, COLK_PLAIN_FWD, st);
    if (s != AZ_OK) return s;
  }
  return AZ_OK;
}

az_status az_fft_backward(az_fft f, void* stream) {
  if (!f) return fail(AZ_ERR_INVALID, "az_fft_backward: null argument");
  if (!(f->direction & AZ_FFT_BACKWARD)) return fail(AZ_ERR_INVALID, "FFT was not planned for backward transforms");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int last = f->dim - 1;
  if (f->work_bytes > 0 && f->work == nullptr) {
    if (cudaMalloc(&f->work, f->work_bytes) != cudaSuccess) {
      cudaGetLastError();
      f->work = nullptr;
      return fail(AZ_ERR_NOMEM, "az_fft_backward: work area");
    }
    f->owns_work = true;
  }
  const void* src = f->u_hat;
  for (int ax = f->dim - f->nt; ax < last; ++ax) {
    az_status s = fft_axis(f, ax, src, f->work, COLK_PLAIN_INV, st);
    if (s != AZ_OK) return s;
    src = f->work;
  }
  long long lines = f->n_vars;
  for (int a = 0; a < last; ++a) lines *= f->shape[a];
  RealRowArgs r{};
  r.in = src;
  r.out = f->u;
  r.tw = f->tw[last];
  r.nlines = lines;
  r.in_line = f->nh;
  r.out_line = f->shape[last];
  const int v = tuned_variant(f->prec, int(f->shape[last]), 1) & 1;  // plan bit only
  cudaError_t ce = f->ks[last]->c2r(v, r, unsigned(cdiv(lines, 2 * f->ks[last]->tiles[v].nlpr)), st);
  if (ce != cudaSuccess) return cuda_fail(ce, "fft c2r pass");
  return AZ_OK;
}
