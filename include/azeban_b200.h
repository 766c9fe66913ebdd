/*
 * azeban_b200 -- C ABI of the B200-native spectral-viscosity incompressible
 * Euler right-hand side, its SSP-RK3 stepper and its real FFTs.
 *
 * Every entry point returns az_status (AZ_OK == 0) and never exits the
 * process; az_last_error_string() describes the last failure of the calling
 * thread.  Array arguments are DEVICE pointers in the layouts of the
 * reference (row-major, spectral arrays [n_vars][N][(N)][N/2+1] complex,
 * r2c along the last axis; include/azeban/grid.hpp:89-99).  Complex values
 * are interleaved (re, im) pairs of the solve's precision.  Streams are
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root).
 */
#ifndef AZEBAN_B200_H_
#define AZEBAN_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AZ_OK = 0,
  AZ_ERR_INVALID = 1,     /* bad argument (shape, null pointer, key) */
  AZ_ERR_UNSUPPORTED = 2, /* a size with no compiled transform length */
  AZ_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  AZ_ERR_NOMEM = 4,       /* device allocation failed */
  AZ_ERR_NONFINITE = 5,   /* the CFL reduction met Inf or NaN */
  AZ_ERR_TIMEOUT = 6      /* a bounded wait inside a kernel ran out; that pass is incomplete */
} az_status;

typedef enum { AZ_PREC_F64 = 0, AZ_PREC_F32 = 1 } az_precision;

typedef enum {
  AZ_VISC_NONE = 0,          /* NoViscosity, spectral_viscosity.hpp:125-128 */
  AZ_VISC_SMOOTH_CUTOFF = 1, /* SmoothCutoff1D, spectral_viscosity.hpp:56-77 */
  AZ_VISC_STEP = 2,          /* Step1D, spectral_viscosity.hpp:40-54 */
  AZ_VISC_QUADRATIC = 3      /* Quadratic, spectral_viscosity.hpp:103-123 */
} az_visc_type;

/* Viscosity as the reference's factory leaves it: eps already divided by
 * N^{2s-1} and k0 = m0 N^theta (spectral_viscosity_factory.hpp:29-89). */
typedef struct {
  int type;        /* az_visc_type */
  double eps;
  double s;        /* SmoothCutoff / Step */
  double k0;       /* SmoothCutoff / Step */
  long long N;     /* Quadratic */
} az_visc;

/* Replaces Grid<Dim> + the IncompressibleEuler<Dim, Visc, NoForcing>
 * constructor (include/azeban/grid.hpp:30-53,
 * include/azeban/equations/incompressible_euler.hpp:56-96). */
typedef struct {
  int dim;               /* 2 or 3 */
  long long N_phys;      /* N, even */
  long long N_phys_pad;  /* M >= N, a supported transform length */
  int precision;         /* az_precision; AZ_PREC_F32 = FP32 bulk, FP64 CFL */
  az_visc visc;
  int batch;             /* ensemble members of this N, >= 1; arrays are [batch][d][...] */
} az_euler_desc;

typedef struct az_euler_s* az_euler;
typedef struct az_rk3_s* az_rk3;
typedef struct az_sim_s* az_sim;
typedef struct az_fft_s* az_fft;

/* Last error of the calling thread ("" if none). */
const char* az_last_error_string(void);

/* Transform lengths with compiled kernels, written to out[0..*n) (capacity cap). */
az_status az_supported_lengths(int* out, int cap, int* n);

/* ---- Equation<Dim> (include/azeban/equations/equation.hpp:27-56) -------- */

/* IncompressibleEuler ctor; allocates its workspace
 * (incompressible_euler.hpp:56-96, src/azeban/memory/workspace.cpp:41-69). */
az_status az_euler_create(const az_euler_desc* desc, az_euler* out);
az_status az_euler_destroy(az_euler eq);

/* Equation<Dim>::dudt (incompressible_euler.hpp:103-120): dudt_hat <- RHS(u_hat).
 * dudt_hat may equal u_hat.  t, dt, C are accepted for interface parity
 * (they only feed forcing, which this path does not have). */
az_status az_euler_dudt(az_euler eq, void* dudt_hat, const void* u_hat, double t, double dt,
                        double C, void* stream);

/* Equation<Dim>::dt (incompressible_euler.hpp:122-124): C / (N u_max) of the
 * last dudt, per member (out[batch]).  Synchronises the stream. */
az_status az_euler_dt(az_euler eq, double C, void* stream, double* out);

/* Equation<Dim>::n_vars / visc (equation.hpp:44-46). */
int az_euler_n_vars(az_euler eq);
double az_euler_visc(az_euler eq);

/* Bytes of device workspace the equation holds. */
size_t az_euler_workspace_size(az_euler eq);

/* Kinetic energy 1/2 <|u|^2> and enstrophy 1/2 <|curl u|^2> of every member
 * of u_hat (host arrays of length batch), summed in FP64 with compensated
 * sums in a fixed order, for any precision of the solve.  No counterpart in
 * this form in the reference, which writes spectra of these quantities
 * (src/azeban/operations/energy_spectrum.cpp, enstrophy_spectrum.cpp).
 * Synchronises the stream. */
az_status az_euler_diagnostics(az_euler eq, const void* u_hat, void* stream, double* energy,
                               double* enstrophy);

/* ---- TimeIntegrator<Dim> / SSP_RK3<Dim> (include/azeban/evolution/time_integrator.hpp:30-60,
 *      include/azeban/evolution/ssp_rk3.hpp:28-76) ---------------------- */

/* SSP_RK3 ctor: allocates the stage arrays u1, u2 (ssp_rk3.hpp:39-42). */
az_status az_rk3_create(az_euler eq, az_rk3* out);
az_status az_rk3_destroy(az_rk3 ts);

/* SSP_RK3::integrate (ssp_rk3.hpp:48-64): one step of every member in place;
 * dt = min(equation dt(C), max_dt) of each member is written to dt_out[batch]
 * (host memory).  Synchronises the stream. */
az_status az_rk3_integrate(az_rk3 ts, double t, double max_dt, double C, void* u_hat,
                           void* stream, double* dt_out);

/* ---- Simulation<Dim> (include/azeban/simulation.hpp:30-93, src/azeban/simulation.cpp:89-102) */

/* Simulation ctor from an initial state (copied into the simulation). */
az_status az_sim_create(az_rk3 ts, double C, const void* u_hat_init, void* stream, az_sim* out);
az_status az_sim_destroy(az_sim sim);

/* Simulation::simulate_until: each member steps with its own dt until its
 * clock reaches t; the step size and the clock stay on the device. */
az_status az_sim_simulate_until(az_sim sim, double t, void* stream);

/* Exactly nsteps SSP-RK3 steps of every member (max_dt = viscous cap), with
 * no host synchronisation: the timed unit of the benchmark. */
az_status az_sim_steps(az_sim sim, int nsteps, void* stream);

/* Device pointer of the state [batch][d][...] (Simulation::u()). */
void* az_sim_u(az_sim sim);

/* Per-member clock, step count and last dt (host arrays of length batch).
 * Any pointer may be NULL.  Synchronises the stream. */
az_status az_sim_state(az_sim sim, void* stream, double* time, long long* nsteps, double* dt);

/* One member (slot) of a batched simulation, for continuous batching (no
 * counterpart in the reference, whose closest is the per-sample loop of
 * src/azeban/run_from_config.cpp:81-102).  member_start copies a state into
 * the slot and restarts its clock at 0 with end t_end; the slot then steps
 * with every step of the simulation (or of a group holding it) until its
 * clock reaches t_end, and is skipped afterwards.  member_stop frees the slot
 * (it is skipped until started again). */
az_status az_sim_member_start(az_sim sim, int member, const void* u_hat_member, double t_end,
                              void* stream);
az_status az_sim_member_stop(az_sim sim, int member, void* stream);

/* ---- groups of simulations (no counterpart in the reference) ------------ */

typedef struct az_group_s* az_group;

/* Several simulations of any dimension, size and precision advanced together:
 * one SSP-RK3 step of all of them is captured once as a graph with one branch
 * per simulation, so their work overlaps on the device.  The simulations must
 * outlive the group. */
az_status az_group_create(az_sim* sims, int n, az_group* out);
az_status az_group_destroy(az_group g);
/* nsteps graph launches; a member whose clock reached its end is skipped. */
az_status az_group_steps(az_group g, int nsteps, void* stream);
/* nsteps steps of members [0, nactive[i]) of simulation i only (none when
 * nactive[i] is 0), each simulation on its own branch; members past the
 * prefix are not touched, so every started member must lie inside it.  The
 * kernels launch over the prefix rounded up to a power of two (a step graph
 * per rounded prefix is captured on first use): a continuous-batching loop
 * then pays for the slots in use, not for every slot of every pool. */
az_status az_group_steps_active(az_group g, int nsteps, const int* nactive, void* stream);
/* Sets every member's end to t (no step). */
az_status az_group_set_end(az_group g, double t, void* stream);
/* simulate_until for every member of every simulation of the group; each
 * chunk of steps launches only the simulations with unfinished members, over
 * their members up to the last unfinished one. */
az_status az_group_simulate_until(az_group g, double t, void* stream);

/* ---- FFT<Dim> (include/azeban/operations/fft.hpp:37-121,
 *      make_fft src/azeban/operations/fft_factory.cpp:10-48) ----------- */

enum { AZ_FFT_FORWARD = 1, AZ_FFT_BACKWARD = 2 }; /* fft.hpp:28 */

typedef struct {
  int dim;                 /* 1, 2 or 3 */
  long long n_vars;        /* data_dim_: transforms batched over the first axis */
  long long shape[3];      /* real-space extents of the dim axes */
  int transform_last;      /* number of trailing axes transformed (1..dim) */
  int precision;           /* az_precision */
  int direction;           /* AZ_FFT_FORWARD | AZ_FFT_BACKWARD */
} az_fft_desc;

/* make_fft + FFT::initialize(u_hat, u): binds the arrays.  The work area
 * (backward transforms over more than one axis only) is allocated on the
 * first backward transform unless az_fft_set_work_area gave one. */
az_status az_fft_create(const az_fft_desc* desc, void* u_hat, void* u, az_fft* out);
az_status az_fft_destroy(az_fft fft);
/* FFT::set_work_area (fft.hpp:84): a caller-owned device buffer of
 * az_fft_work_area_size bytes, used instead of an allocation of its own. */
az_status az_fft_set_work_area(az_fft fft, void* work);
/* FFT::forward: u_hat <- unnormalised r2c(u) (fft.hpp:95). */
az_status az_fft_forward(az_fft fft, void* stream);
/* FFT::backward: u <- unnormalised c2r(u_hat) (fft.hpp:96); u_hat is kept. */
az_status az_fft_backward(az_fft fft, void* stream);
/* FFT::get_work_area_size (fft.hpp:93). */
size_t az_fft_work_area_size(az_fft fft);

/* ---- tuning table (no reference counterpart; the reference's nearest is
 *      optimal_fft_size reading a benchmark file, src/azeban/operations/fft.cpp:63-108) */

/* Kernel variant used for transform length L of a precision by one pass
 * kind: 0 column passes, 1 contiguous-axis passes, 2 epilogue pass of 3-D
 * solves (and of FFT<Dim>), 3-5 the same of 2-D solves.  Bit 0 picks the
 * radix plan (0: at most 24 elements per thread; 1: wide, fewer shared-memory
 * exchanges).  Bit 1: for column passes of solves (kinds 0, 3), the
 * two-tile kernel that overlaps one tile's input copies with the other's
 * transform; for contiguous-axis passes (kinds 1, 4), the bulk-copy kernel.
 * Kinds 0, 1, 3, 4 take variants 0-3, the epilogue kinds 0-1 (plain FFT<Dim>
 * transforms use bit 0 only).  Applies to solves and FFTs created
 * afterwards. */
az_status az_tune_set(int precision, int L, int kind, int variant);
az_status az_tune_get(int precision, int L, int kind, int* variant);

/* ---- per-pass timing (no reference counterpart; replaces the reference's
 *      Profiler, include/azeban/profiler.hpp:35-135, for the transform passes) */

/* When on, every pass launch of a right-hand side is bracketed by two CUDA
 * events on its stream. */
az_status az_profile_enable(int on);
/* Sums per pass id (0 inverse x, 1 inverse y, 2 product, 3 forward y,
 * 4 forward x + projection + stage) of event-timed milliseconds, algorithmic
 * bytes (one read of every input and one write of every output) and launch
 * counts since the last read; npass >= 5.  Waits for the recorded events. */
az_status az_profile_read(double* ms, double* bytes, long long* launches, int npass);

/* ---- failure detection (no reference counterpart: the reference has no
 *      in-kernel waits and aborts on errors, src/azeban/logging.hpp:24-32) */

/* Polls of the bounded wait with which the product pass waits for its bulk
 * copy (default 2^22).  A wait that runs out flags the member's error word;
 * the kernel then waits for the copy to land and returns, and the next call
 * that reads the error word (az_euler_dt, az_rk3_integrate, simulate_until,
 * az_euler_noalloc_status) returns AZ_ERR_TIMEOUT.  0 makes every such wait
 * run out at once: the way the tests exercise that path without a fault.
 * Applies to launches (and graph captures) made after the call. */
az_status az_debug_set_wait_limit(int polls);
int az_debug_get_wait_limit(void);

/* ---- leray (src/azeban/operations/leray.cpp:28-116) --------------------- */

/* In-place projection of u_hat [batch][dim][N]([N])[N/2+1] onto divergence-free
 * fields; the |k| = 0 mode is set to zero.  Used when building initial data
 * (include/azeban/init/initializer.hpp:68-75). */
az_status az_leray(int dim, long long N, int precision, void* u_hat, int batch, void* stream);

/* ---- initial data (include/azeban/init/initializer.hpp:48-75) ------------
 * The physical field is sampled on the device; az_fft_forward and az_leray
 * then give the spectral state, as Initializer::initialize does. */

enum {
  AZ_INIT_TAYLOR_GREEN = 0,          /* src/azeban/init/taylor_green.cpp:29-46 (2-D), :146-184 (3-D),
                                        with its perturbation modes (deltas) */
  AZ_INIT_TAYLOR_GREEN_WORKLOAD = 1, /* (sin x cos y, -cos x sin y[, 0]) with cos z in 3-D (no counterpart) */
  AZ_INIT_DOUBLE_SHEAR_LAYER = 2,    /* src/azeban/init/double_shear_layer.cpp:25-43, v = delta sin(2 pi x + phi) */
  AZ_INIT_GAUSSIAN_NOISE = 3         /* independent standard normals (the random fields' white noise) */
};

typedef struct {
  int kind;            /* AZ_INIT_* */
  int dim;             /* 2 or 3 */
  long long N;         /* grid points per axis */
  int precision;       /* az_precision of the field */
  int batch;           /* members; the field is [batch][dim][N]..[N] real */
  double rho, delta;   /* double shear layer */
  const double* deltas;  /* Taylor-Green perturbation amplitudes, host [batch][8 (2-D) | 24 (3-D)], or NULL */
  const double* phases;  /* double-shear-layer phases, host [batch], or NULL: drawn from the random stream */
  unsigned long long seed;  /* key of the random stream */
  long long member0;        /* member b draws from stream (seed, member0 + b) */
} az_init_desc;

/* Samples the physical field of every member into u (device).  Random values
 * (shear-layer phases when phases is NULL, Gaussian noise) come from the
 * counter-based Philox4x32-10 stream (seed, member): value c of a stream is a
 * function of (seed, member, c) alone.  The call waits for the stream only
 * when deltas or phases are given (their copy to the device). */
az_status az_init_physical(const az_init_desc* desc, void* u, void* stream);
/* u_hat [batch][dim][N]([N])[N/2+1] *= |n|^exponent per mode (n the integer
 * wavevector), 0 at n = 0: the amplitude envelope of a random field. */
az_status az_init_envelope(int dim, long long N, int precision, void* u_hat, int batch, double exponent,
                           void* stream);
/* Scales every member of u_hat to kinetic energy 1/2 <|u|^2> = target
 * (FP64 compensated sums on the device; nothing returns to the host). */
az_status az_init_normalize_energy(int dim, long long N, int precision, void* u_hat, int batch, double target,
                                   void* stream);
/* Value index of stream (seed, member) as a uniform double in [0, 1): the
 * draw the shear-layer phase takes (index 0), for the host. */
az_status az_random_uniform(unsigned long long seed, unsigned long long member, unsigned long long index,
                            double* out);
/* The block function of the stream: Philox4x32-10 of counter[4] under
 * key[2] (Salmon et al., SC 2011); stream (seed, member) block c has counter
 * (c lo, c hi, member lo, member hi) and key (seed lo, seed hi). */
az_status az_philox4x32_10(const unsigned* counter, const unsigned* key, unsigned* out);

/* ---- measurement (no counterpart in the reference) ----------------------- */

/* Times one radix-16 DFT stage of FP32 complex columns held in shared memory,
 * over ctas CTAs of 128 columns, done with the transform passes' butterflies
 * (method 0) or as a DFT-as-GEMM stage on the tensor pipe (method 1: the
 * 32x32 real form of the DFT matrix times the columns, mma.sync m16n8k8 TF32
 * with a three-term head/tail split for FP32 accuracy).  Writes the time per
 * column and stage in ns and the largest error of one stage relative to the
 * largest output (FP64 DFT reference). */
az_status az_bench_radix16_stage(int method, int ctas, double* ns_per_column_stage, double* max_rel_err);

/* Times the 384-point FP32 transform of the wide plan (radix 16, one
 * exchange, radix 24; 8 threads per column) over ctas CTAs of 32 columns held
 * in registers, with the exchange between the stages done through shared
 * memory as the transform passes do (method 0) or as a lane transpose with
 * warp shuffles among each column's 8 consecutive lanes (method 1: two CTAs
 * per SM as method 0; method 2: registers uncapped, one CTA per SM).  Writes
 * the time per column transform in ns and the largest error of one transform
 * relative to the largest output (FP64 DFT reference). */
az_status az_bench_exchange384(int method, int ctas, double* ns_per_column, double* max_rel_err);

/* ---- right-hand side without allocation (no counterpart in the reference) */

/* Size of the one device array that az_euler_dudt_noalloc takes its scratch from. */
#define AZ_NOALLOC_SCRATCH_BYTES (64LL * 1024 * 1024)

/* One right-hand side of one solve, the work of az_euler_dudt with batch 1,
 * that allocates nothing: no cudaMalloc, no cudaFree, no allocating library
 * call.  It has no counterpart in the reference.  It is for callers that
 * cannot let a library allocate device memory, such as a host code that owns
 * all device memory through its own pool under a fixed cap.  The scratch is
 * one file-scope device array of AZ_NOALLOC_SCRATCH_BYTES, held by every GPU
 * that loads the library until the process exits.  That bounds the sizes: at
 * 3/2 padding, 3-D up to N = 64 and 2-D up to N = 1024, in either precision;
 * a larger size returns AZ_ERR_UNSUPPORTED.  Each call looks up the array's
 * device address on the current device; the first call on a device may load
 * the library's device code to do so, so make it before any stream capture.  Every
 * call shares the array, so calls that overlap on the GPU race.  The call
 * does not wait for the GPU: device-side failures are read with
 * az_euler_noalloc_status. */
az_status az_euler_dudt_noalloc(int dim, long long N_phys, long long N_phys_pad, int precision,
                                const az_visc* visc, void* dudt_hat, const void* u_hat, void* stream);

/* Device-side status of the last az_euler_dudt_noalloc on the current device,
 * read from the control block in the same fixed array (no allocation):
 * AZ_OK, AZ_ERR_NONFINITE (the CFL reduction met Inf or NaN) or
 * AZ_ERR_TIMEOUT (a bounded wait ran out; the output is incomplete).
 * Synchronises the stream.  It has no counterpart in the reference. */
az_status az_euler_noalloc_status(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AZEBAN_B200_H_ */
