// Plain-old-data types shared by the CUDA kernels and the host runtime.
#pragma once

#include <cstdint>

namespace azb {

// Per-solve control block, resident in device memory.  Holds the CFL maximum
// of the current right-hand side, the step size and the solve's own clock, so
// a whole SSP-RK3 step runs without a host round trip.
struct alignas(64) Ctrl {
  unsigned long long umax64;  // max |u_i| over the padded grid, FP64 bits
  unsigned int umax32;        // the same, FP32 bits (FP32-bulk solves)
  int skip;                   // 1: this solve is finished, kernels return at once
  double dt;                  // step size of the current SSP-RK3 step
  double time;                // the solve's clock (Simulation::time_)
  double t_end;               // target of simulate_until
  double max_dt;              // min(t_end - time, viscous cap) of this step
  long long nsteps;           // completed steps
  int err;                    // bit 0: non-finite value met in the CFL reduction;
                              // bit 1: a bounded wait on a bulk copy ran out
  int pad_;
};

enum ViscType : int { VISC_NONE = 0, VISC_SMOOTH_CUTOFF = 1, VISC_STEP = 2, VISC_QUADRATIC = 3 };

// Viscosity parameters as the reference's factory leaves them
// (eps already divided by N^{2s-1}, k0 = m0 N^theta).
struct Visc {
  int type;
  int pad_;
  double eps;
  double s;
  double k0;
  long long N;
};

enum Mode : int { MODE_DUDT = 0, MODE_RK1 = 1, MODE_RK2 = 2, MODE_RK3 = 3 };

}  // namespace azb
