"""Where the FP32-bulk trajectory error comes from.

The FP32 form's error against FP64 grows over a trajectory faster than a
one-off rounding of the initial state would make it (the "floor" the bench
reports).  This test shows the excess is what any FP32 evaluation of the same
right-hand sides produces, not a defect of this library's kernels: the
oracle's single-precision evaluation (pocketfft float32 transforms, float32
products, FP64 per-mode arithmetic: dudt_slabs(single=True)) stepped with
SSP-RK3 and its state kept in complex64 after every stage, as the FP32-bulk
form keeps it, lands within a factor of two of it.  Taylor-Green 3-D N = 32 (the bench's field) to azeban t = 1/(2 pi)
and t = 1 (t = 1 and 2 pi on [0, 2 pi)^3).

Tolerance: the library's FP32 error at most twice the single-precision
oracle's, plus 1e-7.
"""

import math

import numpy as np
import pytest
import torch

import azeban_b200 as az
from oracle import euler_oracle as ora
from tests.gpu_helpers import rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu

VISC = {"type": "Smooth Cutoff", "eps": 0.05}
C = 0.2


def _round32(u):
    return u.astype(np.complex64).astype(np.complex128)


def _single_precision_step(eq, u, max_dt):
    """SSP_RK3::integrate (ssp_rk3.hpp:48-64) on single-precision right-hand
    sides, each stage's result stored in complex64."""
    d1 = eq.dudt_slabs(u, single=True)
    dt = min(eq.dt(C), max_dt)
    u1 = _round32(u + dt * d1)
    d2 = eq.dudt_slabs(u1, single=True)
    u2 = _round32(0.75 * u + 0.25 * (u1 + dt * d2))
    d3 = eq.dudt_slabs(u2, single=True)
    return _round32((2.0 / 3.0) * (u2 + dt * d3) + (1.0 / 3.0) * u), dt


@pytest.mark.parametrize("N", [32, 64])
def test_fp32_trajectory_error_is_single_precision_error(N):
    g = ora.Grid(3, N)
    visc = ora.make_viscosity(VISC, g)
    u0 = ora.initialize(ora.taylor_green_workload(3, N))
    eq64 = ora.IncompressibleEuler(g, visc)
    eq32 = ora.IncompressibleEuler(g, visc)
    cap = C * 2.0 / (eq64.visc() * (math.pi * N) ** 2)
    ag = az.Grid(3, N)
    sim = az.Simulation(ag, C, az.SSP_RK3(az.IncompressibleEuler(ag, az.make_viscosity(VISC, ag), "f32")),
                        to_dev(u0, "f32"))
    ref = ora.Simulation(g, C, ora.SSP_RK3(eq64), u0)
    u32, time = _round32(u0), 0.0
    for t_out in (1.0 / (2 * math.pi), 1.0):
        ref.simulate_until(t_out)
        while time < t_out:
            u32, dt = _single_precision_step(eq32, u32, min(t_out - time, cap))
            time += dt
        time = t_out
        sim.simulate_until(t_out)
        e_single = rel_l2(u32, ref.u_)
        e_lib = rel_l2(to_host(sim.u()), ref.u_)
        assert e_lib <= 2.0 * e_single + 1e-7, f"t={t_out}: library {e_lib:.3e}, single-precision oracle {e_single:.3e}"
