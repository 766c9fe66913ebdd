"""Edge cases of the right-hand side and the stepper, against the oracle.

- A zero field: dudt is exactly zero and dt(C) = C / (N u_max) is +inf, as
  the reference's double arithmetic gives (incompressible_euler.hpp:122-124);
  SSP_RK3::integrate then steps with max_dt (ssp_rk3.hpp:55), so
  simulate_until advances a zero state by the viscous cap of
  simulation.cpp:91-93 and the clock lands on t exactly.
- Members of one batch that finish at different step counts: a Taylor-Green
  member beside a zero member; each keeps its own clock, dt and step count on
  the device, the finished member is skipped, and each matches its own
  oracle solve.

Tolerances as the other FP64 tests: 1e-9 relative L2 at the final time.
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


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 16)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_zero_field_dudt_and_dt(dim, N, prec):
    g = az.Grid(dim, N)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC, g), prec)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.zeros(g.shape_fourier(dim), dtype=cdt, device="cuda")
    out = torch.full_like(u, 1.0)
    eq.dudt(out, u)
    assert torch.count_nonzero(out).item() == 0
    assert eq.dt(C) == math.inf
    og = ora.Grid(dim, N)
    oeq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC, og))
    oeq.dudt(np.zeros(og.shape_fourier(dim), dtype=np.complex128))
    assert oeq.dt(C) == math.inf


def _oracle_run(N, u0, t_end):
    g = ora.Grid(3, N)
    sim = ora.Simulation(g, C, ora.SSP_RK3(ora.IncompressibleEuler(g, ora.make_viscosity(VISC, g))), u0)
    sim.simulate_until(t_end)
    return sim.u_, len(sim.dts)


def test_zero_field_simulate_until():
    N, t_end = 16, 0.05
    u0 = np.zeros(ora.Grid(3, N).shape_fourier(3), dtype=np.complex128)
    ref, nsteps_ref = _oracle_run(N, u0, t_end)
    g = az.Grid(3, N)
    sim = az.Simulation(g, C, az.SSP_RK3(az.IncompressibleEuler(g, az.make_viscosity(VISC, g))), to_dev(u0))
    sim.simulate_until(t_end)
    times, nsteps, _ = sim.state()
    assert times[0] == t_end
    assert nsteps[0] == nsteps_ref
    assert torch.count_nonzero(sim.u()).item() == 0
    assert not np.any(ref)


def test_members_finish_at_different_step_counts():
    N, t_end = 16, 0.3
    tg = ora.initialize(ora.taylor_green_workload(3, N))
    zero = np.zeros_like(tg)
    ref_tg, n_tg = _oracle_run(N, tg, t_end)
    _, n_zero = _oracle_run(N, zero, t_end)
    assert n_tg != n_zero
    g = az.Grid(3, N)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC, g), "f64", 2)
    sim = az.Simulation(g, C, az.SSP_RK3(eq), to_dev(np.stack([tg, zero])))
    sim.simulate_until(t_end)
    times, nsteps, _ = sim.state()
    assert times == [t_end, t_end]
    assert list(nsteps) == [n_tg, n_zero]
    u = to_host(sim.u())
    assert rel_l2(u[0], ref_tg) <= 1e-9
    assert not np.any(u[1])
