"""The CUDA path against the committed golden fixtures (tests/golden/*.npz,
written by tests/golden/make_golden.py with the CPU oracle, FP64): each
fixture's stored input goes through the library and its output is compared
with the stored output, so the comparison does not depend on the oracle
running alongside.

  dudt_<d>d_n<N>   one right-hand side: relative L2 <= 1e-12, dt(C = 0.2)
                   within 1e-13 (incompressible_euler.hpp:103-124)
  traj_*           simulate_until(t_end) from the stored initial state
                   (simulation.cpp:89-102, ssp_rk3.hpp:48-64): the same
                   number of steps, the last dt within 1e-10, the final
                   state within 1e-9
  traj_tg3d_n64    the same through a fingerprint of the final state (the
                   modes with |n_i| <= 8, the norm of each component) from
                   the Taylor-Green initial state the oracle generates
"""

import os

import numpy as np
import pytest
import torch

import azeban_b200 as az
from oracle import euler_oracle as ora
from tests.golden.make_golden import VISC, low_modes
from tests.gpu_helpers import rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def _dim_n(name):
    dim = int(name.split("_")[1][0]) if name.startswith("dudt") else int(name.split("_")[1][-2])
    return dim, int(name.rsplit("_n", 1)[1])


@pytest.mark.parametrize("name", ["dudt_2d_n16", "dudt_2d_n32", "dudt_2d_n64", "dudt_3d_n8", "dudt_3d_n16",
                                  "dudt_3d_n32"])
def test_dudt_matches_golden(name):
    data = _load(name)
    dim, N = _dim_n(name)
    g = az.Grid(dim, N)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC, g))
    d_u = to_dev(data["u_hat"])
    d_out = torch.empty_like(d_u)
    eq.dudt(d_out, d_u, 0.0, 0.0, 0.2)
    assert rel_l2(to_host(d_out), data["dudt"]) <= 1e-12
    dt = float(data["dt"])
    assert abs(eq.dt(0.2) - dt) <= 1e-13 * dt


def _simulate(dim, N, u0, t_end):
    g = az.Grid(dim, N)
    sim = az.Simulation(g, 0.2, az.SSP_RK3(az.IncompressibleEuler(g, az.make_viscosity(VISC, g))), to_dev(u0))
    sim.simulate_until(t_end)
    times, nsteps, dts = sim.state()
    return to_host(sim.u()), times[0], nsteps[0], dts[0]


@pytest.mark.parametrize("name", ["traj_tg2d_n64", "traj_dsl2d_n64", "traj_tg3d_n16", "traj_tg3d_n32"])
def test_trajectory_matches_golden(name):
    data = _load(name)
    dim, N = _dim_n(name)
    t_end = float(data["t_end"])
    u, time, nsteps, last_dt = _simulate(dim, N, data["u0"], t_end)
    assert time == t_end
    assert nsteps == len(data["dts"])
    assert abs(last_dt - data["dts"][-1]) <= 1e-10 * abs(data["dts"][-1])
    assert rel_l2(u, data["u_final"]) <= 1e-9


def test_trajectory_fingerprint_tg3d_n64():
    data = _load("traj_tg3d_n64")
    t_end = float(data["t_end"])
    u0 = ora.initialize(ora.taylor_green_workload(3, 64))
    u, time, nsteps, last_dt = _simulate(3, 64, u0, t_end)
    assert nsteps == len(data["dts"])
    assert abs(last_dt - data["dts"][-1]) <= 1e-10 * abs(data["dts"][-1])
    assert rel_l2(low_modes(u), data["u_final_low"]) <= 1e-9
    norms = np.sqrt(np.sum(np.abs(u.reshape(3, -1)) ** 2, axis=1))
    np.testing.assert_allclose(norms, data["u_final_norms"], rtol=1e-10)
