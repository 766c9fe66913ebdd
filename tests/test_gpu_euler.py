"""Parity of the CUDA right-hand side, SSP-RK3 step and simulate_until with
the CPU oracle (a restatement of include/azeban/equations/incompressible_euler.hpp,
include/azeban/evolution/ssp_rk3.hpp and src/azeban/simulation.cpp).

Tolerances (relative L2 over the flat spectral array):
  FP64:  1e-12 per right-hand side / step, 1e-9 at the final time;
  FP32 bulk vs the FP64 oracle: 1e-5.
"""

import math

import numpy as np
import pytest
import torch

import azeban_b200 as az
from oracle import euler_oracle as ora
from tests.gpu_helpers import VISC_CFGS, random_field_hat, rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL64_STEP = 1e-12
TOL64_FINAL = 1e-9
TOL32 = 1e-5


def _pair(dim, N, visc="smooth", prec="f64", batch=1, M=None):
    og = ora.Grid(dim, N, M)
    g = az.Grid(dim, N, M)
    ov = ora.make_viscosity(VISC_CFGS[visc], og)
    v = az.make_viscosity(VISC_CFGS[visc], g)
    return og, g, ora.IncompressibleEuler(og, ov), az.IncompressibleEuler(g, v, prec, batch)


@pytest.mark.parametrize("dim,N", [(2, 16), (2, 32), (2, 64), (2, 128), (3, 8), (3, 16), (3, 32)])
@pytest.mark.parametrize("visc", ["smooth", "step", "quadratic", "none"])
def test_dudt_fp64(dim, N, visc):
    og, g, oeq, eq = _pair(dim, N, visc)
    u_hat = random_field_hat(dim, N, seed=100 * dim + N)
    ref = oeq.dudt(u_hat)
    d_u = to_dev(u_hat)
    d_out = torch.empty_like(d_u)
    eq.dudt(d_out, d_u, 0.0, 0.0, 0.2)
    got = to_host(d_out)
    assert rel_l2(got, ref) <= TOL64_STEP
    # dt(C) from the same right-hand side (incompressible_euler.hpp:116-124)
    assert abs(eq.dt(0.2) - oeq.dt(0.2)) <= 1e-13 * oeq.dt(0.2)


@pytest.mark.parametrize("dim,N,M", [(2, 32, 64), (2, 32, 32), (3, 16, 32), (3, 16, 16), (2, 16, 48)])
def test_dudt_other_padding(dim, N, M):
    """N_phys_pad given explicitly (grid_factory.hpp:60-66)."""
    og, g, oeq, eq = _pair(dim, N, "smooth", M=M)
    u_hat = random_field_hat(dim, N, seed=7)
    ref = oeq.dudt(u_hat)
    d_u = to_dev(u_hat)
    d_out = torch.empty_like(d_u)
    eq.dudt(d_out, d_u)
    assert rel_l2(to_host(d_out), ref) <= TOL64_STEP


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 16)])
def test_dudt_in_place(dim, N):
    """dudt(u, u) is allowed (test/azeban/equations/incompressible_euler.cpp:194)."""
    og, g, oeq, eq = _pair(dim, N)
    u_hat = random_field_hat(dim, N, seed=3)
    ref = oeq.dudt(u_hat)
    d_u = to_dev(u_hat)
    eq.dudt(d_u, d_u)
    assert rel_l2(to_host(d_u), ref) <= TOL64_STEP


@pytest.mark.parametrize("dim,N", [(2, 32), (2, 64), (3, 16), (3, 32)])
def test_dudt_fp32_bulk(dim, N):
    og, g, oeq, eq = _pair(dim, N, prec="f32")
    u_hat = random_field_hat(dim, N, seed=11)
    ref = oeq.dudt(u_hat)
    d_u = to_dev(u_hat, "f32")
    d_out = torch.empty_like(d_u)
    eq.dudt(d_out, d_u)
    assert rel_l2(to_host(d_out), ref) <= TOL32


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 16)])
def test_rk3_step_fp64(dim, N):
    og, g, oeq, eq = _pair(dim, N)
    ts = az.SSP_RK3(eq)
    ots = ora.SSP_RK3(oeq)
    u_hat = random_field_hat(dim, N, seed=5)
    ou = u_hat.copy()
    odt = ots.integrate(0.0, 1.0, 0.2, ou)
    d_u = to_dev(u_hat)
    dt = ts.integrate(0.0, 1.0, 0.2, d_u)
    assert abs(dt - odt) <= 1e-13 * odt
    assert rel_l2(to_host(d_u), ou) <= TOL64_STEP
    # a max_dt below the CFL step is taken as is (ssp_rk3.hpp:55)
    ou2 = u_hat.copy()
    odt2 = ots.integrate(0.0, 0.25 * odt, 0.2, ou2)
    d_u2 = to_dev(u_hat)
    dt2 = ts.integrate(0.0, 0.25 * odt, 0.2, d_u2)
    assert dt2 == odt2
    assert rel_l2(to_host(d_u2), ou2) <= TOL64_STEP


def _tg(dim, N):
    return ora.initialize(ora.taylor_green_workload(dim, N))


@pytest.mark.parametrize("dim,N,t_end", [(2, 64, 1.0), (3, 16, 1.0), (3, 32, 0.25)])
def test_taylor_green_trajectory_fp64(dim, N, t_end):
    """Taylor-Green, SmoothCutoff eps=0.05, C=0.2, SSP-RK3 (the 2-D 64^2 to
    t=1 case is the reference's CPU-runnable configuration)."""
    og, g, oeq, eq = _pair(dim, N)
    u0 = _tg(dim, N)
    osim = ora.Simulation(og, 0.2, ora.SSP_RK3(oeq), u0)
    osim.simulate_until(t_end)
    ts = az.SSP_RK3(eq)
    sim = az.Simulation(g, 0.2, ts, to_dev(u0))
    sim.simulate_until(t_end)
    times, steps, _ = sim.state()
    assert steps[0] == len(osim.dts)
    assert times[0] == t_end
    assert rel_l2(to_host(sim.u()), osim.u_) <= TOL64_FINAL


def test_double_shear_layer_trajectory_fp64():
    """A solve with real nonlinear dynamics: double shear layer 2-D 64^2,
    rho = 0.2, delta = 0.05 (src/azeban/init/double_shear_layer.cpp:25-43)."""
    og, g, oeq, eq = _pair(2, 64)
    u0 = ora.initialize(ora.double_shear_layer(64, 0.2, 0.05))
    osim = ora.Simulation(og, 0.2, ora.SSP_RK3(oeq), u0)
    osim.simulate_until(0.5)
    sim = az.Simulation(g, 0.2, az.SSP_RK3(eq), to_dev(u0))
    sim.simulate_until(0.5)
    assert sim.state()[1][0] == len(osim.dts)
    assert rel_l2(to_host(sim.u()), osim.u_) <= TOL64_FINAL


@pytest.mark.parametrize("dim,N,t_end", [(2, 64, 1.0), (3, 32, 0.25)])
def test_fp32_bulk_trajectory_vs_fp64(dim, N, t_end):
    og, g, oeq, _ = _pair(dim, N)
    eq32 = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), "f32")
    u0 = _tg(dim, N) if dim == 3 else ora.initialize(ora.double_shear_layer(N, 0.2, 0.05))
    osim = ora.Simulation(og, 0.2, ora.SSP_RK3(oeq), u0)
    osim.simulate_until(t_end)
    sim = az.Simulation(g, 0.2, az.SSP_RK3(eq32), to_dev(u0, "f32"))
    sim.simulate_until(t_end)
    assert rel_l2(to_host(sim.u()), osim.u_) <= TOL32


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_members_match_single(prec):
    """Each member of a batched solve equals the same solve alone."""
    dim, N, B = 2, 32, 5
    g = az.Grid(dim, N)
    v = az.make_viscosity(VISC_CFGS["smooth"], g)
    fields = [random_field_hat(dim, N, seed=50 + b) for b in range(B)]
    eqB = az.IncompressibleEuler(g, v, prec, batch=B)
    simB = az.Simulation(g, 0.2, az.SSP_RK3(eqB), to_dev(np.stack(fields), prec))
    simB.simulate_until(0.1)
    outB = to_host(simB.u())
    tB, nB, _ = simB.state()
    for b in range(B):
        eq1 = az.IncompressibleEuler(g, v, prec)
        sim1 = az.Simulation(g, 0.2, az.SSP_RK3(eq1), to_dev(fields[b], prec))
        sim1.simulate_until(0.1)
        assert sim1.state()[1][0] == nB[b]
        np.testing.assert_array_equal(to_host(sim1.u()), outB[b])


def test_viscosity_known_answer_shear():
    """Known answer adapted from test/azeban/equations/spectral_viscosity.cpp:54-104:
    a shear flow u = (f(y), 0) has u.grad u = 0, so each mode evolves by the
    SSP-RK3 amplification of its viscosity factor alone."""
    N = 64
    g = az.Grid(2, N)
    cfg = {"type": "Smooth Cutoff", "eps": 0.05, "m0": 0.5}
    visc = az.make_viscosity(cfg, g)
    ovisc = ora.make_viscosity(cfg, ora.Grid(2, N))
    y = 2 * np.pi * np.arange(N) / N
    f = sum(np.sin(m * y + 0.3 * m) / m for m in (1, 3, 7, 12, 20))
    u = np.stack([np.tile(f, (N, 1)), np.zeros((N, N))])
    u_hat = ora.fft_forward(u)
    eq = az.IncompressibleEuler(g, visc)
    sim = az.Simulation(g, 0.2, az.SSP_RK3(eq), to_dev(u_hat))
    sim.simulate_until(0.01)
    _, _, _ = sim.state()
    got = to_host(sim.u())
    k2 = 2 * np.pi * np.arange(N // 2 + 1)
    nu = ovisc.eval(np.abs(k2))
    for m in (1, 3, 7, 12, 20):
        expect = u_hat[0, 0, m] * math.exp(nu[m] * 0.01)
        assert abs(got[0, 0, m] - expect) ** 2 <= 1e-7 * abs(u_hat[0, 0, m]) ** 2


def test_leray_divergence_2d_double_shear_layer():
    """leray() then the central-difference divergence is < 1e-10 for the
    double shear layer, N = 32, rho = 0.2, delta = 0.05
    (test/azeban/operations/leray.cpp:9-40)."""
    N = 32
    u = ora.double_shear_layer(N, 0.2, 0.05)
    u_hat = to_dev(ora.fft_forward(u))
    az.leray(u_hat)
    phys = ora.fft_backward(to_host(u_hat), N) / N ** 2
    div = ((np.roll(phys[0], -1, axis=0) - np.roll(phys[0], 1, axis=0)) / N
           + (np.roll(phys[1], -1, axis=1) - np.roll(phys[1], 1, axis=1)) / N)
    assert np.abs(div).max() < 1e-10


@pytest.mark.parametrize("dim", [2, 3])
def test_leray_matches_oracle(dim):
    """Random field: the device projection equals the oracle's and removes
    the spectral divergence."""
    N = 32
    rng = np.random.default_rng(dim)
    u = rng.standard_normal((dim,) + (N,) * dim)
    u_hat = to_dev(ora.fft_forward(u))
    az.leray(u_hat)
    ref = ora.leray(ora.fft_forward(u))
    got = to_host(u_hat)
    assert rel_l2(got, ref) <= 1e-14
    ks = np.meshgrid(*([ora.signed_index(N)] * (dim - 1) + [np.arange(N // 2 + 1)]), indexing="ij")
    dspec = sum(1j * 2 * np.pi * ks[a] * got[a] for a in range(dim))
    assert np.abs(dspec).max() <= 1e-10 * np.abs(got).max() * N


def test_wrong_number_of_variables_raises():
    g = az.Grid(2, 16)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g))
    bad = torch.zeros((3, 16, 9), dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError):
        eq.dudt(bad, bad)


def test_unsupported_padding_raises():
    g = az.Grid(2, 16, 20)
    with pytest.raises(az.AzebanError):
        az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g))


@pytest.mark.parametrize("dim,N,prec,batch", [(2, 64, "f64", 1), (3, 32, "f64", 3), (3, 32, "f32", 2), (2, 128, "f32", 4)])
def test_energy_enstrophy_fp64_sums(dim, N, prec, batch):
    """FP64 compensated diagnostics equal correctly rounded sums; a member's
    value is the same alone and inside a batch."""
    g = az.Grid(dim, N)
    v = az.make_viscosity(VISC_CFGS["smooth"], g)
    fields = [random_field_hat(dim, N, seed=70 + b) for b in range(batch)]
    eq = az.IncompressibleEuler(g, v, prec, batch=batch)
    dev = to_dev(np.stack(fields) if batch > 1 else fields[0], prec)
    E, W = eq.diagnostics(dev)
    E = E if batch > 1 else [E]
    W = W if batch > 1 else [W]
    for b in range(batch):
        rounded = to_host(dev[b] if batch > 1 else dev)
        e_ref, w_ref = ora.energy_enstrophy(rounded)
        assert abs(E[b] - e_ref) <= 1e-14 * e_ref
        assert abs(W[b] - w_ref) <= 1e-14 * w_ref
        alone = az.IncompressibleEuler(g, v, prec)
        e1, w1 = alone.diagnostics(to_dev(fields[b], prec))
        assert e1 == E[b] and w1 == W[b]
