"""The device generators of initial data against the oracle.

az_init_physical samples each field in a kernel of the library; the
spectral state follows from the library's FFT and Leray projection.  These
tests compare both the physical samples and the spectral states with the
oracle's restatement of the reference's initialisers
(src/azeban/init/taylor_green.cpp:29-46, :146-184,
src/azeban/init/double_shear_layer.cpp:25-43, initializer.hpp:68-75), and
check the counter-based random stream (Philox4x32-10) against the published
known-answer vectors of its authors.

Tolerances: physical samples 4e-15 absolute (sin, cos, tanh may differ by an
ulp between the device and numpy); spectral states 1e-13 relative L2.
"""

import ctypes as ct
import math

import numpy as np
import pytest
import torch

import azeban_b200 as az
from azeban_b200 import _lib
from azeban_b200 import init as azinit
from oracle import euler_oracle as ora
from tests.gpu_helpers import rel_l2, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,N", [(2, 64), (2, 256), (3, 32), (3, 128)])
def test_taylor_green_workload(dim, N):
    phys = azinit.physical(_lib.AZ_INIT_TAYLOR_GREEN_WORKLOAD, dim, N)[0].cpu().numpy()
    ref = ora.taylor_green_workload(dim, N)
    assert np.abs(phys - ref).max() <= 4e-15
    assert rel_l2(to_host(azinit.taylor_green(dim, N)), ora.initialize(ref)) <= 1e-13


@pytest.mark.parametrize("dim,N", [(2, 64), (3, 32)])
def test_taylor_green_reference_with_perturbation(dim, N):
    """The reference's Taylor-Green and its perturbation modes, two members
    with different amplitudes (and one without)."""
    rng = np.random.default_rng(dim * N)
    nd = 8 if dim == 2 else 24
    deltas = [list(rng.uniform(-0.025, 0.025, nd) / (4 if dim == 2 else 8)), [0.0] * nd]
    phys = azinit.physical(_lib.AZ_INIT_TAYLOR_GREEN, dim, N, batch=2, deltas=deltas).cpu().numpy()
    got = to_host(azinit.taylor_green_reference(dim, N, deltas=deltas))
    for b in range(2):
        ref = ora.taylor_green_reference(dim, N, deltas[b])
        assert np.abs(phys[b] - ref).max() <= 4e-15
        assert rel_l2(got[b], ora.initialize(ref)) <= 1e-13
    np.testing.assert_allclose(phys[1], ora.taylor_green_reference(dim, N), atol=4e-15, rtol=0)


@pytest.mark.parametrize("N,rho", [(64, 0.2), (128, math.pi / 15), (64, 0.0)])
def test_double_shear_layer_reference_and_phases(N, rho):
    """phi = 0 is the reference's DoubleShearLayer; given phases and phases
    drawn from the stream (seed, member) both match the oracle's field at
    those phases."""
    phases = [0.0, 1.3, 5.9]
    phys = azinit.physical(_lib.AZ_INIT_DOUBLE_SHEAR_LAYER, 2, N, batch=3, rho=rho, delta=0.05,
                           phases=phases).cpu().numpy()
    spec = to_host(azinit.double_shear_layer(N, rho, 0.05, phases))
    for b, ph in enumerate(phases):
        ref = ora.double_shear_layer(N, rho, 0.05, ph)
        assert np.abs(phys[b] - ref).max() <= 4e-15
        assert rel_l2(spec[b], ora.initialize(ref)) <= 1e-13
    seed = 2024
    drawn = to_host(azinit.double_shear_layer(N, rho, 0.05, None, seed=seed, member0=5, batch=3))
    for b in range(3):
        ph = azinit.shear_layer_phase(seed, 5 + b)
        assert 0.0 <= ph < 2 * math.pi
        assert rel_l2(drawn[b], ora.initialize(ora.double_shear_layer(N, rho, 0.05, ph))) <= 1e-13


def test_gaussian_noise_stream():
    """Standard normals, a function of (seed, member, position) only: the
    same in a batch as alone, different between members and seeds."""
    dim, N = 3, 32
    a = azinit.physical(_lib.AZ_INIT_GAUSSIAN_NOISE, dim, N, batch=4, seed=11).cpu().numpy()
    alone = azinit.physical(_lib.AZ_INIT_GAUSSIAN_NOISE, dim, N, batch=1, seed=11, member0=2).cpu().numpy()
    np.testing.assert_array_equal(a[2], alone[0])
    other = azinit.physical(_lib.AZ_INIT_GAUSSIAN_NOISE, dim, N, batch=1, seed=12).cpu().numpy()
    assert not np.array_equal(a[0], other[0]) and not np.array_equal(a[0], a[1])
    x = a.ravel()
    assert abs(x.mean()) < 0.02 and abs(x.var() - 1.0) < 0.02
    assert abs(np.corrcoef(x[:-1], x[1:])[0, 1]) < 0.02


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_fractional_brownian_energy_divergence_and_batch(prec):
    N = 32
    u = azinit.fractional_brownian(3, N, 0.75, seed=5, precision=prec, batch=3)
    g = az.Grid(3, N)
    eq = az.IncompressibleEuler(g, az.make_viscosity({"type": "Smooth Cutoff", "eps": 0.05}, g), prec, 3)
    e, _ = eq.diagnostics(u.contiguous())
    for v in e:
        assert abs(v - 1.0) < (1e-12 if prec == "f64" else 1e-5)
    h = to_host(u)
    ks = np.meshgrid(ora.signed_index(N), ora.signed_index(N), np.arange(N // 2 + 1), indexing="ij")
    for b in range(3):
        div = sum(ks[a] * h[b][a] for a in range(3))
        assert np.abs(div).max() <= (1e-10 if prec == "f64" else 1e-4) * np.abs(h[b]).max()
    one = azinit.fractional_brownian(3, N, 0.75, seed=5, precision=prec, batch=1, member0=1)
    np.testing.assert_array_equal(to_host(one), h[1])
