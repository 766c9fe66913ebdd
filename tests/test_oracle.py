"""Pins the CPU oracle against the known answers of the reference's own tests
(CPU only, no GPU).  The reference cannot be built here (zisa, FFTW, Boost,
NetCDF are absent), so these known-answer tests and the committed golden
fixtures are what anchor the oracle.
"""

import math
import os

import numpy as np
import pytest

from oracle import euler_oracle as ora
from oracle.mt19937 import MT19937

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# --- FFT vs a naive DFT (test/azeban/operations/fft.cpp:35-349) -------------

def _dft_axis(x, axis, half=False):
    n = x.shape[axis]
    k = np.arange(n // 2 + 1 if half else n)[:, None]
    j = np.arange(n)[None, :]
    xi = -2 * np.pi * (k * j % n) / n
    W = np.cos(xi) + 1j * np.sin(xi)
    return np.moveaxis(np.tensordot(W, np.moveaxis(x, axis, 0), axes=(1, 0)), 0, axis)


@pytest.mark.parametrize("dim,n,nvars,nt", [
    (1, 128, 1, 1), (1, 128, 2, 1), (2, 128, 1, 2), (2, 128, 2, 2), (2, 128, 1, 1), (2, 128, 2, 1),
    (3, 32, 1, 3), (3, 32, 2, 3), (3, 32, 1, 2), (3, 32, 2, 1)])
def test_fft_vs_naive_dft(dim, n, nvars, nt):
    shape = (nvars,) + (n,) * dim
    u = MT19937().uniform(-1.0, 1.0, int(np.prod(shape))).reshape(shape)
    ref = _dft_axis(u.astype(complex), dim, half=True)
    for ax in range(dim - 1, dim - nt, -1):
        ref = _dft_axis(ref, ax)
    got = ora.fft_forward(u, nt)
    assert np.abs(got.real - ref.real).max() <= 1e-8
    assert np.abs(got.imag - ref.imag).max() <= 1e-8
    back = ora.fft_backward(got, n, nt) / n ** nt
    assert np.abs(back - u).max() <= 1e-8


# --- zero padding (test/azeban/operations/copy_to_padded.cpp:8-177) --------

def _to_real_k(k, n):
    return k - n if k >= n // 2 + 1 else k


def _check_padded(unpadded, padded):
    d = unpadded.ndim
    N = unpadded.shape[0]
    M = padded.shape[0]
    m = {}
    for idx in np.ndindex(*unpadded.shape):
        m[tuple(_to_real_k(i, N) for i in idx)] = unpadded[idx]
    for idx in np.ndindex(*padded.shape):
        kv = tuple(_to_real_k(i, M) for i in idx)
        if kv in m:
            assert padded[idx] == m[kv]
        else:
            assert padded[idx] == 0


@pytest.mark.parametrize("dim,N", [(2, 8), (2, 16), (2, 32), (2, 64), (3, 8), (3, 16)])
def test_zero_padding_map(dim, N):
    rng = MT19937()
    for M in (N, 3 * N // 2, 2 * N):
        shp = (N,) * (dim - 1) + (N // 2 + 1,)
        vals = rng.uniform(-1, 1, 2 * int(np.prod(shp)))
        u = (vals[0::2] + 1j * vals[1::2]).reshape(shp)
        dst = (M,) * (dim - 1) + (M // 2 + 1,)
        _check_padded(u, ora.copy_to_padded(u, dst))


@pytest.mark.parametrize("N", [128, 256, 512, 1024])
def test_zero_padding_map_large_2d_index_rule(N):
    """The index rule at the configs' sizes, vectorised."""
    for M in (N, 3 * N // 2, 2 * N):
        mp = ora.pad_index_map_full(N, M)
        for i in range(M):
            kv = _to_real_k(i, M)
            if mp[i] >= 0:
                assert _to_real_k(int(mp[i]), N) == kv
            else:
                assert not (-(N // 2) + 1 <= kv <= N // 2)


# --- Leray (test/azeban/operations/leray.cpp:9-40) --------------------------

def test_leray_divergence_double_shear_layer():
    N = 32
    u = ora.double_shear_layer(N, 0.2, 0.05)
    u_hat = ora.leray(ora.fft_forward(u))
    v = ora.fft_backward(u_hat, N) / N ** 2
    div = ((np.roll(v[0], -1, 0) - np.roll(v[0], 1, 0)) / N + (np.roll(v[1], -1, 1) - np.roll(v[1], 1, 1)) / N)
    assert np.abs(div).max() < 1e-10


def test_leray_spectral_divergence_3d():
    N = 16
    u = np.random.default_rng(1).standard_normal((3, N, N, N))
    u_hat = ora.leray(ora.fft_forward(u))
    ks = np.meshgrid(ora.signed_index(N), ora.signed_index(N), np.arange(N // 2 + 1), indexing="ij")
    div = sum(1j * ks[a] * u_hat[a] for a in range(3))
    assert np.abs(div).max() <= 1e-10 * np.abs(u_hat).max()


# --- viscosity (test/azeban/equations/spectral_viscosity.cpp:35-153) --------

def _verify_monotone(visc, N):
    last = visc.Qk(0.0)
    assert 0 <= last <= 1
    for i in range(1, N):
        v = visc.Qk(2 * np.pi * i)
        assert v >= last and 0 <= v <= 1
        last = v


@pytest.mark.parametrize("N", [16, 64, 256, 1024, 4096])
def test_viscosity_monotone(N):
    for visc in (ora.Step1D(0.05, 1, 0), ora.Step1D(0.05, 1, math.sqrt(N)), ora.Step1D(0.05, 1, N),
                 ora.SmoothCutoff1D(0.05, 1, 1), ora.SmoothCutoff1D(0.05, 1, math.sqrt(N)),
                 ora.SmoothCutoff1D(0.05, 1, N), ora.Quadratic(0.05, N)):
        _verify_monotone(visc, N)


def test_viscosity_factory_scaling():
    """eps_N = eps / N^{2s-1}, k0 = m0 N^theta (spectral_viscosity_factory.hpp:29-89)."""
    g = ora.Grid(3, 256)
    v = ora.make_viscosity({"type": "Smooth Cutoff", "eps": 0.05}, g)
    assert v.eps == 0.05 / 256 and abs(v.k0 - 2 * np.pi * 16) < 1e-12 and v.s == 1
    v = ora.make_viscosity({"type": "Step", "eps": 0.05, "s": 2, "m0": 1}, g)
    assert abs(v.eps - 0.05 / 256 ** 3) < 1e-20 and abs(v.k0 - 256 ** 0.75) < 1e-9
    q = ora.make_viscosity({"type": "Quadratic", "eps": 0.05}, g)
    assert q.eps == 0.05 / 256 and q.N == 256


def test_viscosity_known_answer_shear_flow():
    """Adapted tracer known answer (spectral_viscosity.cpp:54-104): with
    u = (f(y), 0), u.grad u = 0 and each mode follows exp(nu(|k|) t)."""
    N = 32
    g = ora.Grid(2, N)
    visc = ora.make_viscosity({"type": "Smooth Cutoff", "eps": 0.05, "m0": 0.5}, g)
    y = 2 * np.pi * np.arange(N) / N
    modes = (1, 3, 7, 12)
    f = sum(np.sin(m * y + 0.3 * m) / m for m in modes)
    u_hat = ora.fft_forward(np.stack([np.tile(f, (N, 1)), np.zeros((N, N))]))
    sim = ora.Simulation(g, 0.2, ora.SSP_RK3(ora.IncompressibleEuler(g, visc)), u_hat)
    sim.simulate_until(0.01)
    for m in modes:
        expect = u_hat[0, 0, m] * math.exp(visc.eval(2 * np.pi * m) * 0.01)
        assert abs(sim.u_[0, 0, m] - expect) ** 2 <= 1e-7 * abs(u_hat[0, 0, m]) ** 2


# --- the right-hand side, independently restated --------------------------

@pytest.mark.parametrize("dim,N", [(2, 16), (2, 32), (3, 8), (3, 12)])
def test_rhs_equals_projected_advection(dim, N):
    """For a divergence-free field the divergence form i k.(u (x) u) used by
    the reference equals the advective form u.grad u on the padded grid, so
    -P(u.grad u) + nu u_hat must equal dudt.  The identity needs a padded
    spectrum that is Hermitian, so the Nyquist planes (index N/2, whose
    mirror the padding drops) are cleared."""
    rng = np.random.default_rng(dim * 10 + N)
    u_hat = ora.leray(ora.fft_forward(rng.standard_normal((dim,) + (N,) * dim)))
    for ax in range(1, dim + 1):
        sl = [slice(None)] * (dim + 1)
        sl[ax] = N // 2
        u_hat[tuple(sl)] = 0
    g = ora.Grid(dim, N)
    visc = ora.make_viscosity({"type": "Smooth Cutoff", "eps": 0.05}, g)
    eq = ora.IncompressibleEuler(g, visc)
    got = eq.dudt(u_hat)
    M = g.N_phys_pad
    pad = eq.pad(u_hat)
    kM = [2 * np.pi * np.where(np.arange(M) >= M // 2 + 1, np.arange(M) - M, np.arange(M))] * (dim - 1)
    kM.append(2 * np.pi * np.arange(M // 2 + 1))
    KM = np.meshgrid(*kM, indexing="ij")
    scale = 1.0 / (N ** dim)  # physical values of the N^d-scaled spectrum
    u = ora.fft_backward(pad, M) * scale
    grads = [[ora.fft_backward((1j * KM[b] * pad[a])[None], M)[0] * scale for b in range(dim)] for a in range(dim)]
    adv = np.stack([sum(u[b] * grads[a][b] for b in range(dim)) for a in range(dim)])
    adv_hat = ora.fft_forward(adv) * (N ** dim / M ** dim)
    ret = [ora.retained_index_map(N, M)] * (dim - 1) + [np.arange(N // 2 + 1)]
    adv_hat = adv_hat[np.ix_(range(dim), *ret)]
    kN = [2 * np.pi * ora.signed_index(N)] * (dim - 1) + [2 * np.pi * np.arange(N // 2 + 1)]
    K = np.meshgrid(*kN, indexing="ij")
    k2 = sum(k * k for k in K)
    with np.errstate(divide="ignore", invalid="ignore"):
        kdot = sum(K[a] * adv_hat[a] for a in range(dim)) / k2
    proj = np.stack([adv_hat[a] - K[a] * kdot for a in range(dim)])
    nu = visc.eval(np.sqrt(k2))
    expect = np.where(k2 == 0, 0, -proj + nu * u_hat)
    assert ora.rel_l2(got, expect) <= 1e-11


# --- convergence (test/azeban/equations/incompressible_euler.cpp:44-93) -----

def test_convergence_rate_double_shear_layer_2d():
    def solve(N):
        g = ora.Grid(2, N)
        eq = ora.IncompressibleEuler(g, ora.SmoothCutoff1D(0.05 / N, 1, 1))
        u0 = ora.initialize(ora.double_shear_layer(N, 0.2, 0.05))
        sim = ora.Simulation(g, 0.2, ora.SSP_RK3(eq), u0)
        sim.simulate_until(0.1)
        return sim.u_

    ref = solve(128)
    Ns = [16, 32, 64]
    errs = [ora.L2(solve(N), ref) for N in Ns]
    rate = (math.log(errs[0]) - math.log(errs[-1])) / math.log(Ns[-1] / Ns[0])
    assert rate >= 1


# --- golden fixtures produced by tests/golden/make_golden.py ---------------

def _golden_files():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz")) if os.path.isdir(GOLDEN) else []


@pytest.mark.parametrize("fname", _golden_files())
def test_oracle_reproduces_golden(fname):
    from tests.golden import make_golden
    data = np.load(os.path.join(GOLDEN, fname))
    fresh = make_golden.CASES[fname.replace(".npz", "")]()
    for key in data.files:
        if data[key].dtype.kind in "fc":
            assert ora.rel_l2(fresh[key], data[key]) <= 1e-13, key
        else:
            np.testing.assert_array_equal(fresh[key], data[key])


# --- the bounded-memory right-hand side (used for 3-D N = 512) ---------------

@pytest.mark.parametrize("N,M,visc", [(16, 24, "Smooth Cutoff"), (24, 36, "Step"), (32, 48, "Quadratic"),
                                      (16, 32, "Smooth Cutoff"), (64, 96, "Smooth Cutoff")])
def test_dudt_slabs_equals_dudt(N, M, visc):
    """dudt_slabs evaluates the same right-hand side slab by slab: equal to
    dudt() up to rounding, and the same u_max_ (so the same dt)."""
    rng = np.random.default_rng(N + M)
    u_hat = ora.leray(ora.fft_forward(rng.standard_normal((3, N, N, N))))
    g = ora.Grid(3, N, M)
    eq = ora.IncompressibleEuler(g, ora.make_viscosity({"type": visc, "eps": 0.05}, g))
    ref = eq.dudt(u_hat)
    umax = eq.u_max_
    got = eq.dudt_slabs(u_hat, xchunk=7, zchunk=5, colchunk=1000)
    assert ora.rel_l2(got, ref) <= 1e-14
    assert eq.u_max_ == umax
