"""Pins the oracle's pointwise stages against the reference's own code.

The reference's pointwise headers (include/azeban/equations/
incompressible_euler_functions.hpp:26-112, spectral_viscosity.hpp:27-128,
include/azeban/operations/copy_to_padded_functions.hpp:9-63, complex.hpp) are
compiled here, unmodified, into oracle/_ref by oracle/build_ref.sh (with
stand-ins for the absent ZisaCore/ZisaMemory/fmt headers), and driven per
point / per mode by the reference's CPU glue (incompressible_euler.hpp:168-213,
:230-347).  These tests compare the numpy oracle with that code at the
workloads' index ranges (N = 256, M = 384 in 3-D; N = 512, M = 768 in 2-D):
the padding map, the four viscosity laws, the computeB scaling and products,
and the per-mode projection, viscosity and right-hand side.  The transforms
themselves are FFTW / cuFFT in the reference (not in its tree); they are
pinned by the reference's FFT-vs-DFT test (tests/test_oracle.py).

CPU only.  Skipped where neither the built library nor the reference tree is
present.
"""

import math

import numpy as np
import pytest

from oracle import euler_oracle as ora
from oracle import ref_pointwise as refp

LIB = refp.load()
pytestmark = pytest.mark.skipif(LIB is None, reason="the reference sources are not present to build oracle/_ref")

VISCS = [{"type": "Smooth Cutoff", "eps": 0.05}, {"type": "Step", "eps": 0.05},
         {"type": "Quadratic", "eps": 0.05}, {"type": "None"},
         {"type": "Smooth Cutoff", "eps": 0.3, "s": 2.0, "theta": 0.25, "m0": 3.0}]


@pytest.mark.parametrize("N,M", [(8, 12), (16, 24), (64, 96), (256, 384), (512, 768), (1024, 1536),
                                 (32, 32), (32, 64), (34, 384)])
def test_padding_map_is_the_references(N, M):
    assert np.array_equal(ora.pad_index_map_full(N, M), refp.pad_index_map(LIB, False, N, M))
    Nh, Mh = N // 2 + 1, M // 2 + 1
    assert np.array_equal(ora.pad_index_map_compact(Nh, Mh), refp.pad_index_map(LIB, True, Nh, Mh))


@pytest.mark.parametrize("cfg", VISCS)
@pytest.mark.parametrize("N", [64, 256, 512])
def test_viscosity_laws_are_the_references(cfg, N):
    """nu(|k|) for every |k| that the retained modes of a 3-D grid of N take
    (every sum of three squared signed indices) and a sweep to the padded
    range.  Equal up to the last bits of the libm calls (numpy's exp and pow
    against the C library's): per value, 1e-15 relative plus 2 ulp of the
    cutoff factor Q in 1 - exp(-(k/k0)^18), whose cancellation at small k
    turns an ulp of exp into a large relative difference of a tiny value."""
    g = ora.Grid(3, N)
    visc = ora.make_viscosity(cfg, g)
    s2 = np.unique(ora.signed_index(N).astype(float) ** 2)
    n2 = np.unique((s2[:, None] + s2[None, :]).ravel())
    n2 = np.unique((n2[:, None] + (np.arange(N // 2 + 1.0) ** 2)[None, :]).ravel())
    k = np.concatenate([2 * math.pi * np.sqrt(n2), np.linspace(0, 2 * math.pi * N, 4097)])
    ref = refp.visc_eval(LIB, visc, k)
    got = visc.eval(k)
    eps, sexp = float(getattr(visc, "eps", 0.0)), float(getattr(visc, "s", 1.0))
    scale = eps * np.power(k, 2 * sexp) * 4.5e-16
    assert np.all(np.abs(got - ref) <= 1e-15 * np.abs(ref) + scale)
    assert np.array_equal(got == 0, ref == 0) or getattr(visc, "kind", "") == "smooth_cutoff"


@pytest.mark.parametrize("dim,N,M", [(2, 512, 768), (3, 256, 384), (3, 128, 192), (2, 64, 96)])
def test_compute_B_is_the_references(dim, N, M):
    """The scaling 1/(N^{d/2} M^{d/2}) and the products in the reference's
    order, on a block of padded physical values of the workload's size."""
    rng = np.random.default_rng(N)
    u = rng.standard_normal((dim,) + (64,) * dim) * float(N) ** dim
    g = ora.Grid(dim, N, M)
    eq = ora.IncompressibleEuler(g, ora.NoViscosity())
    assert eq.norm() == refp.norm(LIB, dim, N, M)
    assert np.array_equal(eq.compute_B(u), refp.compute_B(LIB, u, refp.norm(LIB, dim, N, M)))


def _modes(dim, N, count, rng):
    """Signed and padded indices of retained modes: every edge index (0,
    N/2, N/2+1, N-1 and the last compact bin) plus random ones."""
    edge = np.array([0, 1, N // 2 - 1, N // 2, N // 2 + 1, N - 1])
    full = [np.concatenate([edge, rng.integers(0, N, count)]) for _ in range(dim - 1)]
    last = np.concatenate([np.array([0, 1, N // 2 - 1, N // 2]), rng.integers(0, N // 2 + 1, count + 2)])
    n = len(last)
    full = [np.resize(f, n) for f in full]
    return full + [last]


@pytest.mark.parametrize("dim,N,M", [(3, 256, 384), (3, 512, 768), (2, 512, 768), (2, 256, 384)])
@pytest.mark.parametrize("cfg", VISCS)
def test_per_mode_rhs_is_the_references(dim, N, M, cfg):
    """The per-mode part of computeDudt (the projection L = (I - k k^T/|k|^2)
    (i k.B_hat), nu(|k|) u_hat, and 0 at |k| = 0) of the oracle equals the
    reference's incompressible_euler_{2,3}d_compute_L plus its CPU glue, at
    the workload index ranges, on random B_hat and u_hat."""
    rng = np.random.default_rng(N + dim)
    g = ora.Grid(dim, N, M)
    visc = ora.make_viscosity(cfg, g)
    idx = _modes(dim, N, 20000, rng)
    signed = np.stack([ora.signed_index(N)[i] for i in idx[:-1]] + [idx[-1]])
    nb = dim * (dim + 1) // 2
    n = signed.shape[1]
    B = (rng.standard_normal((nb, n)) + 1j * rng.standard_normal((nb, n))) * float(N) ** dim
    u = (rng.standard_normal((dim, n)) + 1j * rng.standard_normal((dim, n))) * float(N) ** dim
    B[:, :3] = 0.0  # include exact zeros
    ref = refp.dudt_modes(LIB, signed, B, u, visc)
    got = ora.dudt_modes(visc, signed, B, u)
    assert np.array_equal(got, ref) or np.abs(got - ref).max() <= 4e-16 * np.abs(ref).max()
    # the |k| = 0 mode is exactly zero in both
    zero = (signed == 0).all(axis=0)
    assert zero.any() and (ref[:, zero] == 0).all() and (got[:, zero] == 0).all()


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 16)])
def test_whole_compute_dudt_is_the_references(dim, N):
    """The oracle's compute_dudt over the whole retained grid, reading B_hat
    at the padded indices (i_B = i >= N/2+1 ? M - N + i : i), equals the
    reference's per-mode code fed the same padded B_hat entries."""
    rng = np.random.default_rng(7 * N)
    g = ora.Grid(dim, N)
    visc = ora.make_viscosity({"type": "Smooth Cutoff", "eps": 0.05}, g)
    eq = ora.IncompressibleEuler(g, visc)
    M = g.N_phys_pad
    nb = dim * (dim + 1) // 2
    bshape = (nb,) + (M,) * (dim - 1) + (M // 2 + 1,)
    B_hat = rng.standard_normal(bshape) + 1j * rng.standard_normal(bshape)
    u_hat = rng.standard_normal(g.shape_fourier(dim)) + 1j * rng.standard_normal(g.shape_fourier(dim))
    got = eq.compute_dudt(B_hat, u_hat)
    grids = np.meshgrid(*([np.arange(N)] * (dim - 1) + [np.arange(N // 2 + 1)]), indexing="ij")
    signed = [ora.signed_index(N)[gi.ravel()] for gi in grids[:-1]] + [grids[-1].ravel()]
    padded = [ora.retained_index_map(N, M)[gi.ravel()] for gi in grids[:-1]] + [grids[-1].ravel()]
    Bm = np.stack([B_hat[(c,) + tuple(padded)] for c in range(nb)])
    um = u_hat.reshape(dim, -1)
    ref = refp.dudt_modes(LIB, np.stack(signed), Bm, um, visc).reshape(got.shape)
    assert np.array_equal(got, ref) or np.abs(got - ref).max() <= 4e-16 * np.abs(ref).max()
