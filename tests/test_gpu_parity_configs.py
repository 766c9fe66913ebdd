"""Parity with the oracle at the workloads' own shapes.

The other GPU tests compare against the oracle at small N.  These run the
right-hand side and one SSP-RK3 step at the sizes the workloads use, so every
kernel runs at its real tile counts, grid shapes and transform lengths:

  3-D N = 128 (M = 192) and N = 256 (M = 384, the headline), batch 1 and 4,
      the Taylor-Green workload field and seeded random fields;
  2-D N = 128, 256, 512 (M up to 768) at the double-shear-layer ensemble
      batches (256, 192, 64 members), one phase per member;
  3-D N = 512 (M = 768), one right-hand side, against the oracle's
      bounded-memory form (dudt_slabs, the same right-hand side evaluated
      slab by slab).

Reference: IncompressibleEuler::dudt (include/azeban/equations/incompressible_euler.hpp:103-124),
SSP_RK3::integrate (include/azeban/evolution/ssp_rk3.hpp:48-64).

Tolerances, relative L2 over the flat spectral array of each member:
  FP64 vs the FP64 oracle: 1e-12 per right-hand side and per step;
  FP32 bulk vs the FP64 oracle: 1e-5 per step; per right-hand side 1e-5 or
      twice the error of the same right-hand side evaluated in single
      precision by pocketfft (the oracle's dudt_single), whichever is larger.
      The workload fields cancel strongly (the Taylor-Green and shear-layer
      nonlinear terms are mostly pressure gradient, removed by the
      projection), so any FP32 evaluation of their right-hand side lands
      near or above 1e-5 (TG 256^3: about 1.6e-5; DSL 256^2: 8.5e-6); the
      second bound checks that this library's FP32 path is as accurate as a
      standard FP32 FFT on them.  Random fields stay at the plain 1e-5;
  dt: 1e-13 relative (FP64), 1e-5 (FP32 bulk, whose CFL maximum is taken over
      FP32 velocity values).
"""

import math
import os

import numpy as np
import pytest
import torch

import azeban_b200 as az
from oracle import euler_oracle as ora
from tests.gpu_helpers import rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5
TOL_DT64 = 1e-13
TOL_DT32 = 1e-5
VISC = {"type": "Smooth Cutoff", "eps": 0.05}
C_CFL = 0.2

ora.set_workers(os.cpu_count() or 1)


def random_hat_3d(N, seed, slope=1.5):
    """Seeded divergence-free 3-D spectrum with every retained mode populated:
    Gaussian half-spectrum coefficients with a decaying envelope, made
    Hermitian-consistent by a c2r / r2c round trip, Leray-projected and
    scaled to unit RMS velocity."""
    rng = np.random.default_rng(seed)
    Nh = N // 2 + 1
    c = rng.standard_normal((3, N, N, Nh)) + 1j * rng.standard_normal((3, N, N, Nh))
    s = ora.signed_index(N).astype(float)
    k2 = s[:, None, None] ** 2 + s[None, :, None] ** 2 + np.arange(Nh, dtype=float)[None, None, :] ** 2
    c *= (1.0 + np.sqrt(k2)) ** (-slope)
    u = ora.fft_backward(c, N)
    del c
    u_hat = ora.leray(ora.fft_forward(u))
    del u
    w = np.where((np.arange(Nh) == 0) | (2 * np.arange(Nh) == N), 1.0, 2.0)
    rms = math.sqrt((w * np.abs(u_hat) ** 2).sum() / 3.0) / N ** 3
    return u_hat / rms


def tg_hat(dim, N):
    return ora.initialize(ora.taylor_green_workload(dim, N))


def dsl_hat(N, phase):
    return ora.initialize(ora.double_shear_layer(N, math.pi / 15, 0.05, phase))


def oracle_eq(dim, N):
    g = ora.Grid(dim, N)
    return ora.IncompressibleEuler(g, ora.make_viscosity(VISC, g), slabs=(dim == 3))


def gpu_eq(dim, N, prec, batch):
    g = az.Grid(dim, N)
    return az.IncompressibleEuler(g, az.make_viscosity(VISC, g), prec, batch)


_FIELDS = {}


def field_3d(N, which):
    key = (N, which)
    if key not in _FIELDS:
        _FIELDS[key] = tg_hat(3, N) if which == "tg" else random_hat_3d(N, seed=1000 + 17 * N + which)
    return _FIELDS[key]


_RHS = {}


def single_precision_error(eq, u_hat, ref):
    """Relative L2 error of the right-hand side evaluated in single precision
    (pocketfft float32, from the FP32-rounded input) against FP64."""
    u32 = u_hat.astype(np.complex64).astype(np.complex128)
    return rel_l2(eq.dudt_single(u32), ref)


def tol32_rhs(e32):
    return max(TOL32, 2.0 * e32)


def oracle_rhs_3d(N, which):
    """Oracle right-hand side, dt(C) and single-precision conditioning of one
    field (cached per module)."""
    key = (N, which)
    if key not in _RHS:
        eq = oracle_eq(3, N)
        u = field_3d(N, which)
        out = eq.dudt(u)
        dt = eq.dt(C_CFL)
        _RHS[key] = (out, dt, single_precision_error(eq, u, out))
    return _RHS[key]


def _check_members(got, refs, tol, what):
    """tol: one tolerance, or one per member."""
    tols = tol if isinstance(tol, (list, tuple)) else [tol] * len(refs)
    for b, ref in enumerate(refs):
        err = rel_l2(got[b], ref)
        assert err <= tols[b], f"{what}: member {b} relative L2 {err:.3e} > {tols[b]:.2e}"


# ---------------------------------------------------------------------------
# 3-D, N = 128 and 256
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("N", [128, 256])
@pytest.mark.parametrize("which", ["tg", 1])
def test_dudt_3d_config_batch1(N, which):
    u_hat = field_3d(N, which)
    ref, dt_ref, e32 = oracle_rhs_3d(N, which)
    for prec, tol, tol_dt in (("f64", TOL64, TOL_DT64), ("f32", tol32_rhs(e32), TOL_DT32)):
        eq = gpu_eq(3, N, prec, 1)
        d_u = to_dev(u_hat, prec)
        d_out = torch.empty_like(d_u)
        eq.dudt(d_out, d_u, 0.0, 0.0, C_CFL)
        err = rel_l2(to_host(d_out), ref)
        assert err <= tol, f"{prec} N={N} field={which}: relative L2 {err:.3e}"
        dt = eq.dt(C_CFL)
        assert abs(dt - dt_ref) <= tol_dt * dt_ref, f"{prec} dt {dt!r} vs oracle {dt_ref!r}"
        del eq, d_u, d_out
        torch.cuda.empty_cache()


@pytest.mark.parametrize("N", [128, 256])
def test_dudt_3d_config_batch4(N):
    """Four different members in one batched right-hand side (the bench's
    batch), each against its own oracle result."""
    which = ["tg", 1, 2, 3]
    refs = [oracle_rhs_3d(N, w)[0] for w in which]
    dts = [oracle_rhs_3d(N, w)[1] for w in which]
    tol32 = [tol32_rhs(oracle_rhs_3d(N, w)[2]) for w in which]
    for prec, tol, tol_dt in (("f64", [TOL64] * 4, TOL_DT64), ("f32", tol32, TOL_DT32)):
        eq = gpu_eq(3, N, prec, 4)
        d_u = torch.stack([to_dev(field_3d(N, w), prec) for w in which]).contiguous()
        d_out = torch.empty_like(d_u)
        eq.dudt(d_out, d_u, 0.0, 0.0, C_CFL)
        got = to_host(d_out)
        _check_members(got, refs, tol, f"{prec} N={N} batch 4")
        for b, dt in enumerate(eq.dt(C_CFL)):
            assert abs(dt - dts[b]) <= tol_dt * dts[b]
        del eq, d_u, d_out, got
        torch.cuda.empty_cache()


@pytest.mark.parametrize("N,batch", [(128, 4), (256, 1)])
def test_rk3_step_3d_config(N, batch):
    """One SSP-RK3 step of every member against the oracle's integrate."""
    which = ["tg", 1, 2, 3][:batch]
    refs, dts = [], []
    for w in which:
        oeq = oracle_eq(3, N)
        u = field_3d(N, w).copy()
        dts.append(ora.SSP_RK3(oeq).integrate(0.0, 1.0, C_CFL, u))
        refs.append(u)
    for prec, tol, tol_dt in (("f64", TOL64, TOL_DT64), ("f32", TOL32, TOL_DT32)):
        eq = gpu_eq(3, N, prec, batch)
        ts = az.SSP_RK3(eq)
        d_u = torch.stack([to_dev(field_3d(N, w), prec) for w in which]).contiguous()
        if batch == 1:
            d_u = d_u[0].contiguous()
        dt = ts.integrate(0.0, 1.0, C_CFL, d_u)
        dt = [dt] if batch == 1 else dt
        got = to_host(d_u)
        got = got[None] if batch == 1 else got
        _check_members(got, refs, tol, f"{prec} N={N} RK3 step")
        for b in range(batch):
            assert abs(dt[b] - dts[b]) <= tol_dt * dts[b]
        del eq, ts, d_u, got
        torch.cuda.empty_cache()


# ---------------------------------------------------------------------------
# 2-D double-shear-layer ensembles at their batches
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("N,batch", [(128, 256), (256, 192), (512, 64)])
def test_dudt_and_step_2d_ensemble(N, batch):
    rng = np.random.default_rng(N)
    phases = rng.uniform(0.0, 2 * math.pi, batch)
    phases[0] = 0.0  # the reference's DoubleShearLayer itself
    fields = [dsl_hat(N, p) for p in phases]
    oeq = oracle_eq(2, N)
    rhs_ref = [oeq.dudt(f) for f in fields]
    # single-precision conditioning of a few members (the phase barely changes it)
    e32 = max(single_precision_error(oeq, fields[b], rhs_ref[b]) for b in (0, 1, batch - 1))
    step_ref, dt_ref = [], []
    for f in fields:
        u = f.copy()
        dt_ref.append(ora.SSP_RK3(oeq).integrate(0.0, 1.0, C_CFL, u))
        step_ref.append(u)
    for prec, tol, tol_dt in (("f64", TOL64, TOL_DT64), ("f32", tol32_rhs(e32), TOL_DT32)):
        eq = gpu_eq(2, N, prec, batch)
        d_u = torch.stack([to_dev(f, prec) for f in fields]).contiguous()
        d_out = torch.empty_like(d_u)
        eq.dudt(d_out, d_u)
        _check_members(to_host(d_out), rhs_ref, tol, f"{prec} 2-D N={N} rhs")
        ts = az.SSP_RK3(eq)
        dts = ts.integrate(0.0, 1.0, C_CFL, d_u)
        _check_members(to_host(d_u), step_ref, TOL64 if prec == "f64" else TOL32, f"{prec} 2-D N={N} step")
        for b in range(batch):
            assert abs(dts[b] - dt_ref[b]) <= tol_dt * dt_ref[b]


# ---------------------------------------------------------------------------
# 3-D N = 512 (M = 768): the bounded-memory oracle
# ---------------------------------------------------------------------------

def test_dudt_3d_512():
    N = 512
    u_hat = random_hat_3d(N, seed=512)
    oeq = oracle_eq(3, N)
    ref = oeq.dudt(u_hat)
    dt_ref = oeq.dt(C_CFL)
    e32 = single_precision_error(oeq, u_hat, ref)
    for prec, tol, tol_dt in (("f32", tol32_rhs(e32), TOL_DT32), ("f64", TOL64, TOL_DT64)):
        eq = gpu_eq(3, N, prec, 1)
        d_u = to_dev(u_hat, prec)
        eq.dudt(d_u, d_u, 0.0, 0.0, C_CFL)  # in place, as the reference allows
        err = rel_l2(to_host(d_u), ref)
        assert err <= tol, f"{prec} N=512: relative L2 {err:.3e}"
        dt = eq.dt(C_CFL)
        assert abs(dt - dt_ref) <= tol_dt * dt_ref
        del eq, d_u
        torch.cuda.empty_cache()
