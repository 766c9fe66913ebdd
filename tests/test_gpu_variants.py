"""Parity of every kernel variant of the right-hand side with the CPU oracle.

The passes have several kernels: bit 0 of a variant picks the radix plan
(0 std, 1 wide); bit 1 picks the two-tile column kernel for the column
passes and the bulk-copy kernel for the contiguous-axis pass.  The tuning table picks one per
(precision, length, kind); these tests pin each one against the oracle, so a
table entry can never select a kernel whose results differ.  Tolerances as in
test_gpu_euler.py.
"""

import ctypes as ct

import numpy as np
import pytest
import torch

import azeban_b200 as az
from azeban_b200 import _lib
from oracle import euler_oracle as ora
from tests.gpu_helpers import VISC_CFGS, random_field_hat, rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


class _Variants:
    """Sets the tuning table entries of one (precision, length) and restores
    the previous ones on exit."""

    def __init__(self, prec, L, dim, cols, rows, epi):
        self.p = 0 if prec == "f64" else 1
        self.L = L
        kb = 3 if dim == 2 else 0
        self.want = {kb + 0: cols, kb + 1: rows, kb + 2: epi}

    def __enter__(self):
        self.saved = {}
        for kind, v in self.want.items():
            old = ct.c_int()
            _lib.check(_lib.lib.az_tune_get(self.p, self.L, kind, ct.byref(old)))
            self.saved[kind] = old.value
            _lib.check(_lib.lib.az_tune_set(self.p, self.L, kind, v))
        return self

    def __exit__(self, *exc):
        for kind, v in self.saved.items():
            _lib.check(_lib.lib.az_tune_set(self.p, self.L, kind, v))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,N", [(2, 32), (2, 64), (2, 128), (3, 16), (3, 32)])
@pytest.mark.parametrize("cols,rows,epi", [(0, 0, 0), (1, 1, 1), (0, 2, 0), (1, 3, 1), (2, 2, 0), (3, 3, 1)])
def test_dudt_every_variant(prec, dim, N, cols, rows, epi):
    og = ora.Grid(dim, N)
    g = az.Grid(dim, N)
    oeq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))
    u_hat = random_field_hat(dim, N, seed=300 + 10 * dim + N)
    ref = oeq.dudt(u_hat)
    with _Variants(prec, g.N_phys_pad, dim, cols, rows, epi):
        eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), prec)
        d_u = to_dev(u_hat, prec)
        d_out = torch.empty_like(d_u)
        eq.dudt(d_out, d_u, 0.0, 0.0, 0.2)
        got = to_host(d_out)
        dt = eq.dt(0.2)
    assert rel_l2(got, ref) <= TOL[prec]
    rel_dt = 1e-13 if prec == "f64" else 1e-6
    assert abs(dt - oeq.dt(0.2)) <= rel_dt * oeq.dt(0.2)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,N,M", [(2, 32, 48), (2, 64, 96), (2, 128, 192), (2, 256, 384), (3, 16, 24),
                                     (3, 32, 48), (3, 64, 96), (3, 34, 384), (2, 34, 768)])
@pytest.mark.parametrize("rows", [4, 5, 6, 7])
def test_dudt_fused_product_variants(prec, dim, N, M, rows):
    """The fused product pass (bit 2 of the contiguous-axis variant: products
    formed in the forward transform's loads, one work area, gap rows, input
    pair stride, twiddles from powers of two; bit 0 the forward plan, bit 1
    the inverse plan) against the oracle, on both plans of both transforms
    and on heavy padding (M = 384 and 768 with few retained rows)."""
    og = ora.Grid(dim, N, M)
    g = az.Grid(dim, N, M)
    oeq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))
    u_hat = random_field_hat(dim, N, seed=900 + 10 * dim + N)
    ref = oeq.dudt(u_hat)
    with _Variants(prec, M, dim, 0, rows, 0):
        eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), prec)
        d_u = to_dev(u_hat, prec)
        d_out = torch.empty_like(d_u)
        eq.dudt(d_out, d_u, 0.0, 0.0, 0.2)
        got = to_host(d_out)
        dt = eq.dt(0.2)
    assert rel_l2(got, ref) <= TOL[prec]
    rel_dt = 1e-13 if prec == "f64" else 1e-6
    assert abs(dt - oeq.dt(0.2)) <= rel_dt * oeq.dt(0.2)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,N,B", [(2, 32, 7), (3, 16, 3)])
@pytest.mark.parametrize("rows", [2, 3, 5, 7])
def test_bulk_copy_kernel_batch_members_match_single(prec, dim, N, B, rows):
    """With the bulk-copy kernel, each member of a batch equals the same solve
    alone, bit for bit, over a short simulate_until.  Members have different
    amplitudes, so they finish at different steps and the skip flags are
    exercised."""
    g = az.Grid(dim, N)
    v = az.make_viscosity(VISC_CFGS["smooth"], g)
    fields = [random_field_hat(dim, N, seed=900 + b) * (1.0 + 0.5 * b) for b in range(B)]
    with _Variants(prec, g.N_phys_pad, dim, 2, rows, 0):
        eqB = az.IncompressibleEuler(g, v, prec, batch=B)
        simB = az.Simulation(g, 0.2, az.SSP_RK3(eqB), to_dev(np.stack(fields), prec))
        simB.simulate_until(0.02)
        outB = to_host(simB.u())
        _, nB, _ = simB.state()
        for b in range(B):
            eq1 = az.IncompressibleEuler(g, v, prec)
            sim1 = az.Simulation(g, 0.2, az.SSP_RK3(eq1), to_dev(fields[b], prec))
            sim1.simulate_until(0.02)
            assert sim1.state()[1][0] == nB[b]
            np.testing.assert_array_equal(to_host(sim1.u()), outB[b])


@pytest.mark.parametrize("mask", [0, 5, 10, 15])
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,N", [(2, 64), (3, 16), (3, 32)])
def test_dudt_every_row_padding(mask, prec, dim, N, monkeypatch):
    """The intermediates' rows may be padded to whole 128-byte lines
    (AZ_PAD_MASK bits: A1, A2, B1, B2); every combination gives the oracle's
    right-hand side, including the grouped column paths of the inverse x pass
    and the epilogue."""
    monkeypatch.setenv("AZ_PAD_MASK", str(mask))
    og = ora.Grid(dim, N)
    g = az.Grid(dim, N)
    oeq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))
    u_hat = random_field_hat(dim, N, seed=500 + N)
    ref = oeq.dudt(u_hat)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), prec)
    d_u = to_dev(u_hat, prec)
    d_out = torch.empty_like(d_u)
    eq.dudt(d_out, d_u)
    assert rel_l2(to_host(d_out), ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,N,M", [(3, 34, 384), (2, 34, 768)])
def test_dudt_heavy_padding(prec, dim, N, M):
    """Heavy padding (M far above 3N/2): narrow epilogue tiles of a few mode
    columns, a partial last tile (N = 34 gives odd tile counts), and zero rows
    filling most of every padded line."""
    og = ora.Grid(dim, N, M)
    g = az.Grid(dim, N, M)
    oeq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))
    u_hat = random_field_hat(dim, N, seed=700 + 10 * dim + N)
    ref = oeq.dudt(u_hat)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), prec)
    d_u = to_dev(u_hat, prec)
    d_out = torch.empty_like(d_u)
    eq.dudt(d_out, d_u, 0.0, 0.0, 0.2)
    assert rel_l2(to_host(d_out), ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,N,M", [(3, 16, 768), (2, 64, 768), (3, 16, 1536)])
def test_long_line_product_kernels_agree(prec, dim, N, M):
    """Every product-pass kernel at the longest lines (where the chunk sizes
    shrink to keep several CTAs per SM) gives the same right-hand side; the
    padded grid is too large for the oracle, so the kernels are checked
    against each other and the FP32 results against FP64."""
    g = az.Grid(dim, N, M)
    u_hat = random_field_hat(dim, N, seed=900 + dim + N)
    outs = {}
    for p in ("f64", prec):
        for rows in (0, 1, 2, 3):
            with _Variants(p, M, dim, 0, rows, 0):
                eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), p)
                d_u = to_dev(u_hat, p)
                d_out = torch.empty_like(d_u)
                eq.dudt(d_out, d_u, 0.0, 0.0, 0.2)
                outs[(p, rows)] = to_host(d_out)
    ref = outs[("f64", 1)]
    for key, got in outs.items():
        assert rel_l2(got, ref) <= TOL[key[0]], key
