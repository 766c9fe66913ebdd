"""Failure detection without a GPU fault.

The reference aborts on errors (src/azeban/logging.hpp:24-32) and only warns
on a tiny dt (src/azeban/simulation.cpp:96-98); this library turns failures
into status codes.  Two device-side failures are detected:

  * a non-finite velocity, folded into the CFL reduction of the product pass:
    AZ_ERR_NONFINITE.  The tests plant a NaN in one member's host-side input
    state (data, not a fault) and check that the status comes back and that
    the other members of the batch are untouched by it;
  * a bounded wait that runs out (the product pass's wait for its bulk copy):
    AZ_ERR_TIMEOUT.  The tests set the wait's poll limit to 0 through
    az_debug_set_wait_limit, so every such wait gives up at once (the copy
    itself is valid and lands; the kernel waits for it before returning), and
    check that the status comes back and that the next call, with the limit
    restored, is correct again on the same context.
"""

import contextlib
import ctypes as ct

import numpy as np
import pytest
import torch

import azeban_b200 as az
from azeban_b200 import _lib
from oracle import euler_oracle as ora
from tests.gpu_helpers import VISC_CFGS, random_field_hat, rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def tuned(prec, L, kind, variant):
    """Temporarily selects a kernel variant (bit 1 of kinds 1 and 4: the
    bulk-copy product pass, the kernel with the bounded wait)."""
    code = az.precision_code(prec)
    old = ct.c_int()
    _lib.check(_lib.lib.az_tune_get(code, L, kind, ct.byref(old)))
    _lib.check(_lib.lib.az_tune_set(code, L, kind, variant))
    try:
        yield
    finally:
        _lib.check(_lib.lib.az_tune_set(code, L, kind, old.value))


@contextlib.contextmanager
def wait_limit(polls):
    old = _lib.lib.az_debug_get_wait_limit()
    _lib.check(_lib.lib.az_debug_set_wait_limit(polls))
    try:
        yield
    finally:
        _lib.check(_lib.lib.az_debug_set_wait_limit(old))


def _eq(dim, N, prec, batch=1):
    g = az.Grid(dim, N)
    return g, az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), prec, batch)


def _fields(dim, N, n):
    return [random_field_hat(dim, N, seed=500 + i) for i in range(n)]


# ---------------------------------------------------------------------------
# non-finite values
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("dim,N,prec,zpass", [(2, 32, "f64", False), (2, 32, "f32", True),
                                              (3, 16, "f64", True), (3, 16, "f32", False)])
def test_nonfinite_member_is_reported_and_isolated(dim, N, prec, zpass):
    """simulate_until returns AZ_ERR_NONFINITE when one member's state holds a
    NaN; the other members' states equal those of a clean batch bit for bit."""
    g, _ = _eq(dim, N, prec)
    kind = 1 if dim == 3 else 4
    with tuned(prec, g.N_phys_pad, kind, 3 if zpass else 1):
        fields = _fields(dim, N, 4)
        bad = [f.copy() for f in fields]
        bad[2][0][(1,) * dim] = np.nan
        runs = {}
        for name, fs in (("clean", fields), ("bad", bad)):
            _, eq = _eq(dim, N, prec, 4)
            sim = az.Simulation(g, 0.2, az.SSP_RK3(eq), torch.stack([to_dev(f, prec) for f in fs]).contiguous())
            if name == "bad":
                with pytest.raises(_lib.AzebanError) as ei:
                    sim.simulate_until(1.0)
                assert ei.value.status == _lib.AZ_ERR_NONFINITE
            else:
                sim.steps(1)
            runs[name] = (to_host(sim.u()), sim.state())
        (clean, st_clean), (bad_u, st_bad) = runs["clean"], runs["bad"]
        for b in (0, 1, 3):
            assert st_bad[1][b] == 1, "the other members took their step"
            assert np.array_equal(bad_u[b], clean[b]), f"member {b} changed by another member's NaN"
            assert st_bad[0][b] == st_clean[0][b]


@pytest.mark.parametrize("dim,N", [(2, 16), (3, 8)])
def test_nonfinite_rk3_and_dt(dim, N):
    """az_rk3_integrate and az_euler_dt report the NaN too; a following
    right-hand side of finite data clears it."""
    g, eq = _eq(dim, N, "f64")
    u = random_field_hat(dim, N, seed=9)
    bad = u.copy()
    bad[1][(0,) * dim] = np.inf
    d_bad = to_dev(bad)
    with pytest.raises(_lib.AzebanError) as ei:
        az.SSP_RK3(eq).integrate(0.0, 1.0, 0.2, d_bad)
    assert ei.value.status == _lib.AZ_ERR_NONFINITE
    out = torch.empty_like(d_bad)
    eq.dudt(out, to_dev(bad))
    with pytest.raises(_lib.AzebanError):
        eq.dt(0.2)
    eq.dudt(out, to_dev(u))
    og = ora.Grid(dim, N)
    oeq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))
    assert rel_l2(to_host(out), oeq.dudt(u)) <= 1e-12
    assert eq.dt(0.2) > 0


# ---------------------------------------------------------------------------
# bounded waits that run out
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("dim,N,prec", [(3, 32, "f32"), (3, 16, "f64"), (2, 64, "f32")])
def test_bounded_wait_timeout_is_reported(dim, N, prec):
    g = az.Grid(dim, N)
    kind = 1 if dim == 3 else 4
    u = random_field_hat(dim, N, seed=31)
    og = ora.Grid(dim, N)
    ref = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og)).dudt(u)
    with tuned(prec, g.N_phys_pad, kind, 3):
        _, eq = _eq(dim, N, prec)  # kernel variants are fixed when the equation is created
        d_u = to_dev(u, prec)
        out = torch.empty_like(d_u)
        with wait_limit(0):
            eq.dudt(out, d_u)
            with pytest.raises(_lib.AzebanError) as ei:
                eq.dt(0.2)
            assert ei.value.status == _lib.AZ_ERR_TIMEOUT
            # a simulation created (and its step graph captured) under the limit
            sim = az.Simulation(g, 0.2, az.SSP_RK3(eq), d_u)
            with pytest.raises(_lib.AzebanError) as ei:
                sim.simulate_until(0.01)
            assert ei.value.status == _lib.AZ_ERR_TIMEOUT
            del sim
        torch.cuda.synchronize()
        # the context is intact: the next right-hand side is right again
        eq.dudt(out, d_u)
        assert eq.dt(0.2) > 0
        assert rel_l2(to_host(out), ref) <= (1e-12 if prec == "f64" else 1e-5)


def test_wait_limit_rejects_negative():
    assert _lib.lib.az_debug_set_wait_limit(-1) == _lib.AZ_ERR_INVALID
    assert _lib.lib.az_debug_get_wait_limit() > 0
