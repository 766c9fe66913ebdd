"""The right-hand side entry point that allocates nothing.

az_euler_dudt_noalloc serves callers that cannot let a library allocate
device memory (a host code that owns all device memory through its own pool
under a fixed cap): its scratch is one fixed device array inside the library.
Called through the C ABI, it must give the output of the regular entry point
(az_euler_dudt through IncompressibleEuler.dudt) within the FP64 parity
tolerance, on two calls in a row that share that array.

This file sorts last so a run that stops at the first failure has already run
every other test; it also passes alone in a fresh process.
"""

import contextlib
import ctypes as ct
import os

import numpy as np
import pytest
import torch

import azeban_b200 as az
from azeban_b200 import _lib
from tests.gpu_helpers import VISC_CFGS, random_field_hat, rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def _noalloc(dim, N, M, prec, visc, out, inp):
    code = az.precision_code(prec)
    cv = visc.to_c()
    stream = torch.cuda.current_stream().cuda_stream or None
    return _lib.lib.az_euler_dudt_noalloc(dim, N, M, code, ct.byref(cv), out.data_ptr(), inp.data_ptr(),
                                          stream)


@pytest.mark.parametrize("dim,N,prec", [(3, 16, "f64"), (2, 64, "f64"), (3, 32, "f32"),
                                        (3, 64, "f64"), (2, 1024, "f64"), (3, 64, "f32")])
def test_noalloc_matches_regular_entry_point_twice(dim, N, prec):
    g = az.Grid(dim, N)
    visc = az.make_viscosity(VISC_CFGS["smooth"], g)
    eq = az.IncompressibleEuler(g, visc, prec)
    tol = TOL64 if prec == "f64" else TOL32
    for call, seed in enumerate((21, 22)):
        u = to_dev(random_field_hat(dim, N, seed=seed), prec)
        ref = torch.empty_like(u)
        eq.dudt(ref, u)
        out = torch.full_like(u, float("nan"))
        _lib.check(_noalloc(dim, N, g.N_phys_pad, prec, visc, out, u))
        torch.cuda.synchronize()
        got = to_host(out)
        assert np.isfinite(got).all(), f"call {call}"
        assert rel_l2(got, to_host(ref)) <= tol, f"call {call}"


def test_noalloc_second_call_with_other_size():
    """A smaller solve after a larger one: the shared array keeps the last
    call's contents and the entry point must not depend on them."""
    for dim, N in ((3, 32), (2, 16)):
        g = az.Grid(dim, N)
        visc = az.make_viscosity(VISC_CFGS["quadratic"], g)
        eq = az.IncompressibleEuler(g, visc)
        u = to_dev(random_field_hat(dim, N, seed=N))
        ref = torch.empty_like(u)
        eq.dudt(ref, u)
        out = torch.empty_like(u)
        _lib.check(_noalloc(dim, N, g.N_phys_pad, "f64", visc, out, u))
        torch.cuda.synchronize()
        assert rel_l2(to_host(out), to_host(ref)) <= TOL64


def test_noalloc_rejects_sizes_above_its_scratch():
    g = az.Grid(3, 128)
    visc = az.make_viscosity(VISC_CFGS["smooth"], g)
    u = torch.zeros((3, 128, 128, 65), dtype=torch.complex128, device="cuda")
    st = _noalloc(3, 128, 192, "f64", visc, u, u)
    assert st == 2  # AZ_ERR_UNSUPPORTED
    assert "scratch" in _lib.lib.az_last_error_string().decode()


@contextlib.contextmanager
def _pad_mask(mask):
    """Row padding of every intermediate (AZ_PAD_MASK, read per call): the
    largest scratch layout."""
    old = os.environ.get("AZ_PAD_MASK")
    os.environ["AZ_PAD_MASK"] = str(mask)
    try:
        yield
    finally:
        if old is None:
            del os.environ["AZ_PAD_MASK"]
        else:
            os.environ["AZ_PAD_MASK"] = old


@pytest.mark.parametrize("dim,N", [(3, 64), (2, 1024)])
def test_noalloc_largest_layout_fits_or_is_rejected(dim, N):
    """With every intermediate row padded the documented maximum sizes still
    fit the array and match the regular entry point (or, if a layout did not
    fit, the call would return AZ_ERR_UNSUPPORTED without touching memory)."""
    g = az.Grid(dim, N)
    visc = az.make_viscosity(VISC_CFGS["smooth"], g)
    eq = az.IncompressibleEuler(g, visc)
    u = to_dev(random_field_hat(dim, N, seed=77))
    ref = torch.empty_like(u)
    eq.dudt(ref, u)
    out = torch.full_like(u, float("nan"))
    with _pad_mask(15):
        st = _noalloc(dim, N, g.N_phys_pad, "f64", visc, out, u)
    if st == _lib.AZ_ERR_UNSUPPORTED:
        assert "scratch" in _lib.lib.az_last_error_string().decode()
        return
    _lib.check(st)
    _lib.check(_lib.lib.az_euler_noalloc_status(torch.cuda.current_stream().cuda_stream or None))
    assert rel_l2(to_host(out), to_host(ref)) <= TOL64


def test_noalloc_status_reports_device_failures():
    """The device-side status of the last call comes back without an
    allocation: a bounded wait that runs out (poll limit 0) gives
    AZ_ERR_TIMEOUT, a NaN in the state AZ_ERR_NONFINITE, and a clean call
    after them AZ_OK with the right result."""
    dim, N, prec = 3, 32, "f32"
    g = az.Grid(dim, N)
    visc = az.make_viscosity(VISC_CFGS["smooth"], g)
    eq = az.IncompressibleEuler(g, visc, prec)
    stream = torch.cuda.current_stream().cuda_stream or None
    u = to_dev(random_field_hat(dim, N, seed=5), prec)
    out = torch.empty_like(u)
    code = az.precision_code(prec)
    old_v = ct.c_int()
    _lib.check(_lib.lib.az_tune_get(code, g.N_phys_pad, 1, ct.byref(old_v)))
    old_polls = _lib.lib.az_debug_get_wait_limit()
    try:
        _lib.check(_lib.lib.az_tune_set(code, g.N_phys_pad, 1, 3))  # the bulk-copy product pass
        _lib.check(_lib.lib.az_debug_set_wait_limit(0))
        _lib.check(_noalloc(dim, N, g.N_phys_pad, prec, visc, out, u))
        assert _lib.lib.az_euler_noalloc_status(stream) == _lib.AZ_ERR_TIMEOUT
    finally:
        _lib.check(_lib.lib.az_debug_set_wait_limit(old_polls))
        _lib.check(_lib.lib.az_tune_set(code, g.N_phys_pad, 1, old_v.value))
    bad = u.clone()
    bad[0, 1, 1, 1] = float("nan")
    _lib.check(_noalloc(dim, N, g.N_phys_pad, prec, visc, out, bad))
    assert _lib.lib.az_euler_noalloc_status(stream) == _lib.AZ_ERR_NONFINITE
    _lib.check(_noalloc(dim, N, g.N_phys_pad, prec, visc, out, u))
    _lib.check(_lib.lib.az_euler_noalloc_status(stream))
    ref = torch.empty_like(u)
    eq.dudt(ref, u)
    assert rel_l2(to_host(out), to_host(ref)) <= TOL32
