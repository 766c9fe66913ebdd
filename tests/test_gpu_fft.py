"""FFT<Dim> on the GPU against a naive DFT and the oracle.

Mirrors test/azeban/operations/fft.cpp:35-349 of the reference: inputs from a
default-seeded std::mt19937 through uniform_real_distribution(-1, 1), forward
compared with a naive DFT to 1e-8, backward checked as unnormalised (u / n^d).
"""

import numpy as np
import pytest
import torch

import azeban_b200 as az
from oracle.mt19937 import MT19937
from tests.gpu_helpers import rel_l2

pytestmark = pytest.mark.gpu


def naive_dft_axis(x, axis, real=False):
    """O(n^2) DFT along one axis (test/azeban/operations/fft.cpp:35-58)."""
    n = x.shape[axis]
    k = np.arange(n if not real else n // 2 + 1)[:, None]
    j = np.arange(n)[None, :]
    W = np.exp(-2j * np.pi * k * j / n)
    return np.moveaxis(np.tensordot(W, np.moveaxis(x, axis, 0), axes=(1, 0)), 0, axis)


def naive_rfftn(u, nt):
    d = u.ndim - 1
    out = naive_dft_axis(u.astype(np.complex128), d, real=True)
    for ax in range(d - 1, d - nt, -1):
        out = naive_dft_axis(out, ax)
    return out


CASES = [
    (1, 128, 1, (True,)), (1, 128, 2, (True,)),
    (2, 128, 1, (True, True)), (2, 128, 2, (True, True)),
    (2, 128, 1, (False, True)), (2, 128, 2, (False, True)),
    (3, 32, 1, (True, True, True)), (3, 32, 2, (True, True, True)),
    (3, 32, 1, (False, True, True)), (3, 32, 2, (False, False, True)),
]


@pytest.mark.parametrize("dim,n,nvars,transform", CASES)
def test_fft_matches_naive_dft(dim, n, nvars, transform):
    rng = MT19937()
    shape = (nvars,) + (n,) * dim
    u_ref = rng.uniform(-1.0, 1.0, int(np.prod(shape))).reshape(shape)
    nt = sum(transform)
    ref_hat = naive_rfftn(u_ref, nt)
    u = torch.from_numpy(u_ref).cuda()
    u_hat = torch.zeros(shape[:-1] + (n // 2 + 1,), dtype=torch.complex128, device="cuda")
    fft = az.make_fft(u_hat, u, az.FFT_FORWARD | az.FFT_BACKWARD, *transform)
    fft.forward()
    h_hat = u_hat.cpu().numpy()
    assert np.abs(h_hat.real - ref_hat.real).max() <= 1e-8
    assert np.abs(h_hat.imag - ref_hat.imag).max() <= 1e-8
    u.zero_()
    fft.backward()
    back = u.cpu().numpy() / n ** nt
    assert np.abs(back - u_ref).max() <= 1e-8


@pytest.mark.parametrize("n", [4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_fft_every_length_vs_numpy(n, prec):
    """Every compiled length, 2-D, against numpy.fft (pocketfft)."""
    rng = np.random.default_rng(n)
    rows = 6
    u_np = rng.standard_normal((2, rows, n))
    rdt = torch.float64 if prec == "f64" else torch.float32
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(u_np).to("cuda", rdt)
    u_hat = torch.zeros((2, rows, n // 2 + 1), dtype=cdt, device="cuda")
    fft = az.make_fft(u_hat, u, az.FFT_FORWARD | az.FFT_BACKWARD, False, True)
    fft.forward()
    ref = np.fft.rfft(u_np, axis=-1)
    tol = 1e-13 if prec == "f64" else 2e-6
    assert rel_l2(u_hat.cpu().numpy(), ref) <= tol
    fft.backward()
    assert rel_l2(u.cpu().double().numpy() / n, u_np) <= tol
    # complex axis of the same length
    if n <= 512:
        u2_np = rng.standard_normal((1, n, 8))
        u2 = torch.from_numpy(u2_np).to("cuda", rdt)
        h2 = torch.zeros((1, n, 5), dtype=cdt, device="cuda")
        f2 = az.make_fft(h2, u2)
        f2.forward()
        assert rel_l2(h2.cpu().numpy(), np.fft.rfftn(u2_np, axes=(1, 2))) <= tol
        f2.backward()
        assert rel_l2(u2.cpu().double().numpy() / (8 * n), u2_np) <= tol


def test_fft_unsupported_length_raises():
    u = torch.zeros((1, 10), dtype=torch.float64, device="cuda")
    u_hat = torch.zeros((1, 6), dtype=torch.complex128, device="cuda")
    with pytest.raises(az.AzebanError):
        az.make_fft(u_hat, u)


def test_fft_caller_work_area():
    """FFT::set_work_area (fft.hpp:84): a backward transform through a
    caller-owned work area equals one through the FFT's own (allocated on
    the first backward transform); a forward-only FFT reports its size but
    allocates nothing."""
    rng = np.random.default_rng(5)
    u_np = rng.standard_normal((3, 24, 32, 16))
    u_hat = torch.zeros((3, 24, 32, 9), dtype=torch.complex128, device="cuda")
    u = torch.from_numpy(u_np).cuda()
    own = az.make_fft(u_hat, u)
    own.forward()
    size = own.get_work_area_size()
    assert size == 3 * 24 * 32 * 9 * 16
    ref_hat = u_hat.clone()
    out_own = torch.empty_like(u)
    f_own = az.make_fft(ref_hat.clone(), out_own)
    f_own.backward()
    out_set = torch.empty_like(u)
    f_set = az.make_fft(ref_hat.clone(), out_set)
    work = torch.empty(size, dtype=torch.uint8, device="cuda")
    f_set.set_work_area(work)
    f_set.backward()
    np.testing.assert_array_equal(out_set.cpu().numpy(), out_own.cpu().numpy())
    assert rel_l2(out_set.cpu().numpy() / (24 * 32 * 16), u_np) <= 1e-13
    with pytest.raises(ValueError):
        f_set.set_work_area(torch.empty(size - 1, dtype=torch.uint8, device="cuda"))
