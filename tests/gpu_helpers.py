"""Shared helpers of the GPU parity tests: seeded inputs built with the oracle
(the checker) and conversions between numpy and torch CUDA tensors."""

import math

import numpy as np
import torch

from oracle import euler_oracle as ora

VISC_CFGS = {
    "smooth": {"type": "Smooth Cutoff", "eps": 0.05},
    "step": {"type": "Step", "eps": 0.05},
    "quadratic": {"type": "Quadratic", "eps": 0.05},
    "none": {"type": "None"},
}


def random_field_hat(dim, N, seed, slope=2.0):
    """Seeded divergence-free spectral field with a decaying spectrum and
    every retained mode populated (Hermitian-consistent: the forward
    transform of a real physical field)."""
    rng = np.random.default_rng(seed)
    shape = (dim,) + (N,) * dim
    u = rng.standard_normal(shape)
    u_hat = ora.fft_forward(u)
    kk = [ora.signed_index(N).astype(float)] * (dim - 1) + [np.arange(N // 2 + 1, dtype=float)]
    ks = np.meshgrid(*kk, indexing="ij")
    kmag = np.sqrt(sum(k * k for k in ks))
    u_hat = u_hat * (1.0 + kmag) ** (-slope)
    u_hat = ora.leray(u_hat)
    # unit max velocity, roughly
    phys = ora.fft_backward(u_hat, N) / N ** dim
    u_hat /= max(np.abs(phys).max(), 1e-300)
    return u_hat


def to_dev(a, prec="f64"):
    dt = torch.complex128 if prec == "f64" else torch.complex64
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dt)


def to_host(t):
    return t.detach().to("cpu", dtype=torch.complex128).numpy()


def rel_l2(a, b):
    return ora.rel_l2(np.asarray(a), np.asarray(b))
