"""Initial data for the benchmark workloads, built on the device.

Each generator samples a physical field at x_i = 2 pi i / N (the reference's
sampling, src/azeban/init/taylor_green.cpp:40-41), transforms it with this
library's FFT and Leray-projects it, as Initializer::initialize does
(include/azeban/init/initializer.hpp:68-75).
"""

from __future__ import annotations

import math

import torch

from .core import FFT, FFT_FORWARD, leray

_RDT = {"f64": torch.float64, "f32": torch.float32}
_CDT = {"f64": torch.complex128, "f32": torch.complex64}


def _coords(N, dim, dtype):
    x = (2 * math.pi / N) * torch.arange(N, device="cuda", dtype=torch.float64)
    return [g.to(dtype) for g in torch.meshgrid(*([x] * dim), indexing="ij")]


def spectral(u_phys: torch.Tensor, project: bool = True) -> torch.Tensor:
    """Forward transform of a [(B,) dim, N, ...] physical field (+ Leray)."""
    # [dim, N...] (one member) or [B, dim, N...]
    if u_phys.dim() >= 3 and u_phys.shape[0] in (2, 3) and u_phys.dim() == u_phys.shape[0] + 1:
        flat = u_phys.unsqueeze(0)
        squeeze = True
    else:
        flat = u_phys
        squeeze = False
    B, d = flat.shape[0], flat.shape[1]
    N = flat.shape[-1]
    cdt = torch.complex128 if flat.dtype == torch.float64 else torch.complex64
    u = flat.reshape((B * d,) + tuple(flat.shape[2:])).contiguous()
    u_hat = torch.empty((B * d,) + tuple(flat.shape[2:-1]) + (N // 2 + 1,), dtype=cdt, device="cuda")
    fft = FFT(u_hat, u, FFT_FORWARD)
    fft.forward()
    u_hat = u_hat.reshape((B, d) + tuple(u_hat.shape[1:]))
    if project:
        leray(u_hat)
    return u_hat[0] if squeeze else u_hat


def taylor_green(dim: int, N: int, precision: str = "f64") -> torch.Tensor:
    """Taylor-Green of the workloads: (sin x cos y, -cos x sin y) in 2-D and
    (sin x cos y cos z, -cos x sin y cos z, 0) in 3-D; spectral, [dim, N, ..., N/2+1]."""
    dt = torch.float64
    if dim == 2:
        x, y = _coords(N, 2, dt)
        u = torch.stack([torch.sin(x) * torch.cos(y), -torch.cos(x) * torch.sin(y)])
    else:
        x, y, z = _coords(N, 3, dt)
        u = torch.stack([torch.sin(x) * torch.cos(y) * torch.cos(z),
                         -torch.cos(x) * torch.sin(y) * torch.cos(z),
                         torch.zeros_like(x)])
    return spectral(u.to(_RDT[precision]))


def double_shear_layer(N: int, rho: float, delta: float, phases, precision: str = "f64") -> torch.Tensor:
    """Double shear layer (src/azeban/init/double_shear_layer.cpp:25-43) with a
    phase per member: u = tanh(2 pi (y - 1/4)/rho) for y < 1/2, else
    tanh(2 pi (3/4 - y)/rho); v = delta sin(2 pi x + phi).  [B, 2, N, N/2+1]."""
    i = torch.arange(N, device="cuda", dtype=torch.float64) / N
    x = i[:, None].expand(N, N)
    y = i[None, :].expand(N, N)
    if rho == 0:
        u = torch.where((y - 0.5).abs() < 0.25, 1.0, -1.0)
    else:
        u = torch.where(y < 0.5, torch.tanh(2 * math.pi * (y - 0.25) / rho),
                        torch.tanh(2 * math.pi * (0.75 - y) / rho))
    ph = torch.as_tensor(list(phases), device="cuda", dtype=torch.float64)
    v = delta * torch.sin(2 * math.pi * x[None] + ph[:, None, None])
    field = torch.stack([u[None].expand_as(v), v], dim=1)
    return spectral(field.to(_RDT[precision]).contiguous())


def fractional_brownian(dim: int, N: int, hurst: float = 0.75, seed: int = 0, precision: str = "f64") -> torch.Tensor:
    """Random divergence-free field: Gaussian Fourier coefficients with
    amplitude |n|^-(H + d/2), Leray-projected, normalised to kinetic energy
    1/2 <|u|^2> = 1.  The coefficients come from the forward transform of
    seeded Gaussian white noise, so the spectrum is Hermitian-consistent.
    [dim, N, ..., N/2+1].  (azeban's own BrownianMotion,
    src/azeban/init/brownian_motion.cpp:144-203, draws uniform coefficients;
    this is the Gaussian form of the workloads.)"""
    gen = torch.Generator(device="cuda").manual_seed(int(seed))
    noise = torch.randn((dim,) + (N,) * dim, generator=gen, device="cuda", dtype=torch.float64)
    u_hat = spectral(noise.to(_RDT[precision]), project=False)
    idx = torch.arange(N, device="cuda", dtype=torch.float64)
    signed = torch.where(idx >= N // 2 + 1, idx - N, idx)
    axes = [signed] * (dim - 1) + [torch.arange(N // 2 + 1, device="cuda", dtype=torch.float64)]
    k2 = sum(g * g for g in torch.meshgrid(*axes, indexing="ij"))
    amp = torch.where(k2 > 0, k2.clamp_min(1e-300) ** (-(hurst + dim / 2.0) / 2.0), torch.zeros_like(k2))
    u_hat = u_hat * amp.to(u_hat.real.dtype)
    leray(u_hat)
    # kinetic energy of the unnormalised half spectrum (Parseval)
    w = torch.full((N // 2 + 1,), 2.0, device="cuda", dtype=torch.float64)
    w[0] = 1.0
    if N % 2 == 0:
        w[N // 2] = 1.0
    e = 0.5 * (w * (u_hat.abs().to(torch.float64) ** 2)).sum() / float(N) ** (2 * dim)
    return (u_hat / torch.sqrt(e).to(u_hat.real.dtype)).contiguous()
