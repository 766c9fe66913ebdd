"""Initial data for the workloads and the reference's initialisers, built on
the device.

Each generator samples its physical field in one kernel of the library
(az_init_physical, straight into a device array), transforms it with the
library's FFT and Leray-projects it, as Initializer::initialize does
(include/azeban/init/initializer.hpp:68-75).  Random values (shear-layer
phases, Gaussian coefficients) come from the library's counter-based Philox
stream (seed, member), so a member's field depends only on its seed and
member index, not on the batch it is generated in.
"""

from __future__ import annotations

import ctypes as ct
import math

import torch

from . import _lib
from ._lib import check, lib
from .core import FFT, FFT_FORWARD, _stream_ptr, leray, precision_code

_RDT = {0: torch.float64, 1: torch.float32}


def physical(kind: int, dim: int, N: int, precision="f64", batch: int = 1, rho: float = 0.0,
             delta: float = 0.0, deltas=None, phases=None, seed: int = 0, member0: int = 0,
             stream=None) -> torch.Tensor:
    """The physical field [batch, dim, N, ...] of one generator (az_init_physical)."""
    prec = precision_code(precision)
    u = torch.empty((batch, dim) + (N,) * dim, dtype=_RDT[prec], device="cuda")
    keep = []

    def arr(x, n):
        if x is None:
            return None
        flat = [float(v) for v in x]
        if len(flat) != n:
            raise ValueError(f"expected {n} values, got {len(flat)}")
        a = (ct.c_double * n)(*flat)
        keep.append(a)
        return ct.cast(a, ct.POINTER(ct.c_double))

    nd = 8 if dim == 2 else 24
    desc = _lib.az_init_desc(kind, dim, N, prec, batch, float(rho), float(delta),
                             arr(None if deltas is None else [v for row in deltas for v in row], batch * nd),
                             arr(phases, batch), int(seed) & (2**64 - 1), int(member0))
    check(lib.az_init_physical(ct.byref(desc), u.data_ptr(), _stream_ptr(stream)))
    return u


def spectral(u_phys: torch.Tensor, project: bool = True, batched: bool | None = None) -> torch.Tensor:
    """Forward transform of a [(B,) dim, N, ...] physical field (+ Leray).
    batched: whether axis 0 is the member axis (None: inferred from the rank,
    which cannot tell a batch of three 2-D fields from one 3-D field)."""
    # [dim, N...] (one member) or [B, dim, N...]
    if batched is None:
        batched = not (u_phys.dim() >= 3 and u_phys.shape[0] in (2, 3) and u_phys.dim() == u_phys.shape[0] + 1)
    if not batched:
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
    return spectral(physical(_lib.AZ_INIT_TAYLOR_GREEN_WORKLOAD, dim, N, precision), batched=True)[0]


def taylor_green_reference(dim: int, N: int, precision: str = "f64", deltas=None) -> torch.Tensor:
    """The reference's Taylor-Green (src/azeban/init/taylor_green.cpp:29-46,
    :146-184): (cos x sin y, -sin x cos y) in 2-D, (cos x sin y sin z,
    -sin x cos y sin z, 0) in 3-D, plus the perturbation modes with amplitudes
    deltas [batch][8 or 24] (the reference's draws, already divided by 4 or
    8); spectral, [batch, dim, N, ..., N/2+1] (batch 1 without deltas)."""
    batch = 1 if deltas is None else len(deltas)
    return spectral(physical(_lib.AZ_INIT_TAYLOR_GREEN, dim, N, precision, batch, deltas=deltas), batched=True)


def double_shear_layer(N: int, rho: float, delta: float, phases=None, precision: str = "f64", seed: int = 0,
                       member0: int = 0, batch: int | None = None) -> torch.Tensor:
    """Double shear layer (src/azeban/init/double_shear_layer.cpp:25-43) with a
    phase per member: u = tanh(2 pi (y - 1/4)/rho) for y < 1/2, else
    tanh(2 pi (3/4 - y)/rho); v = delta sin(2 pi x + phi).  phases: given per
    member, or None to draw phi ~ U[0, 2 pi) from stream (seed, member0 + b)
    for `batch` members.  [B, 2, N, N/2+1]."""
    if phases is not None:
        batch = len(phases)
    elif batch is None:
        batch = 1
    return spectral(physical(_lib.AZ_INIT_DOUBLE_SHEAR_LAYER, 2, N, precision, batch, rho=rho, delta=delta,
                             phases=phases, seed=seed, member0=member0), batched=True)


def stream_uniform(seed: int, member: int, index: int = 0) -> float:
    """Value `index` of random stream (seed, member) as a uniform in [0, 1)."""
    out = ct.c_double()
    check(lib.az_random_uniform(int(seed) & (2**64 - 1), int(member), int(index), ct.byref(out)))
    return out.value


def shear_layer_phase(seed: int, member: int = 0) -> float:
    """The phase az_init_physical draws for member `member` of seed `seed`."""
    return 2 * math.pi * stream_uniform(seed, member, 0)


def fractional_brownian(dim: int, N: int, hurst: float = 0.75, seed: int = 0, precision: str = "f64",
                        batch: int = 1, member0: int = 0) -> torch.Tensor:
    """Random divergence-free field: Gaussian Fourier coefficients with
    amplitude |n|^-(H + d/2), Leray-projected, normalised to kinetic energy
    1/2 <|u|^2> = 1.  The coefficients are the forward transform of seeded
    Gaussian white noise (stream (seed, member0 + b)), so the spectrum is
    Hermitian-consistent.  [dim, N, ..., N/2+1] for batch 1, else
    [batch, dim, ...].  (azeban's own BrownianMotion,
    src/azeban/init/brownian_motion.cpp:144-203, draws uniform coefficients;
    this is the Gaussian form of the workloads.)"""
    prec = precision_code(precision)
    noise = physical(_lib.AZ_INIT_GAUSSIAN_NOISE, dim, N, precision, batch, seed=seed, member0=member0)
    u_hat = spectral(noise, project=False, batched=True).contiguous()
    check(lib.az_init_envelope(dim, N, prec, u_hat.data_ptr(), batch, -(hurst + dim / 2.0),
                               _stream_ptr(None)))
    leray(u_hat)
    check(lib.az_init_normalize_energy(dim, N, prec, u_hat.data_ptr(), batch, 1.0, _stream_ptr(None)))
    return u_hat[0] if batch == 1 else u_hat
