"""Host-side mirror of azeban's interfaces for the Euler hot path.

Names, argument meaning and error behaviour follow the reference:
  Grid / make_grid          include/azeban/grid.hpp:30-165, include/azeban/grid_factory.hpp:28-92
  viscosities + factory     include/azeban/equations/spectral_viscosity.hpp:27-128,
                            include/azeban/equations/spectral_viscosity_factory.hpp:29-89
  IncompressibleEuler       include/azeban/equations/incompressible_euler.hpp:39-387
  SSP_RK3                   include/azeban/evolution/ssp_rk3.hpp:28-76
  Simulation                include/azeban/simulation.hpp:30-93, src/azeban/simulation.cpp:89-102
  make_fft / FFT            include/azeban/operations/fft.hpp:37-121, src/azeban/operations/fft_factory.cpp:10-48
  leray                     src/azeban/operations/leray.cpp:28-116
Every computation runs in ``libazeban_b200.so`` on the GPU; arrays are torch
CUDA tensors in the reference's layouts.  Where the reference aborts
(LOG_ERR / AZEBAN_ERR) this module raises ValueError, and a failing library
call raises AzebanError.
"""

from __future__ import annotations

import ctypes as ct
import math

import torch

from . import _lib
from ._lib import AzebanError, check, lib

PI = math.pi

_CDT = {0: torch.complex128, 1: torch.complex64}
_RDT = {0: torch.float64, 1: torch.float32}


def precision_code(precision) -> int:
    if precision in (0, "f64", "fp64", "double", torch.float64, torch.complex128):
        return _lib.AZ_PREC_F64
    if precision in (1, "f32", "fp32", "float", "fp32_bulk", torch.float32, torch.complex64):
        return _lib.AZ_PREC_F32
    raise ValueError(f"unknown precision {precision!r}")


def _stream_ptr(stream) -> int | None:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream if s.cuda_stream else None


def _check_tensor(t, name, dtype, shape):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must have dtype {dtype}, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


# ---------------------------------------------------------------------------
# Grid
# ---------------------------------------------------------------------------

def next_good_size(nmin: int) -> int:
    """Smallest 2^a 3^b 5^c 7^d >= nmin (src/azeban/operations/fft.cpp:27-61)."""
    best = None
    p7 = 1
    while True:
        p5 = p7
        while True:
            p3 = p5
            while True:
                p2 = p3
                while p2 < nmin:
                    p2 *= 2
                best = p2 if best is None else min(best, p2)
                if p3 >= nmin:
                    break
                p3 *= 3
            if p5 >= nmin:
                break
            p5 *= 5
        if p7 >= nmin:
            break
        p7 *= 7
    return best


class Grid:
    """Grid<Dim> (include/azeban/grid.hpp:30-53): N_phys, N_phys_pad (3N/2 by
    default), N_fourier = N/2+1, N_fourier_pad = M/2+1."""

    def __init__(self, dim: int, N_phys: int, N_phys_pad: int | None = None):
        if dim not in (1, 2, 3):
            raise ValueError("dim must be 1, 2 or 3")
        self.dim = int(dim)
        self.N_phys = int(N_phys)
        self.N_phys_pad = int(3 * self.N_phys // 2 if N_phys_pad is None else N_phys_pad)
        self.N_fourier = self.N_phys // 2 + 1
        self.N_fourier_pad = self.N_phys_pad // 2 + 1

    def shape_phys(self, n_vars):
        return (n_vars,) + (self.N_phys,) * self.dim

    def shape_fourier(self, n_vars):
        return (n_vars,) + (self.N_phys,) * (self.dim - 1) + (self.N_fourier,)

    def shape_phys_pad(self, n_vars):
        return (n_vars,) + (self.N_phys_pad,) * self.dim

    def shape_fourier_pad(self, n_vars):
        return (n_vars,) + (self.N_phys_pad,) * (self.dim - 1) + (self.N_fourier_pad,)

    def __repr__(self):
        return f"Grid(dim={self.dim}, N_phys={self.N_phys}, N_phys_pad={self.N_phys_pad})"


def make_grid(config: dict, dim: int) -> Grid:
    """Grid from the JSON "grid" object (include/azeban/grid_factory.hpp:28-92)."""
    if ("N_phys" in config) == ("N_fourier" in config):
        raise ValueError('Grid config must contain either "N_phys" or "N_fourier", but not both')
    n = int(config["N_phys"]) if "N_phys" in config else 2 * (int(config["N_fourier"]) - 1)
    g = Grid(dim, n)
    has_pp, has_fp = "N_phys_pad" in config, "N_fourier_pad" in config
    if has_pp and has_fp:
        raise ValueError('Grid config may contain "N_phys_pad" or "N_fourier_pad", but not both')
    if has_pp or has_fp:
        val = config["N_phys_pad" if has_pp else "N_fourier_pad"]
        if isinstance(val, str):
            g.N_phys_pad = next_good_size(-(-3 * g.N_phys // 2))
        elif has_pp:
            g.N_phys_pad = int(val)
        else:
            g.N_phys_pad = 2 * (int(val) - 1)
        g.N_fourier_pad = g.N_phys_pad // 2 + 1
    return g


# ---------------------------------------------------------------------------
# Spectral viscosity
# ---------------------------------------------------------------------------

class SmoothCutoff1D:
    """-eps k^{2s} (1 - exp(-(|k|/k0)^18)) (spectral_viscosity.hpp:56-77)."""

    def __init__(self, eps, s, k0):
        self.eps, self.s, self.k0 = float(eps), float(s), float(k0)

    def to_c(self):
        return _lib.az_visc(_lib.AZ_VISC_SMOOTH_CUTOFF, self.eps, self.s, self.k0, 0)


class Step1D:
    """-eps k^{2s} [|k| > k0] (spectral_viscosity.hpp:40-54)."""

    def __init__(self, eps, s, k0):
        self.eps, self.s, self.k0 = float(eps), float(s), float(k0)

    def to_c(self):
        return _lib.az_visc(_lib.AZ_VISC_STEP, self.eps, self.s, self.k0, 0)


class Quadratic:
    """-eps max(0, (k/2pi)^2 - N) (spectral_viscosity.hpp:103-123)."""

    def __init__(self, eps, N):
        self.eps, self.N = float(eps), int(N)

    def to_c(self):
        return _lib.az_visc(_lib.AZ_VISC_QUADRATIC, self.eps, 0.0, 0.0, self.N)


class NoViscosity:
    """nu = 0 (spectral_viscosity.hpp:125-128)."""

    eps = 0.0

    def to_c(self):
        return _lib.az_visc(_lib.AZ_VISC_NONE, 0.0, 0.0, 0.0, 0)


def make_viscosity(config: dict, grid: Grid):
    """The "visc" object of the equation config (src/azeban/equations/equation_factory.cpp:25-58,
    spectral_viscosity_factory.hpp:29-89): eps_N = eps / N^{2s-1},
    k0 = m0 N^theta, defaults s = 1, theta = (2s-1)/(2s), m0 = 2 pi."""
    typ = config.get("type")
    if typ in ("Smooth Cutoff", "Step"):
        if "eps" not in config:
            raise ValueError('Smooth Cutoff Viscosity expects "eps" parameter in config')
        s = float(config.get("s", 1.0))
        theta = float(config.get("theta", (2 * s - 1) / (2 * s)))
        m0 = float(config.get("m0", 2 * PI))
        eps = float(config["eps"])
        epsN = eps / math.pow(float(grid.N_phys), 2 * s - 1)
        mN = m0 * math.pow(float(grid.N_phys), theta)
        return (SmoothCutoff1D if typ == "Smooth Cutoff" else Step1D)(epsN, s, mN)
    if typ == "Quadratic":
        if "eps" not in config:
            raise ValueError('Quadratic Viscosity expects "eps" parameter in config')
        return Quadratic(float(config["eps"]) / grid.N_phys, grid.N_phys)
    if typ == "None":
        return NoViscosity()
    raise ValueError(f"Unknown viscosity type: {typ}")


# ---------------------------------------------------------------------------
# Equation
# ---------------------------------------------------------------------------

class IncompressibleEuler:
    """Equation<Dim> of the spectral-viscosity incompressible Euler RHS with
    no forcing, for ``batch`` ensemble members of one resolution.

    Arrays are [batch, dim, N, (N,) N/2+1] complex tensors (the batch axis is
    omitted when batch == 1 and the tensor has dim+1 axes)."""

    def __init__(self, grid: Grid, visc, precision="f64", batch: int = 1):
        if grid.dim not in (2, 3):
            raise ValueError("Incompressible Euler is only implemented for 2D and 3D")
        self.grid = grid
        self.visc_ = visc
        self.precision = precision_code(precision)
        self.batch = int(batch)
        desc = _lib.az_euler_desc(grid.dim, grid.N_phys, grid.N_phys_pad, self.precision,
                                  visc.to_c(), self.batch)
        h = ct.c_void_p()
        check(lib.az_euler_create(ct.byref(desc), ct.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.az_euler_destroy(h)
            self._h = None

    @property
    def cdtype(self):
        return _CDT[self.precision]

    def shape(self):
        s = self.grid.shape_fourier(self.grid.dim)
        return s if self.batch == 1 else (self.batch,) + s

    def _check(self, t, name):
        base = self.grid.shape_fourier(self.grid.dim)
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"{name} must be a CUDA tensor")
        if t.dim() == len(base) + 1:
            shp = (self.batch,) + base
        elif self.batch == 1 and t.dim() == len(base):
            shp = base
        else:
            raise ValueError(f"{name} must have shape {(self.batch,) + base}")
        if t.shape[-len(base)] != self.grid.dim:
            raise ValueError("Wrong number of variables")
        _check_tensor(t, name, self.cdtype, shp)

    def n_vars(self) -> int:
        return lib.az_euler_n_vars(self._h)

    def visc(self) -> float:
        return lib.az_euler_visc(self._h)

    def workspace_size(self) -> int:
        return lib.az_euler_workspace_size(self._h)

    def dudt(self, dudt_hat, u_hat, t=0.0, dt=0.0, C=0.0, stream=None):
        """Equation::dudt (incompressible_euler.hpp:103-120); dudt_hat may be u_hat."""
        self._check(dudt_hat, "dudt_hat")
        self._check(u_hat, "u_hat")
        check(lib.az_euler_dudt(self._h, dudt_hat.data_ptr(), u_hat.data_ptr(), float(t), float(dt),
                                float(C), _stream_ptr(stream)))

    def diagnostics(self, u_hat, stream=None):
        """Kinetic energy and enstrophy per member (FP64, compensated sums)."""
        self._check(u_hat, "u_hat")
        e = (ct.c_double * self.batch)()
        w = (ct.c_double * self.batch)()
        check(lib.az_euler_diagnostics(self._h, u_hat.data_ptr(), _stream_ptr(stream), e, w))
        return (e[0], w[0]) if self.batch == 1 else (list(e), list(w))

    def dt(self, C: float, stream=None):
        """Equation::dt (incompressible_euler.hpp:122-124), per member."""
        out = (ct.c_double * self.batch)()
        check(lib.az_euler_dt(self._h, float(C), _stream_ptr(stream), out))
        return out[0] if self.batch == 1 else list(out)


class SSP_RK3:
    """Shu-Osher SSP-RK3 (include/azeban/evolution/ssp_rk3.hpp:28-76)."""

    def __init__(self, equation: IncompressibleEuler):
        self.equation_ = equation
        h = ct.c_void_p()
        check(lib.az_rk3_create(equation._h, ct.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.az_rk3_destroy(h)
            self._h = None

    def equation(self):
        return self.equation_

    def integrate(self, t, max_dt, C, u, stream=None):
        """One step in place; returns dt (a list per member when batched)."""
        self.equation_._check(u, "u")
        out = (ct.c_double * self.equation_.batch)()
        check(lib.az_rk3_integrate(self._h, float(t), float(max_dt), float(C), u.data_ptr(),
                                   _stream_ptr(stream), out))
        return out[0] if self.equation_.batch == 1 else list(out)


class Simulation:
    """Simulation<Dim>: owns the state and advances it with the time stepper
    (src/azeban/simulation.cpp:89-102).  Each member keeps its own clock on
    the device."""

    def __init__(self, grid: Grid, C: float, timestepper: SSP_RK3, u_init, stream=None):
        self.grid = grid
        self.C_ = float(C)
        self.timestepper_ = timestepper
        eq = timestepper.equation_
        eq._check(u_init, "u_init")
        self._shape = tuple(u_init.shape)
        self._dtype = u_init.dtype
        h = ct.c_void_p()
        check(lib.az_sim_create(timestepper._h, self.C_, u_init.data_ptr(), _stream_ptr(stream),
                                ct.byref(h)))
        self._h = h
        self._keep = u_init  # the copy is enqueued on the stream; keep the source alive

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.az_sim_destroy(h)
            self._h = None

    def simulate_until(self, t, stream=None):
        check(lib.az_sim_simulate_until(self._h, float(t), _stream_ptr(stream)))

    def simulate_for(self, t, stream=None):
        self.simulate_until(max(self.time_all(stream)) + t, stream)

    def steps(self, n: int, stream=None):
        check(lib.az_sim_steps(self._h, int(n), _stream_ptr(stream)))

    def member_start(self, member: int, u_hat_member, t_end: float, stream=None):
        """Copies one member's state into slot `member` and restarts its clock
        at 0 with end t_end (continuous batching)."""
        base = self.grid.shape_fourier(self.grid.dim)
        _check_tensor(u_hat_member, "u_hat_member", self._dtype, base)
        check(lib.az_sim_member_start(self._h, int(member), u_hat_member.data_ptr(), float(t_end),
                                      _stream_ptr(stream)))

    def member_stop(self, member: int, stream=None):
        """Frees slot `member`: it is skipped until started again."""
        check(lib.az_sim_member_stop(self._h, int(member), _stream_ptr(stream)))

    def u(self):
        """A torch view of the device state (valid while the Simulation lives)."""
        ptr = lib.az_sim_u(self._h)
        return _tensor_from_ptr(ptr, self._shape, self._dtype)

    def state(self, stream=None):
        B = self.timestepper_.equation_.batch
        tm = (ct.c_double * B)()
        ns = (ct.c_longlong * B)()
        dt = (ct.c_double * B)()
        check(lib.az_sim_state(self._h, _stream_ptr(stream), tm, ns, dt))
        return list(tm), list(ns), list(dt)

    def time(self, stream=None):
        return self.state(stream)[0][0]

    def time_all(self, stream=None):
        return self.state(stream)[0]


class Group:
    """Several simulations (any dimension, size, precision) advanced together:
    steps() replays one captured graph per SSP-RK3 step with a branch per
    simulation; steps(active=...) and simulate_until() launch, per
    simulation, a step graph over its active member prefix only (none for a
    finished simulation), each on its own stream."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ct.c_void_p * len(self.sims))(*[s._h for s in self.sims])
        h = ct.c_void_p()
        check(lib.az_group_create(arr, len(self.sims), ct.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.az_group_destroy(h)
            self._h = None

    def steps(self, n: int, stream=None, active=None):
        """n SSP-RK3 steps.  active: optional per-simulation counts; only
        members [0, active[i]) of simulation i are launched (none for 0), so
        every started member must lie inside its prefix."""
        if active is None:
            check(lib.az_group_steps(self._h, int(n), _stream_ptr(stream)))
            return
        if len(active) != len(self.sims):
            raise ValueError("active needs one count per simulation")
        arr = (ct.c_int * len(self.sims))(*[int(a) for a in active])
        check(lib.az_group_steps_active(self._h, int(n), arr, _stream_ptr(stream)))

    def set_end(self, t: float, stream=None):
        check(lib.az_group_set_end(self._h, float(t), _stream_ptr(stream)))

    def simulate_until(self, t: float, stream=None):
        check(lib.az_group_simulate_until(self._h, float(t), _stream_ptr(stream)))


def _tensor_from_ptr(ptr, shape, dtype):
    """Wraps device memory owned by the library as a torch tensor (no copy)."""
    numel = 1
    for s in shape:
        numel *= s
    itemsize = torch.empty((), dtype=dtype).element_size()

    class _Holder:
        __cuda_array_interface__ = {
            "shape": (numel * itemsize,),
            "typestr": "|u1",
            "data": (int(ptr), False),
            "version": 3,
        }

    raw = torch.as_tensor(_Holder(), device="cuda")
    return raw.view(dtype).view(shape)


# ---------------------------------------------------------------------------
# FFT
# ---------------------------------------------------------------------------

FFT_FORWARD = _lib.AZ_FFT_FORWARD
FFT_BACKWARD = _lib.AZ_FFT_BACKWARD


class FFT:
    """FFT<Dim> bound to (u_hat, u) (fft.hpp:37-121): forward() u_hat <- r2c(u),
    backward() u <- c2r(u_hat), both unnormalised, batched over axis 0."""

    def __init__(self, u_hat, u, direction=FFT_FORWARD | FFT_BACKWARD, transform=None):
        dim = u.dim() - 1
        if dim < 1 or dim > 3:
            raise ValueError("u must have 2 to 4 axes (n_vars + 1..3 spatial)")
        transform = tuple(transform) if transform is not None else (True,) * dim
        if len(transform) != dim:
            raise ValueError("one transform flag per axis")
        nt = sum(bool(t) for t in transform)
        if nt == 0 or tuple(bool(t) for t in transform) != (False,) * (dim - nt) + (True,) * nt:
            raise ValueError("only trailing axes can be transformed")
        prec = precision_code(u.dtype)
        if u_hat.dtype != _CDT[prec]:
            raise ValueError("u_hat and u precisions differ")
        exp_hat = tuple(u.shape[:-1]) + (u.shape[-1] // 2 + 1,)
        _check_tensor(u, "u", _RDT[prec], tuple(u.shape))
        _check_tensor(u_hat, "u_hat", _CDT[prec], exp_hat)
        self.u_hat, self.u_ = u_hat, u
        self.direction = int(direction)
        shape = (ct.c_longlong * 3)(*(list(u.shape[1:]) + [0] * (3 - dim)))
        desc = _lib.az_fft_desc(dim, u.shape[0], shape, nt, prec, self.direction)
        h = ct.c_void_p()
        check(lib.az_fft_create(ct.byref(desc), u_hat.data_ptr(), u.data_ptr(), ct.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.az_fft_destroy(h)
            self._h = None

    def is_forward(self):
        return bool(self.direction & FFT_FORWARD)

    def is_backward(self):
        return bool(self.direction & FFT_BACKWARD)

    def get_work_area_size(self):
        return lib.az_fft_work_area_size(self._h)

    def set_work_area(self, work: torch.Tensor):
        """FFT::set_work_area (fft.hpp:84): a device tensor of at least
        get_work_area_size() bytes, used instead of an allocation of the
        FFT's own; kept alive by the FFT."""
        if not isinstance(work, torch.Tensor) or not work.is_cuda or not work.is_contiguous():
            raise ValueError("work must be a contiguous CUDA tensor")
        if work.numel() * work.element_size() < self.get_work_area_size():
            raise ValueError("work area too small")
        check(lib.az_fft_set_work_area(self._h, work.data_ptr()))
        self._work = work

    def forward(self, stream=None):
        check(lib.az_fft_forward(self._h, _stream_ptr(stream)))

    def backward(self, stream=None):
        check(lib.az_fft_backward(self._h, _stream_ptr(stream)))


def make_fft(u_hat, u, direction=FFT_FORWARD | FFT_BACKWARD, *transform):
    """make_fft<Dim>(u_hat, u, direction, transform_x, ...) (fft_factory.hpp:27-60)."""
    return FFT(u_hat, u, direction, transform if transform else None)


def leray(u_hat, stream=None):
    """leray(u_hat) in place (src/azeban/operations/leray.cpp:28-116); accepts
    [dim, N, (N,) N/2+1] or a batch of them."""
    dim = None
    nd = u_hat.dim()
    for d in (2, 3):
        if nd in (d + 1, d + 2) and u_hat.shape[-d - 1] == d:
            dim = d
            break
    if dim is None:
        raise ValueError("u_hat must be [(batch,) dim, N, (N,) N/2+1] with dim in {2, 3}")
    batch = 1 if nd == dim + 1 else u_hat.shape[0]
    prec = precision_code(u_hat.dtype)
    if not u_hat.is_cuda or not u_hat.is_contiguous():
        raise ValueError("u_hat must be a contiguous CUDA tensor")
    check(lib.az_leray(dim, u_hat.shape[-2], prec, u_hat.data_ptr(), batch, _stream_ptr(stream)))
    return u_hat
