"""CPU oracle for the spectral-viscosity incompressible Euler path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: the parity tests, the
smoke check and the CPU-baseline leg of ``bench.py`` import it.  The product
(``azeban_b200`` and its CUDA library) never imports, links or calls it.

It restates, in FP64 numpy, the reference's CPU path for one right-hand side
and its SSP-RK3 stepper.  Every function cites the reference file:line it
follows (paths relative to the reference project root).

Conventions kept from the reference:
  * periodic domain [0,1)^d, wavenumber of index n is k = 2*pi*n
    (include/azeban/equations/incompressible_euler.hpp:247-249, :310-313);
  * spectral arrays are UNNORMALISED forward DFTs (carry N^d), inverse
    transforms are unnormalised too (include/azeban/operations/fft.hpp:80-107);
  * layout [n_vars, N, (N,) N/2+1], r2c along the last axis
    (include/azeban/grid.hpp:89-99).

The transforms use ``scipy.fft`` (pocketfft) with unnormalised conventions;
the reference calls FFTW 3.3.9 / cuFFT (src/azeban/operations/fftwfft.cpp:257-269,
src/azeban/cuda/operations/cufft.cpp:133-149), whose sources are not part of
the reference.  Both c2r implementations ignore the imaginary part of the DC
and Nyquist bins of the real axis; pocketfft does the same.
"""

from __future__ import annotations

import math
import os

import numpy as np

try:  # scipy.fft gives multi-threaded pocketfft; numpy.fft is the fallback.
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

PI = math.pi

_WORKERS = int(os.environ.get("AZ_ORACLE_WORKERS", "1"))


def set_workers(n: int) -> None:
    """Number of threads the oracle's transforms may use (CPU baseline)."""
    global _WORKERS
    _WORKERS = max(1, int(n))


def _irfftn(x, s, axes):
    if _sfft is not None:
        return _sfft.irfftn(x, s=s, axes=axes, norm="forward", workers=_WORKERS)
    return np.fft.irfftn(x, s=s, axes=axes, norm="forward")


def _rfftn(x, axes):
    if _sfft is not None:
        return _sfft.rfftn(x, axes=axes, norm="backward", workers=_WORKERS)
    return np.fft.rfftn(x, axes=axes, norm="backward")


# Single-axis and partial transforms of the slab-wise right-hand side, with
# the same unnormalised conventions (inverse unscaled, forward unscaled).
def _ifftn(x, axes):
    if _sfft is not None:
        return _sfft.ifftn(x, axes=axes, norm="forward", workers=_WORKERS)
    return np.fft.ifftn(x, axes=axes, norm="forward")


def _irfft(x, n, axis):
    if _sfft is not None:
        return _sfft.irfft(x, n=n, axis=axis, norm="forward", workers=_WORKERS)
    return np.fft.irfft(x, n=n, axis=axis, norm="forward")


def _rfft(x, axis):
    if _sfft is not None:
        return _sfft.rfft(x, axis=axis, norm="backward", workers=_WORKERS)
    return np.fft.rfft(x, axis=axis, norm="backward")


def _fft(x, axis):
    if _sfft is not None:
        return _sfft.fft(x, axis=axis, norm="backward", workers=_WORKERS)
    return np.fft.fft(x, axis=axis, norm="backward")


# --------------------------------------------------------------------------
# Grid (include/azeban/grid.hpp:30-165, include/azeban/grid_factory.hpp:28-92)
# --------------------------------------------------------------------------

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
    """Sizes and shapes of one solve (include/azeban/grid.hpp:30-53)."""

    def __init__(self, dim: int, N_phys: int, N_phys_pad: int | None = None):
        self.dim = int(dim)
        self.N_phys = int(N_phys)
        self.N_phys_pad = int(3 * N_phys // 2 if N_phys_pad is None else N_phys_pad)
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


def make_grid(config: dict, dim: int) -> Grid:
    """Grid from the JSON "grid" object (include/azeban/grid_factory.hpp:28-92)."""
    if ("N_phys" in config) == ("N_fourier" in config):
        raise ValueError('Grid config must contain either "N_phys" or "N_fourier", but not both')
    if "N_phys" in config:
        n = int(config["N_phys"])
    else:
        n = 2 * (int(config["N_fourier"]) - 1)
    g = Grid(dim, n)
    has_pp, has_fp = "N_phys_pad" in config, "N_fourier_pad" in config
    if has_pp and has_fp:
        raise ValueError('Grid config may contain "N_phys_pad" or "N_fourier_pad", but not both')
    if has_pp or has_fp:
        key = "N_phys_pad" if has_pp else "N_fourier_pad"
        val = config[key]
        if isinstance(val, str):
            g.N_phys_pad = next_good_size(-(-3 * g.N_phys // 2))
        elif has_pp:
            g.N_phys_pad = int(val)
        else:
            g.N_phys_pad = 2 * (int(val) - 1)
        g.N_fourier_pad = g.N_phys_pad // 2 + 1
    return g


# --------------------------------------------------------------------------
# Spectral viscosity (include/azeban/equations/spectral_viscosity.hpp:27-128,
# include/azeban/equations/spectral_viscosity_factory.hpp:29-89)
# --------------------------------------------------------------------------

class SmoothCutoff1D:
    """nu(k) = -eps k^{2s} (1 - exp(-(|k|/k0)^18)) (spectral_viscosity.hpp:27-38, :56-77)."""

    kind = "smooth_cutoff"

    def __init__(self, eps, s, k0):
        self.eps, self.s, self.k0 = float(eps), float(s), float(k0)

    def Qk(self, k):
        k1 = np.abs(k) / self.k0
        k2 = k1 * k1
        k4 = k2 * k2
        k8 = k4 * k4
        k16 = k8 * k8
        k18 = k16 * k2
        return 1.0 - np.exp(-k18)

    def eval(self, k):
        return -self.eps * np.power(k, 2 * self.s) * self.Qk(k)


class Step1D:
    """nu(k) = -eps k^{2s} [|k| > k0] (spectral_viscosity.hpp:40-54)."""

    kind = "step"

    def __init__(self, eps, s, k0):
        self.eps, self.s, self.k0 = float(eps), float(s), float(k0)

    def Qk(self, k):
        return np.where(np.abs(k) > self.k0, 1.0, 0.0)

    def eval(self, k):
        return -self.eps * np.power(k, 2 * self.s) * self.Qk(k)


class Quadratic:
    """nu(k) = -eps max(0, (k/2pi)^2 - N) (spectral_viscosity.hpp:103-123)."""

    kind = "quadratic"

    def __init__(self, eps, N):
        self.eps, self.N = float(eps), int(N)

    def Qk(self, k):
        sqrtN = math.sqrt(self.N)
        absk = np.abs(k / (2 * PI))
        with np.errstate(divide="ignore", invalid="ignore"):
            q = 1.0 - self.N / (absk * absk)
        return np.where(absk >= sqrtN, q, 0.0)

    def eval(self, k):
        knorm = k / (2 * PI)
        return -self.eps * np.maximum(0.0, knorm * knorm - self.N)


class NoViscosity:
    """nu = 0 (spectral_viscosity.hpp:125-128)."""

    kind = "none"
    eps = 0.0

    def Qk(self, k):
        return np.zeros_like(np.asarray(k, dtype=np.float64))

    def eval(self, k):
        return np.zeros_like(np.asarray(k, dtype=np.float64))


def _s_theta_m0(cfg):
    s = float(cfg.get("s", 1.0))
    theta = float(cfg.get("theta", (2 * s - 1) / (2 * s)))
    m0 = float(cfg.get("m0", 2 * PI))
    return s, theta, m0


def make_viscosity(cfg: dict, grid: Grid):
    """Viscosity from the JSON "visc" object (src/azeban/equations/equation_factory.cpp:25-58,
    spectral_viscosity_factory.hpp:29-89)."""
    typ = cfg.get("type")
    if typ in ("Smooth Cutoff", "Step"):
        if "eps" not in cfg:
            raise ValueError('Smooth Cutoff Viscosity expects "eps" parameter in config')
        s, theta, m0 = _s_theta_m0(cfg)
        eps = float(cfg["eps"])
        epsN = eps / math.pow(float(grid.N_phys), 2 * s - 1)
        mN = m0 * math.pow(float(grid.N_phys), theta)
        return (SmoothCutoff1D if typ == "Smooth Cutoff" else Step1D)(epsN, s, mN)
    if typ == "Quadratic":
        if "eps" not in cfg:
            raise ValueError('Quadratic Viscosity expects "eps" parameter in config')
        return Quadratic(float(cfg["eps"]) / grid.N_phys, grid.N_phys)
    if typ == "None":
        return NoViscosity()
    raise ValueError(f"Unknown viscosity type: {typ}")


# --------------------------------------------------------------------------
# Zero padding (include/azeban/operations/copy_to_padded_functions.hpp:9-63,
# src/azeban/operations/copy_to_padded.cpp:301-328)
# --------------------------------------------------------------------------

def pad_index_map_full(src_n: int, dst_n: int) -> np.ndarray:
    """For each dst index along a full axis: the src index, or -1 for a zero
    (pad_full_dim, copy_to_padded_functions.hpp:36-51).  The Nyquist src index
    src_n/2 stays on the positive side."""
    out = np.full(dst_n, -1, dtype=np.int64)
    for i in range(dst_n):
        if i < src_n // 2 + 1:
            out[i] = i
        elif i < src_n // 2 + 1 + dst_n - src_n:
            out[i] = -1
        else:
            out[i] = i + src_n - dst_n
    return out


def pad_index_map_compact(src_n: int, dst_n: int) -> np.ndarray:
    """Compact (r2c) axis: dst index i copies src index i if i < src_n
    (pad_compact_dim, copy_to_padded_functions.hpp:22-34)."""
    out = np.full(dst_n, -1, dtype=np.int64)
    out[: min(src_n, dst_n)] = np.arange(min(src_n, dst_n))
    return out


def copy_to_padded(src: np.ndarray, dst_shape) -> np.ndarray:
    """Zero-pad one spectral component; all axes full except the last, which
    is compact (copy_to_padded.cpp:301-328 for 3-D, :294-299 for 2-D)."""
    d = src.ndim
    dst = np.zeros(dst_shape, dtype=src.dtype)
    maps = []
    for ax in range(d):
        if ax == d - 1:
            maps.append(pad_index_map_compact(src.shape[ax], dst_shape[ax]))
        else:
            maps.append(pad_index_map_full(src.shape[ax], dst_shape[ax]))
    sel_dst = [np.nonzero(m >= 0)[0] for m in maps]
    sel_src = [m[m >= 0] for m in maps]
    dst[np.ix_(*sel_dst)] = src[np.ix_(*sel_src)]
    return dst


def retained_index_map(n: int, m: int) -> np.ndarray:
    """Index into the padded axis read for retained index i of the unpadded
    axis: i >= n/2+1 ? m - n + i : i (incompressible_euler.hpp:294-299)."""
    i = np.arange(n)
    return np.where(i >= n // 2 + 1, m - n + i, i)


def signed_index(n: int) -> np.ndarray:
    """i >= n/2+1 ? i - n : i (incompressible_euler.hpp:302-309)."""
    i = np.arange(n)
    return np.where(i >= n // 2 + 1, i - n, i)


# --------------------------------------------------------------------------
# Transforms (FFT<Dim>::forward/backward, include/azeban/operations/fft.hpp:80-107)
# --------------------------------------------------------------------------

def fft_backward(u_hat: np.ndarray, n: int, naxes: int | None = None) -> np.ndarray:
    """Unnormalised inverse real transform over the trailing ``naxes`` axes;
    axis 0 is the variable index."""
    d = u_hat.ndim - 1 if naxes is None else naxes
    axes = tuple(range(u_hat.ndim - d, u_hat.ndim))
    return _irfftn(u_hat, s=(n,) * d, axes=axes)


def fft_forward(u: np.ndarray, naxes: int | None = None) -> np.ndarray:
    """Unnormalised forward real transform over the trailing ``naxes`` axes."""
    d = u.ndim - 1 if naxes is None else naxes
    axes = tuple(range(u.ndim - d, u.ndim))
    return _rfftn(u, axes=axes)


def max_norm(u: np.ndarray) -> float:
    """max_i |u_i| over the flat array (include/azeban/operations/norm.hpp:72-83)."""
    return float(np.max(np.abs(u)))


# --------------------------------------------------------------------------
# Incompressible Euler right-hand side
# (include/azeban/equations/incompressible_euler.hpp:39-387,
#  include/azeban/equations/incompressible_euler_functions.hpp:26-112)
# --------------------------------------------------------------------------

class IncompressibleEuler:
    """Equation<Dim> for the spectral-viscosity incompressible Euler RHS
    with no forcing (include/azeban/forcing/no_forcing.hpp:28-44)."""

    def __init__(self, grid: Grid, visc, slabs: bool = False):
        self.grid = grid
        self.visc_ = visc
        self.u_max_ = 0.0
        # 3-D: evaluate dudt() with the bounded-memory dudt_slabs()
        self.slabs = bool(slabs) and grid.dim == 3
        d = grid.dim
        N, M = grid.N_phys, grid.N_phys_pad
        kk = [2 * PI * signed_index(N).astype(np.float64)] * (d - 1) + [
            2 * PI * np.arange(N // 2 + 1, dtype=np.float64)]
        grids = np.meshgrid(*kk, indexing="ij")
        # k1*k1 + k2*k2 (+ k3*k3) in that order (incompressible_euler.hpp:249, :313)
        absk2 = grids[0] * grids[0]
        for g in grids[1:]:
            absk2 = absk2 + g * g
        self._k = grids
        self._absk2 = absk2
        self._nu = visc.eval(np.sqrt(absk2))
        self._ret = [retained_index_map(N, M)] * (d - 1) + [np.arange(N // 2 + 1)]

    def n_vars(self) -> int:
        return self.grid.dim

    def visc(self) -> float:
        return float(getattr(self.visc_, "eps", 0.0))

    def dt(self, C: float) -> float:
        """C / (N_phys * u_max_) (incompressible_euler.hpp:122-124), in IEEE
        double arithmetic as the reference computes it: +inf for a zero field
        (SSP_RK3::integrate then takes max_dt, ssp_rk3.hpp:55)."""
        with np.errstate(divide="ignore"):
            return float(np.float64(C) / (np.float64(self.grid.N_phys) * np.float64(self.u_max_)))

    # -- pieces of dudt, exposed so tests can check each stage -------------
    def pad(self, u_hat):
        """copy_to_padded per component (incompressible_euler.hpp:112-114)."""
        shp = self.grid.shape_fourier_pad(self.n_vars())
        return np.stack([copy_to_padded(u_hat[c], shp[1:]) for c in range(u_hat.shape[0])])

    def physical(self, u_hat):
        """Padded inverse transform, N^d-scaled (incompressible_euler.hpp:115)."""
        return fft_backward(self.pad(u_hat), self.grid.N_phys_pad)

    def norm(self) -> float:
        """1 / (N^{d/2} M^{d/2}) as computeB forms it: the integer powers of
        the square roots by repeated multiplication (incompressible_euler.hpp:171-173)."""
        d = self.grid.dim
        sn, sm = math.sqrt(self.grid.N_phys), math.sqrt(self.grid.N_phys_pad)
        pn, pm = sn, sm
        for _ in range(d - 1):
            pn, pm = sn * pn, sm * pm
        return 1.0 / (pn * pm)

    def compute_B(self, u):
        """Scale by 1/(N^{d/2} M^{d/2}) then the symmetric product in the
        reference's component order (incompressible_euler.hpp:168-213,
        incompressible_euler_functions.hpp:26-45)."""
        d = self.grid.dim
        norm = self.norm()
        v = [norm * u[c] for c in range(d)]
        if d == 2:
            return np.stack([v[0] * v[0], v[0] * v[1], v[1] * v[1]])
        return np.stack([v[0] * v[0], v[1] * v[0], v[1] * v[1],
                         v[2] * v[0], v[2] * v[1], v[2] * v[2]])

    def compute_dudt(self, B_hat, u_hat):
        """L = (I - k k^T/|k|^2)(i k . B_hat), dudt = -L + nu(|k|) u_hat,
        zero at |k| = 0 (incompressible_euler.hpp:230-347,
        incompressible_euler_functions.hpp:47-112)."""
        with np.errstate(divide="ignore", invalid="ignore"):
            return self._compute_dudt(B_hat, u_hat)

    def _compute_dudt(self, B_hat, u_hat):
        d = self.grid.dim
        if d == 2:
            Bs = B_hat[np.ix_(range(3), self._ret[0], self._ret[1])]
            k1, k2 = self._k
            return _dudt_modes_2d(Bs, u_hat, k1, k2, self._absk2, self._nu)
        Bs = B_hat[np.ix_(range(6), self._ret[0], self._ret[1], self._ret[2])]
        k1, k2, k3 = self._k
        return _dudt_modes_3d(Bs, u_hat, k1, k2, k3, self._absk2, self._nu)

    def dudt_modes(self, signed_idx, B_modes, u_modes):
        """The per-mode right-hand side for a list of modes (see dudt_modes)."""
        return dudt_modes(self.visc_, signed_idx, B_modes, u_modes)

    def dudt_single(self, u_hat):
        """The same right-hand side with the padded transforms and the
        products in single precision (pocketfft float32 and float32
        products; the per-mode projection and viscosity stay FP64).  Not the
        reference: a measure of how far any FP32 evaluation of a given
        field's right-hand side lands from FP64, which the FP32-bulk parity
        tests use as the conditioning of that field (fields whose nonlinear
        terms cancel strongly carry FP32 errors above 1e-5 whatever the
        FFT).  Leaves u_max_ unchanged."""
        if self.grid.dim == 3:
            keep = self.u_max_
            out = self.dudt_slabs(u_hat, single=True)
            self.u_max_ = keep
            return out
        d = self.grid.dim
        M = self.grid.N_phys_pad
        up = self.pad(u_hat).astype(np.complex64)
        u = _irfftn(up, s=(M,) * d, axes=tuple(range(1, d + 1)))
        norm = np.float32(self.norm())
        v = [norm * u[c] for c in range(d)]
        B = np.stack([v[0] * v[0], v[0] * v[1], v[1] * v[1]])
        B_hat = _rfftn(B, axes=tuple(range(1, d + 1)))
        return self.compute_dudt(B_hat.astype(np.complex128), u_hat)

    def dudt_slabs(self, u_hat, xchunk=16, zchunk=16, colchunk=1 << 16, single=False):
        """The same right-hand side as dudt() for 3-D, with bounded memory.

        The padded transforms are split by axis: inverse along x and y per
        chunk of z wavenumbers, then per chunk of x planes the c2r along z,
        max |u|, B = u (x) u and the r2c along z and forward transform along
        y (kept at the retained rows), then the forward transform along x and
        the per-mode L and viscosity per chunk of (y, z) columns.  The padded
        physical field never exists whole: the largest array is the
        y-transformed product spectrum [6][M][N][N/2+1].  Used for sizes whose
        padded arrays do not fit in host memory at once (N = 512, M = 768).
        The transform order is the one pocketfft's irfftn / rfftn use, so the
        result equals dudt() up to rounding.  Sets u_max_."""
        if self.grid.dim != 3:
            raise ValueError("dudt_slabs is for 3-D solves")
        N, M = self.grid.N_phys, self.grid.N_phys_pad
        Nh, Mh = N // 2 + 1, M // 2 + 1
        pmap = pad_index_map_full(N, M)
        dsel, ssel = np.nonzero(pmap >= 0)[0], pmap[pmap >= 0]
        ret = retained_index_map(N, M)
        cdt = np.complex64 if single else np.complex128
        norm = np.float32(self.norm()) if single else self.norm()
        xs = [np.arange(a, min(a + xchunk, M)) for a in range(0, M, xchunk)]
        # 1. inverse along x and y of the padded spectrum, per z-wavenumber chunk
        T = [np.empty((3, len(xc), M, Nh), dtype=cdt) for xc in xs]
        for k0 in range(0, Nh, zchunk):
            ks = slice(k0, min(k0 + zchunk, Nh))
            src = u_hat[:, :, :, ks].astype(cdt)
            pad = np.zeros((3, M, M, src.shape[-1]), dtype=cdt)
            pad[np.ix_(range(3), dsel, dsel, range(src.shape[-1]))] = src[np.ix_(range(3), ssel, ssel,
                                                                                 range(src.shape[-1]))]
            t = _ifftn(pad, axes=(1, 2))
            for i, xc in enumerate(xs):
                T[i][:, :, :, ks] = t[:, xc]
            del pad, t
        # 2. per x chunk: c2r along z, max |u|, products, r2c along z, forward y
        W = np.empty((6, M, N, Nh), dtype=cdt)
        umax = 0.0
        for i, xc in enumerate(xs):
            ext = np.zeros((3, len(xc), M, Mh), dtype=cdt)
            ext[..., :Nh] = T[i]
            T[i] = None
            u = _irfft(ext, M, axis=3)
            del ext
            umax = max(umax, float(np.max(np.abs(u))))
            v = [norm * u[c] for c in range(3)]
            del u
            B = np.stack([v[0] * v[0], v[1] * v[0], v[1] * v[1], v[2] * v[0], v[2] * v[1], v[2] * v[2]])
            del v
            Bz = _rfft(B, axis=3)[..., :Nh]
            del B
            W[:, xc] = _fft(Bz, axis=2)[:, :, ret, :]
            del Bz
        self.u_max_ = umax / float(M ** 3)
        # 3. forward along x per column chunk, then the per-mode right-hand side
        W = W.reshape(6, M, N * Nh)
        out = np.empty_like(u_hat)
        out_f = out.reshape(3, N, N * Nh)
        u_f = u_hat.reshape(3, N, N * Nh)
        k1 = (2 * PI * signed_index(N).astype(np.float64))[:, None]
        for c0 in range(0, N * Nh, colchunk):
            cs = slice(c0, min(c0 + colchunk, N * Nh))
            Bx = _fft(W[:, :, cs], axis=1)[:, ret, :].astype(np.complex128)
            col = np.arange(cs.start, cs.stop)
            k2 = (2 * PI * signed_index(N).astype(np.float64)[col // Nh])[None, :]
            k3 = (2 * PI * (col % Nh).astype(np.float64))[None, :]
            absk2 = k1 * k1 + k2 * k2 + k3 * k3
            nu = self.visc_.eval(np.sqrt(absk2))
            out_f[:, :, cs] = _dudt_modes_3d(Bx, u_f[:, :, cs], k1, k2, k3, absk2, nu)
        return out

    def dudt(self, u_hat, t=0.0, dt=0.0, C=0.0):
        """One right-hand side (incompressible_euler.hpp:103-120).  Returns a
        new array; sets u_max_ as the reference does."""
        if self.slabs:
            return self.dudt_slabs(u_hat)
        d = self.grid.dim
        u = self.physical(u_hat)
        self.u_max_ = max_norm(u) / float(self.grid.N_phys_pad ** d)
        B = self.compute_B(u)
        B_hat = fft_forward(B)
        return self.compute_dudt(B_hat, u_hat)


def dudt_modes(visc, signed_idx, B_modes, u_modes):
    """The per-mode right-hand side for a list of modes: signed indices
    [dim, n] (the last one the compact index), B_hat at those modes
    [d(d+1)/2, n], u_hat [dim, n] (incompressible_euler.hpp:230-347)."""
    d = len(signed_idx)
    ks = [2 * PI * np.asarray(signed_idx[c], dtype=np.float64) for c in range(d)]
    absk2 = ks[0] * ks[0]
    for k in ks[1:]:
        absk2 = absk2 + k * k
    nu = visc.eval(np.sqrt(absk2))
    if d == 2:
        return _dudt_modes_2d(B_modes, u_modes, ks[0], ks[1], absk2, nu)
    return _dudt_modes_3d(B_modes, u_modes, ks[0], ks[1], ks[2], absk2, nu)


def _dudt_modes_2d(Bs, u_hat, k1, k2, absk2, nu):
    """Per retained mode in 2-D: b = i k.B_hat, L = (I - k k^T/|k|^2) b,
    dudt = -L + nu u_hat, zero at |k| = 0 (incompressible_euler_functions.hpp:47-71,
    incompressible_euler.hpp:230-281).  Bs: (B11, B12, B22) at the modes."""
    B11, B12, B22 = Bs[0], Bs[1], Bs[2]
    b1 = 1j * k1 * B11 + 1j * k2 * B12
    b2 = 1j * k1 * B12 + 1j * k2 * B22
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / absk2
        k11, k12, k22 = k1 * k1 * inv, k1 * k2 * inv, k2 * k2 * inv
        L = [(1.0 - k11) * b1 + (0.0 - k12) * b2,
             (0.0 - k12) * b1 + (1.0 - k22) * b2]
        zero = absk2 == 0
        out = np.empty(u_hat.shape, dtype=np.complex128)
        for c in range(2):
            out[c] = np.where(zero, 0.0, -L[c] + nu * u_hat[c])
    return out


def _dudt_modes_3d(Bs, u_hat, k1, k2, k3, absk2, nu):
    """Per retained mode: b = i k.B_hat, L = (I - k k^T/|k|^2) b, dudt = -L + nu u_hat,
    zero at |k| = 0 (incompressible_euler_functions.hpp:73-112, incompressible_euler.hpp:283-347).
    Bs holds the six products at the retained modes in the reference's order
    (B11, B21, B22, B31, B32, B33); the wavenumber arrays broadcast against them."""
    B11, B21, B22, B31, B32, B33 = (Bs[c] for c in range(6))
    b1 = 1j * k1 * B11 + 1j * k2 * B21 + 1j * k3 * B31
    b2 = 1j * k1 * B21 + 1j * k2 * B22 + 1j * k3 * B32
    b3 = 1j * k1 * B31 + 1j * k2 * B32 + 1j * k3 * B33
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / absk2
        k11, k12, k13 = k1 * k1 * inv, k1 * k2 * inv, k1 * k3 * inv
        k22, k23, k33 = k2 * k2 * inv, k2 * k3 * inv, k3 * k3 * inv
        L = [(1.0 - k11) * b1 + (0.0 - k12) * b2 + (0.0 - k13) * b3,
             (0.0 - k12) * b1 + (1.0 - k22) * b2 + (0.0 - k23) * b3,
             (0.0 - k13) * b1 + (0.0 - k23) * b2 + (1.0 - k33) * b3]
        zero = absk2 == 0
        out = np.empty(u_hat.shape, dtype=np.complex128)
        for c in range(3):
            out[c] = np.where(zero, 0.0, -L[c] + nu * u_hat[c])
    return out


def axpby(a, x, b, y):
    """y <- a x + b y (include/azeban/operations/axpby.hpp:28-56)."""
    y *= b
    y += a * x
    return y


class SSP_RK3:
    """Shu-Osher SSP-RK3 (include/azeban/evolution/ssp_rk3.hpp:48-64)."""

    def __init__(self, equation: IncompressibleEuler):
        self.equation_ = equation

    def integrate(self, t, max_dt, C, u):
        eq = self.equation_
        u1 = eq.dudt(u, t, max_dt, C)
        dt = min(eq.dt(C), max_dt)
        axpby(1.0, u, dt, u1)
        u2 = eq.dudt(u1, t, dt, C)
        axpby(1.0, u1, dt, u2)
        axpby(3.0 / 4, u, 1.0 / 4, u2)
        u1b = eq.dudt(u2, t, dt, C)
        axpby(1.0, u2, dt, u1b)
        axpby(2.0 / 3, u1b, 1.0 / 3, u)
        return dt


class Simulation:
    """Owns the state and loops integrate (src/azeban/simulation.cpp:89-102)."""

    def __init__(self, grid: Grid, C: float, timestepper: SSP_RK3, u_hat: np.ndarray):
        self.grid = grid
        self.C_ = float(C)
        self.timestepper_ = timestepper
        self.u_ = np.array(u_hat, dtype=np.complex128, copy=True)
        self.time_ = 0.0
        self.dts = []

    def simulate_until(self, t, max_steps=None):
        eq = self.timestepper_.equation_
        steps = 0
        while self.time_ < t:
            eps = eq.visc()
            cap = self.C_ * 2.0 / (eps * (PI * self.grid.N_phys) ** 2) if eps != 0 else math.inf
            max_dt = min(t - self.time_, cap)
            dt = self.timestepper_.integrate(t, max_dt, self.C_, self.u_)
            self.dts.append(dt)
            self.time_ += dt
            steps += 1
            if max_steps is not None and steps >= max_steps:
                return steps
        self.time_ = t
        return steps


# --------------------------------------------------------------------------
# Initial data (src/azeban/init/taylor_green.cpp:29-76,146-206,
# src/azeban/init/double_shear_layer.cpp:25-66, src/azeban/operations/leray.cpp:28-116)
# --------------------------------------------------------------------------

def leray(u_hat: np.ndarray) -> np.ndarray:
    """Divergence-free projection in place (src/azeban/operations/leray.cpp:28-116)."""
    d = u_hat.ndim - 1
    N = u_hat.shape[1]
    kk = [2 * PI * signed_index(N).astype(np.float64)] * (d - 1) + [
        2 * PI * np.arange(u_hat.shape[-1], dtype=np.float64)]
    ks = np.meshgrid(*kk, indexing="ij")
    absk2 = ks[0] * ks[0]
    for g in ks[1:]:
        absk2 = absk2 + g * g
    zero = absk2 == 0
    with np.errstate(divide="ignore", invalid="ignore"):
        old = [u_hat[c].copy() for c in range(d)]
        for a in range(d):
            acc = np.zeros_like(old[0])
            for b in range(d):
                coef = (1.0 if a == b else 0.0) - (ks[a] * ks[b]) / absk2
                acc = acc + coef * old[b]
            u_hat[a] = np.where(zero, 0.0, acc)
    return u_hat


def _coords(N, d):
    x = 2 * PI / N * np.arange(N, dtype=np.float64)
    return np.meshgrid(*([x] * d), indexing="ij")


def taylor_green_reference(dim: int, N: int, deltas=None) -> np.ndarray:
    """azeban's own Taylor-Green field (taylor_green.cpp:29-46 in 2-D,
    :146-184 in 3-D), physical space, with its perturbation modes of
    amplitudes deltas (8 in 2-D: d * 4 + {ss, sc, cs, cc} of (2x, 2y); 24 in
    3-D: d * 8 + the eight sin/cos products of (2x, 2y, 2z)), or none."""
    if dim == 2:
        x, y = _coords(N, 2)
        u = [1.0 * np.cos(x) * np.sin(y), -1.0 * np.sin(x) * np.cos(y)]
        if deltas is not None:
            # left to right, as the reference multiplies: delta * f(2x) * g(2y)
            fs = [(np.sin, np.sin), (np.sin, np.cos), (np.cos, np.sin), (np.cos, np.cos)]
            for d in range(2):
                for t, (f, g) in enumerate(fs):
                    u[d] = u[d] + deltas[t + 4 * d] * f(2 * x) * g(2 * y)
        return np.stack(u)
    x, y, z = _coords(N, 3)
    u = [1.0 * np.cos(x) * np.sin(y) * np.sin(z), -1.0 * np.sin(x) * np.cos(y) * np.sin(z),
         0.0 * np.sin(x) * np.sin(y) * np.cos(z)]
    if deltas is not None:
        fx = [np.sin(2 * x), np.cos(2 * x)]
        fy = [np.sin(2 * y), np.cos(2 * y)]
        fz = [np.sin(2 * z), np.cos(2 * z)]
        for d in range(3):
            for t in range(8):
                # delta * f(2x) * g(2y) * h(2z), left to right; t = 4 a + 2 b + c
                a, b, c = t >> 2, (t >> 1) & 1, t & 1
                u[d] = u[d] + deltas[t + 8 * d] * fx[a] * fy[b] * fz[c]
    return np.stack(u)


def taylor_green_workload(dim: int, N: int) -> np.ndarray:
    """The Taylor-Green field of the benchmark workloads, sampled at
    x_i = 2 pi i / N: (sin x cos y, -cos x sin y) in 2-D and
    (sin x cos y cos z, -cos x sin y cos z, 0) in 3-D."""
    if dim == 2:
        x, y = _coords(N, 2)
        return np.stack([np.sin(x) * np.cos(y), -np.cos(x) * np.sin(y)])
    x, y, z = _coords(N, 3)
    return np.stack([np.sin(x) * np.cos(y) * np.cos(z),
                     -np.cos(x) * np.sin(y) * np.cos(z),
                     0.0 * x])


def double_shear_layer(N: int, rho: float, delta: float, phase: float = 0.0) -> np.ndarray:
    """azeban's DoubleShearLayer (double_shear_layer.cpp:25-43) with an added
    phase phi in v = delta sin(2 pi x + phi); phi = 0 is the reference field."""
    i = np.arange(N, dtype=np.float64)
    x = (i / N)[:, None] * np.ones((1, N))
    y = np.ones((N, 1)) * (i / N)[None, :]
    if rho == 0:
        u = np.where(np.abs(y - 0.5) < 0.25, 1.0, -1.0)
    else:
        u = np.where(y < 0.5, np.tanh(2 * PI * (y - 0.25) / rho), np.tanh(2 * PI * (0.75 - y) / rho))
    v = delta * np.sin(2 * PI * x + phase)
    return np.stack([u, v])


def initialize(u_phys: np.ndarray) -> np.ndarray:
    """Forward transform then Leray projection (include/azeban/init/initializer.hpp:68-75)."""
    return leray(fft_forward(u_phys))


# --------------------------------------------------------------------------
# L2 helper (test/azeban/utils.hpp:61-111)
# --------------------------------------------------------------------------

def L2(u_hat: np.ndarray, u_ref_hat: np.ndarray) -> float:
    """Physical-space L2 difference via Parseval after padding u_hat to the
    reference grid and rescaling (test/azeban/utils.hpp:61-111)."""
    d = u_hat.ndim - 1
    N, Nr = u_hat.shape[1], u_ref_hat.shape[1]
    pad = np.stack([copy_to_padded(u_hat[c], u_ref_hat.shape[1:]) for c in range(u_hat.shape[0])])
    pad = pad * (float(Nr) / N) ** d
    diff2 = np.abs(pad - u_ref_hat) ** 2
    err = diff2[..., 0].sum() + 2 * diff2[..., 1:].sum()
    return math.sqrt(err) / Nr ** d


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b||_2 / ||b||_2 over the flat arrays."""
    nb = np.linalg.norm(np.ravel(b))
    return float(np.linalg.norm(np.ravel(a - b)) / (nb if nb > 0 else 1.0))


# --------------------------------------------------------------------------
# Diagnostics (Parseval on the half spectrum; exact-rounded sums)
# --------------------------------------------------------------------------

def energy_enstrophy(u_hat: np.ndarray):
    """1/2 <|u|^2> and 1/2 <|curl u|^2> of one unnormalised r2c spectrum
    [d, N, (N,) N/2+1], summed with math.fsum (correctly rounded)."""
    d = u_hat.ndim - 1
    N = u_hat.shape[1]
    kk = [2 * PI * signed_index(N).astype(np.float64)] * (d - 1) + [
        2 * PI * np.arange(u_hat.shape[-1], dtype=np.float64)]
    ks = np.meshgrid(*kk, indexing="ij")
    k2 = sum(k * k for k in ks)
    last = np.arange(u_hat.shape[-1])
    w = np.where((last == 0) | (2 * last == N), 1.0, 2.0)
    a2 = sum(np.abs(u_hat[c]) ** 2 for c in range(d))
    scale = 1.0 / float(N) ** (2 * d)
    e = 0.5 * scale * math.fsum((w * a2).ravel())
    z = 0.5 * scale * math.fsum((w * k2 * a2).ravel())
    return e, z
