"""ctypes binding of oracle/_ref/libazeban_ref.so: the reference's own
pointwise functions compiled here (see oracle/build_ref.sh).

TEST INFRASTRUCTURE ONLY: the parity tests use it to pin the numpy oracle's
pointwise stages (padding map, viscosity laws, the computeB scaling and
products, the per-mode projection and right-hand side) against the
reference's code.
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libazeban_ref.so")
BUILD = os.path.join(HERE, "build_ref.sh")

_P = ct.POINTER(ct.c_double)
_PI = ct.POINTER(ct.c_int)


def load(reference_root: str = "/root/reference"):
    """The compiled library, built from the reference tree first if it is
    missing and the tree is there; None if neither."""
    if not os.path.exists(LIB):
        if not os.path.isdir(os.path.join(reference_root, "include", "azeban")):
            return None
        subprocess.run(["sh", BUILD, reference_root], check=True, capture_output=True)
    lib = ct.CDLL(LIB)
    lib.azref_norm.restype = ct.c_double
    lib.azref_norm.argtypes = [ct.c_int, ct.c_longlong, ct.c_longlong]
    lib.azref_compute_B.restype = None
    lib.azref_compute_B.argtypes = [ct.c_int, ct.c_longlong, ct.c_double, _P, _P]
    lib.azref_dudt_modes.restype = None
    lib.azref_dudt_modes.argtypes = [ct.c_int, ct.c_longlong, _PI, _P, _P, ct.c_int, ct.c_double, ct.c_double,
                                     ct.c_double, ct.c_longlong, _P]
    lib.azref_visc_eval.restype = None
    lib.azref_visc_eval.argtypes = [ct.c_int, ct.c_double, ct.c_double, ct.c_double, ct.c_longlong,
                                    ct.c_longlong, _P, _P]
    lib.azref_pad_index.restype = ct.c_longlong
    lib.azref_pad_index.argtypes = [ct.c_int, ct.c_longlong, ct.c_longlong, ct.c_longlong]
    return lib


def _dp(a):
    return a.ctypes.data_as(_P)


VISC_CODES = {"smooth_cutoff": 1, "step": 2, "quadratic": 3, "none": 0}


def visc_args(visc):
    """(type, eps, s, k0, N) of an oracle viscosity object."""
    kind = getattr(visc, "kind", "none")
    return (VISC_CODES[kind], float(getattr(visc, "eps", 0.0)), float(getattr(visc, "s", 0.0)),
            float(getattr(visc, "k0", 0.0)), int(getattr(visc, "N", 0)))


def norm(lib, dim, N, M):
    return lib.azref_norm(dim, N, M)


def compute_B(lib, u: np.ndarray, norm_: float) -> np.ndarray:
    """u [dim, ...] real -> B [dim(dim+1)/2, ...]."""
    dim = u.shape[0]
    flat = np.ascontiguousarray(u.reshape(dim, -1), dtype=np.float64)
    n = flat.shape[1]
    B = np.empty((dim * (dim + 1) // 2, n), dtype=np.float64)
    lib.azref_compute_B(dim, n, norm_, _dp(flat), _dp(B))
    return B.reshape((B.shape[0],) + u.shape[1:])


def dudt_modes(lib, idx: np.ndarray, B_hat: np.ndarray, u_hat: np.ndarray, visc) -> np.ndarray:
    """idx [dim, n] signed indices, B_hat [nb, n], u_hat [dim, n] complex -> dudt [dim, n]."""
    dim, n = idx.shape
    ii = np.ascontiguousarray(idx, dtype=np.int32)
    Bc = np.ascontiguousarray(B_hat, dtype=np.complex128)
    uc = np.ascontiguousarray(u_hat, dtype=np.complex128)
    out = np.empty((dim, n), dtype=np.complex128)
    t, eps, s, k0, N = visc_args(visc)
    lib.azref_dudt_modes(dim, n, ii.ctypes.data_as(_PI), Bc.ctypes.data_as(_P), uc.ctypes.data_as(_P),
                         t, eps, s, k0, N, out.ctypes.data_as(_P))
    return out


def visc_eval(lib, visc, k: np.ndarray) -> np.ndarray:
    kk = np.ascontiguousarray(k, dtype=np.float64).ravel()
    out = np.empty_like(kk)
    t, eps, s, k0, N = visc_args(visc)
    lib.azref_visc_eval(t, eps, s, k0, N, kk.size, _dp(kk), _dp(out))
    return out.reshape(np.shape(k))


def pad_index_map(lib, compact: bool, src_n: int, dst_n: int) -> np.ndarray:
    return np.array([lib.azref_pad_index(int(compact), src_n, dst_n, i) for i in range(dst_n)], dtype=np.int64)
