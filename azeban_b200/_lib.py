"""ctypes binding of ``libazeban_b200.so`` (the C ABI in include/azeban_b200.h).

The library is the product: if it is missing this module raises at import,
there is no fallback path.
"""

from __future__ import annotations

import ctypes as ct
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libazeban_b200.so")

AZ_OK = 0
AZ_ERR_INVALID, AZ_ERR_UNSUPPORTED, AZ_ERR_CUDA, AZ_ERR_NOMEM, AZ_ERR_NONFINITE, AZ_ERR_TIMEOUT = 1, 2, 3, 4, 5, 6
AZ_PREC_F64, AZ_PREC_F32 = 0, 1
AZ_VISC_NONE, AZ_VISC_SMOOTH_CUTOFF, AZ_VISC_STEP, AZ_VISC_QUADRATIC = 0, 1, 2, 3
AZ_FFT_FORWARD, AZ_FFT_BACKWARD = 1, 2
AZ_NOALLOC_SCRATCH_BYTES = 64 * 1024 * 1024

STATUS_NAMES = {0: "AZ_OK", 1: "AZ_ERR_INVALID", 2: "AZ_ERR_UNSUPPORTED", 3: "AZ_ERR_CUDA",
                4: "AZ_ERR_NOMEM", 5: "AZ_ERR_NONFINITE", 6: "AZ_ERR_TIMEOUT"}

# Every entry point include/azeban_b200.h declares.
EXPORTS = [
    "az_last_error_string", "az_supported_lengths",
    "az_euler_create", "az_euler_destroy", "az_euler_dudt", "az_euler_dt", "az_euler_n_vars",
    "az_euler_visc", "az_euler_workspace_size",
    "az_rk3_create", "az_rk3_destroy", "az_rk3_integrate",
    "az_sim_create", "az_sim_destroy", "az_sim_simulate_until", "az_sim_steps", "az_sim_u",
    "az_sim_state",
    "az_fft_create", "az_fft_destroy", "az_fft_forward", "az_fft_backward", "az_fft_work_area_size",
    "az_fft_set_work_area",
    "az_leray", "az_profile_enable", "az_profile_read", "az_euler_dudt_noalloc",
    "az_tune_set", "az_tune_get", "az_euler_diagnostics",
    "az_sim_member_start", "az_sim_member_stop", "az_group_create", "az_group_destroy",
    "az_group_steps", "az_group_steps_active", "az_group_set_end", "az_group_simulate_until",
    "az_debug_set_wait_limit", "az_debug_get_wait_limit", "az_euler_noalloc_status",
    "az_init_physical", "az_init_envelope", "az_init_normalize_energy", "az_random_uniform",
    "az_philox4x32_10", "az_bench_radix16_stage", "az_bench_exchange384",
]


class AzebanError(RuntimeError):
    """A non-zero az_status, with the library's error string."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class az_visc(ct.Structure):
    _fields_ = [("type", ct.c_int), ("eps", ct.c_double), ("s", ct.c_double),
                ("k0", ct.c_double), ("N", ct.c_longlong)]


class az_euler_desc(ct.Structure):
    _fields_ = [("dim", ct.c_int), ("N_phys", ct.c_longlong), ("N_phys_pad", ct.c_longlong),
                ("precision", ct.c_int), ("visc", az_visc), ("batch", ct.c_int)]


AZ_INIT_TAYLOR_GREEN, AZ_INIT_TAYLOR_GREEN_WORKLOAD, AZ_INIT_DOUBLE_SHEAR_LAYER, AZ_INIT_GAUSSIAN_NOISE = 0, 1, 2, 3


class az_init_desc(ct.Structure):
    _fields_ = [("kind", ct.c_int), ("dim", ct.c_int), ("N", ct.c_longlong), ("precision", ct.c_int),
                ("batch", ct.c_int), ("rho", ct.c_double), ("delta", ct.c_double),
                ("deltas", ct.POINTER(ct.c_double)), ("phases", ct.POINTER(ct.c_double)),
                ("seed", ct.c_ulonglong), ("member0", ct.c_longlong)]


class az_fft_desc(ct.Structure):
    _fields_ = [("dim", ct.c_int), ("n_vars", ct.c_longlong), ("shape", ct.c_longlong * 3),
                ("transform_last", ct.c_int), ("precision", ct.c_int), ("direction", ct.c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python azeban_b200/build.py` "
            "(there is no CPU fallback)")
    lib = ct.CDLL(LIB_PATH)
    P, I, D, LL, SZ = ct.c_void_p, ct.c_int, ct.c_double, ct.c_longlong, ct.c_size_t
    sig = {
        "az_last_error_string": (ct.c_char_p, []),
        "az_supported_lengths": (I, [ct.POINTER(I), I, ct.POINTER(I)]),
        "az_euler_create": (I, [ct.POINTER(az_euler_desc), ct.POINTER(P)]),
        "az_euler_destroy": (I, [P]),
        "az_euler_dudt": (I, [P, P, P, D, D, D, P]),
        "az_euler_dt": (I, [P, D, P, ct.POINTER(D)]),
        "az_euler_n_vars": (I, [P]),
        "az_euler_visc": (D, [P]),
        "az_euler_workspace_size": (SZ, [P]),
        "az_rk3_create": (I, [P, ct.POINTER(P)]),
        "az_rk3_destroy": (I, [P]),
        "az_rk3_integrate": (I, [P, D, D, D, P, P, ct.POINTER(D)]),
        "az_sim_create": (I, [P, D, P, P, ct.POINTER(P)]),
        "az_sim_destroy": (I, [P]),
        "az_sim_simulate_until": (I, [P, D, P]),
        "az_sim_steps": (I, [P, I, P]),
        "az_sim_u": (P, [P]),
        "az_sim_state": (I, [P, P, ct.POINTER(D), ct.POINTER(LL), ct.POINTER(D)]),
        "az_fft_create": (I, [ct.POINTER(az_fft_desc), P, P, ct.POINTER(P)]),
        "az_fft_destroy": (I, [P]),
        "az_fft_forward": (I, [P, P]),
        "az_fft_backward": (I, [P, P]),
        "az_fft_work_area_size": (SZ, [P]),
        "az_fft_set_work_area": (I, [P, P]),
        "az_leray": (I, [I, LL, I, P, I, P]),
        "az_profile_enable": (I, [I]),
        "az_profile_read": (I, [ct.POINTER(D), ct.POINTER(D), ct.POINTER(LL), I]),
        "az_euler_dudt_noalloc": (I, [I, LL, LL, I, ct.POINTER(az_visc), P, P, P]),
        "az_tune_set": (I, [I, I, I, I]),
        "az_tune_get": (I, [I, I, I, ct.POINTER(I)]),
        "az_euler_diagnostics": (I, [P, P, P, ct.POINTER(D), ct.POINTER(D)]),
        "az_sim_member_start": (I, [P, I, P, D, P]),
        "az_sim_member_stop": (I, [P, I, P]),
        "az_group_create": (I, [ct.POINTER(P), I, ct.POINTER(P)]),
        "az_group_destroy": (I, [P]),
        "az_group_steps": (I, [P, I, P]),
        "az_group_steps_active": (I, [P, I, ct.POINTER(I), P]),
        "az_group_set_end": (I, [P, D, P]),
        "az_group_simulate_until": (I, [P, D, P]),
        "az_debug_set_wait_limit": (I, [I]),
        "az_debug_get_wait_limit": (I, []),
        "az_euler_noalloc_status": (I, [P]),
        "az_init_physical": (I, [ct.POINTER(az_init_desc), P, P]),
        "az_init_envelope": (I, [I, LL, I, P, I, D, P]),
        "az_init_normalize_energy": (I, [I, LL, I, P, I, D, P]),
        "az_random_uniform": (I, [ct.c_ulonglong, ct.c_ulonglong, ct.c_ulonglong, ct.POINTER(D)]),
        "az_philox4x32_10": (I, [ct.POINTER(ct.c_uint), ct.POINTER(ct.c_uint), ct.POINTER(ct.c_uint)]),
        "az_bench_radix16_stage": (I, [I, I, ct.POINTER(D), ct.POINTER(D)]),
        "az_bench_exchange384": (I, [I, I, ct.POINTER(D), ct.POINTER(D)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != AZ_OK:
        msg = lib.az_last_error_string().decode(errors="replace")
        raise AzebanError(status, msg)


def supported_lengths():
    n = ct.c_int(0)
    check(lib.az_supported_lengths(None, 0, ct.byref(n)))
    buf = (ct.c_int * n.value)()
    check(lib.az_supported_lengths(buf, n.value, ct.byref(n)))
    return list(buf)
