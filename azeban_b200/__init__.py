"""azeban_b200: B200-native spectral-viscosity incompressible Euler RHS,
SSP-RK3 stepper and real FFTs behind azeban's interfaces.

The compute runs in the in-tree CUDA library ``libazeban_b200.so`` (sm_100a),
reached through its C ABI (include/azeban_b200.h).
"""

from ._lib import AzebanError, supported_lengths
from .core import (FFT, FFT_BACKWARD, FFT_FORWARD, Grid, Group, IncompressibleEuler, NoViscosity,
                   Quadratic, Simulation, SmoothCutoff1D, SSP_RK3, Step1D, leray, make_fft,
                   make_grid, make_viscosity, next_good_size, precision_code)

from . import tune as _tune

_tune.load_table()

__all__ = [
    "AzebanError", "supported_lengths", "FFT", "FFT_BACKWARD", "FFT_FORWARD", "Grid", "Group",
    "IncompressibleEuler", "NoViscosity", "Quadratic", "Simulation", "SmoothCutoff1D", "SSP_RK3",
    "Step1D", "leray", "make_fft", "make_grid", "make_viscosity", "next_good_size",
    "precision_code",
]
