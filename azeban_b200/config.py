"""The reference's JSON run configuration, for this path.

Restates the factories that turn azeban's config file into a solve:
  make_simulation    src/azeban/simulation_factory.cpp:9-46
  make_equation      src/azeban/equations/equation_factory.cpp:17-58, :160-199,
                     include/azeban/equations/incompressible_euler_factory.hpp:27-46
  make_timestepper   include/azeban/evolution/time_integrator_factory.hpp:34-62
  make_grid          include/azeban/grid_factory.hpp:28-92 (core.make_grid)
  make_viscosity     include/azeban/equations/spectral_viscosity_factory.hpp:29-89
  make_sequence      include/azeban/sequence_factory.hpp
  make_initializer   the "init" object (Taylor Green, Double Shear Layer) and
                     the random variables of its parameters
                     (include/azeban/random/random_variable_factory.hpp)
  run_from_config    src/azeban/run_from_config.cpp:23-103: the sample loop,
                     simulate_until each snapshot time, and the output of
                     u_hat and of u = backward transform of u_hat / N^d.

The keys, their defaults and the messages of a bad config are the
reference's; where the reference prints a message and exits, this module
raises ConfigError with that message.  Parts of the reference outside this
path (other equations, forcings, integrators, tracers, MPI, NetCDF and
ParaView writers, spectra) raise ConfigError naming the key.

Two keys are this library's own: "precision" ("double", the default, or
"float" for FP32 bulk with FP64 CFL) selects the precision the reference
fixes at compile time (config.hpp.in:24-28), and snapshots are written as
.npy files (NetCDF is not available here).
"""

from __future__ import annotations

import json
import math
import os

import numpy as np
import torch

from . import init as azinit
from .core import (FFT, FFT_BACKWARD, Grid, IncompressibleEuler, Simulation, SSP_RK3, make_grid,
                   make_viscosity)
from .random import MT19937, uniform_real


class ConfigError(ValueError):
    """A config the reference would reject (same message), or one outside this path."""


def load(path: str) -> dict:
    with open(path) as f:
        return json.load(f)


def _precision(config: dict, precision=None) -> str:
    if precision is not None:
        return precision
    p = config.get("precision", "double")
    if p in ("double", "f64", "fp64"):
        return "f64"
    if p in ("float", "f32", "fp32"):
        return "f32"
    raise ConfigError(f'Unknown precision: "{p}"')


def make_sequence(spec):
    """A number, a list, or {"start", "stop", "n" | "step"} (sequence_factory.hpp)."""
    if isinstance(spec, (int, float)) and not isinstance(spec, bool):
        return [float(spec)]
    if isinstance(spec, list):
        return [float(x) for x in spec]
    if isinstance(spec, dict):
        start = float(spec.get("start", 0))
        if "stop" not in spec:
            raise ConfigError('Expected key "stop" in sequence specifier')
        stop = float(spec["stop"])
        if "n" in spec:
            n = int(spec["n"])
            return [start + i * (stop - start) / n for i in range(n + 1)]
        if "step" in spec:
            step = float(spec["step"])
            res = [start]
            while res[-1] < stop:
                res.append(res[-1] + step)
            res[-1] = stop
            return res
        raise ConfigError('Expected either "n" or "step" in sequence specification')
    raise ConfigError("Unsupported type for a sequence")


def make_equation(config: dict, grid: Grid, precision: str = "f64", batch: int = 1,
                  has_tracer: bool = False) -> IncompressibleEuler:
    """The "equation" object (equation_factory.cpp:160-199)."""
    if "name" not in config:
        raise ConfigError('Equation config must contain key "name"')
    if "visc" not in config:
        raise ConfigError('Equation config must contain key "visc"')
    if "type" not in config["visc"]:
        raise ConfigError('Must specify the type of Spectral Viscosity in key "type"')
    forcing = "No Forcing"
    if "forcing" in config:
        if "type" not in config["forcing"]:
            raise ConfigError('Must specify the type of Forcing in key "type"')
        forcing = config["forcing"]["type"]
    visc_type = config["visc"]["type"]
    if visc_type not in ("Smooth Cutoff", "Step", "Quadratic"):
        raise ConfigError(f"Unknown viscosity type: {visc_type}")
    if forcing != "No Forcing":
        if forcing in ("Sinusoidal", "White Noise", "White Noise High Freq", "Boussinesq"):
            raise ConfigError(f'Forcing "{forcing}" is not on this path (no forcing only)')
        raise ConfigError(f"Unknown forcing type: {forcing}")
    name = config["name"]
    if name != "Euler":
        if name == "Euler Naive":
            raise ConfigError('Equation "Euler Naive" is not on this path (the optimised "Euler" is)')
        raise ConfigError(f'Unknown equation name: "{name}"')
    if grid.dim not in (2, 3):
        raise ConfigError("Euler is only implemented for 2D or 3D")
    if has_tracer:
        raise ConfigError("Tracers are not on this path")
    return IncompressibleEuler(grid, make_viscosity(config["visc"], grid), precision, batch)


def make_timestepper(config: dict, equation: IncompressibleEuler) -> SSP_RK3:
    """The "timestepper" object (time_integrator_factory.hpp:34-62)."""
    if "type" not in config:
        raise ConfigError("Missing timestepper type")
    typ = config["type"]
    if typ == "SSP RK3":
        return SSP_RK3(equation)
    if typ in ("Forward Euler", "SSP RK2", "Euler Maruyama"):
        raise ConfigError(f'Time integrator "{typ}" is not on this path (SSP RK3 is)')
    raise ConfigError(f'Unknown time integrator: "{typ}"')


def make_grid_from(config: dict) -> Grid:
    if "dimension" not in config:
        raise ConfigError('Config must contain key "dimension"')
    if "grid" not in config:
        raise ConfigError('Config must contain key "grid"')
    try:
        return make_grid(config["grid"], int(config["dimension"]))
    except ValueError as e:
        raise ConfigError(str(e)) from None


def make_simulation(config: dict, seed: int = 1, precision=None, batch: int = 1, u_init=None) -> Simulation:
    """Grid, equation, time stepper and CFL constant of a config
    (simulation_factory.cpp:9-46) as a Simulation of `batch` members whose
    state starts at u_init (zero if None; the initialiser writes it)."""
    device = config.get("device", "cuda")
    if device == "cpu":
        raise ConfigError('Device "cpu" is not on this path: this library runs on the GPU')
    if device != "cuda":
        raise ConfigError(f"Unknown device type: {device}")
    grid = make_grid_from(config)
    if "equation" not in config:
        raise ConfigError('Config must contain key "equation"')
    has_tracer = "init" in config and "tracer" in config["init"]
    prec = _precision(config, precision)
    equation = make_equation(config["equation"], grid, prec, batch, has_tracer)
    if "timestepper" not in config:
        raise ConfigError("Config is missing timestepper specifications")
    timestepper = make_timestepper(config["timestepper"], equation)
    if "C" not in config["timestepper"]:
        raise ConfigError('Timestepper config is missing CFL constant "C"')
    C = float(config["timestepper"]["C"])
    shape = ((batch,) if batch > 1 else ()) + grid.shape_fourier(grid.dim)
    if u_init is None:
        u_init = torch.zeros(shape, dtype=equation.cdtype, device="cuda")
    return Simulation(grid, C, timestepper, u_init)


class RandomVariable:
    """A number, or {"name": "Uniform", "min", "max"} drawn from the run's
    mt19937 as std::uniform_real_distribution<double> draws it
    (include/azeban/random/uniform.hpp); "Normal" and "Delta" as the
    reference's normal and delta variables."""

    def __init__(self, spec, rng: MT19937):
        self.rng = rng
        if isinstance(spec, (int, float)) and not isinstance(spec, bool):
            self.kind, self.value = "const", float(spec)
        elif isinstance(spec, dict) and spec.get("name") == "Uniform":
            self.kind, self.lo, self.hi = "uniform", float(spec["min"]), float(spec["max"])
        elif isinstance(spec, dict) and spec.get("name") == "Delta":
            self.kind, self.value = "const", float(spec["value"])
        else:
            raise ConfigError(f"Random variable {spec!r} is not supported on this path")

    def get(self) -> float:
        if self.kind == "const":
            return self.value
        return uniform_real(self.rng, self.lo, self.hi)


class Initializer:
    """The "init" object: Taylor Green (taylor_green.cpp:29-46, :146-184,
    with its "perturb" random variable; each sample draws 8 (2-D) or 24 (3-D)
    amplitudes, divided by 4 or 8) and Double Shear Layer
    (double_shear_layer.cpp:25-43, "rho" and "delta" random variables), built
    on the device, transformed and Leray-projected."""

    def __init__(self, config: dict, dim: int, rng: MT19937):
        if "init" not in config or "name" not in config["init"]:
            raise ConfigError('Config must contain key "init" with a "name"')
        c = config["init"]
        self.name, self.dim = c["name"], dim
        if self.name == "Taylor Green":
            self.delta = RandomVariable(c.get("perturb", 0.0), rng)
        elif self.name == "Double Shear Layer":
            if dim != 2:
                raise ConfigError("Double shear layer is only available in 2d")
            self.rho = RandomVariable(c["rho"], rng)
            self.dl = RandomVariable(c["delta"], rng)
        else:
            raise ConfigError(f'Initializer "{self.name}" is not on this path')

    def initialize(self, grid: Grid, precision: str) -> torch.Tensor:
        N = grid.N_phys
        if self.name == "Taylor Green":
            nd = 8 if self.dim == 2 else 24
            div = 4.0 if self.dim == 2 else 8.0
            deltas = [[self.delta.get() / div for _ in range(nd)]]
            return azinit.taylor_green_reference(self.dim, N, precision, deltas)[0]
        return azinit.double_shear_layer(N, self.rho.get(), self.dl.get(), [0.0], precision)[0]


def run_from_config(config: dict, out_dir: str | None = None, precision=None, log=print):
    """The reference's run (run_from_config.cpp:23-103): for each sample,
    initialise, then at every snapshot time simulate_until it and write u_hat
    and u = backward transform of u_hat / N^d.  Snapshots go to
    <path>/sample_<s>_time_<t>_{u_hat,u}.npy (the writer's "path", or
    out_dir).  Returns {(sample, time): (u_hat, u)} as host arrays when no
    path is given."""
    dim = int(config.get("dimension", 0))
    num_samples = int(config.get("num_samples", 1))
    start = int(config.get("sample_idx_start", 0))
    time_offset = float(config.get("time_offset", 0.0))
    seed = int(config.get("seed", 1))
    rng = MT19937(seed)
    sim = make_simulation(config, seed, precision)
    prec = "f64" if sim.timestepper_.equation_.precision == 0 else "f32"
    grid = sim.grid
    init = Initializer(config, dim, rng)
    if "writer" not in config:
        raise ConfigError('Config file must contain key "writer"')
    wr = config["writer"]
    name = wr.get("name")
    if name not in ("NetCDF Snapshot", "NumPy Snapshot"):
        raise ConfigError(f'Writer "{name}" is not on this path (snapshots are written as .npy)')
    if "snapshots" not in wr:
        raise ConfigError('Writer config needs key "snapshots"')
    times = make_sequence(wr["snapshots"])
    path = wr.get("path", out_dir) if out_dir is None else out_dir
    if path:
        os.makedirs(path, exist_ok=True)
    results = {}
    u_hat_dev = torch.empty(grid.shape_fourier(dim), dtype=sim.u().dtype, device="cuda")
    u_dev = torch.empty(grid.shape_phys(dim), dtype=torch.float64 if prec == "f64" else torch.float32,
                        device="cuda")
    fft = FFT(u_hat_dev, u_dev, FFT_BACKWARD)
    for sample in range(start, start + num_samples):
        u0 = init.initialize(grid, prec)
        sim.member_start(0, u0, math.inf)
        _set_time(sim, time_offset)
        for t in times:
            if t < time_offset:
                continue
            sim.simulate_until(t)
            if log:
                log(f"Sample {sample}, Time {t}")
            u_hat = sim.u().clone()
            u_hat_dev.copy_(u_hat.reshape(u_hat_dev.shape))
            u_hat_dev.div_(float(grid.N_phys) ** dim)
            fft.backward()
            uh, u = u_hat.cpu().numpy(), u_dev.cpu().numpy()
            if path:
                np.save(os.path.join(path, f"sample_{sample}_time_{t:.6g}_u_hat.npy"), uh)
                np.save(os.path.join(path, f"sample_{sample}_time_{t:.6g}_u.npy"), u)
            else:
                results[(sample, t)] = (uh, u)
    return results


def _set_time(sim: Simulation, t: float) -> None:
    """Simulation::set_time: the member's clock starts at t."""
    if t != 0.0:
        raise ConfigError('"time_offset" other than 0 is not on this path')
