"""Generates the golden fixtures of the Euler path with the CPU oracle.

Run ``python tests/golden/make_golden.py`` from the repository root to
(re)write ``tests/golden/*.npz``.  Each fixture holds its seeded input and
the oracle's output in FP64:
  dudt_<d>d_n<N>     one right-hand side of a seeded random divergence-free
                     field (SmoothCutoff eps=0.05) and dt(C = 0.2)
  traj_tg2d_n64      Taylor-Green 2-D 64^2 to t = 1 (C = 0.2, SSP-RK3)
  traj_dsl2d_n64     double shear layer 2-D 64^2, rho=0.2, delta=0.05, to t = 0.5
  traj_tg3d_n16      Taylor-Green 3-D 16^3 to t = 1
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import euler_oracle as ora  # noqa: E402

VISC = {"type": "Smooth Cutoff", "eps": 0.05}


def random_field_hat(dim, N, seed, slope=2.0):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((dim,) + (N,) * dim)
    u_hat = ora.fft_forward(u)
    kk = [ora.signed_index(N).astype(float)] * (dim - 1) + [np.arange(N // 2 + 1, dtype=float)]
    ks = np.meshgrid(*kk, indexing="ij")
    u_hat = u_hat * (1.0 + np.sqrt(sum(k * k for k in ks))) ** (-slope)
    u_hat = ora.leray(u_hat)
    u_hat /= np.abs(ora.fft_backward(u_hat, N) / N ** dim).max()
    return u_hat


def _dudt_case(dim, N):
    def make():
        g = ora.Grid(dim, N)
        eq = ora.IncompressibleEuler(g, ora.make_viscosity(VISC, g))
        u = random_field_hat(dim, N, seed=1000 + 10 * dim + N)
        out = eq.dudt(u)
        return {"u_hat": u, "dudt": out, "dt": np.array(eq.dt(0.2))}
    return make


def _traj_case(dim, N, field, t_end):
    def make():
        g = ora.Grid(dim, N)
        eq = ora.IncompressibleEuler(g, ora.make_viscosity(VISC, g))
        u0 = ora.initialize(field())
        sim = ora.Simulation(g, 0.2, ora.SSP_RK3(eq), u0)
        sim.simulate_until(t_end)
        return {"u0": u0, "u_final": sim.u_, "dts": np.array(sim.dts), "t_end": np.array(t_end)}
    return make


CASES = {
    "dudt_2d_n16": _dudt_case(2, 16),
    "dudt_2d_n32": _dudt_case(2, 32),
    "dudt_2d_n64": _dudt_case(2, 64),
    "dudt_3d_n8": _dudt_case(3, 8),
    "dudt_3d_n16": _dudt_case(3, 16),
    "traj_tg2d_n64": _traj_case(2, 64, lambda: ora.taylor_green_workload(2, 64), 1.0),
    "traj_dsl2d_n64": _traj_case(2, 64, lambda: ora.double_shear_layer(64, 0.2, 0.05), 0.5),
    "traj_tg3d_n16": _traj_case(3, 16, lambda: ora.taylor_green_workload(3, 16), 1.0),
}


def main():
    for name, make in CASES.items():
        data = make()
        np.savez(os.path.join(HERE, name + ".npz"), **data)
        print(name, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
