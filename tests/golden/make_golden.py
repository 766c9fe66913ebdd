"""Generates the golden fixtures of the Euler path with the CPU oracle.

Run ``python tests/golden/make_golden.py`` from the repository root to
(re)write ``tests/golden/*.npz``.  Each fixture holds its seeded input and
the oracle's output in FP64:
  dudt_<d>d_n<N>     one right-hand side of a seeded random divergence-free
                     field (SmoothCutoff eps=0.05) and dt(C = 0.2)
  traj_tg2d_n64      Taylor-Green 2-D 64^2 to t = 1 (C = 0.2, SSP-RK3)
  traj_dsl2d_n64     double shear layer 2-D 64^2, rho=0.2, delta=0.05, to t = 0.5
  traj_tg3d_n16      Taylor-Green 3-D 16^3 to t = 1
  traj_tg3d_n32      Taylor-Green 3-D 32^3 to t = 1
  traj_tg3d_n64      Taylor-Green 3-D 64^3 to t = 1, as a fingerprint of the
                     final state (the modes with |n_i| <= 8 on every axis, the
                     L2 norm of each component) and the dt sequence
The 3-D 32^3 and 64^3 fixtures are written compressed (np.savez_compressed).
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


def low_modes(u_hat, K=8):
    """The modes of a [d][N]..[N/2+1] spectrum with |n| <= K on every axis
    (signed indices on the full axes, 0..K on the compact one)."""
    N = u_hat.shape[1]
    full = np.r_[0:K + 1, N - K:N]
    out = u_hat
    for ax in range(1, u_hat.ndim - 1):
        out = np.take(out, full, axis=ax)
    return np.ascontiguousarray(out[..., :K + 1])


def _traj_fingerprint_case(dim, N, field, t_end):
    def make():
        full = _traj_case(dim, N, field, t_end)()
        u = full["u_final"]
        norms = np.sqrt(np.sum(np.abs(u.reshape(dim, -1)) ** 2, axis=1))
        return {"u_final_low": low_modes(u), "u_final_norms": norms, "dts": full["dts"], "t_end": full["t_end"]}
    return make


CASES = {
    "dudt_2d_n16": _dudt_case(2, 16),
    "dudt_2d_n32": _dudt_case(2, 32),
    "dudt_2d_n64": _dudt_case(2, 64),
    "dudt_3d_n8": _dudt_case(3, 8),
    "dudt_3d_n16": _dudt_case(3, 16),
    "dudt_3d_n32": _dudt_case(3, 32),
    "traj_tg2d_n64": _traj_case(2, 64, lambda: ora.taylor_green_workload(2, 64), 1.0),
    "traj_dsl2d_n64": _traj_case(2, 64, lambda: ora.double_shear_layer(64, 0.2, 0.05), 0.5),
    "traj_tg3d_n16": _traj_case(3, 16, lambda: ora.taylor_green_workload(3, 16), 1.0),
    "traj_tg3d_n32": _traj_case(3, 32, lambda: ora.taylor_green_workload(3, 32), 1.0),
    "traj_tg3d_n64": _traj_fingerprint_case(3, 64, lambda: ora.taylor_green_workload(3, 64), 1.0),
}
COMPRESSED = {"dudt_3d_n32", "traj_tg3d_n32", "traj_tg3d_n64"}


def main(names=None):
    for name, make in CASES.items():
        if names and name not in names:
            continue
        data = make()
        save = np.savez_compressed if name in COMPRESSED else np.savez
        save(os.path.join(HERE, name + ".npz"), **data)
        print(name, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
