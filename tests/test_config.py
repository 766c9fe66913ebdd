"""The reference's JSON run configuration (azeban_b200.config).

Keys, defaults and error messages follow src/azeban/simulation_factory.cpp
:9-46, src/azeban/equations/equation_factory.cpp:160-199,
include/azeban/evolution/time_integrator_factory.hpp:34-62,
include/azeban/grid_factory.hpp:28-92 and include/azeban/sequence_factory.hpp;
the run loop follows src/azeban/run_from_config.cpp:23-103.  The host-side
parsing runs on CPU; building and running solves needs the GPU.
"""

import math
import os

import numpy as np
import pytest
import torch

from azeban_b200 import config as cfg
from azeban_b200.random import MT19937, uniform_real
from oracle import euler_oracle as ora
from oracle.mt19937 import MT19937 as OracleMT

# The keys and values of the reference's experiments/TechnicalReport/N256/config.json
# (the 256^3 Taylor-Green run of its performance logs).
TG_N256 = {
    "output": "tg_N256_time", "device": "cuda", "dimension": 3, "num_samples": 1, "seed": 1, "time": 5,
    "snapshots": {"start": 0, "stop": 5, "n": 50},
    "grid": {"N_phys": 256, "N_phys_pad": ""},
    "equation": {"name": "Euler", "visc": {"type": "Quadratic", "eps": 0.05}},
    "timestepper": {"type": "SSP RK3", "C": 0.5},
    "init": {"name": "Taylor Green", "perturb": {"name": "Uniform", "min": -0.025, "max": 0.025}},
}


def test_grid_of_the_technical_report_config():
    g = cfg.make_grid_from(TG_N256)
    assert (g.dim, g.N_phys, g.N_phys_pad, g.N_fourier) == (3, 256, 384, 129)
    assert cfg.make_sequence(TG_N256["snapshots"])[:3] == [0.0, 0.1, 0.2]
    assert len(cfg.make_sequence(TG_N256["snapshots"])) == 51


def test_sequences():
    assert cfg.make_sequence(0.5) == [0.5]
    assert cfg.make_sequence([0, 1]) == [0.0, 1.0]
    assert cfg.make_sequence({"start": 0, "stop": 1, "step": 0.3}) == [0.0, 0.3, 0.6, 0.8999999999999999, 1.0]
    with pytest.raises(cfg.ConfigError, match='Expected key "stop"'):
        cfg.make_sequence({"n": 3})
    with pytest.raises(cfg.ConfigError, match='"n" or "step"'):
        cfg.make_sequence({"stop": 1})


@pytest.mark.parametrize("mutate,msg", [
    (lambda c: c.pop("grid"), 'Config must contain key "grid"'),
    (lambda c: c.pop("dimension"), 'Config must contain key "dimension"'),
    (lambda c: c.pop("equation"), 'Config must contain key "equation"'),
    (lambda c: c["equation"].pop("name"), 'Equation config must contain key "name"'),
    (lambda c: c["equation"].pop("visc"), 'Equation config must contain key "visc"'),
    (lambda c: c["equation"]["visc"].pop("type"), 'Must specify the type of Spectral Viscosity in key "type"'),
    (lambda c: c["equation"]["visc"].update(type="Magic"), "Unknown viscosity type: Magic"),
    (lambda c: c["equation"].update(name="Burgers"), 'Unknown equation name: "Burgers"'),
    (lambda c: c["equation"].update(forcing={"type": "Sinusoidal"}), "not on this path"),
    (lambda c: c["equation"].update(forcing={}), 'Must specify the type of Forcing in key "type"'),
    (lambda c: c.update(device="cpu"), "runs on the GPU"),
    (lambda c: c.update(device="tpu"), "Unknown device type: tpu"),
    (lambda c: c["grid"].update(N_fourier=129), 'either "N_phys" or "N_fourier"'),
])
def test_bad_configs_rejected_with_the_references_messages(mutate, msg):
    import copy
    c = copy.deepcopy(TG_N256)
    mutate(c)
    with pytest.raises(cfg.ConfigError, match=msg):
        cfg.make_simulation(c)


def test_timestepper_errors():
    with pytest.raises(cfg.ConfigError, match="Missing timestepper type"):
        cfg.make_timestepper({}, None)
    with pytest.raises(cfg.ConfigError, match='Unknown time integrator: "RK4"'):
        cfg.make_timestepper({"type": "RK4"}, None)
    with pytest.raises(cfg.ConfigError, match="not on this path"):
        cfg.make_timestepper({"type": "SSP RK2"}, None)


def test_random_draws_are_the_references():
    """The run's std::mt19937 and uniform_real_distribution<double> draws
    (the initialisers' random parameters) equal the oracle's restatement,
    which is pinned bit for bit against libstdc++."""
    a = MT19937(7)
    o = OracleMT(7)
    assert [uniform_real(a, -0.025, 0.025) for _ in range(50)] == list(o.uniform(-0.025, 0.025, 50))
    g = MT19937()
    for _ in range(9999):
        g()
    assert g() == 4123659995  # the C++ standard's check value of std::mt19937


# ---------------------------------------------------------------------------
# solves built from a config (GPU)
# ---------------------------------------------------------------------------

def _config(dim, N, init, visc="Smooth Cutoff", snapshots=(0.01, 0.02)):
    return {"device": "cuda", "dimension": dim, "seed": 3, "grid": {"N_phys": N, "N_phys_pad": ""},
            "equation": {"name": "Euler", "visc": {"type": visc, "eps": 0.05}},
            "timestepper": {"type": "SSP RK3", "C": 0.2}, "init": init,
            "writer": {"name": "NetCDF Snapshot", "snapshots": list(snapshots)}}


def _oracle_run(conf, u0, t):
    og = ora.make_grid(conf["grid"], conf["dimension"])
    eq = ora.IncompressibleEuler(og, ora.make_viscosity(conf["equation"]["visc"], og))
    sim = ora.Simulation(og, conf["timestepper"]["C"], ora.SSP_RK3(eq), u0)
    sim.simulate_until(t)
    return sim


@pytest.mark.gpu
def test_make_simulation_matches_oracle():
    conf = _config(3, 16, {"name": "Taylor Green"}, visc="Quadratic")
    sim = cfg.make_simulation(conf)
    u0 = ora.initialize(ora.taylor_green_reference(3, 16))
    sim.u().copy_(torch.from_numpy(u0).cuda())
    sim.simulate_until(0.02)
    osim = _oracle_run(conf, u0, 0.02)
    assert ora.rel_l2(sim.u().cpu().numpy(), osim.u_) <= 1e-9
    assert sim.state()[1][0] == len(osim.dts)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,init", [
    (2, {"name": "Double Shear Layer", "rho": 0.2, "delta": 0.05}),
    (2, {"name": "Taylor Green", "perturb": {"name": "Uniform", "min": -0.025, "max": 0.025}}),
    (3, {"name": "Taylor Green", "perturb": {"name": "Uniform", "min": -0.025, "max": 0.025}}),
])
def test_run_from_config_snapshots_match_oracle(tmp_path, dim, init):
    """Two samples, two snapshot times: each u_hat equals the oracle's run of
    the same config (same random draws), and each u is the backward
    transform of u_hat / N^d (run_from_config.cpp:86-99)."""
    N = 32 if dim == 2 else 16
    conf = _config(dim, N, init)
    conf["num_samples"] = 2
    out = str(tmp_path / "snap")
    cfg.run_from_config(conf, out_dir=out, log=None)
    rng = OracleMT(conf["seed"])
    for sample in range(2):
        if init["name"] == "Taylor Green":
            nd = 8 if dim == 2 else 24
            deltas = rng.uniform(-0.025, 0.025, nd) / (4 if dim == 2 else 8)
            u0 = ora.initialize(ora.taylor_green_reference(dim, N, deltas))
        else:
            u0 = ora.initialize(ora.double_shear_layer(N, 0.2, 0.05))
        og = ora.make_grid(conf["grid"], dim)
        eq = ora.IncompressibleEuler(og, ora.make_viscosity(conf["equation"]["visc"], og))
        sim = ora.Simulation(og, 0.2, ora.SSP_RK3(eq), u0)
        for t in conf["writer"]["snapshots"]:
            sim.simulate_until(t)
            uh = np.load(os.path.join(out, f"sample_{sample}_time_{t:.6g}_u_hat.npy"))
            u = np.load(os.path.join(out, f"sample_{sample}_time_{t:.6g}_u.npy"))
            assert ora.rel_l2(uh, sim.u_) <= 1e-9
            phys = ora.fft_backward(sim.u_ / float(N) ** dim, N)
            assert ora.rel_l2(u, phys) <= 1e-9
