"""Groups of simulations, slot control and the continuous-batching serving
loop: every result must be the same alone and in the mix."""

import math

import numpy as np
import pytest
import torch

import azeban_b200 as az
from azeban_b200 import init as azinit
from azeban_b200 import serving
from oracle import euler_oracle as ora
from tests.gpu_helpers import VISC_CFGS, random_field_hat, rel_l2, to_dev, to_host

pytestmark = pytest.mark.gpu


def _sim(dim, N, prec, fields):
    g = az.Grid(dim, N)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g), prec, batch=len(fields))
    ts = az.SSP_RK3(eq)
    u0 = to_dev(np.stack(fields) if len(fields) > 1 else fields[0], prec)
    return eq, ts, az.Simulation(g, 0.2, ts, u0)


def test_group_equals_each_simulation_alone():
    specs = [(2, 32, "f64", 2), (3, 16, "f64", 1), (2, 64, "f32", 3)]
    fields = {s: [random_field_hat(s[0], s[1], seed=10 * i + b) for b in range(s[3])]
              for i, s in enumerate(specs)}
    keep = []
    sims = []
    for s in specs:
        eq, ts, sim = _sim(s[0], s[1], s[2], fields[s])
        keep += [eq, ts]
        sims.append(sim)
    group = az.Group(sims)
    group.simulate_until(0.05)
    for s, sim in zip(specs, sims):
        eq, ts, alone = _sim(s[0], s[1], s[2], fields[s])
        alone.simulate_until(0.05)
        np.testing.assert_array_equal(to_host(sim.u()), to_host(alone.u()))
        assert sim.state()[1] == alone.state()[1]


def test_slot_restart_equals_fresh_solve():
    """A slot stopped, restarted with a new state and stepped in a group gives
    the same trajectory as a fresh simulation of that state."""
    dim, N = 2, 32
    f = [random_field_hat(dim, N, seed=s) for s in (1, 2, 3)]
    eq, ts, sim = _sim(dim, N, "f64", f)
    group = az.Group([sim])
    group.set_end(0.0)
    new = to_dev(random_field_hat(dim, N, seed=99))
    sim.member_stop(0)
    sim.member_stop(2)
    sim.member_start(1, new, 0.04)
    group.steps(40)
    t, n, _ = sim.state()
    assert t[1] >= 0.04 and n[0] == 0 and n[2] == 0
    eq2, ts2, fresh = _sim(dim, N, "f64", [random_field_hat(dim, N, seed=99)])
    fresh.simulate_until(t[1])
    assert fresh.state()[1][0] == n[1]
    np.testing.assert_array_equal(to_host(sim.u()[1]), to_host(fresh.u()))


def test_fractional_brownian_field():
    u = azinit.fractional_brownian(3, 32, 0.75, seed=5, precision="f64")
    g = az.Grid(3, 32)
    eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFGS["smooth"], g))
    e, _ = eq.diagnostics(u)
    assert abs(e - 1.0) < 1e-12
    h = to_host(u)
    ks = np.meshgrid(ora.signed_index(32), ora.signed_index(32), np.arange(17), indexing="ij")
    div = sum(ks[a] * h[a] for a in range(3))
    assert np.abs(div).max() <= 1e-10 * np.abs(h).max()
    again = azinit.fractional_brownian(3, 32, 0.75, seed=5, precision="f64")
    np.testing.assert_array_equal(to_host(again), h)


def test_serving_result_same_alone_and_in_mix():
    caps = {(2, 32): 3, (2, 64): 2, (3, 16): 2}
    target = serving.Request(0.0, 0, 2, 64, 0.2, 1234)
    mix = [serving.Request(0.00, 1, 2, 32, 0.3, 11), serving.Request(0.00, 2, 3, 16, 0.25, 12),
           serving.Request(0.02, 0, 2, 64, 0.2, 1234), serving.Request(0.03, 3, 2, 64, 0.15, 13),
           serving.Request(0.05, 4, 2, 32, 0.1, 14), serving.Request(0.06, 5, 3, 16, 0.3, 15)]
    loop = serving.ServingLoop(caps, "f32")
    _, st_alone, res_alone = loop.run([target], keep_results=True)
    loop2 = serving.ServingLoop(caps, "f32")
    rec, st_mix, res_mix = loop2.run(mix, keep_results=True)
    assert st_mix["completed"] == len(mix)
    np.testing.assert_array_equal(res_alone[0].cpu().numpy(), res_mix[0].cpu().numpy())
    assert st_mix["p99_s"] >= st_mix["p50_s"] > 0


def test_serving_matches_oracle_fp64():
    """A served FP64 double-shear-layer request equals the oracle's solve of
    the same initial state to the trajectory tolerance."""
    caps = {(2, 32): 2}
    req = serving.Request(0.0, 0, 2, 32, 0.3, 77)
    loop = serving.ServingLoop(caps, "f64")
    _, _, res = loop.run([req], keep_results=True)
    u0 = to_host(serving.initial_state(req, "f64"))
    og = ora.Grid(2, 32)
    osim = ora.Simulation(og, 0.2, ora.SSP_RK3(ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))), u0)
    osim.simulate_until(0.3)
    got = res[0].cpu().numpy()
    # the slot's last step is clamped to land on t_end, as simulate_until's is
    assert rel_l2(got, osim.u_) <= 1e-9


def test_group_active_prefix_steps_match_full_steps():
    """Steps over each simulation's active prefix give the members inside it
    exactly what full steps give, leave the members past it untouched, and
    skip a simulation whose prefix is empty."""
    dim, N, B = 2, 32, 5
    f = [random_field_hat(dim, N, seed=40 + b) for b in range(B)]
    g3 = [random_field_hat(3, 16, seed=60 + b) for b in range(2)]
    eq, ts, sim = _sim(dim, N, "f64", f)
    eq2, ts2, ref = _sim(dim, N, "f64", f)
    eq3, ts3, other = _sim(3, 16, "f64", g3)
    grp = az.Group([sim, other])
    full = az.Group([ref])
    for gg in (grp, full):
        gg.set_end(1.0)
    for s in (sim, ref):
        s.member_stop(3)
        s.member_stop(4)
    before_other = to_host(other.u())
    grp.steps(6, active=[3, 0])
    full.steps(6)
    got, want = to_host(sim.u()), to_host(ref.u())
    np.testing.assert_array_equal(got[:3], want[:3])
    np.testing.assert_array_equal(got[3:], np.stack(f[3:]))
    np.testing.assert_array_equal(to_host(other.u()), before_other)
    assert sim.state()[1] == ref.state()[1] == [6, 6, 6, 0, 0]
    assert other.state()[1] == [0, 0]
    with pytest.raises(az.AzebanError):
        grp.steps(1, active=[B + 1, 0])
