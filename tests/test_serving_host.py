"""Host logic of the serving loop, on CPU: the request stream, the cost
model and the slot plan (the device side is in test_gpu_serving.py)."""

import numpy as np
import pytest

from azeban_b200 import serving as sv


def test_member_step_bytes_is_the_pass_model():
    # 3-D 256^3 FP32: 1,991.0 M complex elements per member-step (five
    # passes of one read and one write, x3 right-hand sides, plus the two
    # state reads of the stage combinations), 8 bytes each
    assert sv.member_step_bytes(3, 256, "f32") == pytest.approx(15.93e9, rel=2e-3)
    assert sv.member_step_bytes(3, 256, "f64") == pytest.approx(2 * sv.member_step_bytes(3, 256, "f32"))
    # cost grows with N^d (times the log-free pass model)
    assert sv.member_step_bytes(2, 128) / sv.member_step_bytes(2, 64) == pytest.approx(4.0, rel=0.05)
    assert sv.member_step_bytes(3, 128) / sv.member_step_bytes(3, 64) == pytest.approx(8.0, rel=0.05)


def test_poisson_stream_rate_classes_and_seed():
    a = sv.poisson_stream(200.0, 60.0, seed=11)
    b = sv.poisson_stream(200.0, 60.0, seed=11)
    assert [(r.arrival, r.dim, r.N, r.t_end, r.seed) for r in a] == \
           [(r.arrival, r.dim, r.N, r.t_end, r.seed) for r in b]
    assert abs(len(a) - 12000) < 5 * np.sqrt(12000)
    t = np.array([r.arrival for r in a])
    assert np.all(np.diff(t) > 0) and t[-1] <= 60.0
    assert all(0.25 <= r.t_end <= 1.0 for r in a)
    assert len({r.rid for r in a}) == len(a)
    # class frequencies proportional to 1/cost
    cost = np.array([sv.member_step_bytes(d, n) for d, n in sv.CLASSES])
    p = (1 / cost) / (1 / cost).sum()
    counts = np.array([sum(1 for r in a if (r.dim, r.N) == c) for c in sv.CLASSES])
    expect = p * len(a)
    big = expect > 50
    assert np.all(np.abs(counts[big] - expect[big]) < 5 * np.sqrt(expect[big]))


def test_plan_capacities_fit_the_budget():
    budget = int(40e9)
    caps = sv.plan_capacities(budget, "f32")
    assert set(caps) == set(sv.CLASSES)
    used = sum(sv.pool_bytes(d, n, "f32", c) for (d, n), c in caps.items())
    assert used <= budget
    # equal weights: each class gets about the same share of the budget
    shares = [sv.pool_bytes(d, n, "f32", c) for (d, n), c in caps.items()]
    per = [sv.pool_bytes(d, n, "f32", 1) for (d, n) in caps]
    assert all(budget / len(caps) - s < p for s, p in zip(shares, per))
    # a class too large for its share still gets the minimum
    tiny = sv.plan_capacities(int(1e9), "f32", minimum=1)
    assert tiny[(3, 256)] == 1
    weighted = sv.plan_capacities(budget, "f32", weights={c: (4.0 if c == (2, 64) else 1.0) for c in sv.CLASSES})
    assert weighted[(2, 64)] > caps[(2, 64)]
