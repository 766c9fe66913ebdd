"""Continuous-batching serving loop for ensemble solves.

Requests (one solve each: a 2-D double shear layer or a 3-D fractional
Brownian field, an N, an end time and a seed) arrive over time.  Each size
class (dim, N) owns a pool of slots: one batched IncompressibleEuler /
SSP_RK3 / Simulation whose members are the slots.  All pools are advanced
together, one SSP-RK3 step per tick (``Group``): each pool's step launches
over its lowest slots only, up to the highest slot in use (slots are handed
out lowest first), so a tick costs what the admitted solves cost, not what
every slot of every pool would; a slot whose clock reached its end is skipped
on the device.  Between ticks the
host admits waiting requests into free slots (their state is generated on the
device straight into the slot) and retires finished ones, so requests that
arrive while others run join at the next step and their work overlaps.

Admission is by HBM footprint: the pools' capacities are fixed at start-up
from a memory budget (``plan_capacities``), and a request waits until its
class has a free slot.  Each member's arithmetic does not depend on the other
members (every kernel works per member), so a result is the same alone and in
the mix.

The reference's closest counterpart is its per-sample loop
(src/azeban/run_from_config.cpp:81-102) and the split of ensemble samples over
ranks (src/azeban.cpp:131-152).
"""

from __future__ import annotations

import heapq
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import init as azinit
from .core import SSP_RK3, Grid, Group, IncompressibleEuler, Simulation, make_viscosity

VISC = {"type": "Smooth Cutoff", "eps": 0.05}
CLASSES = [(2, 64), (2, 128), (2, 256), (2, 512), (3, 64), (3, 128), (3, 256)]


def member_step_bytes(dim: int, N: int, precision: str = "f32") -> float:
    """Algorithmic HBM bytes of one SSP-RK3 step of one member (the pass
    model: one read and one write of every pass's input and output)."""
    M, Nh = 3 * N // 2, N // 2 + 1
    cs = 8 if precision == "f32" else 16
    if dim == 3:
        rhs = (3 * (N * N * Nh + M * N * Nh) + 3 * (M * N * Nh + M * M * Nh) + 9 * M * M * Nh
               + 6 * (M * M * Nh + M * N * Nh) + 6 * M * N * Nh + 3 * N * N * Nh * 2.67)
    else:
        rhs = 2 * (N * Nh + M * Nh) + 5 * M * Nh + 3 * M * Nh + 2 * N * Nh * 2.67
    return 3 * rhs * cs


def pool_bytes(dim: int, N: int, precision: str, capacity: int) -> int:
    """Device bytes of one pool: workspace plus four state arrays (u, u1, u2
    and the simulation's copy), per member times capacity."""
    M, Nh = 3 * N // 2, N // 2 + 1
    cs = 8 if precision == "f32" else 16
    if dim == 3:
        work = (6 * M * N * Nh + 3 * M * M * Nh + 6 * M * M * Nh) * cs
        state = 3 * N * N * Nh * cs
    else:
        work = (2 * M * Nh + 3 * M * Nh) * cs
        state = 2 * N * Nh * cs
    return int(capacity * (work + 4 * state))


def plan_capacities(budget_bytes: int, precision: str, weights=None, minimum: int = 1) -> dict:
    """Slots per class: the budget split in proportion to each class's
    expected concurrency weight, at least `minimum` slots per class."""
    weights = weights or {c: 1.0 for c in CLASSES}
    total_w = sum(weights.values())
    caps = {}
    for c in CLASSES:
        share = budget_bytes * weights[c] / total_w
        per = pool_bytes(c[0], c[1], precision, 1)
        caps[c] = max(minimum, int(share // per))
    return caps


@dataclass(order=True)
class Request:
    arrival: float
    rid: int = field(compare=False)
    dim: int = field(compare=False)
    N: int = field(compare=False)
    t_end: float = field(compare=False)
    seed: int = field(compare=False)


def poisson_stream(rate: float, duration: float, seed: int = 0, classes=CLASSES, precision: str = "f32"):
    """Poisson arrivals at `rate` per second for `duration` seconds; class
    probability proportional to 1/cost (cost = member-step bytes), t_end ~
    U[0.25, 1], a seed per request."""
    rng = np.random.default_rng(seed)
    cost = np.array([member_step_bytes(d, n, precision) for d, n in classes])
    p = (1.0 / cost) / (1.0 / cost).sum()
    reqs = []
    t = 0.0
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        c = classes[rng.choice(len(classes), p=p)]
        reqs.append(Request(t, rid, c[0], c[1], float(rng.uniform(0.25, 1.0)), int(rng.integers(0, 2**31))))
        rid += 1
    return reqs


def initial_state(req: Request, precision: str):
    """The request's initial spectral state, generated on the device."""
    if req.dim == 2:
        phase = float(np.random.default_rng(req.seed).uniform(0.0, 2 * math.pi))
        return azinit.double_shear_layer(req.N, math.pi / 15, 0.05, [phase], precision)[0]
    return azinit.fractional_brownian(3, req.N, 0.75, req.seed, precision)


class ServingLoop:
    def __init__(self, capacities: dict, precision: str = "f32", C: float = 0.2):
        self.precision = precision
        self.C = C
        self.pools = {}
        sims = []
        for cls, cap in capacities.items():
            if cap < 1:
                continue
            dim, N = cls
            g = Grid(dim, N)
            eq = IncompressibleEuler(g, make_viscosity(VISC, g), precision, batch=cap)
            ts = SSP_RK3(eq)
            zeros = torch.zeros((cap,) + g.shape_fourier(dim), dtype=eq.cdtype, device="cuda")
            sim = Simulation(g, C, ts, zeros)
            for b in range(cap):
                sim.member_stop(b)
            # free slots as a min-heap: admissions take the lowest slot, which
            # keeps the pool's active prefix short
            self.pools[cls] = {"eq": eq, "ts": ts, "sim": sim, "free": list(range(cap)),
                               "active": {}, "cap": cap}
            sims.append(sim)
        torch.cuda.synchronize()
        self.group = Group(sims)

    def run(self, requests, keep_results: bool = False, wall_limit: float | None = None):
        """Serves `requests` (their arrival times are seconds from the start);
        returns per-request records and aggregate statistics."""
        pending = sorted(requests)
        queue = []  # admitted in arrival order per class
        records = {}
        results = {}
        steps_done = 0
        member_steps = 0
        t0 = time.perf_counter()
        i = 0
        while i < len(pending) or queue or any(p["active"] for p in self.pools.values()):
            now = time.perf_counter() - t0
            if wall_limit is not None and now > wall_limit:
                break
            while i < len(pending) and pending[i].arrival <= now:
                heapq.heappush(queue, pending[i])
                i += 1
            # admit FIFO while slots are free
            waiting = []
            while queue:
                r = heapq.heappop(queue)
                pool = self.pools.get((r.dim, r.N))
                if pool is None:
                    raise ValueError(f"no pool for class {(r.dim, r.N)}")
                if pool["free"]:
                    slot = heapq.heappop(pool["free"])
                    u0 = initial_state(r, self.precision)
                    pool["sim"].member_start(slot, u0, r.t_end)
                    pool["active"][slot] = r
                    records[r.rid] = {"arrival": r.arrival, "admitted": time.perf_counter() - t0,
                                      "class": (r.dim, r.N), "t_end": r.t_end}
                else:
                    waiting.append(r)
            for r in waiting:
                heapq.heappush(queue, r)
            if not any(p["active"] for p in self.pools.values()):
                if i < len(pending):
                    time.sleep(max(0.0, min(0.01, pending[i].arrival - (time.perf_counter() - t0))))
                continue
            self.group.steps(1, active=[max(p["active"]) + 1 if p["active"] else 0
                                        for p in self.pools.values()])
            steps_done += 1
            member_steps += sum(len(p["active"]) for p in self.pools.values())
            # retire finished members
            for cls, pool in self.pools.items():
                if not pool["active"]:
                    continue
                times, nsteps, _ = pool["sim"].state()
                done = [s for s in pool["active"] if times[s] >= pool["active"][s].t_end]
                for slot in done:
                    r = pool["active"].pop(slot)
                    rec = records[r.rid]
                    rec["finish"] = time.perf_counter() - t0
                    rec["steps"] = int(nsteps[slot])
                    if keep_results:
                        results[r.rid] = pool["sim"].u()[slot].clone()
                    pool["sim"].member_stop(slot)
                    heapq.heappush(pool["free"], slot)
        wall = time.perf_counter() - t0
        lat = np.array([r["finish"] - r["arrival"] for r in records.values() if "finish" in r])
        done_steps = sum(r.get("steps", 0) for r in records.values())
        stats = {
            "requests": len(requests), "completed": int(len(lat)), "wall_s": wall, "ticks": steps_done,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "member_steps": done_steps, "member_steps_per_s": done_steps / wall if wall > 0 else None,
        }
        return records, stats, results
