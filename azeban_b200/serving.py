"""Continuous-batching serving loop for ensemble solves.

Requests (one solve each: a 2-D double shear layer or a 3-D fractional
Brownian field, an N, an end time and a seed) arrive over time.  Each size
class (dim, N) owns a pool of slots: one batched IncompressibleEuler /
SSP_RK3 / Simulation whose members are the slots, stepped on its own CUDA
stream.  The pools advance independently: as soon as a pool's step is done
the host retires its finished members, admits waiting requests of its class
into free slots (their state is generated on the device straight into the
slot) and launches its next SSP-RK3 step, so a small solve does not wait for
the step of a large one, and the pools' work overlaps on the device.  A
pool's step launches over its lowest slots only, up to the highest slot in
use (slots are handed out lowest first), so it costs what the admitted
solves cost, not what every slot would; a slot whose clock reached its end
is skipped on the device.  Two measures keep small solves from queueing
behind large ones: the pools of cheap classes step on high-priority streams
(their few CTAs are scheduled ahead of a large solve's as SMs free up), and a
pool launches several steps at once when its step is cheap (up to
``STEP_BYTES`` of modelled HBM traffic per launch), so the host loop is not
what paces it; a member that reaches its end inside such a launch is skipped
for the rest of it (its last step lands on its end time).

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
# Modelled HBM bytes of one launch of a pool's steps (the steps per launch
# are chosen to stay near it), and the per-member-step cost below which a
# class's pool gets a high-priority stream.
STEP_BYTES = 2e9
CHEAP_BYTES = 1e9


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
        # phase ~ U[0, 2 pi) from the counter-based stream (seed, 0), drawn on the device
        return azinit.double_shear_layer(req.N, math.pi / 15, 0.05, None, precision, seed=req.seed)[0]
    return azinit.fractional_brownian(3, req.N, 0.75, req.seed, precision)


class ServingLoop:
    def __init__(self, capacities: dict, precision: str = "f32", C: float = 0.2):
        self.precision = precision
        self.C = C
        self.pools = {}
        for cls, cap in capacities.items():
            if cap < 1:
                continue
            dim, N = cls
            g = Grid(dim, N)
            eq = IncompressibleEuler(g, make_viscosity(VISC, g), precision, batch=cap)
            ts = SSP_RK3(eq)
            zeros = torch.zeros((cap,) + g.shape_fourier(dim), dtype=eq.cdtype, device="cuda")
            cheap = member_step_bytes(dim, N, precision) < CHEAP_BYTES
            stream = torch.cuda.Stream(priority=-1 if cheap else 0)
            with torch.cuda.stream(stream):
                sim = Simulation(g, C, ts, zeros)
                for b in range(cap):
                    sim.member_stop(b)
            # free slots as a min-heap: admissions take the lowest slot, which
            # keeps the pool's active prefix short
            self.pools[cls] = {"eq": eq, "ts": ts, "sim": sim, "free": list(range(cap)),
                               "active": {}, "cap": cap, "stream": stream, "group": Group([sim]),
                               "step_bytes": member_step_bytes(dim, N, precision)}
        torch.cuda.synchronize()
        self._warm()

    def _warm(self):
        """Captures every prefix step graph of every pool (steps over slots
        that are all stopped change nothing) and runs each class's
        initial-data generator once, so no capture or first-use cost lands
        inside the serving loop."""
        for (dim, N), pool in self.pools.items():
            st = pool["stream"]
            n = 1
            while True:
                pool["group"].steps(1, stream=st, active=[min(n, pool["cap"])])
                if n >= pool["cap"]:
                    break
                n *= 2
            with torch.cuda.stream(st):
                initial_state(Request(0.0, -1, dim, N, 1.0, 0), self.precision)
        torch.cuda.synchronize()

    def run(self, requests, keep_results: bool = False, wall_limit: float | None = None):
        """Serves `requests` (their arrival times are seconds from the start);
        returns per-request records and aggregate statistics ("ticks" counts
        pool steps)."""
        pending = sorted(requests)
        queues = {cls: [] for cls in self.pools}  # waiting requests per class, by arrival
        inflight = {cls: None for cls in self.pools}  # event of the pool's step in flight
        records = {}
        results = {}
        steps_done = 0
        t0 = time.perf_counter()
        i = 0
        while True:
            now = time.perf_counter() - t0
            if wall_limit is not None and now > wall_limit:
                break
            while i < len(pending) and pending[i].arrival <= now:
                r = pending[i]
                i += 1
                if (r.dim, r.N) not in self.pools:
                    raise ValueError(f"no pool for class {(r.dim, r.N)}")
                heapq.heappush(queues[(r.dim, r.N)], r)
            busy = False
            for cls, pool in self.pools.items():
                ev = inflight[cls]
                if ev is not None:
                    if not ev.query():
                        busy = True
                        continue
                    inflight[cls] = None
                    self._retire(pool, records, results, keep_results, t0)
                self._admit(pool, queues[cls], records, t0)
                if pool["active"]:
                    st = pool["stream"]
                    k = int(STEP_BYTES // (pool["step_bytes"] * len(pool["active"])))
                    k = max(1, min(16, k))
                    with torch.cuda.stream(st):
                        pool["group"].steps(k, stream=st, active=[max(pool["active"]) + 1])
                        ev = torch.cuda.Event()
                        ev.record(st)
                    inflight[cls] = ev
                    steps_done += 1
                    busy = True
            if not busy:
                if i >= len(pending) and not any(queues.values()):
                    break
                if i < len(pending):
                    time.sleep(max(0.0, min(0.01, pending[i].arrival - (time.perf_counter() - t0))))
        wall = time.perf_counter() - t0
        torch.cuda.synchronize()  # the kept results were copied on the pools' streams
        lat = np.array([r["finish"] - r["arrival"] for r in records.values() if "finish" in r])
        done_steps = sum(r.get("steps", 0) for r in records.values())
        stats = {
            "requests": len(requests), "completed": int(len(lat)), "wall_s": wall, "ticks": steps_done,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "member_steps": done_steps, "member_steps_per_s": done_steps / wall if wall > 0 else None,
        }
        # per class: time to solution, and the part of it spent waiting for a slot
        per = {}
        for cls in sorted({r["class"] for r in records.values() if "finish" in r}):
            rs = [r for r in records.values() if "finish" in r and r["class"] == cls]
            tot = np.array([r["finish"] - r["arrival"] for r in rs])
            wait = np.array([r["admitted"] - r["arrival"] for r in rs])
            per[f"{cls[0]}D-{cls[1]}"] = {"n": len(rs), "p50_s": float(np.percentile(tot, 50)),
                                          "p99_s": float(np.percentile(tot, 99)),
                                          "wait_p99_s": float(np.percentile(wait, 99))}
        stats["per_class"] = per
        return records, stats, results

    def _admit(self, pool, queue, records, t0):
        """Waiting requests of the pool's class into its free slots (lowest
        first), on the pool's stream."""
        st = pool["stream"]
        while queue and pool["free"]:
            r = heapq.heappop(queue)
            slot = heapq.heappop(pool["free"])
            with torch.cuda.stream(st):
                u0 = initial_state(r, self.precision)
                pool["sim"].member_start(slot, u0, r.t_end, stream=st)
            pool["active"][slot] = r
            records[r.rid] = {"arrival": r.arrival, "admitted": time.perf_counter() - t0,
                              "class": (r.dim, r.N), "t_end": r.t_end}

    def _retire(self, pool, records, results, keep_results, t0):
        """Members of the pool whose clock reached their end: recorded, their
        slots freed (the pool's step has completed)."""
        st = pool["stream"]
        times, nsteps, _ = pool["sim"].state(stream=st)
        for slot in [s for s in pool["active"] if times[s] >= pool["active"][s].t_end]:
            r = pool["active"].pop(slot)
            rec = records[r.rid]
            rec["finish"] = time.perf_counter() - t0
            rec["steps"] = int(nsteps[slot])
            if keep_results:
                with torch.cuda.stream(st):
                    results[r.rid] = pool["sim"].u()[slot].clone()
            pool["sim"].member_stop(slot, stream=st)
            heapq.heappush(pool["free"], slot)
