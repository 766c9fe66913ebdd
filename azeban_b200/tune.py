"""Autotuner for the radix plans of the transform passes.

For one workload (dimension, N, padded M, precision, batch) it runs SSP-RK3
steps of a Simulation with every kernel variant, times each pass with the
library's per-pass CUDA events (az_profile_*), and keeps, for each pass kind
(column passes, contiguous-axis product pass, epilogue pass), the fastest
variant.
Results go into a JSON tuning table that ``azeban_b200`` loads at import
(``tuning.json`` beside this file) and applies with az_tune_set.

The reference's closest counterpart picks the padded FFT size from a
benchmark file (src/azeban/operations/fft.cpp:63-108).

Usage on a GPU: ``python -m azeban_b200.tune --out azeban_b200/tuning.json``.
"""

from __future__ import annotations

import argparse
import ctypes as ct
import json
import os

import torch

from . import _lib
from .core import SSP_RK3, Grid, IncompressibleEuler, Simulation, make_viscosity, precision_code

TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
KIND_PASSES = {0: (0, 1, 3), 1: (2,), 2: (4,)}  # pass ids per tuned kind (+3 for 2-D solves)
VISC = {"type": "Smooth Cutoff", "eps": 0.05}


# Kernel variants: bit 0 picks the radix plan (0 std, 1 wide); bit 1 picks
# the two-tile column kernel (column passes) or the bulk-copy kernel
# (contiguous-axis pass).  Runs 4-7 time the fused product pass (bit 2 of
# the contiguous-axis variant; its bit 1 is then the inverse transform's
# plan); the other passes repeat runs 0-3 there.  The epilogue has plan
# variants only.
RUNS = (0, 1, 2, 3, 4, 5, 6, 7)


def _kind_variant(kind0: int, run: int) -> int:
    if kind0 == 1:
        return run
    return run & 3 if kind0 == 0 else run & 1


def _set_all(prec: int, L: int, run: int) -> None:
    for kind in range(6):
        _lib.check(_lib.lib.az_tune_set(prec, L, kind, _kind_variant(kind % 3, run)))


def _time_passes(eq, u, reps):
    """Per-pass times averaged over SSP-RK3 steps of a Simulation: the first
    pass of stage 1 reads the caller-layout state and those of stages 2 and 3
    the stepper's component-innermost buffers, as in every run (a plain dudt
    times the first layout only)."""
    sim = Simulation(eq.grid, 0.2, SSP_RK3(eq), u)
    sim.steps(2)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.az_profile_enable(1))
    sim.steps(reps)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.az_profile_enable(0))
    ms = (ct.c_double * 5)()
    by = (ct.c_double * 5)()
    nl = (ct.c_longlong * 5)()
    _lib.check(_lib.lib.az_profile_read(ms, by, nl, 5))
    return [ms[i] / nl[i] if nl[i] else 0.0 for i in range(5)]


def autotune(dim: int, N: int, precision="f32", batch: int = 1, M: int | None = None, reps: int = 5):
    """Measures both plan variants of one workload and applies the winners;
    returns the table entries."""
    prec = precision_code(precision)
    g = Grid(dim, N, M)
    L = g.N_phys_pad
    visc = make_viscosity(VISC, g)
    shape = ((batch,) if batch > 1 else ()) + g.shape_fourier(dim)
    cdt = torch.complex128 if prec == 0 else torch.complex64
    gen = torch.Generator(device="cuda").manual_seed(1234)
    u = (torch.randn(shape, dtype=cdt, device="cuda", generator=gen) * (N ** dim) * 1e-3).contiguous()
    per_run = {}
    for run in RUNS:
        _set_all(prec, L, run)
        eq = IncompressibleEuler(g, visc, precision, batch)
        per_run[run] = _time_passes(eq, u, reps)
        del eq
    entries = []
    kbase = 3 if dim == 2 else 0
    for kind0, passes in KIND_PASSES.items():
        kind = kbase + kind0
        t = {}
        for run, times in per_run.items():
            v = _kind_variant(kind0, run)
            ms = sum(times[p] for p in passes)
            t[v] = min(t.get(v, ms), ms)
        if all(x == 0.0 for x in t.values()):
            continue
        best = min(t, key=t.get)
        _lib.check(_lib.lib.az_tune_set(prec, L, kind, best))
        entries.append({"precision": prec, "L": L, "kind": kind, "variant": best,
                        "workload": f"{dim}-D N={N} M={L} batch={batch}",
                        "ms_per_rhs": {str(v): t[v] for v in sorted(t)}})
    return entries


def load_table(path: str = TABLE) -> int:
    """Applies a saved tuning table; returns the number of entries."""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        entries = json.load(f)
    n = 0
    for e in entries:
        if _lib.lib.az_tune_set(int(e["precision"]), int(e["L"]), int(e["kind"]), int(e["variant"])) == 0:
            n += 1
    return n


WORKLOADS = [
    # (dim, N, precision, batch): the configs' sizes
    (3, 256, "f32", 4), (3, 256, "f64", 1), (3, 128, "f32", 1), (3, 128, "f64", 1),
    (3, 64, "f32", 4), (3, 64, "f64", 4), (3, 512, "f32", 1),
    (2, 128, "f32", 64), (2, 256, "f32", 32), (2, 512, "f32", 16), (2, 64, "f64", 1),
    (2, 64, "f32", 64), (2, 512, "f64", 4),
]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args(argv)
    table = {}
    for dim, N, prec, batch in WORKLOADS:
        for e in autotune(dim, N, prec, batch, reps=args.reps):
            table[(e["precision"], e["L"], e["kind"])] = e
            print(json.dumps(e), flush=True)
    with open(args.out, "w") as f:
        json.dump(list(table.values()), f, indent=1)


if __name__ == "__main__":
    main()
