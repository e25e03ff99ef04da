"""Autotuner of the solver's launch schedule.

Two options of the K_r^{-1} operator decide how the PCG iterations reach the GPU
but not what they compute: ``checkEvery`` (iterations queued behind the device's
active flag between two host reads of the PCG state) and ``useGraphs`` (replay
the iteration bodies from captured CUDA graphs or launch them one by one).  The
best pair depends on the problem size (small N is launch-bound, large N is not)
and on the host, so it is measured: each candidate times a few K_r^{-1} actions
on a fixed vector after a warm-up, and the fastest wins.  The candidates must
produce bitwise-identical results, which the tuner checks.
"""
from __future__ import annotations

import time

import torch

from .core import QSystem, make_explicit_krinv_compact, start_vector

__all__ = ["tune_krinv_schedule"]

DEFAULT_CANDIDATES = ((2, 1), (4, 1), (8, 1), (16, 1), (4, 0))


def tune_krinv_schedule(sys: QSystem, precision="mixed", tolCG=1e-10, maxitCG=3000, candidates=DEFAULT_CANDIDATES,
                        reps=4, seed=7):
    """Return ``(best, table)``: ``best`` = {"checkEvery": c, "useGraphs": g} of the fastest
    candidate (pass it as keyword arguments to make_explicit_krinv_compact) and ``table``
    the seconds per K_r^{-1} action of every candidate."""
    v = start_vector(seed, sys.nr).reshape(-1, 1)
    ref = None
    table = []
    for every, graphs in candidates:
        op, _ = make_explicit_krinv_compact(sys, tolCG, maxitCG, precision=precision, checkEvery=int(every),
                                            useGraphs=int(graphs))
        y = op(v)  # warm-up (graph capture, workspaces)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            y = op(v)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / reps
        if ref is None:
            ref = y.clone()
        elif not torch.equal(y, ref):
            raise RuntimeError("launch-schedule candidates gave different results (checkEvery=%d, useGraphs=%d)"
                               % (every, graphs))
        table.append({"checkEvery": int(every), "useGraphs": int(graphs), "seconds": dt})
        del op
    best = min(table, key=lambda r: r["seconds"])
    return {"checkEvery": best["checkEvery"], "useGraphs": best["useGraphs"]}, table
