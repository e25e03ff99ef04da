"""Autotuner of the solver's launch schedule and pass tile shapes.

Three options of the K_r^{-1} operator decide how its work reaches the GPU but not
what a mode computes: ``checkEvery`` (PCG iterations queued behind the device's
active flag between two host reads of the PCG state), ``useGraphs`` (replay the
iteration bodies from captured CUDA graphs or launch them one by one) and
``passColumns`` (columns of the 6D grid per CTA in the pass A/C kernels of the
inner solves; alternatives are compiled for 2N = 6, 8, 10, the sizes of the
Bloch-path workload).  The best combination depends on the problem size (small N is
launch-bound, large N is not) and on the host, so it is measured: each candidate
times a few K_r^{-1} actions on a fixed vector after a warm-up, and the fastest
wins.  Candidates that differ only in the schedule must give bitwise-identical
results; a different tile shape regroups the grid reductions (their summation
order), so those results must agree to ``rtol``.  The tuner checks both.
"""
from __future__ import annotations

import time

import torch

from .core import QSystem, make_explicit_krinv_compact, start_vector

__all__ = ["tune_krinv_schedule", "DEFAULT_CANDIDATES", "COLUMN_CANDIDATES"]

DEFAULT_CANDIDATES = ((2, 1), (4, 1), (8, 1), (16, 1), (4, 0))
# passColumns values per grid length 2N (0 = the built-in default)
COLUMN_CANDIDATES = {6: (0, 4, 6), 8: (0, 2, 4), 10: (0, 2, 4)}


def tune_krinv_schedule(sys: QSystem, precision="mixed", tolCG=1e-10, maxitCG=3000, candidates=DEFAULT_CANDIDATES,
                        reps=4, seed=7, columns=None, rtol=1e-7, **opts):
    """Return ``(best, table)``: ``best`` = {"checkEvery", "useGraphs", "passColumns"} of the
    fastest candidate (pass it as keyword arguments to make_explicit_krinv_compact) and
    ``table`` the seconds per K_r^{-1} action of every candidate.  ``opts``: further K_r^{-1}
    options held fixed over the candidates (e.g. ``refineTarget``)."""
    if columns is None:
        columns = COLUMN_CANDIDATES.get(2 * sys.N, (0,))
    v = start_vector(seed, sys.nr).reshape(-1, 1)
    ref, table = {}, []
    for cols in columns:
        for every, graphs in candidates:
            op, _ = make_explicit_krinv_compact(sys, tolCG, maxitCG, precision=precision, checkEvery=int(every),
                                                useGraphs=int(graphs), passColumns=int(cols), **opts)
            y = op(v)  # warm-up (graph capture, workspaces)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                y = op(v)
            torch.cuda.synchronize()
            dt = (time.perf_counter() - t0) / reps
            if cols not in ref:
                ref[cols] = y.clone()
            elif not torch.equal(y, ref[cols]):
                raise RuntimeError("launch-schedule candidates gave different results (checkEvery=%d, useGraphs=%d, "
                                   "passColumns=%d)" % (every, graphs, cols))
            first = ref[columns[0]]
            diff = float(torch.linalg.norm(y - first) / torch.linalg.norm(first))
            if diff > rtol:
                raise RuntimeError("tile-shape candidates disagree (passColumns=%d: %.3e)" % (cols, diff))
            table.append({"checkEvery": int(every), "useGraphs": int(graphs), "passColumns": int(cols), "seconds": dt})
            del op
    best = min(table, key=lambda r: r["seconds"])
    return {k: best[k] for k in ("checkEvery", "useGraphs", "passColumns")}, table
