"""Result and checkpoint formats of the reference's experiment drivers, for B200 results.

The reference stores one checkpoint per Bloch point (``qres`` + ``signature``, reused
only when the signature matches and the stored solve converged: exp4/run_exp4_medium.m:37-62)
and writes CSV tables whose column names are MATLAB ``writetable`` variable names
(exp4/write_exp4_outputs.m:5-41, exp1/run_fig1bc_method.m:185-206).  This module writes
the same records from this library's solves so that the reference's ``load`` calls and
plotting scripts read them: checkpoints as MAT-file version 5 (``scipy.io.savemat``;
MATLAB's ``load`` reads it -- the reference's ``-v7.3`` is HDF5, for which no writer is
installed here), with the reference's struct and field names.
"""
from __future__ import annotations

import csv
import os
from dataclasses import dataclass, field

import numpy as np

__all__ = ["exp4_checkpoint_signature", "signatures_equal_exp4", "QResult", "save_q_checkpoint",
           "load_q_checkpoint", "write_exp4_spectrum_csv", "write_exp4_timing_csv",
           "write_exp4_selected_csv", "write_fig1bc_csv", "make_exp1bc_signature"]

SIGNATURE_FIELDS = ("version", "medium", "modelType", "materialParameters", "gpuProduction", "N",
                    "pathSubintervals", "nev", "p", "tolLanczos", "tolCG", "pointIndex", "q", "selectedMode")


def exp4_checkpoint_signature(numerics: dict, medium: str, modelType: str, materialParameters, N: int,
                              pathSubintervals: int, nev: int, p: int, tolLanczos: float, tolCG: float,
                              q, pointIndex: int, selectedMode: int = 0) -> dict:
    """exp4/exp4_checkpoint_signature.m:1-23 -- the configuration subset that makes a
    q-point checkpoint valid (``numerics`` stands for the struct of problem/solver/mass
    settings the reference nests there)."""
    return {"numerics": dict(numerics), "version": 6, "medium": str(medium), "modelType": str(modelType),
            "materialParameters": np.asarray(materialParameters, dtype=np.float64).reshape(1, -1),
            "gpuProduction": True, "N": int(N), "pathSubintervals": int(pathSubintervals), "nev": int(nev),
            "p": int(p), "tolLanczos": float(tolLanczos), "tolCG": float(tolCG), "pointIndex": int(pointIndex),
            "q": np.asarray(q, dtype=np.float64).reshape(1, 3), "selectedMode": int(selectedMode)}


def _scalar(v):
    a = np.asarray(v)
    return a.reshape(-1)[0].item() if a.size == 1 else a


def _numerics_equal(a, b):
    if isinstance(a, dict) or isinstance(b, dict):
        if not (isinstance(a, dict) and isinstance(b, dict)) or set(a) != set(b):
            return False
        return all(_numerics_equal(a[k], b[k]) for k in a)
    xa, xb = np.asarray(a), np.asarray(b)
    if xa.dtype.kind in "USO" or xb.dtype.kind in "USO":
        return str(_scalar(a)) == str(_scalar(b))
    return xa.shape == xb.shape and bool(np.array_equal(xa, xb, equal_nan=True))


def signatures_equal_exp4(a: dict, b: dict) -> bool:
    """exp4/signatures_equal_exp4.m:1-24 -- strict compatibility of two signatures."""
    if any(k not in a or k not in b for k in SIGNATURE_FIELDS):
        return False
    if "numerics" not in a or "numerics" not in b or not _numerics_equal(a["numerics"], b["numerics"]):
        return False
    ma = np.asarray(a["materialParameters"], dtype=np.float64).reshape(-1)
    mb = np.asarray(b["materialParameters"], dtype=np.float64).reshape(-1)
    if ma.size != mb.size:
        return False
    qa = np.asarray(a["q"], dtype=np.float64).reshape(-1)
    qb = np.asarray(b["q"], dtype=np.float64).reshape(-1)
    return (_scalar(a["version"]) == _scalar(b["version"]) and str(_scalar(a["medium"])) == str(_scalar(b["medium"]))
            and str(_scalar(a["modelType"])) == str(_scalar(b["modelType"]))
            and bool(_scalar(a["gpuProduction"])) == bool(_scalar(b["gpuProduction"]))
            and (ma.size == 0 or np.max(np.abs(ma - mb)) < 1e-13)
            and all(_scalar(a[k]) == _scalar(b[k]) for k in ("N", "pathSubintervals", "nev", "p", "tolLanczos",
                                                              "tolCG", "pointIndex", "selectedMode"))
            and qa.size == qb.size and np.max(np.abs(qa - qb)) < 1e-14)


@dataclass
class QResult:
    """The ``qres`` struct of exp4/solve_exp4_qpoint.m:48-64 (host arrays)."""
    pointIndex: int
    q: np.ndarray
    lam: np.ndarray                        # stored as field ``lambda``
    outerSteps: int
    wallTimeSeconds: float
    converged: bool
    numConverged: int
    maxRelativeInverseRitzResidual: float
    cgAverageIterations: float
    cgMaxIterations: int = 0
    cgMaxRelativeResidual: float = 0.0
    finalRestart: int = 0
    selectedMode: int = 0
    selectedLambda: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))
    Xselected: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))

    def to_struct(self) -> dict:
        d = {k: getattr(self, k) for k in self.__dataclass_fields__ if k != "lam"}
        d["lambda"] = np.asarray(self.lam, dtype=np.float64).reshape(-1, 1)
        d["q"] = np.asarray(self.q, dtype=np.float64).reshape(3, 1)
        d["converged"] = bool(self.converged)
        return d

    @classmethod
    def from_struct(cls, s: dict) -> "QResult":
        g = lambda k, dflt=None: s[k] if k in s else dflt  # noqa: E731
        return cls(pointIndex=int(_scalar(g("pointIndex"))), q=np.asarray(g("q"), dtype=np.float64).reshape(-1),
                   lam=np.asarray(g("lambda"), dtype=np.float64).reshape(-1), outerSteps=int(_scalar(g("outerSteps"))),
                   wallTimeSeconds=float(_scalar(g("wallTimeSeconds"))), converged=bool(_scalar(g("converged"))),
                   numConverged=int(_scalar(g("numConverged"))),
                   maxRelativeInverseRitzResidual=float(_scalar(g("maxRelativeInverseRitzResidual"))),
                   cgAverageIterations=float(_scalar(g("cgAverageIterations"))),
                   cgMaxIterations=int(_scalar(g("cgMaxIterations", 0))),
                   cgMaxRelativeResidual=float(_scalar(g("cgMaxRelativeResidual", 0.0))),
                   finalRestart=int(_scalar(g("finalRestart", 0))), selectedMode=int(_scalar(g("selectedMode", 0))),
                   selectedLambda=np.asarray(g("selectedLambda", np.zeros((0, 0)))),
                   Xselected=np.asarray(g("Xselected", np.zeros((0, 0)))))


def _loadmat_struct(obj):
    """scipy's mat_struct (struct_as_record=False) -> nested dict."""
    if hasattr(obj, "_fieldnames"):
        return {k: _loadmat_struct(getattr(obj, k)) for k in obj._fieldnames}
    return obj


def save_q_checkpoint(path: str, qres: QResult, signature: dict) -> None:
    """``save(ckFile,'qres','signature')`` of exp4/run_exp4_medium.m:83-86, as MAT-file v5."""
    from scipy.io import savemat
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    savemat(path, {"qres": qres.to_struct(), "signature": signature}, do_compression=True,
            long_field_names=True, oned_as="column")


def load_q_checkpoint(path: str, signature: dict, tolLanczos: float):
    """The reuse rule of exp4/run_exp4_medium.m:41-62: the stored qres if the file exists,
    its signature equals ``signature``, the selected mode matches (with its eigenvector
    stored when one is selected) and the stored solve converged with
    maxRelativeInverseRitzResidual <= tolLanczos; otherwise None."""
    from scipy.io import loadmat
    if not os.path.exists(path):
        return None
    C = loadmat(path, struct_as_record=False, squeeze_me=True)
    if "qres" not in C or "signature" not in C:
        return None
    qs, sig = _loadmat_struct(C["qres"]), _loadmat_struct(C["signature"])
    q = QResult.from_struct(qs)
    sel = int(signature["selectedMode"])
    mode_ok = q.selectedMode == sel and (sel == 0 or (np.size(q.Xselected) > 0 and np.size(q.selectedLambda) > 0))
    resid_ok = q.converged and np.isfinite(q.maxRelativeInverseRitzResidual) and \
        q.maxRelativeInverseRitzResidual <= tolLanczos
    if signatures_equal_exp4(sig, signature) and mode_ok and resid_ok:
        return q
    return None


def _write_table(path, header, rows):
    """MATLAB ``writetable`` layout: a header of variable names, one row per record."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(header)
        for r in rows:
            w.writerow(["%.17g" % v if isinstance(v, (float, np.floating)) else v for v in r])


def write_exp4_spectrum_csv(path, qPlot, lambdaPlot):
    """exp4/write_exp4_outputs.m:5-17: columns point, mode, q1, q2, q3, lambda (qPlot 3 x P,
    lambdaPlot nev x P, one row per plotted point and mode)."""
    qPlot = np.asarray(qPlot, dtype=np.float64).reshape(3, -1)
    lam = np.asarray(lambdaPlot, dtype=np.float64)
    rows = [(ip + 1, j + 1, qPlot[0, ip], qPlot[1, ip], qPlot[2, ip], lam[j, ip])
            for ip in range(qPlot.shape[1]) for j in range(lam.shape[0])]
    _write_table(path, ["point", "mode", "q1", "q2", "q3", "lambda"], rows)


def write_exp4_selected_csv(path, selected):
    """exp4/write_exp4_outputs.m:19-30: one row per selected mode (dicts with label,
    pointIndex, modeIndex, lambda6D, lambdaLWRQ, deltaLambda, eta3D, nuLWRQ, lwrqIdentityError)."""
    rows = [(s["label"], s["pointIndex"], s["modeIndex"], s["lambda6D"], s["lambdaLWRQ"], s["deltaLambda"],
             s["eta3D"], s["nuLWRQ"], s["lwrqIdentityError"]) for s in selected]
    _write_table(path, ["label", "point", "mode", "lambda6D", "lambdaLWRQ", "relDiff", "eta3D", "nuLWRQ",
                        "identity"], rows)


def write_exp4_timing_csv(path, qres_list, loadedFromCheckpoint):
    """exp4/write_exp4_outputs.m:32-40: qpoint, wall_s, outer, mhat_avg, max_ritz, from_checkpoint."""
    rows = [(i + 1, q.wallTimeSeconds, q.outerSteps, q.cgAverageIterations, q.maxRelativeInverseRitzResidual,
             int(bool(c))) for i, (q, c) in enumerate(zip(qres_list, loadedFromCheckpoint))]
    _write_table(path, ["qpoint", "wall_s", "outer", "mhat_avg", "max_ritz", "from_checkpoint"], rows)


def write_fig1bc_csv(path, scaleResults):
    """exp1/run_fig1bc_method.m:185-206 (write_fig1bc_csv): one row per N with N, NF, status,
    lin, wall, observedLin, observedWall, outer, setup, plateau, maxPlateau, gpuFree (GiB);
    missing fields are written as NaN, as the reference initialises them."""
    nan = float("nan")
    rows = []
    for r in scaleResults:
        g = lambda *ks: next((float(r[k]) for k in ks if k in r), nan)  # noqa: E731
        gpu = r.get("gpuAvailableAfterMethodSetupBytes")
        rows.append((int(r["N"]), int(r["NF"]), str(r["status"]), g("plotLinearIterations"), g("plotWallSeconds"),
                     g("observedLinearIterations", "totalLinearSolverIterations"),
                     g("observedWallSeconds", "solverWallSeconds"), g("outerSteps"), g("methodSetupSeconds"),
                     g("totalPlateauAccepts"), g("maxPlateauAcceptedResidual"),
                     nan if gpu is None else float(gpu) / 2 ** 30))
    _write_table(path, ["N", "NF", "status", "lin", "wall", "observedLin", "observedWall", "outer", "setup",
                        "plateau", "maxPlateau", "gpuFree"], rows)


def make_exp1bc_signature(method: str, N: int, settings: dict) -> dict:
    """exp1/make_exp1bc_signature.m:1-44: version 6 for method A, 4 for B/C, kind
    'fig1bc-hybrid-lowmem', method, N and the solver settings (``settings`` holds the
    remaining fields under the reference's names: numEig, P, T, epsC, alpha, q, tolKr,
    tolMhat, lanczosTol, ...)."""
    m = str(method).upper()
    s = {"version": 6 if m == "A" else 4, "kind": "fig1bc-hybrid-lowmem", "method": m, "N": int(N)}
    for k, v in settings.items():
        s[k] = np.asarray(v, dtype=np.float64) if isinstance(v, (list, tuple)) else v
    return s
