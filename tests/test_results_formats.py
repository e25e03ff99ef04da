"""CPU tests of the result/checkpoint formats (exp4/exp4_checkpoint_signature.m,
exp4/run_exp4_medium.m:37-62, exp4/write_exp4_outputs.m, exp1/run_fig1bc_method.m:185-206):
a checkpoint written here loads through scipy.io.loadmat with the reference's struct and
field names, is reused only under the reference's rule, and the CSV tables carry the
reference's column names."""
import csv

import numpy as np
from scipy.io import loadmat

from fame_b200 import results as R


def _sig(q=(0.1, 0.2, 0.3), point=3, mode=0, N=5):
    return R.exp4_checkpoint_signature({"problem": "golden", "solver": "explicit-mixed", "mass": "fft6d"},
                                       "cos12", "separable_cos", [12.0], N, 4, 10, 40, 1e-8, 1e-10, q, point, mode)


def _qres(converged=True, resid=1e-9, mode=0):
    lam = np.linspace(0.01, 0.1, 10)
    X = np.ones((6, 1), dtype=np.complex128) if mode else np.zeros((0, 0))
    return R.QResult(pointIndex=3, q=np.array([0.1, 0.2, 0.3]), lam=lam, outerSteps=40, wallTimeSeconds=0.11,
                     converged=converged, numConverged=10, maxRelativeInverseRitzResidual=resid,
                     cgAverageIterations=13.9, selectedMode=mode,
                     selectedLambda=np.array([lam[mode - 1]]) if mode else np.zeros((0, 0)), Xselected=X)


def test_checkpoint_round_trip_with_reference_field_names(tmp_path):
    path = str(tmp_path / "checkpoint" / "cos12_q003.mat")
    sig = _sig()
    R.save_q_checkpoint(path, _qres(), sig)
    C = loadmat(path, struct_as_record=False, squeeze_me=True)
    q = C["qres"]
    for name in ("pointIndex", "q", "lambda", "outerSteps", "wallTimeSeconds", "converged", "numConverged",
                 "maxRelativeInverseRitzResidual", "cgAverageIterations", "selectedMode", "Xselected"):
        assert name in q._fieldnames, name
    assert np.allclose(q.__dict__["lambda"], np.linspace(0.01, 0.1, 10))
    s = C["signature"]
    assert set(R.SIGNATURE_FIELDS) <= set(s._fieldnames) and "numerics" in s._fieldnames
    assert s.version == 6 and s.medium == "cos12" and s.numerics.mass == "fft6d"
    got = R.load_q_checkpoint(path, sig, tolLanczos=1e-8)
    assert got is not None and np.allclose(got.lam, np.linspace(0.01, 0.1, 10)) and got.outerSteps == 40


def test_checkpoint_reuse_rule(tmp_path):
    path = str(tmp_path / "c.mat")
    R.save_q_checkpoint(path, _qres(), _sig())
    assert R.load_q_checkpoint(path, _sig(q=(0.1, 0.2, 0.3000001)), 1e-8) is None   # q differs
    assert R.load_q_checkpoint(path, _sig(N=4), 1e-8) is None                         # N differs
    assert R.load_q_checkpoint(path, _sig(mode=2), 1e-8) is None                      # selected mode differs
    assert R.load_q_checkpoint(str(tmp_path / "missing.mat"), _sig(), 1e-8) is None
    R.save_q_checkpoint(path, _qres(converged=False), _sig())
    assert R.load_q_checkpoint(path, _sig(), 1e-8) is None                            # not converged
    R.save_q_checkpoint(path, _qres(resid=1e-6), _sig())
    assert R.load_q_checkpoint(path, _sig(), 1e-8) is None                            # residual above tol
    R.save_q_checkpoint(path, _qres(mode=2), _sig(mode=2))
    assert R.load_q_checkpoint(path, _sig(mode=2), 1e-8).selectedMode == 2


def test_csv_tables_have_reference_columns(tmp_path):
    qPlot = np.array([[0, 0.25], [0, 0], [0, 0]])
    lam = np.arange(20, dtype=float).reshape(10, 2)
    p = str(tmp_path / "Exp4_cos12_spectrum.csv")
    R.write_exp4_spectrum_csv(p, qPlot, lam)
    rows = list(csv.reader(open(p)))
    assert rows[0] == ["point", "mode", "q1", "q2", "q3", "lambda"] and len(rows) == 21
    assert rows[11][:2] == ["2", "1"] and float(rows[11][5]) == 1.0
    p = str(tmp_path / "Exp4_cos12_timing.csv")
    R.write_exp4_timing_csv(p, [_qres(), _qres()], [False, True])
    rows = list(csv.reader(open(p)))
    assert rows[0] == ["qpoint", "wall_s", "outer", "mhat_avg", "max_ritz", "from_checkpoint"] and rows[2][-1] == "1"
    p = str(tmp_path / "Exp4_cos12_selected.csv")
    R.write_exp4_selected_csv(p, [dict(label="A", pointIndex=1, modeIndex=10, lambda6D=0.1, lambdaLWRQ=0.1,
                                       deltaLambda=0.0, eta3D=0.1, nuLWRQ=0.07, lwrqIdentityError=1e-16)])
    assert list(csv.reader(open(p)))[0] == ["label", "point", "mode", "lambda6D", "lambdaLWRQ", "relDiff",
                                            "eta3D", "nuLWRQ", "identity"]
    p = str(tmp_path / "fig1bc.csv")
    R.write_fig1bc_csv(p, [dict(N=5, NF=10 ** 6, status="ok", plotLinearIterations=560, plotWallSeconds=0.11,
                                totalLinearSolverIterations=560, solverWallSeconds=0.11, outerSteps=40)])
    rows = list(csv.reader(open(p)))
    assert rows[0] == ["N", "NF", "status", "lin", "wall", "observedLin", "observedWall", "outer", "setup",
                       "plateau", "maxPlateau", "gpuFree"]
    assert rows[1][:3] == ["5", "1000000", "ok"] and rows[1][8] == "nan"
    s = R.make_exp1bc_signature("c", 5, {"numEig": 10, "q": [0.05, 0.04, 0.03]})
    assert s["version"] == 4 and s["method"] == "C" and R.make_exp1bc_signature("A", 5, {})["version"] == 6
