"""GPU parity of method A (the original shift-invert comparison path): the K symbol,
the MINRES-solved shift-invert operator and the device eigensolve, against the
oracle's dense N=1 problem and against method C on the GPU."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _sys(N, dev, q=(0.13, 0.21, 0.17)):
    import fame_b200 as F
    P = F.configs.P_REFERENCE
    E = O.material_smooth_exp(N)
    m = F.MassBackend(torch.as_tensor(E, device=dev), N)
    return F, E, O.build_q_system(N, P, q, E), F.build_q_system(m, P, q)


def test_apply_K_original_vs_oracle(cuda_device):
    F, E, S, sg = _sys(2, cuda_device)
    x = O.start_vector(5, 3 * S.NF)
    y = F.apply_K_original(torch.as_tensor(x, device=cuda_device), sg).cpu().numpy()
    assert rel(y, O.apply_K_original(x, S)) < 1e-14


def test_osi_top_vs_dense_n1(cuda_device):
    """T x (device MINRES, true relative residual 1e-11) vs (K - sigma M)^{-1} M x solved densely."""
    F, E, S, sg = _sys(1, cuda_device)
    sigma = 1e-4
    op, getStats, meta = F.make_A_eigs_top_preconditioned(sg, sigma, E.mean(), tol=1e-11)
    x = O.start_vector(3, 3 * S.NF)
    y = op(torch.as_tensor(x, device=cuda_device)).cpu().numpy()
    K, M3 = O.dense_original_operators(S)
    yd = np.linalg.solve(K - sigma * M3, M3 @ x)
    assert rel(y, yd) < 1e-9
    st = getStats()
    assert st["topVectorApplications"] == 1 and st["failures"] == 0 and st["maxTrueRelres"] <= 1e-11
    # the oracle's restated MINRES needs a similar number of iterations
    _, it, _ = O.osi_top_apply(x, S, sigma, sigma * E.mean(), tol=1e-11)
    assert st["totalMINRESIterations"] <= 2 * it + 5


def test_osi_eigs_vs_dense_n1(cuda_device):
    """The 10 eigenvalues above the shift vs the dense original GEVP; eigenvectors
    M-normalised with K x = lambda M x."""
    F, E, S, sg = _sys(1, cuda_device)
    lam, X, info, stats = F.eigs_method_A(sg, nev=10, sigma=1e-4, epsMean=E.mean(), epsMax=E.max(), tol=1e-10,
                                          p=40, tolMinres=1e-11, return_vectors=True)
    assert info["converged"]
    ev = O.dense_original_gevp(S)
    ref = ev[ev > 1e-10][:10]
    assert np.max(np.abs(lam - ref) / ref) < 1e-9
    K, M3 = O.dense_original_operators(S)
    Xh = X.cpu().numpy()
    for j in range(10):
        x = Xh[:, j]
        assert abs(np.vdot(x, M3 @ x) - 1.0) < 1e-9
        res = np.linalg.norm(K @ x - lam[j] * (M3 @ x))
        assert res / (np.linalg.norm(K @ x) + lam[j] * np.linalg.norm(M3 @ x)) < 1e-8


def test_method_a_matches_method_c_n3(cuda_device):
    """Method A and method C (both on the GPU) give the same 10 smallest positive
    eigenvalues (exp1/check_fig1bc_results.m:23-25 checks 1e-7); MINRES at the
    reference's tolerance 1e-10 (exp1/make_config_A_fig1a.m:61)."""
    F, E, S, sg = _sys(3, cuda_device)
    lamA, _, infoA, statsA = F.eigs_method_A(sg, nev=10, sigma=1e-4, epsMean=E.mean(), epsMax=E.max(), tol=1e-10,
                                             p=40, tolMinres=1e-10)
    assert infoA["converged"] and statsA["failures"] == 0 and statsA["maxTrueRelres"] <= 1e-9
    op, _ = F.make_explicit_krinv_compact(sg, 1e-12, 3000, precision="fp64")
    v0 = F.start_vector(F.configs.SEED, sg.nr)
    _, theta, _, infoC = F.Lanczos(op, None, None, sg.nr, 10, 1e-10, 30, 40, v0)
    lamC = np.sort(1.0 / theta)
    assert np.max(np.abs(lamA - lamC) / lamC) < 1e-8, (lamA, lamC)
