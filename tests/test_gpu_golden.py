"""GPU vs the committed golden fixtures (the oracle's frozen outputs)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(G, name + ".npz")))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_mass_vs_fixture(cuda_device):
    import fame_b200 as F
    d = load("mass_n2")
    m = F.MassBackend(torch.as_tensor(d["E"], device=cuda_device), 2)
    y = m.MscalarOp(torch.as_tensor(d["x"], device=cuda_device)).cpu().numpy()
    assert rel(y, d["y"]) < 1e-13
    y32 = m.MscalarOp(torch.as_tensor(d["x"], device=cuda_device).to(torch.complex64)).cpu().numpy()
    assert rel(y32, d["y"]) < 2e-6


def test_basis_vs_fixture(cuda_device):
    import fame_b200 as F
    d = load("basis_n2_golden")
    m = F.MassBackend(F.configs.material_separable_cos(2, device=cuda_device), 2)
    s = F.build_q_system(m, F.configs.P_GOLDEN, F.configs.Q_PHYS)
    np.testing.assert_allclose(s.kLift, d["kLift"], rtol=1e-14, atol=1e-16)
    for k in ("V11", "V12", "V21", "V22", "V31", "V32", "detV1", "W1", "W2"):
        assert rel(getattr(s, k).cpu().numpy(), d[k]) < 1e-10, k
    assert rel(s.invCorthDiag.cpu().numpy(), d["invC"]) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_krinv_and_eigs_vs_fixture(cuda_device, precision):
    import fame_b200 as F
    dk, de = load("krinv_n2_tracking"), load("eigs")
    m = F.MassBackend(torch.as_tensor(load("mass_n2")["E"], device=cuda_device), 2)
    s = F.build_q_system(m, F.configs.P_REFERENCE, F.configs.Q_TRACKING)
    op, _ = F.make_explicit_krinv_compact(s, 1e-12, 3000, precision=precision)
    y = op(torch.as_tensor(dk["b"], device=cuda_device)).cpu().numpy()
    assert rel(y, dk["y"]) < 1e-10
    v0 = F.start_vector(F.configs.SEED, s.nr)
    _, theta, _, info = F.Lanczos(op, None, None, s.nr, 10, 1e-10, 30, 40, v0)
    lam = np.sort(1.0 / theta)
    assert info["converged"]
    assert np.max(np.abs(lam - de["n2_tracking"]) / de["n2_tracking"]) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_n3_benchmark_system_eigs_vs_fixture(cuda_device, precision):
    """The 10 smallest eigenvalues of the N=3 benchmark system (golden-ratio P, separable
    cos material, q = (0.05, 0.04, 0.03)) frozen from the oracle at tol 1e-10, tolCG 1e-12;
    the GPU solve at the same settings, with and without its Rayleigh-Ritz step."""
    import fame_b200 as F
    de = load("eigs")
    m = F.MassBackend(F.configs.material_separable_cos(3, 12.0, device=cuda_device), 3)
    s = F.build_q_system(m, F.configs.P_GOLDEN, F.configs.Q_PHYS)
    op, _ = F.make_explicit_krinv_compact(s, 1e-12, 3000, precision=precision)
    v0 = F.start_vector(F.configs.SEED, s.nr)
    Y, theta, _, info = F.Lanczos(op, None, None, s.nr, 10, 1e-10, 30, 40, v0)
    assert info["converged"]
    ref = de["n3_golden_cos"]
    lam = np.sort(1.0 / (theta.cpu().numpy() if torch.is_tensor(theta) else np.asarray(theta)))
    assert np.max(np.abs(lam - ref) / ref) < 1e-10, lam
    lam_rr, _ = F.rayleigh_ritz(s, Y)
    lam_rr = np.sort(np.asarray(lam_rr))
    assert np.max(np.abs(lam_rr - ref) / ref) < 1e-10, lam_rr


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_reference_kat_n5_tracked_modes(cuda_device, precision):
    """exp3/make_config_experiment4.m:38-52, exp3/solve_tracked_modes_exp4.m:37-42: the
    reference's N=5 tracked modes 11 and 114 (material epsC = 4, alpha = 1.2, P = [I;
    diag(sqrt 2, sqrt 3, sqrt 5)], q = (0.13, 0.21, 0.17)) from its k = 140, p = 188 scan
    (tolLanczos = tolCG = 1e-10).  The reference checks 5e-7; its values carry 13 digits."""
    import fame_b200 as F
    N = 5
    m = F.MassBackend(F.configs.material_smooth_exp(N, 4.0, 1.2, device=cuda_device), N)
    s = F.build_q_system(m, F.configs.P_REFERENCE, F.configs.Q_TRACKING)
    op, _ = F.make_explicit_krinv_compact(s, 1e-10, 3000, precision=precision)
    v0 = F.start_vector(20260831, s.nr)
    _, theta, _, info = F.Lanczos(op, None, None, s.nr, 140, 1e-10, 30, 188, v0)
    assert info["converged"] and info["nconv"] == 140
    lam = np.sort(1.0 / theta)[[10, 113]]
    ref = np.array([1.200090550277e-02, 4.462939906027e-02])
    assert np.max(np.abs(lam - ref) / ref) < 1e-10, lam
