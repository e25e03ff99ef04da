"""GPU parity of the Yee-field LWRQ validation (exp3/compute_yee_lwrq_metrics_exp4.m)
against the oracle, on random fields and on a reconstructed eigenmode."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

KEYS = ("lambdaCrop", "lambda3D", "eta3D", "etaUsing6DLambda", "deltaLambda", "VLWRQ", "nuLWRQ",
        "croppedMass")


def _flat(u):
    return torch.as_tensor(np.asarray(u).reshape(-1, order="F"))


@pytest.mark.parametrize("material", [("exp", 4.0, 1.2), ("cos", 12.0)])
def test_lwrq_random_fields(cuda_device, material):
    import fame_b200 as F
    n, h = 6, 0.0125
    rng = np.random.default_rng(11)
    m = 2 * n + 3
    u = [rng.standard_normal((m, m, m)) + 1j * rng.standard_normal((m, m, m)) for _ in range(3)]
    P = F.configs.P_REFERENCE if material[0] == "exp" else F.configs.P_GOLDEN
    ref, sref = O.compute_yee_lwrq_metrics(*u, 0.05, P, n, h, material, save_spatial=True)
    met, sp = F.compute_yee_lwrq_metrics([_flat(c).to(cuda_device) for c in u], 0.05, P, n, h, material,
                                         save_spatial=True)
    for k in KEYS:
        np.testing.assert_allclose(met[k], ref[k], rtol=1e-11, err_msg=k)
    assert met["deltaPart"] < 1e-13 and met["deltaLWRQIdentity"] < 1e-12
    for k in ("relativeDeviation_z0", "relativeDeviation_x0"):
        np.testing.assert_allclose(sp[k], sref[k], rtol=1e-10, atol=1e-14)


def test_lwrq_of_reconstructed_mode(cuda_device):
    """Mode 1 of the N=2 tracking system (reference material), reconstructed on the Yee grid."""
    import fame_b200 as F
    N, n, h = 2, 8, 0.05
    E = O.material_smooth_exp(N)
    m = F.MassBackend(torch.as_tensor(E, device=cuda_device), N)
    sg = F.build_q_system(m, F.configs.P_REFERENCE, F.configs.Q_TRACKING)
    op, _ = F.make_explicit_krinv_compact(sg, 1e-12, 3000)
    Y, theta, _, _ = F.Lanczos(op, None, None, sg.nr, 2, 1e-10, 30, 20, F.start_vector(F.configs.SEED, sg.nr))
    j = int(np.argmax(theta))
    lam6 = 1.0 / theta[j]
    X, _, _ = F.recover_original_eigenvectors(Y[:, j:j + 1].contiguous(), sg, 1e-12, 3000)
    fields, _ = F.reconstruct_three_components(X[:, 0].contiguous(), sg, n, h, method="direct")
    ref, _ = O.compute_yee_lwrq_metrics(*(f.cpu().numpy().reshape((2 * n + 3,) * 3, order="F") for f in fields),
                                        lam6, F.configs.P_REFERENCE, n, h, ("exp", 4.0, 1.2))
    met, _ = F.compute_yee_lwrq_metrics(fields, lam6, F.configs.P_REFERENCE, n, h, ("exp", 4.0, 1.2))
    for k in KEYS:
        np.testing.assert_allclose(met[k], ref[k], rtol=1e-10, err_msg=k)
    assert met["croppedMass"] > 0 and np.isfinite(met["eta3D"])
