"""CPU: the committed golden fixtures are reproduced by the oracle and agree
with the reference's stored known answers."""
import os

import numpy as np

import oracle as O

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PHI = (1 + 5 ** 0.5) / 2
P_GOLDEN = np.vstack([np.eye(3), np.diag([PHI, 1 / PHI, PHI ** 2])])


def load(name):
    return dict(np.load(os.path.join(G, name + ".npz")))


def test_fixture_kat_matches_reference():
    e = load("eigs")
    # exp3/make_config_experiment4.m:38-45, rel 5e-7
    assert np.max(np.abs(e["n2_tracking"][[0, 9]] - e["kat_n2"]) / e["kat_n2"]) < 5e-7


def test_mass_fixture_reproduced():
    d = load("mass_n2")
    y = O.applyMij_fft(d["x"], d["E"], 2)
    assert np.linalg.norm(y - d["y"]) / np.linalg.norm(d["y"]) < 1e-14


def test_basis_fixture_reproduced():
    d = load("basis_n2_golden")
    S = O.build_q_system(2, P_GOLDEN, (0.05, 0.04, 0.03), O.material_separable_cos(2))
    for k in ("V11", "V22", "W1", "W2", "invC"):
        ref = d[k]
        assert np.linalg.norm(getattr(S, k) - ref) / np.linalg.norm(ref) < 1e-14, k


def test_recon_fixture_consistent():
    d = load("recon_n1")
    assert np.linalg.norm(d["taylor6"] - d["direct"]) / np.linalg.norm(d["direct"]) < 1e-2
    u = O.reconstruct_field_direct_blocked(d["coeff"], d["qModes"], d["r"][:50])
    assert np.allclose(u, d["direct"][:50], rtol=1e-13, atol=1e-13)
