"""Pinned synthetic workloads of the eigensolver hot path.

Materials are synthesised on the device in the reference's grid convention
(x_d = 2*pi*j/(2N), column-major 6D order, exp1/build_experiment1_common.m:10-11).
The cut matrix of the benchmark workloads is an axis-block golden-ratio matrix
``[I3; diag(phi, 1/phi, phi^2)]``; the reference's own experiments use
``[I3; diag(sqrt2, sqrt3, sqrt5)]`` (exp1/make_config_exp1bc.m:20-26).
"""
from __future__ import annotations

import math

import numpy as np
import torch

PHI = (1.0 + math.sqrt(5.0)) / 2.0
P_GOLDEN = np.vstack([np.eye(3), np.diag([PHI, 1.0 / PHI, PHI ** 2])])
P_REFERENCE = np.vstack([np.eye(3), np.diag([math.sqrt(2.0), math.sqrt(3.0), math.sqrt(5.0)])])
Q_PHYS = (0.05, 0.04, 0.03)          # exp1/make_config_exp1bc.m:34
Q_TRACKING = (0.13, 0.21, 0.17)          # exp3/make_config_experiment4.m:26
SEED = 20260905                          # exp1/make_config_BC_fig1a.m:42
# Reference KAT: N=2, modes 1 and 10 of the tracking system (exp3/make_config_experiment4.m:38-40)
KAT_N2_LAMBDA = (1.201276300237e-02, 4.496454358674e-02)

# At Gamma (q = 0) the xi = 0 mode has q_xi = 0 and the null-space-free reduction is
# singular (exp1/assemble_K_and_nullspace_free_basis.m:36-42); the Bloch-path
# workload solves that point at this small shift along the first path segment.
GAMMA_SHIFT = np.array([1e-3, 0.0, 0.0])

# Solver settings of the 10-eigenpair workloads (shift 0, Krylov block 40, outer tol 1e-8,
# inner Mhat PCG tol 1e-10).
SOLVE = dict(nev=10, p=40, tol=1e-8, maxRestart=30, tolCG=1e-10, maxitCG=3000)
# Options of the mixed form in these workloads: the FP64 refinement of each Mhat solve stops
# at the reference pcg rule relres <= tolCG (exp1/make_explicit_krinv_compact.m:43), as the
# FP64 form does; the eigenvalues are then refined by Rayleigh-Ritz on the exact K_r.
MIXED_OPTS = dict(refineTarget=1.0)


def _coords(N, device):
    """Six broadcastable coordinate tensors x_1..x_6 in column-major grid order."""
    n = 2 * N
    c = torch.arange(n, dtype=torch.float64, device=device) * (2 * math.pi / n)
    out = []
    for d in range(6):
        shape = [1] * 6
        shape[5 - d] = n  # x_1 varies fastest (last torch dim)
        out.append(c.view(shape))
    return out


def material_separable_cos(N, delta=12.0, device="cuda"):
    """eps = 1 + delta * prod_d (1 + cos x_d)/2 — band-limited (3^6 DFT coefficients)."""
    prod = torch.ones((2 * N,) * 6, dtype=torch.float64, device=device)
    for x in _coords(N, device):
        prod = prod * (1 + torch.cos(x)) / 2
    return (1 + delta * prod).reshape(-1)


def material_smooth_exp(N, epsC=4.0, alpha=1.2, device="cuda"):
    """eps = epsC * exp(alpha/6 * sum cos x_d) (exp1/build_smooth_scalar_material_compact.m:3-6)."""
    s = torch.zeros((2 * N,) * 6, dtype=torch.float64, device=device)
    for x in _coords(N, device):
        s = s + torch.cos(x)
    return (epsC * torch.exp((alpha / 6.0) * s)).reshape(-1)


def material_cos_param(N, delta, a, device="cuda"):
    """eps = 1 + delta * prod_d (1 + a_d cos x_d)/(1 + a_d); returns (eps, [d eps/d theta])
    with theta = (delta, a_1..a_6)."""
    xs = _coords(N, device)
    fac = [(1 + a[d] * torch.cos(xs[d])) / (1 + a[d]) for d in range(6)]
    prod = torch.ones((2 * N,) * 6, dtype=torch.float64, device=device)
    for f in fac:
        prod = prod * f
    grads = [prod.reshape(-1)]
    for d in range(6):
        dfd = (torch.cos(xs[d]) - 1) / (1 + a[d]) ** 2
        grads.append((delta * prod / fac[d] * dfd).reshape(-1))
    return (1 + delta * prod).reshape(-1), grads


def gradient_amplitudes(seed=20260907):
    """a_d ~ U[0.5, 1] from a seeded generator (eigenvalue-gradient workload, N=6)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.5, 1.0, size=6)


def bloch_path(points_per_segment=4):
    """12 q-points on Gamma -> (0.5,0,0) -> (0.5,0.5,0) -> (0.5,0.5,0.5), N round-robin 3,4,5."""
    verts = np.array([[0, 0, 0], [0.5, 0, 0], [0.5, 0.5, 0], [0.5, 0.5, 0.5]], dtype=np.float64)
    qs = []
    for s in range(3):
        for t in range(points_per_segment):
            qs.append(verts[s] + (verts[s + 1] - verts[s]) * t / points_per_segment)
    Ns = [3 + (i % 3) for i in range(len(qs))]
    return qs, Ns
