"""Hellmann-Feynman eigenvalue gradients through the mass-operator adjoint.

For K x = lambda M(theta) x with K independent of theta and x M-normalised,
d lambda / d theta_t = -lambda x^H (dM/dtheta_t) x, and
x^H (dM/dtheta_t) x = NF sum_y (d eps/d theta_t)(y) sum_c |ifftn(x_c)(y)|^2,
evaluated by fame_mass_adjoint.  EigenvalueFunction wraps a full solve
(Lanczos on K_r^{-1}, eigenvector recovery) in a torch.autograd.Function.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from . import configs
from ._lib import call
from .core import MassBackend, build_q_system, make_explicit_krinv_compact, start_vector, Lanczos, _ptr
from .recon import recover_original_eigenvectors

__all__ = ["mass_adjoint", "eigenpairs", "EigenvalueFunction", "eigenvalue_gradients"]


def mass_adjoint(mass: MassBackend, X, dEps):
    """out[j, t] = X[:, j]^H (dM/dtheta_t) X[:, j]; dEps: list of NF real fields (device)."""
    Xc = X.t().contiguous()
    k = Xc.shape[0]
    G = torch.stack([g.reshape(-1) for g in dEps], 0).contiguous()  # nparams x NF
    out = (C.c_double * (k * G.shape[0]))()
    mass.ctx.bind()
    call("fame_mass_adjoint", mass.h, _ptr(Xc), k, _ptr(G), G.shape[0], out)
    return np.array(out[:]).reshape(k, G.shape[0])


def eigenpairs(N, theta, P=None, q=None, nev=10, p=40, tol=1e-8, tolCG=1e-10, precision="mixed",
               device="cuda"):
    """Smallest eigenpairs for the parametrised material eps(theta) = 1 + delta prod (1+a cos)/(1+a)."""
    P = configs.P_GOLDEN if P is None else P
    q = configs.Q_PHYS if q is None else q
    theta = np.asarray(theta, dtype=np.float64)
    eps, grads = configs.material_cos_param(N, float(theta[0]), theta[1:7], device=device)
    mass = MassBackend(eps, N)
    sysq = build_q_system(mass, P, q)
    op, _ = make_explicit_krinv_compact(sysq, tolCG, 3000, precision=precision)
    v0 = start_vector(configs.SEED, sysq.nr)
    Y, th, _, info = Lanczos(op, None, None, sysq.nr, nev, tol, 30, p, v0)
    lam = 1.0 / th
    order = np.argsort(lam)
    return lam[order], Y[:, order.tolist()], sysq, mass, grads, info


def eigenvalue_gradients(N, theta, **kw):
    """(lambda, d lambda / d theta) for the 10 smallest eigenvalues (theta = (delta, a_1..a_6))."""
    lam, Y, sysq, mass, grads, _ = eigenpairs(N, theta, **kw)
    X, MX, _ = recover_original_eigenvectors(Y, sysq, 1e-12, 3000)
    quad = mass_adjoint(mass, X, grads)
    return lam, -lam[:, None] * quad


class EigenvalueFunction(torch.autograd.Function):
    """lambda(theta) with a Hellmann-Feynman backward pass (theta: float64 CPU tensor of 7)."""

    @staticmethod
    def forward(ctx, theta, N, kw):
        lam, dlam = eigenvalue_gradients(N, theta.detach().cpu().numpy(), **(kw or {}))
        ctx.save_for_backward(torch.as_tensor(dlam))
        return torch.as_tensor(lam, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_lam):
        (dlam,) = ctx.saved_tensors
        return grad_lam.to(dlam.dtype) @ dlam, None, None
