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

__all__ = ["mass_adjoint", "eigenpairs", "EigenvalueFunction", "eigenvalue_gradients", "modes_per_chunk"]


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


def modes_per_chunk(NF, nev, device_bytes=None, device=None):
    """Eigenvectors recovered (and their adjoint terms evaluated) together: each mode holds
    X and M X (3 NF complex128 each) plus the recovery's PCG vectors (~6 NF complex128);
    with ``device_bytes`` (default: half of the device's free memory) fewer modes than
    ``nev`` are recovered at a time when they do not fit, the rest recomputed chunk by chunk."""
    per_mode = 12 * NF * 16
    if device_bytes is None:
        free, _ = torch.cuda.mem_get_info(device)
        device_bytes = free // 2
    return int(max(1, min(nev, device_bytes // per_mode)))


def eigenvalue_gradients(N, theta, chunk=None, device_bytes=None, **kw):
    """(lambda, d lambda / d theta) for the smallest eigenvalues (theta = (delta, a_1..a_6)).

    Only the Ritz vectors Y (2NF x nev) are kept from the solve (the Krylov basis is
    released); the original eigenvectors x_j = M^{-1} V y_j are recovered ``chunk`` modes
    at a time (default: as many as fit in ``device_bytes``, see modes_per_chunk) and
    discarded after their adjoint terms are taken, so the gradient's memory does not grow
    with nev."""
    lam, Y, sysq, mass, grads, _ = eigenpairs(N, theta, **kw)
    nev = Y.shape[1]
    chunk = chunk or modes_per_chunk(sysq.NF, nev, device_bytes)
    quad = np.zeros((nev, len(grads)))
    for j0 in range(0, nev, chunk):
        cols = list(range(j0, min(nev, j0 + chunk)))
        X, MX, _ = recover_original_eigenvectors(Y[:, cols].contiguous(), sysq, 1e-12, 3000)
        quad[cols] = mass_adjoint(mass, X, grads)
        del X, MX
    return lam, -lam[:, None] * quad


class EigenvalueFunction(torch.autograd.Function):
    """lambda(theta) with a Hellmann-Feynman backward pass (theta: float64 CPU tensor of 7).

    ``kw`` are eigenvalue_gradients' keywords; with ``recompute=True`` in it, forward keeps
    only theta and lambda and backward repeats the solve (deterministic: the same start
    vector gives the same eigenvectors) to rebuild the eigenvectors, instead of holding
    any solver state between the two passes."""

    @staticmethod
    def forward(ctx, theta, N, kw):
        kw = dict(kw or {})
        recompute = kw.pop("recompute", False)
        th = theta.detach().cpu().numpy()
        if recompute:
            lam = eigenpairs(N, th, **{k: v for k, v in kw.items() if k not in ("chunk", "device_bytes")})[0]
            ctx.N, ctx.kw = N, kw
            ctx.save_for_backward(theta.detach().clone())
            ctx.dlam = None
        else:
            lam, dlam = eigenvalue_gradients(N, th, **kw)
            ctx.dlam = torch.as_tensor(dlam)
        return torch.as_tensor(lam, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_lam):
        dlam = ctx.dlam
        if dlam is None:
            (theta,) = ctx.saved_tensors
            dlam = torch.as_tensor(eigenvalue_gradients(ctx.N, theta.cpu().numpy(), **ctx.kw)[1])
        return grad_lam.to(dlam.dtype) @ dlam, None, None
