"""Method A of the reference: the original shift-invert eigensolve on the full
3NF space (exp1/build_experiment1_q_system_A_only.m,
exp1/build_original_shift_preconditioner_A_only.m,
exp1/make_A_eigs_top_preconditioned.m, exp1/run_method_A_fig1a.m), the
comparison path of the null-space-free methods B and C.

``make_A_eigs_top_preconditioned`` returns the operator of the reference's
``eigs`` call, T x = (K - sigma M)^{-1} M x with the shifted system solved by
preconditioned MINRES on the device; ``eigs_method_A`` returns the eigenvalues
above the shift (lambda = sigma + 1/theta) from the device Lanczos on the
Hermitian form M^(1/2) (K - sigma M)^{-1} M^(1/2) of T.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import call
from .core import QSystem, _ptr, start_vector

__all__ = ["apply_K_original", "make_A_eigs_top_preconditioned", "eigs_method_A", "OsiOperator"]


def apply_K_original(x, sys: QSystem):
    """exp1/build_experiment1_q_system_A_only.m:61-73 (applyK): y = K x on 3NF columns."""
    if x.shape[0] != 3 * sys.NF:
        raise L.FameError(L.FAME_ERR_INVALID, "Kop input must have 3*NF rows.")
    cols = 1 if x.dim() == 1 else x.shape[1]
    xt = x.contiguous() if x.dim() == 1 else x.t().contiguous()
    y = torch.empty_like(xt)
    sys.ctx.bind()
    call("fame_apply_K_original", sys.h, _ptr(xt), _ptr(y), cols)
    return y if x.dim() == 1 else y.t()


class OsiOperator:
    """T x = (K - sigma M)^{-1} M x (exp1/make_A_eigs_top_preconditioned.m:61-75)."""

    def __init__(self, sys: QSystem, sigma, tau, tol=1e-10, maxit=4000):
        if not tau > 0:
            raise ValueError("Preconditioner tau must be finite and positive.")
        self.sys, self.sigma, self.tau, self.tol, self.maxit = sys, float(sigma), float(tau), tol, maxit
        h = C.c_void_p()
        sys.ctx.bind()
        call("fame_osi_create", sys.h, sys.mass.h, self.sigma, self.tau, float(tol), int(maxit), C.byref(h))
        self.h = h

    def __call__(self, x):
        cols = 1 if x.dim() == 1 else x.shape[1]
        xt = x.contiguous() if x.dim() == 1 else x.t().contiguous()
        y = torch.empty_like(xt)
        self.sys.ctx.bind()
        call("fame_osi_apply", self.h, _ptr(xt), _ptr(y), cols)
        return y if x.dim() == 1 else y.t()

    def stats(self):
        s = L.fame_osi_stats()
        call("fame_osi_stats_get", self.h, C.byref(s))
        return dict(topVectorApplications=s.topApplications, totalMINRESIterations=s.minresIterations,
                    cycles=s.cycles, maxTrueRelres=s.maxTrueRelres, failures=s.failures,
                    totalPlateauAccepts=s.plateauAccepts)

    def close(self):
        if getattr(self, "h", None):
            L.lib.fame_osi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_A_eigs_top_preconditioned(sys: QSystem, sigma, epsMean, tol=1e-10, maxit=4000):
    """exp1/make_A_eigs_top_preconditioned.m:1-75 — (Top, getStats, meta) with
    tau = sigma * mean(eps) (cfg.shift.preconditionerTauMode = 'sigma-times-mean-epsilon')."""
    tau = float(sigma) * float(epsMean)
    if not np.isfinite(tau):
        raise ValueError("sigma and epsMean must be finite")
    op = OsiOperator(sys, sigma, tau, tol, maxit)
    meta = dict(sigma=float(sigma), tolMINRES=tol, maxitMINRESPerSegment=maxit,
                preconditioner="spectral-(K+tauI)", tau=tau,
                factorization="none; exact modewise Fourier-symbol inverse")
    return op, op.stats, meta


def eigs_method_A(sys: QSystem, nev=10, sigma=1e-4, epsMean=None, epsMax=None, tol=1e-10, maxiter=300, p=40,
                  tolMinres=1e-10, maxitMinres=4000, v0=None, return_vectors=False, op=None):
    """exp1/run_method_A_fig1a.m:9-50 with the shift check of exp1/run_fig1a_A_only.m:66-72
    (sigma < min|q|^2 / max eps).  Returns (lambda ascending, X (3NF x nev, M-normalised)
    or None, Lanczos info, MINRES statistics)."""
    if epsMean is None or epsMax is None:
        raise ValueError("epsMean and epsMax of the material are required")
    bound = sys.minQq / float(epsMax)
    if not sigma < bound:
        raise ValueError("Unsafe shift: sigma=%.3e >= lower bound %.3e." % (sigma, bound))
    if op is None:
        op = OsiOperator(sys, sigma, float(sigma) * float(epsMean), tolMinres, maxitMinres)
    n = 3 * sys.NF
    v0c = (start_vector(20260906, n) if v0 is None else v0).contiguous()
    lam = (C.c_double * nev)()
    X = torch.empty(nev, n, dtype=torch.complex128, device=v0c.device) if return_vectors else None
    info = L.fame_lanczos_info()
    sys.ctx.bind()
    call("fame_osi_eigs", op.h, int(nev), float(tol), int(maxiter), int(p), _ptr(v0c), lam, _ptr(X),
         C.byref(info))
    return (np.array(lam[:]), X.t() if X is not None else None,
            dict(steps=info.steps, restarts=info.restarts, converged=bool(info.converged), nconv=info.nconv,
                 maxWantedResidual=info.maxWantedResidual), op.stats())
