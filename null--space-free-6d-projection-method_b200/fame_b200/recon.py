"""Eigenvector recovery, Fourier diagnostics and Yee-field reconstruction
(host mirror of the reference functions; all compute in libfame_b200.so)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import FameError, call
from .core import QSystem, _ptr, default_context

__all__ = ["compute_yee_lwrq_metrics", "reconstruct_fields_direct_grid", "recover_original_eigenvectors", "compute_fourier_diagnostics", "build_projected_q_modes",
           "build_yee_points", "build_yee_block_partition", "reconstruct_field_direct_blocked",
           "reconstruct_field_direct_grid", "taylor_on_blocks", "reconstruct_field_taylor_multi",
           "reconstruct_field_taylor_single", "reconstruct_three_components"]


def recover_original_eigenvectors(Y, sys: QSystem, tol=1e-12, maxit=3000, precision="fp64"):
    """exp2/recover_original_eigenvectors_exp2.m:12-57 — X = M^{-1} V Y, M-normalised.

    Returns ``(X, MX, info)`` with X, MX of shape (3NF, k) (column-major views).
    """
    Yc = Y.t().contiguous() if Y.dim() == 2 else Y.reshape(1, -1).contiguous()
    k = Yc.shape[0]
    if Yc.shape[1] != sys.nr:
        raise FameError(L.FAME_ERR_INVALID, "Y must have 2*NF rows")
    X = torch.empty(k, sys.ndof, dtype=torch.complex128, device=Y.device)
    MX = torch.empty_like(X)
    its = (C.c_int * max(k, 1))()
    rr = (C.c_double * max(k, 1))()
    sys.ctx.bind()
    call("fame_recover_eigvecs", sys.h, sys.mass.h, _ptr(Yc), k, float(tol), int(maxit),
         L.FAME_PREC_MIXED if precision == "mixed" else L.FAME_PREC_FP64, _ptr(X), _ptr(MX), its, rr)
    return X.t(), MX.t(), dict(iterations=list(its[:k]), relativeResiduals=list(rr[:k]))


def compute_fourier_diagnostics(X, MX, lam, sys: QSystem):
    """exp2/compute_fourier_diagnostics_exp2.m:10-27 — GEVP residual, divergence, Rayleigh."""
    Xc, MXc = X.t().contiguous(), MX.t().contiguous()
    k = Xc.shape[0]
    lam = np.asarray(lam, dtype=np.float64).reshape(-1)
    lamc = (C.c_double * k)(*lam)
    res, div, ray = (C.c_double * k)(), (C.c_double * k)(), (C.c_double * k)()
    sys.ctx.bind()
    call("fame_fourier_diagnostics", sys.h, _ptr(Xc), _ptr(MXc), lamc, k, res, div, ray)
    res, div, ray = np.array(res[:]), np.array(div[:]), np.array(ray[:])
    return dict(resGEVP=res, divRelative2=div, rayleigh=ray, maxResGEVP=float(res.max()),
                maxDivRelative2=float(div.max()))


def _fourier_xi(N, device):
    n = 2 * N
    f = torch.cat([torch.arange(0, N), torch.arange(-N, 0)]).to(device=device, dtype=torch.float64)
    return f, n


def build_projected_q_modes(sys: QSystem):
    """exp2/build_projected_q_modes.m:4-10 — NF x 3 projected wave vectors (device,
    column-major storage: ``q[:, c]`` contiguous)."""
    dev = torch.device("cuda", sys.ctx.device)
    f, n = _fourier_xi(sys.N, dev)
    Q = torch.zeros(3, (2 * sys.N) ** 6, dtype=torch.float64, device=dev)
    for ell in range(6):
        shape = [1] * 6
        shape[5 - ell] = n  # axis 1 fastest
        xi = (f.view(shape) + float(sys.kLift[ell])).expand((n,) * 6).reshape(-1)
        for c in range(3):
            if sys.P[ell, c] != 0.0:
                Q[c] += float(sys.P[ell, c]) * xi
    return Q.t()


def build_yee_points(n, h, device=None):
    """exp2/build_yee_edge_points_plus.m:11-17 — the three staggered plus-grids
    (each M x 3, column-major) and the per-axis coordinates of each grid."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    idx = torch.arange(-(n + 1), n + 2, dtype=torch.float64, device=dev)
    m = idx.numel()
    I = idx.view(1, 1, m).expand(m, m, m).reshape(-1)   # fastest
    J = idx.view(1, m, 1).expand(m, m, m).reshape(-1)
    K = idx.view(m, 1, 1).expand(m, m, m).reshape(-1)
    pts, axes = [], []
    for comp in range(3):
        sh = [0.0, 0.0, 0.0]
        sh[comp] = 0.5
        R = torch.stack([h * (I + sh[0]), h * (J + sh[1]), h * (K + sh[2])], 0)  # 3 x M
        pts.append(R.t())
        axes.append(tuple(h * (idx + sh[d]) for d in range(3)))
    return pts, axes, (m, m, m)


def build_yee_block_partition(szPlus, nBlocks, device=None):
    """exp2/build_yee_block_partition_exp3.m:1-31 in CSR form (blockPtr, blockIds), 0-based."""
    m = szPlus[0]
    base, rem = divmod(m, nBlocks)
    groups, s = [], 0
    for b in range(nBlocks):
        ln = base + (1 if b < rem else 0)
        groups.append(np.arange(s, s + ln))
        s += ln
    ids, ptr = [], [0]
    for k in range(nBlocks):
        for j in range(nBlocks):
            for i in range(nBlocks):
                I, J, K = np.meshgrid(groups[i], groups[j], groups[k], indexing="ij")
                blk = (I + m * J + m * m * K).reshape(-1, order="F")
                ids.append(blk)
                ptr.append(ptr[-1] + blk.size)
    dev = device or torch.device("cuda", torch.cuda.current_device())
    return (torch.as_tensor(np.asarray(ptr, dtype=np.int64), device=dev),
            torch.as_tensor(np.concatenate(ids).astype(np.int64), device=dev))


def _pts(R):
    Rc = R.t().contiguous()  # 3 x M
    return Rc, Rc.shape[1]


def reconstruct_field_direct_blocked(coeff, qModes, rPoints, ctx=None):
    """exp2/reconstruct_field_direct_blocked_exp3.m:1-29 — u = exp(i R Q^T) c (any cut matrix)."""
    ctx = ctx or default_context()
    Qc = qModes.t().contiguous()
    Rc, M = _pts(rPoints)
    c = coeff.reshape(-1).contiguous()
    u = torch.empty(M, dtype=torch.complex128, device=c.device)
    call("fame_reconstruct_direct", ctx.bind(), _ptr(c), _ptr(Qc), c.numel(), _ptr(Rc), M, _ptr(u))
    return u


def reconstruct_field_direct_grid(coeff, sys: QSystem, axes, tensor_cores=False):
    """The direct sum on a tensor grid for an axis-block cut matrix (factorised GEMMs).

    ``tensor_cores=True``: the three complex GEMMs as split-FP32 (3xTF32) tcgen05 products
    (``fame_reconstruct_direct_grid_3xtf32``); FP64 CUDA-core GEMMs otherwise.
    """
    xs, ys, zs = (a.contiguous() for a in axes)
    c = coeff.reshape(-1).contiguous()
    u = torch.empty(xs.numel() * ys.numel() * zs.numel(), dtype=torch.complex128, device=c.device)
    sys.ctx.bind()
    call("fame_reconstruct_direct_grid_3xtf32" if tensor_cores else "fame_reconstruct_direct_grid", sys.h, _ptr(c),
         _ptr(xs), xs.numel(), _ptr(ys), ys.numel(), _ptr(zs), zs.numel(), _ptr(u))
    return u


def reconstruct_fields_direct_grid(coeff, sys: QSystem, axes_list, tensor_cores=False):
    """The factorised direct sum for several field components in one call (each GEMM one
    launch over all components; exp2/reconstruct_three_components_exp3.m reconstructs them
    one after another).  ``coeff``: the component-stacked coefficients (ncomp x NF, e.g. a
    recovered 3NF eigenvector); ``axes_list``: per component (xs, ys, zs) of equal sizes.
    Returns one field per component (views of one buffer)."""
    nc = len(axes_list)
    xs = torch.cat([a[0] for a in axes_list]).contiguous()
    ys = torch.cat([a[1] for a in axes_list]).contiguous()
    zs = torch.cat([a[2] for a in axes_list]).contiguous()
    nx, ny, nz = (axes_list[0][d].numel() for d in range(3))
    c = coeff.reshape(-1).contiguous()
    if c.numel() != nc * sys.NF:
        raise ValueError("coeff must hold ncomp x NF coefficients")
    M = nx * ny * nz
    u = torch.empty(nc * M, dtype=torch.complex128, device=c.device)
    sys.ctx.bind()
    call("fame_reconstruct_direct_grid_fields", sys.h, _ptr(c), nc, _ptr(xs), nx, _ptr(ys), ny, _ptr(zs), nz,
         int(bool(tensor_cores)), _ptr(u))
    return [u[i * M:(i + 1) * M] for i in range(nc)]


def taylor_on_blocks(coeff, qModes, rPoints, p, blocks, fixedCenter=None, ctx=None, tensor_cores=False):
    """exp2/taylor_on_blocks_exp3.m:1-97 — ``blocks`` = (blockPtr, blockIds) CSR tensors.

    ``tensor_cores``: block moments as 3xTF32 tensor-core GEMMs (split-FP32) instead of FP64.
    """
    ctx = ctx or default_context()
    Qc = qModes.t().contiguous()
    Rc, M = _pts(rPoints)
    c = coeff.reshape(-1).contiguous()
    ptr, ids = blocks
    u = torch.zeros(M, dtype=torch.complex128, device=c.device)
    fc = (C.c_double * 3)(*fixedCenter) if fixedCenter is not None else None
    call("fame_taylor_on_blocks_3xtf32" if tensor_cores else "fame_taylor_on_blocks", ctx.bind(), _ptr(c), _ptr(Qc),
         c.numel(), _ptr(Rc), M, int(p),
         _ptr(ptr), _ptr(ids), ptr.numel() - 1, fc, _ptr(u))
    return u


def reconstruct_field_taylor_multi(coeff, qModes, rPoints, p, blocks, tensor_cores=False):
    """exp2/reconstruct_field_taylor_multi_exp3.m:1-10."""
    return taylor_on_blocks(coeff, qModes, rPoints, p, blocks, None, tensor_cores=tensor_cores)


def reconstruct_field_taylor_single(coeff, qModes, rPoints, p, r0=(0.0, 0.0, 0.0)):
    """exp2/reconstruct_field_taylor_single_exp3.m:1-10 — one block, fixed center r0."""
    M = rPoints.shape[0]
    dev = rPoints.device
    blocks = (torch.tensor([0, M], dtype=torch.int64, device=dev), torch.arange(M, dtype=torch.int64, device=dev))
    return taylor_on_blocks(coeff, qModes, rPoints, p, blocks, r0)


def reconstruct_three_components(X, sys: QSystem, n, h, method="direct", p=10, nBlocks=4):
    """exp2/reconstruct_three_components_exp3.m:1-42 for one eigenvector X (3NF)."""
    NF = sys.NF
    pts, axes, sz = build_yee_points(n, h)
    out = []
    if method == "direct":
        for c in range(3):
            out.append(reconstruct_field_direct_grid(X[c * NF:(c + 1) * NF], sys, axes[c]))
    else:
        Q = build_projected_q_modes(sys)
        blocks = build_yee_block_partition(sz, nBlocks)
        for c in range(3):
            out.append(taylor_on_blocks(X[c * NF:(c + 1) * NF], Q, pts[c], p, blocks))
    return out, sz


LWRQ_KEYS = ("lambdaCrop", "lambda3D", "eta3D", "etaUsing6DLambda", "deltaLambda", "VLWRQ", "nuLWRQ",
             "deltaPart", "deltaLWRQIdentity", "croppedMass")


def compute_yee_lwrq_metrics(fields, lambda6D, P, n, h, material=("exp", 4.0, 1.2), save_spatial=False, ctx=None):
    """exp3/compute_yee_lwrq_metrics_exp4.m:1-100 on the GPU.

    ``fields``: the three plus-grid components (complex128 device tensors of
    (2n+3)^3 points, x fastest, as returned by the Yee reconstruction).
    ``material``: ("exp", epsC, alpha) or ("cos", delta), sampled on the Yee
    edges with the cut matrix ``P`` (6 x 3).  Returns ``(metrics, spatial)``
    with the reference's field names; ``spatial`` holds the z = 0 and x = 0
    slices of |rho - lambda3D| / |lambda3D| when ``save_spatial``.
    """
    ctx = ctx or default_context()
    m = 2 * n + 3
    us = [f.reshape(-1).to(torch.complex128).contiguous() for f in fields]
    if any(u.numel() != m ** 3 for u in us):
        raise FameError(L.FAME_ERR_INVALID, "fieldPlus size does not match requested n=%d." % n)
    Pc = (C.c_double * 18)(*np.asarray(P, dtype=np.float64).reshape(6, 3).ravel(order="F"))
    kind = 0 if material[0] == "exp" else 1
    mp0 = float(material[1])
    mp1 = float(material[2]) if len(material) > 2 else 0.0
    out = (C.c_double * 10)()
    q = 2 * n + 1
    z0 = (C.c_double * (q * q))() if save_spatial else None
    x0 = (C.c_double * (q * q))() if save_spatial else None
    call("fame_yee_lwrq_metrics", ctx.bind(), _ptr(us[0]), _ptr(us[1]), _ptr(us[2]), int(n), float(h), Pc, kind,
         mp0, mp1, float(lambda6D), out, z0, x0)
    met = dict(h=h, n=n, halfWidth=n * h, lambda6D=lambda6D)
    met.update({k: float(out[i]) for i, k in enumerate(LWRQ_KEYS)})
    spatial = None
    if save_spatial:
        spatial = dict(relativeDeviation_z0=np.ctypeslib.as_array(z0).reshape(q, q, order="F").copy(),
                       relativeDeviation_x0=np.ctypeslib.as_array(x0).reshape(q, q, order="F").copy(),
                       coord=np.arange(-n, n + 1) * h, lambda3D=met["lambda3D"], lambda6D=lambda6D, h=h, n=n)
    return met, spatial
