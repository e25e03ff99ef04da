"""NumPy FP64 restatement of the reference hot path (test infrastructure only).

Every function cites the reference MATLAB file it follows (paths are relative
to the reference project root).  Vectors are 1-D complex128 arrays in the
reference's column-major 6D ordering (axis 1 fastest), component-stacked
``[U1;U2;U3]`` where the reference stacks components.

The MATLAB builtins used by the reference (``fftn``/``ifftn``/``fft``,
``pcg``, ``eig``) are closed; here they are restated from their documented
semantics: ``fftn`` is the unnormalised forward DFT with ``exp(-2*pi*i*k*x/n)``,
``ifftn`` the inverse with the ``1/n`` factor, ``pcg`` is preconditioned CG
with ``x0=0`` that stops on ``||b-A*x||/||b|| <= tol`` after verifying the
recursive residual against the true residual.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

try:  # multi-threaded pocketfft when available (same transform as numpy.fft)
    import scipy.fft as _sfft
except ImportError:  # pragma: no cover
    _sfft = None

#: host threads used by the oracle's FFTs (the CPU baseline sets this)
FFT_WORKERS = 1


def set_fft_workers(n):
    """Number of host threads for the oracle's FFTs (1 = single-threaded)."""
    global FFT_WORKERS
    FFT_WORKERS = max(1, int(n))


def _fftn(a):
    if _sfft is not None and FFT_WORKERS > 1:
        return _sfft.fftn(a, workers=FFT_WORKERS)
    return np.fft.fftn(a)


def _ifftn(a):
    if _sfft is not None and FFT_WORKERS > 1:
        return _sfft.ifftn(a, workers=FFT_WORKERS)
    return np.fft.ifftn(a)

__all__ = [
    "build_fourier_grid_6d", "grid_coordinates", "material_smooth_exp",
    "material_separable_cos", "material_cos_param", "applyMij_fft",
    "build_radix_exact_rank1_plan_scalar", "build_exact_rank1_scalar_kernel_fft",
    "applyMij_rank1_exact", "rank1_exact_fft_scatter", "rank1_exact_ifft_gather",
    "mass_stencil_bandlimited", "MassOp", "assemble_K_and_nullspace_free_basis",
    "QSystem", "build_q_system", "apply_V_blockdiag", "apply_VH_blockdiag",
    "solveV1_blockdiag", "solveV1H_blockdiag", "apply_Mhat_C_scalar_compact",
    "pcg", "make_explicit_krinv_compact", "make_nested_krinv_instrumented",
    "Lanczos", "recover_original_eigenvectors", "compute_fourier_diagnostics",
    "start_vector", "build_projected_q_modes", "build_yee_points",
    "build_yee_block_partition", "build_multi_index_list_3d",
    "taylor_coeff_alpha", "taylor_on_blocks", "reconstruct_field_taylor_multi",
    "reconstruct_field_taylor_single", "reconstruct_field_direct_blocked",
    "reconstruct_component_taylor_batch", "solve_modes", "dense_reduced_operator",
    "mass_adjoint_quadratic", "set_fft_workers", "apply_cropped_A", "yee_material",
    "separable_conv3_same", "compute_lwrq", "compute_yee_lwrq_metrics",
    "apply_K_original", "apply_shift_preconditioner", "minres", "osi_top_apply",
    "dense_original_operators", "dense_original_gevp", "apply_Kr_exact", "rayleigh_ritz_Kr",
]


# ---------------------------------------------------------------------------
# Grid and material
# ---------------------------------------------------------------------------

def build_fourier_grid_6d(N: int, T=None):
    """exp1/build_fourier_grid_6d.m:1-30 — per-axis frequencies [0..N-1,-N..-1].

    Returns ``Xi``: a list of six flat NF-vectors (column-major ndgrid), each
    scaled by 2*pi/T_d.
    """
    n = 2 * N
    if T is None:
        T = np.full(6, 2 * np.pi)
    freq1 = np.concatenate([np.arange(0, N), np.arange(-N, 0)]).astype(np.float64)
    Xi = []
    for d in range(6):
        shape = [1] * 6
        shape[d] = n
        J = np.broadcast_to(freq1.reshape(shape), (n,) * 6)
        Xi.append(((2 * np.pi / T[d]) * J).reshape(-1, order="F").copy())
    return Xi


def grid_coordinates(N: int):
    """exp1/build_experiment1_common.m:10-11 — x_d = 2*pi*j/(2N) on an ndgrid."""
    n = 2 * N
    c = np.arange(n) / n * 2 * np.pi
    out = []
    for d in range(6):
        shape = [1] * 6
        shape[d] = n
        out.append(np.broadcast_to(c.reshape(shape), (n,) * 6))
    return out


def material_smooth_exp(N: int, epsC=4.0, alpha=1.2):
    """exp1/build_smooth_scalar_material_compact.m:3-6 — epsC*exp(alpha/6*sum cos x_d).

    Returned flat in column-major order (length NF).
    """
    xs = grid_coordinates(N)
    phi = (alpha / 6.0) * sum(np.cos(x) for x in xs)
    return (epsC * np.exp(phi)).reshape(-1, order="F")


def material_separable_cos(N: int, delta=12.0):
    """Band-limited material eps = 1 + delta*prod_d (1+cos x_d)/2 (flat, column-major)."""
    xs = grid_coordinates(N)
    prod = np.ones((2 * N,) * 6)
    for x in xs:
        prod = prod * (1 + np.cos(x)) / 2
    return (1 + delta * prod).reshape(-1, order="F")


def material_cos_param(N: int, delta, a):
    """eps = 1 + delta*prod_d (1 + a_d cos x_d)/(1 + a_d) (flat, column-major).

    Parametrised material of the eigenvalue-gradient workload; returns
    ``(eps, [d eps/d delta, d eps/d a_1, ..., d eps/d a_6])``.
    """
    xs = grid_coordinates(N)
    fac = [(1 + a[d] * np.cos(xs[d])) / (1 + a[d]) for d in range(6)]
    prod = np.ones((2 * N,) * 6)
    for f in fac:
        prod = prod * f
    eps = 1 + delta * prod
    grads = [prod]
    for d in range(6):
        # d/da [(1 + a cos x)/(1 + a)] = (cos x - 1)/(1 + a)^2
        dfd = (np.cos(xs[d]) - 1) / (1 + a[d]) ** 2
        grads.append(delta * prod / fac[d] * dfd)
    flat = lambda g: np.asarray(g).reshape(-1, order="F")
    return flat(eps), [flat(g) for g in grads]


# ---------------------------------------------------------------------------
# Mass operator
# ---------------------------------------------------------------------------

def _grid(x, N):
    return x.reshape((2 * N,) * 6, order="F")


def applyMij_fft(x, E, N):
    """exp1/applyMij_fft.m:1-24 — y = fftn(E .* ifftn(X)), column by column.

    ``x`` is (NF,) or (NF, nrhs); ``E`` is the real-space material, flat (NF,).
    """
    Eg = _grid(E, N)
    if x.ndim == 1:
        return _fftn(Eg * _ifftn(_grid(x, N))).reshape(-1, order="F")
    return np.stack([applyMij_fft(x[:, j], E, N) for j in range(x.shape[1])], axis=1)


def build_radix_exact_rank1_plan_scalar(N: int, dim: int = 6):
    """exp1/build_radix_exact_rank1_plan_scalar.m:18-63 (0-based indices here)."""
    nGrid = 2 * N
    B = 2 * nGrid - 1
    NF = nGrid ** dim
    z = np.array([B ** j for j in range(dim)], dtype=np.int64)
    M = nGrid * B ** (dim - 1)
    s = nGrid - 1
    idx = np.arange(NF, dtype=np.int64)
    tmp = idx.copy()
    code = np.zeros(NF, dtype=np.int64)
    for j in range(dim):
        code += (tmp % nGrid) * z[j]
        tmp //= nGrid
    shift = (s * int(z.sum())) % M
    target = (code + shift) % M
    return dict(N=N, dim=dim, nGrid=nGrid, B=B, NF=NF, M=M, z=z, shiftCode=shift,
                inputIdx=code, targetIdx=target, embeddingRatio=M / NF)


def build_exact_rank1_scalar_kernel_fft(E, plan):
    """exp1/build_exact_rank1_scalar_kernel_fft.m:9-37 — decode residues, FFT length M."""
    N, nGrid, B, M, dim = plan["N"], plan["nGrid"], plan["B"], plan["M"], plan["dim"]
    Ehat = np.fft.fftn(_grid(E, N)).reshape(-1, order="F")
    code = np.arange(M, dtype=np.int64)
    tmp = code.copy()
    res = np.zeros(M, dtype=np.int64)
    stride = 1
    s = nGrid - 1
    for _ in range(dim):
        digit = tmp % B
        tmp //= B
        res += ((digit - s) % nGrid) * stride
        stride *= nGrid
    h = Ehat[res] / plan["NF"]
    return np.fft.fft(h)


def rank1_exact_fft_scatter(x, plan):
    """exp1/rank1_exact_fft_scatter.m:1-13."""
    x = x.reshape(plan["NF"], -1)
    if x.shape[0] != plan["NF"]:
        raise ValueError("rank1_exact_fft_scatter:BadSize")
    emb = np.zeros((plan["M"], x.shape[1]), dtype=np.complex128)
    emb[plan["inputIdx"], :] = x
    return np.fft.fft(emb, axis=0)


def rank1_exact_ifft_gather(Y, plan):
    """exp1/rank1_exact_ifft_gather.m:1-11."""
    if Y.shape[0] != plan["M"]:
        raise ValueError("rank1_exact_ifft_gather:BadSize")
    return np.fft.ifft(Y, axis=0)[plan["targetIdx"], :]


def applyMij_rank1_exact(x, kernelFFT, plan):
    """exp1/applyMij_rank1_exact.m:1-6."""
    one = x.ndim == 1
    X = rank1_exact_fft_scatter(x, plan)
    y = rank1_exact_ifft_gather(kernelFFT[:, None] * X, plan)
    return y[:, 0] if one else y


def mass_stencil_bandlimited(x, N, delta=12.0):
    """Closed form of the mass operator for eps = 1 + delta*prod (1+cos)/2.

    That material has DFT coefficients only at offsets {-1,0,1}^6, so
    M = I + delta * (x) circ[1/4, 1/2, 1/4] along every axis (no aliasing for
    2N >= 3).  Independent of any FFT.
    """
    X = _grid(x, N)
    Y = X.copy()
    for d in range(6):
        Y = 0.5 * Y + 0.25 * np.roll(Y, 1, axis=d) + 0.25 * np.roll(Y, -1, axis=d)
    return (X + delta * Y).reshape(-1, order="F")


class MassOp:
    """exp1/build_mass_backend_large_scalar.m:27-46 — the four mass handles."""

    def __init__(self, E, N):
        self.E, self.N, self.NF = E, N, (2 * N) ** 6
        self.applies = 0

    def scalar(self, x):  # MscalarOp
        self.applies += 1 if x.ndim == 1 else x.shape[1]
        return applyMij_fft(x, self.E, self.N)

    def full(self, U):  # Mop: 3NF -> 3NF, component-first
        n = self.NF
        return np.concatenate([self.scalar(U[k * n:(k + 1) * n]) for k in range(3)])

    def inverse_scalar(self, x):
        """M^{-1} x = fftn(ifftn(x) ./ E): on the (2N)^6 grid the convolution of
        exp1/applyMij_fft.m:11 is diagonal in real space, so its inverse is exact."""
        return applyMij_fft(x, 1.0 / self.E, self.N)


# ---------------------------------------------------------------------------
# Null-space-free basis
# ---------------------------------------------------------------------------

def assemble_K_and_nullspace_free_basis(P, k, Xi, tol=1e-13):
    """exp1/assemble_K_and_nullspace_free_basis.m:18-105.

    Returns dict with q1,q2,q3 (projected wave vectors), Qq=|q|^2, V11..V32.
    Raises on a (near-)zero projected mode, as the reference does (:36-42).
    """
    q = [np.zeros_like(Xi[0]) for _ in range(3)]
    for ell in range(6):
        s = Xi[ell] + k[ell]
        for c in range(3):
            q[c] = q[c] + P[ell, c] * s
    q1, q2, q3 = q
    Qq = np.abs(q1) ** 2 + np.abs(q2) ** 2 + np.abs(q3) ** 2
    if Qq.min() <= tol:
        raise ValueError("zero projected Fourier mode (Gamma point): min|q|^2=%.3e" % Qq.min())
    sq = np.sqrt(Qq)
    Qs = q1 + q2 + q3
    denom = 3 * Qq - np.abs(Qs) ** 2
    reg = denom > tol
    u = {key: np.zeros(q1.shape, dtype=np.complex128) for key in
         ("11", "21", "31", "12", "22", "32")}
    s1 = 1.0 / np.sqrt(Qq[reg] * denom[reg])
    u["11"][reg] = (Qq[reg] - q1[reg] * np.conj(Qs[reg])) * s1
    u["21"][reg] = (Qq[reg] - q2[reg] * np.conj(Qs[reg])) * s1
    u["31"][reg] = (Qq[reg] - q3[reg] * np.conj(Qs[reg])) * s1
    s2 = 1.0 / np.sqrt(denom[reg])
    u["12"][reg] = (np.conj(q3[reg]) - np.conj(q2[reg])) * s2
    u["22"][reg] = (np.conj(q1[reg]) - np.conj(q3[reg])) * s2
    u["32"][reg] = (np.conj(q2[reg]) - np.conj(q1[reg])) * s2
    # singular branch (:75-91): q parallel to (1,1,1)
    for m in np.nonzero(~reg)[0]:
        qv = np.array([q1[m], q2[m], q3[m]], dtype=np.float64)
        qh = qv / np.linalg.norm(qv)
        a = np.zeros(3)
        a[np.argmin(np.abs(qh))] = 1
        z1 = a - qh * (qh @ a)
        z1 /= np.linalg.norm(z1)
        z2 = np.cross(qh, z1)
        z2 /= np.linalg.norm(z2)
        u["11"][m], u["21"][m], u["31"][m] = z1
        u["12"][m], u["22"][m], u["32"][m] = z2
    V = {key: u[key] * sq for key in u}
    return dict(q1=q1, q2=q2, q3=q3, Qq=Qq, sqrtQq=sq, nsingular=int((~reg).sum()),
                V11=V["11"], V21=V["21"], V31=V["31"], V12=V["12"], V22=V["22"], V32=V["32"])


def apply_V_blockdiag(x, S):
    """exp1/apply_V_blockdiag.m:1-17 — 2n -> 3n."""
    n = S.NF
    x1, x2 = x[:n], x[n:2 * n]
    return np.concatenate([S.V11 * x1 + S.V12 * x2, S.V21 * x1 + S.V22 * x2,
                           S.V31 * x1 + S.V32 * x2])


def apply_VH_blockdiag(x, S):
    """exp1/apply_VH_blockdiag.m:1-16 — 3n -> 2n."""
    n = S.NF
    x1, x2, x3 = x[:n], x[n:2 * n], x[2 * n:]
    c = np.conj
    return np.concatenate([c(S.V11) * x1 + c(S.V21) * x2 + c(S.V31) * x3,
                           c(S.V12) * x1 + c(S.V22) * x2 + c(S.V32) * x3])


def solveV1_blockdiag(x, V11, V12, V21, V22, det, n):
    """exp1/solveV1_blockdiag.m:1-10 — 2x2 Cramer solve y = V1^{-1} x."""
    x1, x2 = x[:n], x[n:2 * n]
    return np.concatenate([(V22 * x1 - V12 * x2) / det, (-V21 * x1 + V11 * x2) / det])


def solveV1H_blockdiag(x, V11, V12, V21, V22, det, n):
    """exp1/solveV1H_blockdiag.m:1-10 — y = V1^{-*} x."""
    c = np.conj
    x1, x2 = x[:n], x[n:2 * n]
    return np.concatenate([(c(V22) * x1 - c(V21) * x2) / c(det),
                           (-c(V12) * x1 + c(V11) * x2) / c(det)])


@dataclass
class QSystem:
    """The q-dependent system (exp1/build_experiment1_q_system.m:1-42)."""
    N: int
    NF: int
    P: np.ndarray
    q: np.ndarray
    kLift: np.ndarray
    mass: MassOp
    q1: np.ndarray
    q2: np.ndarray
    q3: np.ndarray
    Qq: np.ndarray
    V11: np.ndarray
    V12: np.ndarray
    V21: np.ndarray
    V22: np.ndarray
    V31: np.ndarray
    V32: np.ndarray
    detV1: np.ndarray
    W1: np.ndarray
    W2: np.ndarray
    invC: np.ndarray
    sigmaR: np.ndarray
    nsingular: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def nr(self):
        return 2 * self.NF

    def Kop(self, x):
        """exp1/assemble_K_and_nullspace_free_basis.m:110-119."""
        n = self.NF
        q1, q2, q3 = self.q1, self.q2, self.q3
        x1, x2, x3 = x[:n], x[n:2 * n], x[2 * n:]
        a = lambda t: np.abs(t) ** 2
        c = np.conj
        y1 = (a(q2) + a(q3)) * x1 - (q1 * c(q2)) * x2 - (q1 * c(q3)) * x3
        y2 = -(q2 * c(q1)) * x1 + (a(q1) + a(q3)) * x2 - (q2 * c(q3)) * x3
        y3 = -(q3 * c(q1)) * x1 - (q3 * c(q2)) * x2 + (a(q1) + a(q2)) * x3
        return np.concatenate([y1, y2, y3])

    def U0Hop(self, x):
        """exp1/assemble_K_and_nullspace_free_basis.m:121-127."""
        n = self.NF
        s = np.sqrt(self.Qq)
        c = np.conj
        return (c(self.q1 / s) * x[:n] + c(self.q2 / s) * x[n:2 * n]
                + c(self.q3 / s) * x[2 * n:])


def build_q_system(N, P, q, E):
    """exp1/build_experiment1_q_system.m:4-24 plus invC
    (exp1/build_inner_system_operators.m:10-14)."""
    P = np.asarray(P, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    kLift = P @ np.linalg.solve(P.T @ P, q)
    Xi = build_fourier_grid_6d(N)
    B = assemble_K_and_nullspace_free_basis(P, kLift, Xi)
    n = (2 * N) ** 6
    det = B["V11"] * B["V22"] - B["V12"] * B["V21"]
    W = solveV1H_blockdiag(np.concatenate([np.conj(B["V31"]), np.conj(B["V32"])]),
                           B["V11"], B["V12"], B["V21"], B["V22"], det, n)
    W1, W2 = W[:n], W[n:]
    Korth = np.real(1 + np.abs(W1) ** 2 + np.abs(W2) ** 2)
    if Korth.min() <= 0:
        raise ValueError("Korth has a nonpositive diagonal entry.")
    return QSystem(N=N, NF=n, P=P, q=q, kLift=kLift, mass=MassOp(E, N),
                   q1=B["q1"], q2=B["q2"], q3=B["q3"], Qq=B["Qq"],
                   V11=B["V11"], V12=B["V12"], V21=B["V21"], V22=B["V22"],
                   V31=B["V31"], V32=B["V32"], detV1=det, W1=W1, W2=W2,
                   invC=1.0 / np.sqrt(Korth), sigmaR=np.concatenate([B["Qq"], B["Qq"]]),
                   nsingular=B["nsingular"])


def apply_Mhat_C_scalar_compact(x, S):
    """exp1/apply_Mhat_C_scalar_compact.m:8-21."""
    z = S.invC * x
    s = S.mass.scalar(z)
    s = s + np.conj(S.W1) * S.mass.scalar(S.W1 * z)
    s = s + np.conj(S.W2) * S.mass.scalar(S.W2 * z)
    return S.invC * s


# ---------------------------------------------------------------------------
# Krylov solvers
# ---------------------------------------------------------------------------

def pcg(A, b, tol, maxit, M=None):
    """MATLAB ``pcg(A,b,tol,maxit,M,[],zeros)`` restated (closed builtin).

    Returns ``(x, flag, relres, iters)``.  Convergence is tested on the
    recursive residual and confirmed on the true residual ``b - A x`` (the
    true residual then replaces the recursive one), as MATLAB documents.
    """
    n2b = np.linalg.norm(b)
    x = np.zeros_like(b)
    if n2b == 0:
        return x, 0, 0.0, 0
    tolb = tol * n2b
    r = b.copy()
    normr = n2b
    rho = 1.0
    p = None
    best = (x.copy(), normr)
    moresteps = 0
    for ii in range(1, maxit + 1):
        z = M(r) if M is not None else r
        rho1 = rho
        rho = np.vdot(r, z)
        if rho == 0 or not np.isfinite(rho):
            return best[0], 4, best[1] / n2b, ii - 1
        if ii == 1:
            p = z.copy()
        else:
            beta = rho / rho1
            p = z + beta * p
        q = A(p)
        pq = np.vdot(p, q)
        if np.real(pq) <= 0 or not np.isfinite(pq):
            return best[0], 4, best[1] / n2b, ii - 1
        alpha = rho / pq
        x = x + alpha * p
        r = r - alpha * q
        normr = np.linalg.norm(r)
        if normr <= tolb:
            r = b - A(x)
            normr_act = np.linalg.norm(r)
            if normr_act <= tolb:
                return x, 0, normr_act / n2b, ii
            moresteps += 1
            if moresteps >= 3:
                return x, 3, normr_act / n2b, ii
            normr = normr_act
        if normr < best[1]:
            best = (x.copy(), normr)
    rtrue = np.linalg.norm(b - A(best[0]))
    return best[0], 1, rtrue / n2b, maxit


def make_explicit_krinv_compact(S, tolCG=1e-10, maxitCG=1200):
    """exp1/make_explicit_krinv_compact.m:24-80 — K_r^{-1} by the explicit form.

    Returns ``(KrInvOp, getStats)``.
    """
    n = S.NF
    stats = dict(inverseCalls=0, totalMhatIterations=0, maxMhatIterations=0,
                 maxMhatRelativeResidual=0.0, flags=[], iterations=[],
                 relativeResiduals=[])

    def applyOne(qv):
        if qv.shape[0] != 2 * n:
            raise ValueError("Explicit K_r^{-1} input must have 2*NF rows.")
        if not np.all(np.isfinite(qv)):
            raise ValueError("Explicit K_r^{-1} input contains NaN/Inf.")
        r = solveV1H_blockdiag(qv, S.V11, S.V12, S.V21, S.V22, S.detV1, n)
        mr1 = S.mass.scalar(r[:n])
        mr2 = S.mass.scalar(r[n:])
        b = -(np.conj(S.W1) * mr1 + np.conj(S.W2) * mr2)
        bhat = S.invC * b
        u, flag, relres, it = pcg(lambda v: apply_Mhat_C_scalar_compact(v, S), bhat,
                                  tolCG, maxitCG)
        if not np.all(np.isfinite(u)) or (flag != 0 and relres > 10 * tolCG):
            raise RuntimeError("Mhat CG failed: flag=%d relres=%.3e iter=%d" % (flag, relres, it))
        z = S.invC * u
        mr1 = mr1 + S.mass.scalar(S.W1 * z)
        mr2 = mr2 + S.mass.scalar(S.W2 * z)
        y = solveV1_blockdiag(np.concatenate([mr1, mr2]), S.V11, S.V12, S.V21, S.V22,
                              S.detV1, n)
        stats["inverseCalls"] += 1
        stats["totalMhatIterations"] += it
        stats["maxMhatIterations"] = max(stats["maxMhatIterations"], it)
        stats["maxMhatRelativeResidual"] = max(stats["maxMhatRelativeResidual"], relres)
        stats["flags"].append(flag)
        stats["iterations"].append(it)
        stats["relativeResiduals"].append(relres)
        return y

    def op(qv):
        if qv.ndim == 1:
            return applyOne(qv)
        return np.stack([applyOne(qv[:, j]) for j in range(qv.shape[1])], axis=1)

    return op, (lambda: dict(stats))


def make_nested_krinv_instrumented(S, epsC=4.0, tolKr=1e-10, tolM=1e-12, maxitKr=600,
                                   maxitM=1600, useKrPreconditioner=True):
    """exp1/make_nested_krinv_instrumented.m:33-126 — K_r z = V^* M^{-1} V z by
    outer PCG with an inner PCG on the full mass per matvec."""
    stats = dict(inverseCalls=0, totalKrIterations=0, massSolveCalls=0,
                 totalMassIterations=0, krIterations=[], massIterations=[])

    def applyKr(z):
        Vz = apply_V_blockdiag(z, S)
        y, flag, rr, it = pcg(S.mass.full, Vz, tolM, maxitM)
        if not np.all(np.isfinite(y)) or (flag != 0 and rr > 10 * tolM):
            raise RuntimeError("Nested M solve failed")
        stats["massSolveCalls"] += 1
        stats["totalMassIterations"] += it
        stats["massIterations"].append(it)
        return apply_VH_blockdiag(y, S)

    M1 = (lambda r: epsC * (r / S.sigmaR)) if useKrPreconditioner else None

    def applyOne(b):
        if b.shape[0] != S.nr:
            raise ValueError("Nested K_r^{-1} input must have 2*NF rows.")
        x, flag, rr, it = pcg(applyKr, b, tolKr, maxitKr, M1)
        if not np.all(np.isfinite(x)) or (flag != 0 and rr > 10 * tolKr):
            raise RuntimeError("Nested K_r solve failed")
        stats["inverseCalls"] += 1
        stats["totalKrIterations"] += it
        stats["krIterations"].append(it)
        return x

    def op(b):
        if b.ndim == 1:
            return applyOne(b)
        return np.stack([applyOne(b[:, j]) for j in range(b.shape[1])], axis=1)

    return op, (lambda: dict(stats))


def _mgs(Q, r, jj):
    """exp2/Lanczos.m:150-155 — GramSchmitGEP with B = I (modified GS over jj cols)."""
    for kk in range(jj):
        r = r - np.vdot(Q[:, kk], r) * Q[:, kk]
    return r


def Lanczos(fncA, n, k, tol, maxiter, p, v0):
    """exp2/Lanczos.m:1-148 with fncB = fncBinv = identity.

    Returns ``(ev, ew, iter, info)``: Ritz vectors (n x k), Ritz values theta
    (descending), total Lanczos steps, and per-restart info.
    """
    eps0 = np.finfo(np.float64).eps
    v = v0 / math.sqrt(abs(np.vdot(v0, v0)))
    Q = np.zeros((n, p), dtype=np.complex128)
    k0 = k
    Alpha, Beta = [], []
    beta = 0.0
    d = np.zeros(0)
    c = np.zeros(0)
    justRestarted = False
    sizeV = 1
    kk = 0
    info = dict(restart=[], totalIter=[], maxWantedResidual=[], ritzValues=[])
    Usmall = None
    ind = None
    for mm in range(1, maxiter + 1):
        for jj in range(sizeV, p + 1):
            j = jj - 1
            Q[:, j] = v
            Aq = fncA(Q[:, j])
            alpha = float(np.real(np.vdot(Aq, Q[:, j])))
            pr = Aq
            if jj == 1:
                r = pr - alpha * Q[:, j]
            elif justRestarted:
                r = _mgs(Q, pr, jj)
                justRestarted = False
            else:
                r = pr - alpha * Q[:, j] - beta * Q[:, j - 1]
                r = r - np.vdot(Q[:, j - 1], r) * Q[:, j - 1]
            r = r - np.vdot(Q[:, j], r) * Q[:, j]
            r = _mgs(Q, r, jj)
            r = _mgs(Q, r, jj)
            beta2 = float(np.real(np.vdot(r, r)))
            if beta2 <= 0 or math.sqrt(beta2) < 1e-14:
                beta = math.sqrt(max(beta2, 0.0))
                break
            beta = math.sqrt(beta2)
            v = r / beta
            Alpha.append(alpha)
            Beta.append(beta)
            kk += 1
        m1 = len(Alpha)
        H1 = np.diag(Alpha) + np.diag(Beta[:-1], 1) + np.diag(Beta[:-1], -1)
        kd = len(d)
        H = np.zeros((kd + m1, kd + m1))
        H[:kd, :kd] = np.diag(d)
        H[kd:, kd:] = H1
        if kd:
            H[:kd, kd] = c
            H[kd, :kd] = c
        Alpha, Beta = [], []
        dvals, Usmall = np.linalg.eigh(H)
        res = np.abs(beta * Usmall[-1, :])
        ind = np.argsort(-dvals, kind="stable")
        d = dvals[ind]
        res = res[ind]
        wanted = slice(0, min(k0, len(res)))
        info["restart"].append(mm)
        info["totalIter"].append(kk)
        info["maxWantedResidual"].append(float(res[wanted].max()))
        info["ritzValues"].append(d[wanted].copy())
        threshold = tol * np.maximum(eps0 ** (2.0 / 3.0), np.abs(d[wanted]))
        nconv = int(np.count_nonzero(res[wanted] < threshold))
        if nconv >= k0 or mm == maxiter:
            info["converged"] = nconv >= k0
            info["nconv"] = nconv
            break
        k = k0 + min(nconv, (p - k0) // 2)
        if k == 1 and p > 3:
            k = p // 2
        keep = ind[:k]
        Ukeep = Usmall[:, keep]
        Q[:, :k] = Q[:, :Ukeep.shape[0]] @ Ukeep
        d = d[:k]
        c = beta * Ukeep[-1, :]
        justRestarted = True
        sizeV = k + 1
    Ukeep = Usmall[:, ind[:k0]]
    U = Q[:, :Ukeep.shape[0]] @ Ukeep
    return U, d[:k0], kk, info


def start_vector(seed: int, n: int):
    """Counter-based start vector shared with the device generator.

    Element i has real part u(2i) and imaginary part u(2i+1) with
    u(c) = 2*((splitmix64(seed + (c+1)*0x9E3779B97F4A7C15) >> 11) * 2^-53) - 1.
    (The reference draws v0 with MATLAB's Mersenne twister, whose stream
    cannot be reproduced outside MATLAB.)
    """
    with np.errstate(over="ignore"):
        c = np.arange(2 * n, dtype=np.uint64)
        z = np.uint64(seed) + (c + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
    u = 2 * u - 1
    return u[0::2] + 1j * u[1::2]


def recover_original_eigenvectors(Y, S, tol=1e-12, maxit=3000):
    """exp2/recover_original_eigenvectors_exp2.m:12-50 — x = M^{-1} V y, M-normalised."""
    k = Y.shape[1]
    X = np.zeros((3 * S.NF, k), dtype=np.complex128)
    MX = np.zeros_like(X)
    its = []
    for j in range(k):
        rhs = apply_V_blockdiag(Y[:, j], S)
        xj, flag, rr, it = pcg(S.mass.full, rhs, tol, maxit)
        if flag != 0 and rr > 10 * tol:
            raise RuntimeError("recover_original_eigenvectors_exp2:RecoveryCGFailure")
        Mx = S.mass.full(xj)
        nj2 = float(np.real(np.vdot(xj, Mx)))
        s = math.sqrt(nj2)
        X[:, j] = xj / s
        MX[:, j] = Mx / s
        its.append(it)
    return X, MX, dict(iterations=its)


def compute_fourier_diagnostics(X, MX, lam, S):
    """exp2/compute_fourier_diagnostics_exp2.m:10-19."""
    eps = np.finfo(float).eps
    res, div, ray = [], [], []
    D0 = np.sqrt(S.Qq)
    for j in range(X.shape[1]):
        x, Mx = X[:, j], MX[:, j]
        Kx = S.Kop(x)
        ray.append(float(np.real(np.vdot(x, Kx) / np.vdot(x, Mx))))
        den = np.linalg.norm(Kx) + abs(lam[j]) * np.linalg.norm(Mx)
        res.append(np.linalg.norm(Kx - lam[j] * Mx) / max(den, eps))
        div.append(np.linalg.norm(D0 * S.U0Hop(Mx)) / max(np.linalg.norm(Mx), eps))
    return dict(resGEVP=np.array(res), divRelative2=np.array(div), rayleigh=np.array(ray))


def solve_modes(S, nev=10, p=40, tol=1e-8, maxRestart=30, tolCG=1e-10, seed=20260905,
                method="explicit", **kw):
    """exp2/solve_modes_exp3.m:13-52 — inverse Lanczos on K_r^{-1}, lambda = 1/theta."""
    if method == "explicit":
        op, getStats = make_explicit_krinv_compact(S, tolCG, kw.get("maxitCG", 3000))
    else:
        op, getStats = make_nested_krinv_instrumented(S, **kw)
    v0 = start_vector(seed, S.nr)
    Y, theta, steps, info = Lanczos(op, S.nr, nev, tol, maxRestart, p, v0)
    lam = np.real(1.0 / theta)
    order = np.argsort(lam, kind="stable")
    return dict(lam=lam[order], Y=Y[:, order], theta=theta[order], steps=steps,
                info=info, stats=getStats())


def apply_Kr_exact(y, S):
    """K_r y = V^* M^{-1} V y (exp1/make_nested_krinv_instrumented.m:4-13) with the exact
    grid inverse of the mass instead of the inner PCG on M."""
    n = S.NF
    v = apply_V_blockdiag(y, S)
    w = np.concatenate([S.mass.inverse_scalar(v[c * n:(c + 1) * n]) for c in range(3)])
    return apply_VH_blockdiag(w, S)


def rayleigh_ritz_Kr(Y, S):
    """Rayleigh-Ritz refinement of approximate eigenvectors Y (2NF x k) of K_r with the
    exact K_r (no reference counterpart; the reference reports 1/theta of the Lanczos
    Ritz values, exp2/Lanczos.m:140-147).  Returns (lam ascending, Y refined, relres)."""
    Y = np.asarray(Y, dtype=np.complex128)
    Z = np.stack([apply_Kr_exact(Y[:, j], S) for j in range(Y.shape[1])], axis=1)
    G = Y.conj().T @ Z
    B = Y.conj().T @ Y
    G = 0.5 * (G + G.conj().T)
    B = 0.5 * (B + B.conj().T)
    L = np.linalg.cholesky(B)
    Li = np.linalg.inv(L)
    lam, U = np.linalg.eigh(Li @ G @ Li.conj().T)
    R = Li.conj().T @ U
    Yr, Zr = Y @ R, Z @ R
    relres = np.linalg.norm(Zr - Yr * lam, axis=0) / np.linalg.norm(Zr, axis=0)
    return lam, Yr, relres


def dense_reduced_operator(S):
    """Dense K_r = V^* M^{-1} V (small N only; an independent check of the solver)."""
    n = S.NF
    Mdense = np.stack([S.mass.scalar(np.eye(n, dtype=np.complex128)[:, j]) for j in range(n)],
                      axis=1)
    Minv = np.linalg.inv(Mdense)
    V = np.zeros((3 * n, 2 * n), dtype=np.complex128)
    for j in range(2 * n):
        e = np.zeros(2 * n, dtype=np.complex128)
        e[j] = 1
        V[:, j] = apply_V_blockdiag(e, S)
    Minv3 = np.zeros((3 * n, 3 * n), dtype=np.complex128)
    for c in range(3):
        Minv3[c * n:(c + 1) * n, c * n:(c + 1) * n] = Minv
    return V.conj().T @ Minv3 @ V


def mass_adjoint_quadratic(X, dE, N):
    """x^H (dM) x for M(eps) x = fftn(eps .* ifftn(x)) per component.

    x^H fftn(dE .* ifftn(x)) = NF * sum_y dE(y) |ifftn(x)(y)|^2, summed over
    the three field components of each column of X.
    """
    NF = (2 * N) ** 6
    out = np.zeros((X.shape[1], len(dE)))
    for j in range(X.shape[1]):
        dens = np.zeros(NF)
        for c in range(3):
            u = np.fft.ifftn(_grid(X[c * NF:(c + 1) * NF, j], N)).reshape(-1, order="F")
            dens += np.abs(u) ** 2
        for t, g in enumerate(dE):
            out[j, t] = NF * float(np.dot(g, dens))
    return out


# ---------------------------------------------------------------------------
# Yee reconstruction
# ---------------------------------------------------------------------------

def build_projected_q_modes(P, kLift, N):
    """exp2/build_projected_q_modes.m:4-10 — NF x 3 projected wave vectors."""
    Xi = build_fourier_grid_6d(N)
    Q = np.zeros((len(Xi[0]), 3))
    for ell in range(6):
        s = Xi[ell] + kLift[ell]
        for c in range(3):
            Q[:, c] += P[ell, c] * s
    return Q


def build_yee_points(n, h):
    """exp2/build_yee_edge_points_plus.m:11-17 — three staggered plus-grids."""
    idx = np.arange(-(n + 1), n + 2, dtype=np.float64)
    I, J, K = np.meshgrid(idx, idx, idx, indexing="ij")
    I, J, K = (a.reshape(-1, order="F") for a in (I, J, K))
    r1 = h * np.stack([I + 0.5, J, K], axis=1)
    r2 = h * np.stack([I, J + 0.5, K], axis=1)
    r3 = h * np.stack([I, J, K + 0.5], axis=1)
    return r1, r2, r3, (len(idx),) * 3


def build_yee_block_partition(szPlus, nBlocks):
    """exp2/build_yee_block_partition_exp3.m:1-31 (0-based index lists)."""
    m = szPlus[0]
    base, rem = divmod(m, nBlocks)
    groups, s = [], 0
    for b in range(nBlocks):
        ln = base + (1 if b < rem else 0)
        groups.append(np.arange(s, s + ln))
        s += ln
    blocks = []
    for k in range(nBlocks):
        for j in range(nBlocks):
            for i in range(nBlocks):
                I, J, K = np.meshgrid(groups[i], groups[j], groups[k], indexing="ij")
                blocks.append((I + m * J + m * m * K).reshape(-1, order="F"))
    return blocks


def build_multi_index_list_3d(p):
    """exp2/build_multi_index_list_3d_exp3.m:3-14 — a1 outer, a3 inner."""
    return np.array([(a1, a2, a3) for a1 in range(p + 1) for a2 in range(p - a1 + 1)
                     for a3 in range(p - a1 - a2 + 1)], dtype=np.int64)


def taylor_coeff_alpha(alphaList):
    """i^|a| / a! (exp2/taylor_on_blocks_exp3.m:25-29)."""
    out = np.zeros(len(alphaList), dtype=np.complex128)
    for i, a in enumerate(alphaList):
        out[i] = (1j) ** int(sum(a)) * math.exp(-sum(math.lgamma(t + 1) for t in a))
    return out


def taylor_on_blocks(coeff, qModes, rPoints, p, blocks, fixedCenter=None, termBatchSize=32):
    """exp2/taylor_on_blocks_exp3.m:8-79 — multi-center separated Taylor evaluation."""
    coeff = np.asarray(coeff).reshape(-1)
    alphaList = build_multi_index_list_3d(p)
    L = len(alphaList)
    Qx = np.ones((len(coeff), p + 1))
    Qy, Qz = Qx.copy(), Qx.copy()
    for s in range(1, p + 1):
        Qx[:, s] = Qx[:, s - 1] * qModes[:, 0]
        Qy[:, s] = Qy[:, s - 1] * qModes[:, 1]
        Qz[:, s] = Qz[:, s - 1] * qModes[:, 2]
    ca = taylor_coeff_alpha(alphaList)
    u = np.zeros(rPoints.shape[0], dtype=np.complex128)
    for ids in blocks:
        R = rPoints[ids]
        rc = (R.min(0) + R.max(0)) / 2 if fixedCenter is None else np.asarray(fixedCenter, float)
        Rc = R - rc
        cC = coeff * np.exp(1j * (qModes @ rc))
        Rx = np.ones((len(ids), p + 1))
        Ry, Rz = Rx.copy(), Rx.copy()
        for s in range(1, p + 1):
            Rx[:, s] = Rx[:, s - 1] * Rc[:, 0]
            Ry[:, s] = Ry[:, s - 1] * Rc[:, 1]
            Rz[:, s] = Rz[:, s - 1] * Rc[:, 2]
        ub = np.zeros(len(ids), dtype=np.complex128)
        for s0 in range(0, L, termBatchSize):
            aa = alphaList[s0:s0 + termBatchSize]
            Qb = Qx[:, aa[:, 0]] * Qy[:, aa[:, 1]] * Qz[:, aa[:, 2]]
            Rb = Rx[:, aa[:, 0]] * Ry[:, aa[:, 1]] * Rz[:, aa[:, 2]]
            mom = ca[s0:s0 + termBatchSize] * (Qb.T @ cC)
            ub += Rb @ mom
        u[ids] = ub
    return u


def reconstruct_field_taylor_multi(coeff, qModes, rPoints, p, blocks, termBatchSize=32):
    """exp2/reconstruct_field_taylor_multi_exp3.m:1-10."""
    return taylor_on_blocks(coeff, qModes, rPoints, p, blocks, None, termBatchSize)


def reconstruct_field_taylor_single(coeff, qModes, rPoints, p, r0=(0.0, 0.0, 0.0)):
    """exp2/reconstruct_field_taylor_single_exp3.m:1-10."""
    return taylor_on_blocks(coeff, qModes, rPoints, p, [np.arange(rPoints.shape[0])], r0)


def reconstruct_field_direct_blocked(coeff, qModes, rPoints, blockSize=512):
    """exp2/reconstruct_field_direct_blocked_exp3.m:8-15 — u = exp(i R Q^T) c."""
    coeff = np.asarray(coeff).reshape(-1)
    u = np.zeros(rPoints.shape[0], dtype=np.complex128)
    for s in range(0, rPoints.shape[0], blockSize):
        ph = rPoints[s:s + blockSize] @ qModes.T
        u[s:s + blockSize] = np.exp(1j * ph) @ coeff
    return u


def reconstruct_component_taylor_batch(coeffMat, qModes, rPoints, p, blocks):
    """exp3/reconstruct_component_taylor_batch_exp4.m:14-38 — the GEMM form
    (moments = Qalpha^T * (c .* phase), then per-point evaluation)."""
    coeffMat = np.asarray(coeffMat).reshape(qModes.shape[0], -1)
    alphaList = build_multi_index_list_3d(p)
    ca = taylor_coeff_alpha(alphaList)
    Qalpha = np.stack([qModes[:, 0] ** a[0] * qModes[:, 1] ** a[1] * qModes[:, 2] ** a[2]
                       for a in alphaList], axis=1)
    centers = np.stack([(rPoints[ids].min(0) + rPoints[ids].max(0)) / 2 for ids in blocks])
    ph = np.exp(1j * (qModes @ centers.T))  # NF x C
    mom = ca[:, None, None] * np.einsum("fl,fc,fr->lcr", Qalpha, ph, coeffMat)
    u = np.zeros((rPoints.shape[0], coeffMat.shape[1]), dtype=np.complex128)
    for ib, ids in enumerate(blocks):
        Rc = rPoints[ids] - centers[ib]
        phi = np.stack([Rc[:, 0] ** a[0] * Rc[:, 1] ** a[1] * Rc[:, 2] ** a[2]
                        for a in alphaList], axis=1)
        u[ids] = phi @ mom[:, ib, :]
    return u


# ------------------------------------------------------------------ LWRQ (a22)
# Physical validation of a reconstructed Yee field: cropped curl-curl action,
# scalar material on the Yee edges, local Gaussian-window Rayleigh quotient.
# Fields are (m, m, m) arrays on the plus-grid (m = 2n+3), axis 0 = x (the
# column-major order of exp2/build_yee_edge_points_plus.m:11-17).

def _inner(u, dx, dy, dz):
    """u at the interior points shifted by (dx, dy, dz) cells."""
    m = u.shape[0]
    return u[1 + dx:m - 1 + dx, 1 + dy:m - 1 + dy, 1 + dz:m - 1 + dz]


def apply_cropped_A(u1, u2, u3, h):
    """exp3/apply_cropped_A_exp3.m:1-58 — Yee curl-curl on the (2n+1)^3 interior.

    Second differences along one axis and the mixed forward/backward differences
    of the curl-curl operator, scaled by 1/h^2.
    """
    s = _inner

    def second(u, ax):
        e = [0, 0, 0]
        e[ax] = 1
        return 2 * s(u, 0, 0, 0) - s(u, *[-v for v in e]) - s(u, *e)

    def mixed(u, back, fwd):
        # backward difference along `back` of the forward difference along `fwd`
        f = [0, 0, 0]
        f[fwd] = 1
        b = [0, 0, 0]
        b[back] = -1
        fb = [f[i] + b[i] for i in range(3)]
        return s(u, *fb) - s(u, *b) - s(u, *f) + s(u, 0, 0, 0)

    h2 = 1.0 / (h * h)
    A1 = h2 * (second(u1, 1) + second(u1, 2) - mixed(u2, 1, 0) - mixed(u3, 2, 0))
    A2 = h2 * (second(u2, 0) + second(u2, 2) - mixed(u1, 0, 1) - mixed(u3, 2, 1))
    A3 = h2 * (second(u3, 0) + second(u3, 1) - mixed(u1, 0, 2) - mixed(u2, 1, 2))
    return A1, A2, A3


def yee_material(P, n, h, material):
    """exp3/sample_scalar_yee_material_exp4.m:1-21 — eps on the three edge grids.

    material: ("exp", epsC, alpha) -> epsC exp(alpha/6 sum_l cos(P_l . x)), or
    ("cos", delta) -> 1 + delta prod_l (1 + cos(P_l . x))/2.
    """
    idx = np.arange(-n, n + 1, dtype=np.float64) * h
    P = np.asarray(P, dtype=np.float64)
    out = []
    for c in range(3):
        ax = [idx.copy(), idx.copy(), idx.copy()]
        ax[c] = ax[c] + h / 2
        X, Y, Z = np.meshgrid(*ax, indexing="ij")
        if material[0] == "exp":
            S = sum(np.cos(P[l, 0] * X + P[l, 1] * Y + P[l, 2] * Z) for l in range(P.shape[0]))
            out.append(material[1] * np.exp(material[2] / 6.0 * S))
        else:
            prod = np.ones_like(X)
            for l in range(P.shape[0]):
                prod = prod * (1 + np.cos(P[l, 0] * X + P[l, 1] * Y + P[l, 2] * Z)) / 2
            out.append(1.0 + material[1] * prod)
    return out


def separable_conv3_same(X, k):
    """exp3/separable_conv3_same_exp4.m:1-7 — zero-padded separable 3D convolution."""
    R = (len(k) - 1) // 2
    Y = X
    for ax in range(3):
        Z = np.zeros_like(Y)
        L = Y.shape[ax]
        for t in range(len(k)):
            sh = t - R  # Z(i) += k[t] * Y(i - sh)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            if sh >= 0:
                dst[ax] = slice(sh, L)
                src[ax] = slice(0, L - sh)
            else:
                dst[ax] = slice(0, L + sh)
                src[ax] = slice(-sh, L)
            Z[tuple(dst)] += k[t] * Y[tuple(src)]
        Y = Z
    return Y


def compute_lwrq(a, b, h, radius=3, sigma_factor=2.0, mass_floor=1e-14, return_rho=False):
    """exp3/compute_lwrq_exp4.m:12-58 — column-normalised local Gaussian RQ."""
    off = np.arange(-radius, radius + 1) * h
    sigma = sigma_factor * h
    k = np.exp(-(off ** 2) / sigma ** 2)
    den = separable_conv3_same(np.ones_like(a), k)
    if not np.all(np.isfinite(den)) or np.any(den <= 0):
        raise ValueError("Invalid LWRQ column-normalization denominator.")
    E = separable_conv3_same(a / den, k)
    M = separable_conv3_same(b / den, k)
    if not np.all(np.isfinite(M)) or np.any(M <= mass_floor * M.max()):
        raise ValueError("Nonpositive or numerically tiny local LWRQ mass encountered.")
    sumE, sumM = E.sum(), M.sum()
    lam = sumE / sumM
    rho = E / M
    V = np.sum(M * np.abs(rho - lam) ** 2) / (sumM * abs(lam) ** 2)
    sumA, sumB = a.sum(), b.sum()
    tiny = np.finfo(np.float64).eps
    part = max(abs(sumE - sumA) / max(abs(sumA), tiny), abs(sumM - sumB) / max(abs(sumB), tiny))
    return dict(lam=lam, V=V, nu=np.sqrt(max(V, 0.0)), partitionError=part, rho=rho if return_rho else None)


def compute_yee_lwrq_metrics(u1, u2, u3, lambda6D, P, n, h, material, save_spatial=False):
    """exp3/compute_yee_lwrq_metrics_exp4.m:1-100 — scalar LWRQ diagnostics of a
    reconstructed Yee field (u_c: (2n+3)^3 arrays, axis 0 = x)."""
    A1, A2, A3 = apply_cropped_A(u1, u2, u3, h)
    c1, c2, c3 = (_inner(u, 0, 0, 0) for u in (u1, u2, u3))
    e1, e2, e3 = yee_material(P, n, h, material)
    B1, B2, B3 = e1 * c1, e2 * c2, e3 * c3
    a = np.real(np.conj(c1) * A1 + np.conj(c2) * A2 + np.conj(c3) * A3)
    b = np.real(np.conj(c1) * B1 + np.conj(c2) * B2 + np.conj(c3) * B3)
    sumB = b.sum()
    if sumB <= 0:
        raise ValueError("Cropped Yee mass is not positive.")
    lamCrop = a.sum() / sumB
    L = compute_lwrq(a, b, h, return_rho=save_spatial)
    lam3 = float(np.real(L["lam"]))
    dId = abs(lam3 - lamCrop) / max(abs(lamCrop), np.finfo(np.float64).eps)
    nA = np.sqrt(sum(np.sum(np.abs(x) ** 2) for x in (A1, A2, A3)))
    nB = np.sqrt(sum(np.sum(np.abs(x) ** 2) for x in (B1, B2, B3)))

    def rsq(lam):
        return sum(np.sum(np.abs(Ax - lam * Bx) ** 2) for Ax, Bx in ((A1, B1), (A2, B2), (A3, B3)))

    m = dict(h=h, n=n, halfWidth=n * h, lambda6D=lambda6D, lambdaCrop=lamCrop, lambda3D=lam3,
             eta3D=np.sqrt(rsq(lam3)) / (nA + abs(lam3) * nB),
             etaUsing6DLambda=np.sqrt(rsq(lambda6D)) / (nA + abs(lambda6D) * nB),
             deltaLambda=abs(lam3 - lambda6D) / abs(lambda6D), VLWRQ=L["V"], nuLWRQ=L["nu"],
             deltaPart=L["partitionError"], deltaLWRQIdentity=dId, croppedMass=sumB)
    spatial = None
    if save_spatial:
        c = n
        spatial = dict(relativeDeviation_z0=np.abs(L["rho"][:, :, c] - lam3) / abs(lam3),
                       relativeDeviation_x0=np.abs(L["rho"][c, :, :] - lam3) / abs(lam3))
    return m, spatial


# ---------------------------------------------------------------------------
# Method A: original shift-invert on the full 3NF space (comparison path)
# ---------------------------------------------------------------------------

def apply_K_original(x, S):
    """exp1/build_experiment1_q_system_A_only.m:61-73 (applyK): per mode
    K_q = |q|^2 I - q q^*, components stacked [x1; x2; x3]."""
    n = S.NF
    x1, x2, x3 = x[:n], x[n:2 * n], x[2 * n:]
    q1, q2, q3 = S.q1, S.q2, S.q3
    y1 = (np.abs(q2) ** 2 + np.abs(q3) ** 2) * x1 - (q1 * np.conj(q2)) * x2 - (q1 * np.conj(q3)) * x3
    y2 = -(q2 * np.conj(q1)) * x1 + (np.abs(q1) ** 2 + np.abs(q3) ** 2) * x2 - (q2 * np.conj(q3)) * x3
    y3 = -(q3 * np.conj(q1)) * x1 - (q3 * np.conj(q2)) * x2 + (np.abs(q1) ** 2 + np.abs(q2) ** 2) * x3
    return np.concatenate([y1, y2, y3])


def apply_shift_preconditioner(x, S, tau):
    """exp1/build_original_shift_preconditioner_A_only.m:24-54: (K + tau I)^{-1} x mode by mode,
    1/(Q+tau) x + (1/tau - 1/(Q+tau)) q (q^* x) / Q."""
    if not tau > 0:
        raise ValueError("Preconditioner tau must be finite and positive.")
    n = S.NF
    q1, q2, q3 = S.q1, S.q2, S.q3
    Q = np.abs(q1) ** 2 + np.abs(q2) ** 2 + np.abs(q3) ** 2
    invTrans = 1.0 / (Q + tau)
    corr = (1.0 / tau - invTrans) / Q
    x1, x2, x3 = x[:n], x[n:2 * n], x[2 * n:]
    cqx = corr * (np.conj(q1) * x1 + np.conj(q2) * x2 + np.conj(q3) * x3)
    return np.concatenate([invTrans * x1 + q1 * cqx, invTrans * x2 + q2 * cqx, invTrans * x3 + q3 * cqx])


def minres(A, b, tol, maxit, M=None):
    """Preconditioned MINRES for Hermitian A and SPD preconditioner (the callable M
    applies its inverse), x0 = 0, restating the Paige-Saunders recurrences that MATLAB's
    minres implements (the reference's shifted solve, exp1/make_A_eigs_top_preconditioned.m:
    285-286).  Stops when the recursive preconditioned residual norm phibar <= tol*beta1;
    returns (x, iterations, true relative residual)."""
    Minv = M if M is not None else (lambda r: r)
    x = np.zeros_like(b)
    r1 = b.copy()
    y = Minv(r1)
    beta1 = math.sqrt(max(np.real(np.vdot(r1, y)), 0.0))
    if beta1 == 0.0:
        return x, 0, 0.0
    oldb, beta, dbar, epsln, phibar, cs, sn = 0.0, beta1, 0.0, 0.0, beta1, -1.0, 0.0
    w = np.zeros_like(b)
    w2 = np.zeros_like(b)
    r2 = r1.copy()
    it = 0
    for it in range(1, maxit + 1):
        v = y / beta
        y = A(v)
        if it >= 2:
            y = y - (beta / oldb) * r1
        alfa = np.real(np.vdot(v, y))
        y = y - (alfa / beta) * r2
        r1, r2 = r2, y
        y = Minv(r2)
        oldb, beta = beta, math.sqrt(max(np.real(np.vdot(r2, y)), 0.0))
        oldeps = epsln
        delta = cs * dbar + sn * alfa
        gbar = sn * dbar - cs * alfa
        epsln = sn * beta
        dbar = -cs * beta
        gamma = max(math.hypot(gbar, beta), 1e-300)
        cs, sn = gbar / gamma, beta / gamma
        phi = cs * phibar
        phibar = sn * phibar
        w1, w2 = w2, w
        w = (v - oldeps * w1 - delta * w2) / gamma
        x = x + phi * w
        if phibar <= tol * beta1 or beta == 0.0:
            break
    relres = np.linalg.norm(b - A(x)) / np.linalg.norm(b)
    return x, it, relres


def osi_top_apply(x, S, sigma, tau, tol=1e-12, maxit=4000):
    """exp1/make_A_eigs_top_preconditioned.m:61-113: T x = (K - sigma M)^{-1} M x by
    preconditioned MINRES with the spectral preconditioner (K + tau I)^{-1}."""
    rhs = S.mass.full(x)
    A = lambda u: apply_K_original(u, S) - sigma * S.mass.full(u)  # noqa: E731
    return minres(A, rhs, tol, maxit, lambda r: apply_shift_preconditioner(r, S, tau))


def dense_original_operators(S):
    """Dense K (block 3x3 per mode) and M3 = blkdiag(M, M, M) of the original GEVP
    K x = lambda M x (small N only)."""
    n = S.NF
    I3n = np.eye(3 * n, dtype=np.complex128)
    K = np.stack([apply_K_original(I3n[:, j], S) for j in range(3 * n)], axis=1)
    Ms = np.stack([S.mass.scalar(np.eye(n, dtype=np.complex128)[:, j]) for j in range(n)], axis=1)
    M3 = np.zeros((3 * n, 3 * n), dtype=np.complex128)
    for c in range(3):
        M3[c * n:(c + 1) * n, c * n:(c + 1) * n] = Ms
    return K, M3


def dense_original_gevp(S):
    """All eigenvalues (ascending) of K x = lambda M x: NF zeros (gradient fields) and the
    2NF positive eigenvalues that the null-space-free methods compute."""
    K, M3 = dense_original_operators(S)
    Lc = np.linalg.cholesky((M3 + M3.conj().T) / 2)
    Li = np.linalg.inv(Lc)
    H = Li @ ((K + K.conj().T) / 2) @ Li.conj().T
    return np.sort(np.linalg.eigvalsh((H + H.conj().T) / 2))
