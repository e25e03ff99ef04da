"""Host-side mirror of the reference's hot-path interface over the C ABI.

Names, argument meaning and error behaviour follow the reference MATLAB
functions (cited per function).  Arrays are CUDA torch tensors used only as
device buffers: complex vectors are ``torch.complex128`` (``complex64`` for
FP32 entry points), matrices are column-major (``x[:, j]`` is column j, i.e.
``x.T`` is contiguous).  Every operation runs in libfame_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from ._lib import FameError, call

__all__ = [
    "Context", "applyMij_fft", "MassBackend", "apply_V_blockdiag", "apply_VH_blockdiag",
    "solveV1_blockdiag", "solveV1H_blockdiag", "QSystem", "build_q_system",
    "make_explicit_krinv_compact", "make_nested_krinv_instrumented", "KrInv", "Lanczos",
    "start_vector", "FameError", "apply_Mhat_C_scalar_compact", "kernel_launches", "solve_batch",
    "rayleigh_ritz", "rank1_exact_fft_scatter", "rank1_exact_ifft_gather", "tune_batch",
]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _colmajor(x: torch.Tensor, dtype=torch.complex128):
    """Return (tensor, nrows, ncols) with column-major storage on the device."""
    if x.dtype != dtype:
        raise TypeError("expected %s, got %s" % (dtype, x.dtype))
    if not x.is_cuda:
        raise TypeError("expected a CUDA tensor")
    if x.dim() == 1:
        return x.contiguous(), x.shape[0], 1
    if x.dim() != 2:
        raise ValueError("expected a vector or a matrix")
    xt = x.t().contiguous()
    return xt, x.shape[0], x.shape[1]


def _new_colmajor(nrows, ncols, like, dtype=torch.complex128):
    if ncols == 1 and like.dim() == 1:
        return torch.empty(nrows, dtype=dtype, device=like.device), None
    buf = torch.empty(ncols, nrows, dtype=dtype, device=like.device)
    return buf, buf.t()


class Context:
    """Device context (replaces gpu_initialize / wait_for_gpu, exp1/wait_for_gpu.m:5-11).

    Work is queued on torch's current CUDA stream, so results are ordered
    with surrounding torch operations.
    """

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        call("fame_ctx_create", device, C.byref(h))
        self.h = h

    def bind(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        call("fame_ctx_set_stream", self.h, C.c_void_p(s))
        return self.h

    def sync(self):
        call("fame_ctx_sync", self.bind())

    def close(self):
        if self.h:
            L.lib.fame_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = {}


def default_context(device=None) -> Context:
    dev = torch.cuda.current_device() if device is None else device
    if dev not in _default_ctx:
        _default_ctx[dev] = Context(dev)
    return _default_ctx[dev]


def _grid_N(n_rows: int) -> int:
    for N in range(1, 8):
        if (2 * N) ** 6 == n_rows:
            return N
    raise ValueError("row count %d is not (2N)^6 for N in 1..7" % n_rows)


def applyMij_fft(x, Eij, N=None, ctx: Context | None = None):
    """exp1/applyMij_fft.m:1-24 — y = fftn(Eij .* ifftn(x)) per column.

    ``x``: complex128 (FP64) or complex64 (FP32), NF rows; ``Eij``: float64 real-space
    material (NF,) in column-major grid order.
    """
    ctx = ctx or default_context()
    prec = L.FAME_F32 if x.dtype == torch.complex64 else L.FAME_F64
    xc, n, k = _colmajor(x, x.dtype)
    N = N or _grid_N(n)
    E = Eij.contiguous()
    if E.dtype != torch.float64 or E.numel() != n:
        raise ValueError("Eij must be float64 with NF entries")
    y, view = _new_colmajor(n, k, x, x.dtype)
    call("fame_applyMij_fft", ctx.bind(), N, _ptr(E), _ptr(xc), _ptr(y), k, prec)
    return y if view is None else view


class MassBackend:
    """The mass struct of exp1/build_mass_backend_large_scalar.m:27-46.

    Handles ``Mop`` (3NF), ``Mcol3op`` (NF -> [0;0;Mx]), ``Mcols12op``
    (2NF -> [Mx1;Mx2;0]) and ``MscalarOp`` (NF), all the same exact operator.
    """

    def __init__(self, E: torch.Tensor, N: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.N, self.NF = N, (2 * N) ** 6
        self.E = E.contiguous()
        if self.E.dtype != torch.float64 or self.E.numel() != self.NF:
            raise ValueError("E must be float64 with (2N)^6 entries")
        h = C.c_void_p()
        call("fame_mass_create", self.ctx.bind(), N, _ptr(self.E), C.byref(h))
        self.h = h
        self.name = "fft6d-scalar"
        self.info = dict(name=self.name, N=N, NF=self.NF, M=self.NF, MOverNF=1.0)

    def _apply(self, mode, x, rows_in, rows_out):
        prec = L.FAME_F32 if x.dtype == torch.complex64 else L.FAME_F64
        xc, n, k = _colmajor(x, x.dtype)
        if n != rows_in:
            raise FameError(L.FAME_ERR_INVALID, "input must have %d rows" % rows_in)
        y, view = _new_colmajor(rows_out, k, x, x.dtype)
        self.ctx.bind()
        call("fame_mass_apply", self.h, mode, _ptr(xc), _ptr(y), k, prec)
        return y if view is None else view

    def MscalarOp(self, x):
        return self._apply(L.FAME_MASS_SCALAR, x, self.NF, self.NF)

    def Mop(self, U):
        return self._apply(L.FAME_MASS_FULL3, U, 3 * self.NF, 3 * self.NF)

    def Mcol3op(self, x):
        return self._apply(L.FAME_MASS_COL3, x, self.NF, 3 * self.NF)

    def Mcols12op(self, x12):
        return self._apply(L.FAME_MASS_COLS12, x12, 2 * self.NF, 3 * self.NF)

    def applyMij_rank1_exact(self, x, plan):
        """exp1/applyMij_rank1_exact.m:1-6 with the reference plan struct.

        ``plan`` needs ``inputIdx``/``targetIdx`` (1-based uint32, NF each) and ``M``.
        """
        xc, n, k = _colmajor(x)
        if n != self.NF:
            raise FameError(L.FAME_ERR_INVALID, "rank1_exact_fft_scatter:BadSize")
        dev = x.device
        tin = torch.as_tensor(np.asarray(plan["inputIdx"], dtype=np.uint32).view(np.int32)).to(dev)
        ttg = torch.as_tensor(np.asarray(plan["targetIdx"], dtype=np.uint32).view(np.int32)).to(dev)
        y, view = _new_colmajor(n, k, x)
        self.ctx.bind()
        call("fame_applyMij_rank1_exact", self.h, _ptr(tin), _ptr(ttg), int(plan["M"]), _ptr(xc),
             _ptr(y), k)
        return y if view is None else view

    def close(self):
        if getattr(self, "h", None):
            L.lib.fame_mass_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _plan_idx(plan, key, dev):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(plan[key], dtype=np.uint32).ravel()).view(np.int32)).to(dev)


def rank1_exact_fft_scatter(x, plan, ctx: Context | None = None):
    """exp1/rank1_exact_fft_scatter.m:1-13 — Xfft = fft of x embedded at plan.inputIdx (length plan.M).

    ``plan`` needs ``NF``, ``M`` and the 1-based ``inputIdx`` (uint32); x is NF or NF x nrhs
    complex128 on the device; the result is M or M x nrhs.
    """
    ctx = ctx or default_context()
    xc, n, k = _colmajor(x)
    NF, M = int(plan["NF"]), int(plan["M"])
    if n != NF:
        raise FameError(L.FAME_ERR_INVALID, "rank1_exact_fft_scatter:BadSize")
    X, view = _new_colmajor(M, k, x)
    call("fame_rank1_exact_fft_scatter", ctx.bind(), _ptr(xc), k, _ptr(_plan_idx(plan, "inputIdx", x.device)), NF, M,
         _ptr(X))
    return X if view is None else view


def rank1_exact_ifft_gather(Yfft, plan, ctx: Context | None = None):
    """exp1/rank1_exact_ifft_gather.m:1-11 — y = ifft(Yfft) at plan.targetIdx (NF rows)."""
    ctx = ctx or default_context()
    Yc, m, k = _colmajor(Yfft)
    NF, M = int(plan["NF"]), int(plan["M"])
    if m != M:
        raise FameError(L.FAME_ERR_INVALID, "rank1_exact_ifft_gather:BadSize")
    y, view = _new_colmajor(NF, k, Yfft)
    call("fame_rank1_exact_ifft_gather", ctx.bind(), _ptr(Yc), k, _ptr(_plan_idx(plan, "targetIdx", Yfft.device)),
         NF, M, _ptr(y))
    return y if view is None else view


def _map(name, x, diags, n, rows_in, rows_out, ctx):
    ctx = ctx or default_context()
    xc, rows, k = _colmajor(x)
    if rows != rows_in:
        raise FameError(L.FAME_ERR_INVALID, "%s input must have %d rows" % (name, rows_in))
    ds = [d.contiguous() for d in diags]
    for d in ds:
        if d.dtype != torch.complex128 or d.numel() != n:
            raise ValueError("diagonals must be complex128 with n entries")
    y, view = _new_colmajor(rows_out, k, x)
    call(name, ctx.bind(), _ptr(xc), *[_ptr(d) for d in ds], n, k, _ptr(y))
    return y if view is None else view


def apply_V_blockdiag(x, Vdata, ctx=None):
    """exp1/apply_V_blockdiag.m:1-17 — y = V x (2n -> 3n)."""
    n = Vdata["n"]
    return _map("fame_apply_V_blockdiag", x, [Vdata[k] for k in ("V11", "V12", "V21", "V22", "V31", "V32")],
                n, 2 * n, 3 * n, ctx)


def apply_VH_blockdiag(x, Vdata, ctx=None):
    """exp1/apply_VH_blockdiag.m:1-16 — y = V^* x (3n -> 2n)."""
    n = Vdata["n"]
    return _map("fame_apply_VH_blockdiag", x, [Vdata[k] for k in ("V11", "V12", "V21", "V22", "V31", "V32")],
                n, 3 * n, 2 * n, ctx)


def solveV1_blockdiag(x, V11, V12, V21, V22, det, n, ctx=None):
    """exp1/solveV1_blockdiag.m:1-10 — y = V1^{-1} x."""
    return _map("fame_solveV1_blockdiag", x, [V11, V12, V21, V22, det], n, 2 * n, 2 * n, ctx)


def solveV1H_blockdiag(x, V11, V12, V21, V22, det, n, ctx=None):
    """exp1/solveV1H_blockdiag.m:1-10 — y = V1^{-*} x."""
    return _map("fame_solveV1H_blockdiag", x, [V11, V12, V21, V22, det], n, 2 * n, 2 * n, ctx)


_DIAG = {"V11": 0, "V21": 1, "V31": 2, "V12": 3, "V22": 4, "V32": 5, "detV1": 6, "W1": 7, "W2": 8,
         "invCorthDiag": 9, "Qq": 10, "q1": 11, "q2": 12, "q3": 13}


class QSystem:
    """q-dependent null-space-free system (exp1/build_experiment1_q_system.m:1-42).

    Diagonals are materialised lazily as tensors (``sys.V11`` ...); the
    device-resident copies used by the solvers live in the basis handle.
    """

    def __init__(self, mass: MassBackend, P, q):
        self.mass = mass
        self.ctx = mass.ctx
        self.N, self.NF = mass.N, mass.NF
        self.nr, self.ndof = 2 * self.NF, 3 * self.NF
        self.P = np.asarray(P, dtype=np.float64).reshape(6, 3)
        self.qPhys = np.asarray(q, dtype=np.float64).reshape(3)
        Pc = (C.c_double * 18)(*self.P.reshape(-1, order="F"))
        qc = (C.c_double * 3)(*self.qPhys)
        h = C.c_void_p()
        call("fame_basis_create", self.ctx.bind(), self.N, Pc, qc, C.byref(h))
        self.h = h
        info = L.fame_basis_info()
        call("fame_basis_info_get", self.h, C.byref(info))
        self.kLift = np.array(info.kLift[:])
        self.minAbsDetV1 = info.minAbsDetV1
        self.minQq = info.minQq
        self.nsingular = info.nsingular
        self.pivot = info.pivot
        self._cache = {}

    def __getattr__(self, name):
        if name in _DIAG:
            if name not in self._cache:
                real = _DIAG[name] >= 9
                t = torch.empty(self.NF, dtype=torch.float64 if real else torch.complex128,
                                device=torch.device("cuda", self.ctx.device))
                self.ctx.bind()
                call("fame_basis_get", self.h, _DIAG[name], _ptr(t))
                self._cache[name] = t
            return self._cache[name]
        raise AttributeError(name)

    @property
    def Vdata(self):
        d = {k: getattr(self, k) for k in ("V11", "V12", "V21", "V22", "V31", "V32")}
        d["n"], d["nr"] = self.NF, 2 * self.NF
        return d

    @property
    def sigmaR(self):
        return torch.cat([self.Qq, self.Qq])

    def close(self):
        if getattr(self, "h", None):
            L.lib.fame_basis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_q_system(mass: MassBackend, P, q) -> QSystem:
    """exp1/build_experiment1_q_system.m:4-24 (+ invC, exp1/build_inner_system_operators.m:10-14)."""
    return QSystem(mass, P, q)


@dataclass
class KrInvStats:
    inverseCalls: int
    totalIterations: int
    maxIterations: int
    maxRelativeResidual: float
    massSolveCalls: int
    totalMassIterations: int
    refineSteps: int
    fp32Iterations: int
    massApplies: int
    totalInverseTime: float

    @property
    def averageIterations(self):
        return self.totalIterations / self.inverseCalls if self.inverseCalls else float("nan")


class KrInv:
    """A K_r^{-1} action; ``op(q)`` returns K_r^{-1} q column by column."""

    def __init__(self, sys: QSystem, opts: L.fame_krinv_opts):
        self.sys = sys
        self.opts = opts
        h = C.c_void_p()
        sys.ctx.bind()
        call("fame_krinv_create", sys.h, sys.mass.h, C.byref(opts), C.byref(h))
        self.h = h

    def __call__(self, q):
        qc, n, k = _colmajor(q)
        if n != self.sys.nr:
            raise FameError(L.FAME_ERR_INVALID, "K_r^{-1} input must have 2*NF rows")
        y, view = _new_colmajor(n, k, q)
        self.sys.ctx.bind()
        call("fame_krinv_apply", self.h, _ptr(qc), _ptr(y), k)
        return y if view is None else view

    def stats(self) -> KrInvStats:
        s = L.fame_krinv_stats()
        call("fame_krinv_stats_get", self.h, C.byref(s))
        return KrInvStats(s.inverseCalls, s.totalIterations, s.maxIterations, s.maxRelativeResidual,
                          s.massSolveCalls, s.totalMassIterations, s.refineSteps, s.fp32Iterations,
                          s.massApplies, s.totalInverseSeconds)

    def reset_stats(self):
        call("fame_krinv_stats_reset", self.h)

    def close(self):
        if getattr(self, "h", None):
            L.lib.fame_krinv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def apply_Mhat_C_scalar_compact(x, sys: "QSystem"):
    """exp1/apply_Mhat_C_scalar_compact.m:8-21 with the system's W1, W2, invC.

    ``x``: NF-vector, complex128 (FP64) or complex64 (FP32 operator).
    """
    prec = L.FAME_F32 if x.dtype == torch.complex64 else L.FAME_F64
    xc = x.contiguous()
    if xc.dim() != 1 or xc.numel() != sys.NF:
        raise FameError(L.FAME_ERR_INVALID, "Mhat input must be an NF-vector")
    y = torch.empty_like(xc)
    sys.ctx.bind()
    call("fame_apply_Mhat_C_scalar_compact", sys.h, sys.mass.h, _ptr(xc), _ptr(y), prec)
    return y


def kernel_launches() -> int:
    """Kernels launched by libfame_b200.so since it was loaded."""
    return int(L.lib.fame_kernel_launches())


def _opts(**kw) -> L.fame_krinv_opts:
    o = L.fame_krinv_opts()
    call("fame_krinv_default_opts", C.byref(o))
    for k, v in kw.items():
        if v is not None:
            setattr(o, k, v)
    return o


def make_explicit_krinv_compact(sys: QSystem, tolCG=1e-10, maxitCG=1200, precision="fp64", **kw):
    """exp1/make_explicit_krinv_compact.m:1-105 — returns ``(KrInvOp, getStats)``.

    ``precision``: "fp64" (plain) or "mixed" (FP32 mass + PCG inside FP64
    iterative refinement of each Mhat solve).
    """
    o = _opts(kind=L.FAME_KRINV_EXPLICIT, tolCG=tolCG, maxitCG=maxitCG,
              prec_mode=L.FAME_PREC_MIXED if precision == "mixed" else L.FAME_PREC_FP64, **kw)
    op = KrInv(sys, o)
    return op, op.stats


def make_nested_krinv_instrumented(sys: QSystem, epsC=4.0, tolKr=1e-10, tolM=1e-12, maxitKr=600,
                                   maxitM=1600, useKrPreconditioner=True, precision="fp64", **kw):
    """exp1/make_nested_krinv_instrumented.m:1-174 — returns ``(KrInvOp, getStats)``."""
    o = _opts(kind=L.FAME_KRINV_NESTED, tolKr=tolKr, tolM=tolM, maxitKr=maxitKr, maxitM=maxitM,
              epsC=float(epsC), useKrPreconditioner=int(bool(useKrPreconditioner)),
              prec_mode=L.FAME_PREC_MIXED if precision == "mixed" else L.FAME_PREC_FP64, **kw)
    op = KrInv(sys, o)
    return op, op.stats


def start_vector(seed: int, n: int, device=None, ctx: Context | None = None):
    """Counter-based start vector (complex128, device), identical to the oracle's."""
    ctx = ctx or default_context(device)
    v = torch.empty(n, dtype=torch.complex128, device=torch.device("cuda", ctx.device))
    call("fame_start_vector", ctx.bind(), C.c_ulonglong(seed), n, _ptr(v))
    return v


def _is_identity(f):
    """True for None or a callable that returns its argument unchanged (fncB = @(x) x)."""
    if f is None:
        return True
    t = torch.arange(4, dtype=torch.complex128)
    try:
        out = f(t)
    except Exception:
        return False
    return out is t or (isinstance(out, torch.Tensor) and torch.equal(out, t))


def Lanczos(fncA, fncB, fncBinv, n, k, tol, maxiter, p, v0, flag_gpu=True, verbose=False):
    """exp2/Lanczos.m:1-21 — restarted Lanczos for the k largest eigenvalues theta of fncA.

    ``fncA`` must be a K_r^{-1} action from this package (it runs on the
    device without host round trips); ``fncB`` and ``fncBinv`` must be the
    identity, as in every call of the reference's hot path.
    Returns ``(ev, ew, iter, info)`` like the reference.
    """
    if not isinstance(fncA, KrInv):
        raise TypeError("fncA must be a KrInv (make_explicit_krinv_compact / make_nested_krinv_instrumented)")
    if not (_is_identity(fncB) and _is_identity(fncBinv)):
        raise ValueError("only fncB = fncBinv = identity is supported")
    if n != fncA.sys.nr:
        raise FameError(L.FAME_ERR_INVALID, "n must equal 2*NF")
    v0c = v0.contiguous()
    theta = (C.c_double * k)()
    Y = torch.empty(k, n, dtype=torch.complex128, device=v0.device)
    info = L.fame_lanczos_info()
    fncA.sys.ctx.bind()
    call("fame_lanczos", fncA.h, k, float(tol), int(maxiter), int(p), _ptr(v0c), theta, _ptr(Y),
         C.byref(info))
    ew = np.array(theta[:])
    return Y.t(), ew, info.steps, dict(steps=info.steps, restarts=info.restarts,
                                       converged=bool(info.converged), nconv=info.nconv,
                                       maxWantedResidual=info.maxWantedResidual)


def rayleigh_ritz(sys: QSystem, Y):
    """Rayleigh-Ritz refinement with the exact K_r = V^* M^{-1} V (no reference counterpart).

    ``Y``: complex128 device matrix (2NF x k, k <= 32), e.g. the eigenvectors returned by
    ``Lanczos``; it is overwritten with the refined vectors.  Returns ``(lam, relres)``:
    ascending eigenvalues lambda of K_r and ||K_r y - lambda y|| / ||K_r y|| per vector.
    """
    if Y.dim() != 2 or Y.shape[0] != sys.nr or Y.dtype != torch.complex128 or not Y.is_cuda:
        raise FameError(L.FAME_ERR_INVALID, "Y must be a complex128 CUDA matrix with 2*NF rows")
    k = int(Y.shape[1])
    if Y.stride(0) != 1 or Y.stride(1) != sys.nr:
        raise ValueError("Y must be column-major (Y.t() contiguous), as Lanczos returns it")
    lam = (C.c_double * k)()
    rel = (C.c_double * k)()
    sys.ctx.bind()
    call("fame_rayleigh_ritz", sys.h, sys.mass.h, _ptr(Y), k, lam, rel)
    return np.array(lam[:]), np.array(rel[:])


def solve_batch(Ns, materials, qs, P, nev=10, tol=1e-8, maxiter=30, p=40, tolCG=1e-10,
                precision="mixed", seed=None, device=None, tuned=None, **kw):
    """Solve independent Bloch points of uneven size concurrently (one call).

    ``materials[i]`` is the float64 device eps grid of instance i.  ``tuned`` maps a grid
    size N to K_r^{-1} options (``checkEvery``, ``useGraphs``, ``passColumns``, e.g. from
    ``tune_batch``) applied to every instance of that N; other instances use the
    defaults.  Other keyword arguments are K_r^{-1} options of every instance (e.g.
    ``refineTarget``).  Returns ``(lam, infos)`` with lam (count x nev) ascending eigenvalues
    lambda = 1/theta.
    """
    from . import configs
    count = len(Ns)
    dev = torch.cuda.current_device() if device is None else device
    Es = [e.contiguous() for e in materials]
    Earr = (C.c_void_p * count)(*[e.data_ptr() for e in Es])
    Narr = (C.c_int * count)(*[int(n) for n in Ns])
    qarr = (C.c_double * (3 * count))(*np.asarray(qs, dtype=np.float64).reshape(-1))
    Parr = (C.c_double * 18)(*np.asarray(P, dtype=np.float64).reshape(6, 3).reshape(-1, order="F"))
    base = dict(kind=L.FAME_KRINV_EXPLICIT, tolCG=tolCG, maxitCG=3000,
                prec_mode=L.FAME_PREC_MIXED if precision == "mixed" else L.FAME_PREC_FP64, **kw)
    opts = (L.fame_krinv_opts * count)(*[_opts(**base, **((tuned or {}).get(int(n), {}))) for n in Ns])
    theta = (C.c_double * (count * nev))()
    infos = (L.fame_lanczos_info * count)()
    status = (C.c_int * count)()
    torch.cuda.synchronize(dev)
    call("fame_solve_batch_each", dev, count, Narr, Earr, qarr, Parr, opts, nev, float(tol), int(maxiter),
         int(p), C.c_ulonglong(configs.SEED if seed is None else seed), theta, infos, status)
    th = np.array(theta[:]).reshape(count, nev)
    return np.sort(1.0 / th, axis=1), [dict(steps=i.steps, converged=bool(i.converged), nconv=i.nconv)
                                       for i in infos]


def tune_batch(Ns, materials, qs, P, precision="mixed", tolCG=1e-10, **kw):
    """The autotuner (``autotune.tune_krinv_schedule``) run once per distinct grid size of a
    batch, on its first instance: returns ``{N: options}`` for ``solve_batch(tuned=...)``."""
    from .autotune import tune_krinv_schedule
    out = {}
    for n, E, q in zip(Ns, materials, qs):
        n = int(n)
        if n in out:
            continue
        sysq = build_q_system(MassBackend(E, n), P, q)
        out[n] = tune_krinv_schedule(sysq, precision=precision, tolCG=tolCG, **kw)[0]
        torch.cuda.synchronize()
        del sysq
    return out
