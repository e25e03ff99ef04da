"""GPU parity of the Mhat action (exp1/apply_Mhat_C_scalar_compact.m:8-21) against the oracle.

``fame_apply_Mhat_C_scalar_compact`` runs the natural-order prologue/epilogue of the
Mhat chain (passes A/B/C over the three fields z, W1 z, W2 z) -- the chain whose
device time the benchmark reports as its roofline kernel.  It is compared here, in
FP64 and FP32, with the oracle's restatement on the same inputs, for both cut matrices
and both materials, together with the allocation-free entry point that runs the same
chain on static scratch.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

# FP64: rounding of three 6D FFT convolutions; FP32: complex64 passes with FP32 accumulation
TOL = {torch.complex128: 1e-13, torch.complex64: 2e-6}


def _case(N, Pname, material, dev):
    import fame_b200 as F
    Pm = F.configs.P_GOLDEN if Pname == "golden" else F.configs.P_REFERENCE
    q = F.configs.Q_PHYS if Pname == "golden" else F.configs.Q_TRACKING
    E = O.material_separable_cos(N, 12.0) if material == "cos" else O.material_smooth_exp(N)
    S = O.build_q_system(N, Pm, q, E)
    m = F.MassBackend(torch.as_tensor(E, device=dev), N)
    return F, S, m, F.build_q_system(m, Pm, q)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("Pname,material", [("golden", "cos"), ("golden", "exp"), ("reference", "cos"),
                                            ("reference", "exp")])
@pytest.mark.parametrize("N", [2, 3])
def test_mhat_matches_oracle(cuda_device, N, Pname, material, dtype):
    F, S, m, s = _case(N, Pname, material, cuda_device)
    rng = np.random.default_rng(100 + N)
    for _ in range(2):  # two calls on the handle's workspace
        x = rng.standard_normal(S.NF) + 1j * rng.standard_normal(S.NF)
        if dtype == torch.complex64:
            x = x.astype(np.complex64).astype(np.complex128)  # the FP32 operator sees exactly these inputs
        y_ref = O.apply_Mhat_C_scalar_compact(x, S)
        y = F.apply_Mhat_C_scalar_compact(torch.as_tensor(x, device=cuda_device).to(dtype), s)
        err = _rel(y.cpu().numpy().astype(np.complex128), y_ref)
        assert err < TOL[dtype], (N, Pname, material, dtype, err)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_mhat_noalloc_matches_oracle(cuda_device, dtype):
    """The allocation-free entry point against the oracle directly (N=3, golden P)."""
    F, S, m, s = _case(3, "golden", "cos", cuda_device)
    lib = F._lib.lib
    prec = 1 if dtype == torch.complex64 else 0
    rng = np.random.default_rng(7)
    x = rng.standard_normal(S.NF) + 1j * rng.standard_normal(S.NF)
    if dtype == torch.complex64:
        x = x.astype(np.complex64).astype(np.complex128)
    xd = torch.as_tensor(x, device=cuda_device).to(dtype)
    y = torch.full_like(xd, float("nan"))
    s.ctx.bind()
    assert lib.fame_apply_Mhat_C_scalar_compact_noalloc(s.h, m.h, C.c_void_p(xd.data_ptr()),
                                                        C.c_void_p(y.data_ptr()), prec) == 0
    torch.cuda.synchronize()
    err = _rel(y.cpu().numpy().astype(np.complex128), O.apply_Mhat_C_scalar_compact(x, S))
    assert err < TOL[dtype], err


@pytest.mark.parametrize("N", [6, 7])
def test_mhat_hermitian_positive_at_the_largest_grids(cuda_device, N):
    """2N = 12 and 14 (the largest supported grids, NF = 2,985,984 and 7,529,536): Mhat is
    Hermitian positive definite (exp1/apply_Mhat_C_scalar_compact.m:8-21 is B^* (I (x) M) B
    with an isometry B), so <y, Mhat x> = conj(<x, Mhat y>) and <x, Mhat x> > 0, FP64."""
    import fame_b200 as F
    E = F.configs.material_separable_cos(N, 12.0, device=cuda_device)
    m = F.MassBackend(E, N)
    s = F.build_q_system(m, F.configs.P_GOLDEN, F.configs.Q_PHYS)
    x = F.start_vector(11, s.NF)
    y = F.start_vector(12, s.NF)
    Mx = F.apply_Mhat_C_scalar_compact(x, s)
    My = F.apply_Mhat_C_scalar_compact(y, s)
    a = complex(torch.vdot(y, Mx).item())
    b = complex(torch.vdot(x, My).item()).conjugate()
    assert abs(a - b) <= 1e-12 * abs(a)
    q = complex(torch.vdot(x, Mx).item())
    assert abs(q.imag) <= 1e-12 * q.real and q.real > 0
    # the material bounds the Rayleigh quotient: 1 <= eps <= 13 and B is an isometry
    r = q.real / float(torch.vdot(x, x).real.item())
    assert 1.0 - 1e-12 <= r <= 13.0 + 1e-12
