"""GPU parity: 6D mass operator, rank-1 drop-in, basis assembly and maps vs the oracle."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def _rand(n, seed, ncol=None):
    rng = np.random.default_rng(seed)
    shape = (n,) if ncol is None else (n, ncol)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("N", [1, 2, 3])
def test_applyMij_fft_fp64_matches_oracle(cuda_device, N):
    import fame_b200 as F
    NF = (2 * N) ** 6
    E = O.material_smooth_exp(N, 4.0, 1.2)
    x = _rand(NF, 10 + N, 2)
    y_ref = O.applyMij_fft(x, E, N)
    xt = torch.as_tensor(x, device=cuda_device)
    Et = torch.as_tensor(E, device=cuda_device)
    y = F.applyMij_fft(xt, Et, N).cpu().numpy()
    assert _rel(y, y_ref) < 1e-13


@pytest.mark.parametrize("N", [1, 2, 4, 5, 6, 7])
def test_mass_handles_fp64(cuda_device, N):
    import fame_b200 as F
    NF = (2 * N) ** 6
    Et = F.configs.material_separable_cos(N, 12.0, device=cuda_device)
    E = Et.cpu().numpy()
    m = F.MassBackend(Et, N)
    x = _rand(NF, 3)
    y = m.MscalarOp(torch.as_tensor(x, device=cuda_device)).cpu().numpy()
    # closed form of the band-limited material (no FFT involved)
    assert _rel(y, O.mass_stencil_bandlimited(x, N, 12.0)) < 1e-13
    if N <= 4:
        assert _rel(y, O.applyMij_fft(x, E, N)) < 1e-13
    U = _rand(3 * NF, 4)
    MU = m.Mop(torch.as_tensor(U, device=cuda_device)).cpu().numpy()
    ref = np.concatenate([O.mass_stencil_bandlimited(U[k * NF:(k + 1) * NF], N, 12.0) for k in range(3)])
    assert _rel(MU, ref) < 1e-13
    c3 = m.Mcol3op(torch.as_tensor(x, device=cuda_device)).cpu().numpy()
    assert np.all(c3[:2 * NF] == 0) and _rel(c3[2 * NF:], y) < 1e-15
    x12 = _rand(2 * NF, 5)
    c12 = m.Mcols12op(torch.as_tensor(x12, device=cuda_device)).cpu().numpy()
    assert np.all(c12[2 * NF:] == 0)
    assert _rel(c12[:NF], O.mass_stencil_bandlimited(x12[:NF], N, 12.0)) < 1e-13


@pytest.mark.parametrize("N", [1, 2, 3, 5, 6, 7])
def test_mass_fp32(cuda_device, N):
    import fame_b200 as F
    NF = (2 * N) ** 6
    Et = F.configs.material_separable_cos(N, 12.0, device=cuda_device)
    m = F.MassBackend(Et, N)
    x = _rand(NF, 7)
    y32 = m.MscalarOp(torch.as_tensor(x, device=cuda_device).to(torch.complex64)).cpu().numpy()
    assert _rel(y32, O.mass_stencil_bandlimited(x, N, 12.0)) < 2e-6


def test_rank1_dropin_matches_reference_plan(cuda_device):
    import fame_b200 as F
    N = 2
    NF = (2 * N) ** 6
    E = O.material_smooth_exp(N, 4.0, 1.2)
    plan = O.build_radix_exact_rank1_plan_scalar(N)
    kfft = O.build_exact_rank1_scalar_kernel_fft(E, plan)
    x = _rand(NF, 11)
    y_ref = O.applyMij_rank1_exact(x, kfft, plan)
    m = F.MassBackend(torch.as_tensor(E, device=cuda_device), N)
    plan1 = dict(inputIdx=plan["inputIdx"] + 1, targetIdx=plan["targetIdx"] + 1, M=plan["M"])
    y = m.applyMij_rank1_exact(torch.as_tensor(x, device=cuda_device), plan1).cpu().numpy()
    assert _rel(y, y_ref) < 1e-11   # exp1/smoke_test_rank1_lowmem.m:17-23
    bad = dict(plan1, targetIdx=plan1["targetIdx"][::-1].copy())
    with pytest.raises(F.FameError) as e:
        m.applyMij_rank1_exact(torch.as_tensor(x, device=cuda_device), bad)
    assert e.value.status == 1
    with pytest.raises(F.FameError):
        m.applyMij_rank1_exact(torch.as_tensor(x, device=cuda_device), dict(plan1, M=plan["M"] + 1))


@pytest.mark.parametrize("P,q", [("golden", (0.05, 0.04, 0.03)), ("reference", (0.13, 0.21, 0.17))])
def test_basis_and_maps(cuda_device, P, q):
    import fame_b200 as F
    N = 2
    Pm = F.configs.P_GOLDEN if P == "golden" else F.configs.P_REFERENCE
    E = O.material_smooth_exp(N)
    S = O.build_q_system(N, Pm, q, E)
    m = F.MassBackend(torch.as_tensor(E, device=cuda_device), N)
    sysg = F.build_q_system(m, Pm, q)
    np.testing.assert_allclose(sysg.kLift, S.kLift, rtol=1e-14, atol=1e-15)
    errs = {}
    for name in ("V11", "V12", "V21", "V22", "V31", "V32", "detV1", "W1", "W2"):
        errs[name] = _rel(getattr(sysg, name).cpu().numpy(), getattr(S, name))
    assert max(errs.values()) < 1e-10, errs
    assert _rel(sysg.invCorthDiag.cpu().numpy(), S.invC) < 1e-12
    n = S.NF
    x2 = _rand(2 * n, 1, 2)
    x3 = _rand(3 * n, 2, 2)
    t = lambda a: torch.as_tensor(a, device=cuda_device)
    y = F.apply_V_blockdiag(t(x2), sysg.Vdata).cpu().numpy()
    assert _rel(y, np.stack([O.apply_V_blockdiag(x2[:, j], S) for j in range(2)], 1)) < 1e-12
    y = F.apply_VH_blockdiag(t(x3), sysg.Vdata).cpu().numpy()
    assert _rel(y, np.stack([O.apply_VH_blockdiag(x3[:, j], S) for j in range(2)], 1)) < 1e-12
    args = [sysg.V11, sysg.V12, sysg.V21, sysg.V22, sysg.detV1, n]
    y = F.solveV1_blockdiag(t(x2), *args).cpu().numpy()
    ref = np.stack([O.solveV1_blockdiag(x2[:, j], S.V11, S.V12, S.V21, S.V22, S.detV1, n) for j in range(2)], 1)
    assert _rel(y, ref) < 1e-11
    y = F.solveV1H_blockdiag(t(x2), *args).cpu().numpy()
    ref = np.stack([O.solveV1H_blockdiag(x2[:, j], S.V11, S.V12, S.V21, S.V22, S.detV1, n) for j in range(2)], 1)
    assert _rel(y, ref) < 1e-11


def test_gamma_point_is_rejected(cuda_device):
    import fame_b200 as F
    N = 1
    m = F.MassBackend(F.configs.material_separable_cos(N, device=cuda_device), N)
    with pytest.raises(F.FameError) as e:
        F.build_q_system(m, F.configs.P_GOLDEN, (0.0, 0.0, 0.0))
    assert e.value.status == 7  # FAME_ERR_SINGULAR (exp1/assemble_K_and_nullspace_free_basis.m:36-42)


def test_start_vector_matches_oracle(cuda_device):
    import fame_b200 as F
    v = F.start_vector(20260905, 1000).cpu().numpy()
    assert np.array_equal(v, O.start_vector(20260905, 1000))


def test_cached_device_memory_reuse_and_trim(cuda_device):
    """Handles created and destroyed repeatedly take their device memory from the
    library's cached pool (same results each time); fame_device_trim_memory returns it."""
    import fame_b200 as F
    from fame_b200 import _lib as L
    N = 2
    E = torch.as_tensor(O.material_smooth_exp(N), device=cuda_device)
    x = torch.as_tensor(O.start_vector(4, (2 * N) ** 6), device=cuda_device)
    outs = []
    for _ in range(3):
        m = F.MassBackend(E, N)
        outs.append(m.MscalarOp(x).cpu().numpy())
        m.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])
    assert L.lib.fame_device_trim_memory(cuda_device.index or 0) == 0
    m = F.MassBackend(E, N)
    assert np.array_equal(m.MscalarOp(x).cpu().numpy(), outs[0])
    # the library keeps its own pool: the device's default pool keeps its release threshold
    try:
        from cuda.bindings import runtime as rt
    except ImportError:
        from cuda import cudart as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(cuda_device.index or 0)
    assert int(err) == 0
    err, thr = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReleaseThreshold)
    assert int(err) == 0 and int(thr) == 0


@pytest.mark.parametrize("N", [2, 5])
def test_bounded_wait_timeout_is_reported(cuda_device, N):
    """The bounded mbarrier wait of pass B runs out (stage barriers armed for bytes that no
    copy delivers; nothing is in flight), every CTA sets the fault word and returns, the host
    reports FAME_ERR_CUDA at the next synchronisation, and the context stays usable: a mass
    action afterwards matches the oracle."""
    import fame_b200 as F
    from fame_b200 import _lib as L
    E = O.material_separable_cos(N, 12.0)
    m = F.MassBackend(torch.as_tensor(E, device=cuda_device), N)
    m.ctx.bind()
    st = L.lib.fame_selftest_bounded_wait(m.h, 4096)
    assert st == 2 and b"bounded device-side wait" in L.lib.fame_last_error()
    x = O.start_vector(12, (2 * N) ** 6)
    for dtype, tol in ((torch.complex128, 1e-13), (torch.complex64, 2e-6)):
        y = m.MscalarOp(torch.as_tensor(x, device=cuda_device).to(dtype)).cpu().numpy().astype(np.complex128)
        ref = O.applyMij_fft(x.astype(np.complex64).astype(np.complex128) if dtype == torch.complex64 else x, E, N)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < tol
    m.ctx.sync()  # nothing left on the fault word
