"""GPU parity: eigenvector recovery, Fourier diagnostics, Yee-field reconstruction
(direct, factorised direct, multi-center Taylor) and the mass adjoint / eigenvalue
gradients, against the oracle."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _sys(N, dev, material="cos", Pname="golden", q=None):
    import fame_b200 as F
    P = F.configs.P_GOLDEN if Pname == "golden" else F.configs.P_REFERENCE
    q = F.configs.Q_PHYS if q is None else q
    E = O.material_separable_cos(N) if material == "cos" else O.material_smooth_exp(N)
    m = F.MassBackend(torch.as_tensor(E, device=dev), N)
    return F, O.build_q_system(N, P, q, E), F.build_q_system(m, P, q), m


def test_recovery_and_diagnostics(cuda_device):
    F, S, sg, m = _sys(2, cuda_device)
    op, _ = F.make_explicit_krinv_compact(sg, 1e-12, 3000)
    v0 = F.start_vector(F.configs.SEED, sg.nr)
    Y, theta, _, info = F.Lanczos(op, None, None, sg.nr, 4, 1e-10, 30, 40, v0)
    lam = 1.0 / theta
    X, MX, rinfo = F.recover_original_eigenvectors(Y, sg, 1e-12, 3000)
    Yh = Y.cpu().numpy()
    Xo, MXo, _ = O.recover_original_eigenvectors(Yh, S, 1e-12, 3000)
    assert rel(X.cpu().numpy(), Xo) < 1e-9
    assert rel(MX.cpu().numpy(), MXo) < 1e-9
    d = F.compute_fourier_diagnostics(X, MX, lam, sg)
    do = O.compute_fourier_diagnostics(Xo, MXo, lam, S)
    np.testing.assert_allclose(d["resGEVP"], do["resGEVP"], rtol=1e-3, atol=1e-12)
    assert d["maxResGEVP"] < 1e-6
    np.testing.assert_allclose(d["rayleigh"], lam, rtol=1e-9)
    np.testing.assert_allclose(d["rayleigh"], do["rayleigh"], rtol=1e-12)
    np.testing.assert_allclose(d["divRelative2"], do["divRelative2"], rtol=1e-3, atol=1e-12)
    assert np.max(d["divRelative2"]) < 1e-10


@pytest.mark.parametrize("N,n", [(2, 5), (2, 40), (4, 17)])
def test_direct_grid_3xtf32_vs_fp64(cuda_device, N, n):
    """Factorised direct sum with the three complex GEMMs as split-FP32 (3xTF32) tcgen05
    products vs the FP64 GEMMs: relative field error below 4e-6 on all three Yee
    components (random unit coefficients)."""
    F, S, sg, m = _sys(N, cuda_device)
    c = torch.as_tensor(O.start_vector(17, S.NF), device=cuda_device)
    pts, axes, sz = F.build_yee_points(n, 0.0125)
    for comp in range(3):
        u64 = F.reconstruct_field_direct_grid(c, sg, axes[comp]).cpu().numpy()
        utc = F.reconstruct_field_direct_grid(c, sg, axes[comp], tensor_cores=True).cpu().numpy()
        assert rel(utc, u64) < 4e-6, (comp, rel(utc, u64))
        utc2 = F.reconstruct_field_direct_grid(c, sg, axes[comp], tensor_cores=True).cpu().numpy()
        assert np.array_equal(utc, utc2)


@pytest.mark.parametrize("tc", [False, True])
def test_direct_grid_components_in_one_call(cuda_device, tc):
    """The three Yee components reconstructed in one call (each GEMM batched over them)
    equal the component-by-component calls bit for bit, in FP64 and as 3xTF32."""
    F, S, sg, m = _sys(2, cuda_device)
    X = torch.as_tensor(np.concatenate([O.start_vector(20 + c, S.NF) for c in range(3)]), device=cuda_device)
    pts, axes, sz = F.build_yee_points(5, 0.0125)
    us = F.reconstruct_fields_direct_grid(X, sg, axes, tensor_cores=tc)
    for comp in range(3):
        one = F.reconstruct_field_direct_grid(X[comp * S.NF:(comp + 1) * S.NF], sg, axes[comp], tensor_cores=tc)
        assert torch.equal(us[comp], one), comp


def test_direct_sum_plain_and_factorised(cuda_device):
    F, S, sg, m = _sys(2, cuda_device)
    Q = F.build_projected_q_modes(sg)
    np.testing.assert_allclose(Q.cpu().numpy(), O.build_projected_q_modes(F.configs.P_GOLDEN, S.kLift, 2),
                               rtol=1e-14, atol=1e-14)
    c = torch.as_tensor(O.start_vector(5, S.NF), device=cuda_device)
    pts, axes, sz = F.build_yee_points(3, 0.0125)
    r1, _, _, _ = O.build_yee_points(3, 0.0125)
    np.testing.assert_array_equal(pts[0].cpu().numpy(), r1)
    u_ref = O.reconstruct_field_direct_blocked(c.cpu().numpy(), Q.cpu().numpy(), r1)
    u = F.reconstruct_field_direct_blocked(c, Q, pts[0]).cpu().numpy()
    assert rel(u, u_ref) < 1e-12
    ug = F.reconstruct_field_direct_grid(c, sg, axes[0]).cpu().numpy()
    assert rel(ug, u_ref) < 1e-12


def test_taylor_multi_and_single(cuda_device):
    F, S, sg, m = _sys(1, cuda_device)
    Q = F.build_projected_q_modes(sg)
    c = torch.as_tensor(O.start_vector(9, S.NF), device=cuda_device)
    pts, axes, sz = F.build_yee_points(4, 0.0125)
    blocks = F.build_yee_block_partition(sz, 2)
    r1 = pts[0].cpu().numpy()
    ob = O.build_yee_block_partition(sz, 2)
    for p in (0, 2, 3, 6, 10):  # L = 1, 10, 20 (fewer terms than staged modes), 84, 286
        ut = F.reconstruct_field_taylor_multi(c, Q, pts[0], p, blocks).cpu().numpy()
        uo = O.reconstruct_field_taylor_multi(c.cpu().numpy(), Q.cpu().numpy(), r1, p, ob)
        assert rel(ut, uo) < 1e-11, p
        ut = F.reconstruct_field_taylor_multi(c, Q, pts[0], p, blocks, tensor_cores=True).cpu().numpy()
        assert rel(ut, uo) < 2e-6, p
    us = F.reconstruct_field_taylor_single(c, Q, pts[0], 8).cpu().numpy()
    uso = O.reconstruct_field_taylor_single(c.cpu().numpy(), Q.cpu().numpy(), r1, 8)
    assert rel(us, uso) < 1e-11


def test_mass_adjoint_vs_oracle(cuda_device):
    import fame_b200 as F
    N = 2
    a = F.configs.gradient_amplitudes()
    eps, grads = O.material_cos_param(N, 12.0, a)
    m = F.MassBackend(torch.as_tensor(eps, device=cuda_device), N)
    X = np.stack([O.start_vector(20 + j, 3 * (2 * N) ** 6) for j in range(2)], 1)
    out = F.grad.mass_adjoint(m, torch.as_tensor(X, device=cuda_device),
                              [torch.as_tensor(g, device=cuda_device) for g in grads])
    ref = O.mass_adjoint_quadratic(X, grads, N)
    np.testing.assert_allclose(out, ref, rtol=1e-12)


def test_eigenvalue_gradients_fd_and_autograd(cuda_device):
    """Hellmann-Feynman gradient vs central finite differences (step 1e-6), N=2."""
    import fame_b200 as F
    N = 2
    theta = np.concatenate([[12.0], F.configs.gradient_amplitudes()])
    kw = dict(nev=4, tolCG=1e-12, tol=1e-10, precision="fp64")
    lam, dl = F.grad.eigenvalue_gradients(N, theta, **kw)
    h = 1e-6
    for t in (0, 1, 4):
        tp, tm = theta.copy(), theta.copy()
        tp[t] += h
        tm[t] -= h
        fd = (F.grad.eigenpairs(N, tp, **kw)[0] - F.grad.eigenpairs(N, tm, **kw)[0]) / (2 * h)
        np.testing.assert_allclose(dl[:, t], fd, rtol=2e-4, atol=1e-9)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    lam_t = F.grad.EigenvalueFunction.apply(th, N, kw)
    lam_t.sum().backward()
    np.testing.assert_allclose(th.grad.numpy(), dl.sum(0), rtol=1e-12)
    # eigenvectors recovered one mode at a time (as under a small memory budget) and the
    # recompute form (backward repeats the solve) give the same gradients
    _, dl1 = F.grad.eigenvalue_gradients(N, theta, chunk=1, **kw)
    np.testing.assert_allclose(dl1, dl, rtol=1e-12, atol=1e-15)
    assert F.grad.modes_per_chunk((2 * N) ** 6, 4, device_bytes=12 * 16 * (2 * N) ** 6 * 2) == 2
    th2 = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    F.grad.EigenvalueFunction.apply(th2, N, dict(kw, recompute=True)).sum().backward()
    np.testing.assert_allclose(th2.grad.numpy(), dl.sum(0), rtol=1e-12)


def test_batched_bloch_path_matches_single_solves(cuda_device):
    """Instances of uneven N solved concurrently equal one-at-a-time solves."""
    import fame_b200 as F
    Ns = [1, 2, 1, 2]
    qs = [(0.05, 0.04, 0.03), (0.1, 0.02, 0.03), (0.2, 0.1, 0.05), (0.25, 0.25, 0.1)]
    mats = [F.configs.material_separable_cos(N, device=cuda_device) for N in Ns]
    lam, infos = F.solve_batch(Ns, mats, qs, F.configs.P_GOLDEN, nev=6, tol=1e-10, tolCG=1e-12,
                               precision="fp64")
    for i, (N, q) in enumerate(zip(Ns, qs)):
        m = F.MassBackend(mats[i], N)
        s = F.build_q_system(m, F.configs.P_GOLDEN, q)
        op, _ = F.make_explicit_krinv_compact(s, 1e-12, 3000)
        _, th, _, info = F.Lanczos(op, None, None, s.nr, 6, 1e-10, 30, 40, F.start_vector(F.configs.SEED, s.nr))
        assert infos[i]["converged"]
        np.testing.assert_allclose(lam[i], np.sort(1.0 / th), rtol=1e-10)


def test_batched_bloch_path_with_tuned_options(cuda_device):
    """The autotuner's per-N choices (schedule, pass tile shape) reach every instance of that N
    (fame_solve_batch_each) and change only how the work is launched: the eigenvalues equal
    those of the default options."""
    import fame_b200 as F
    Ns = [3, 2, 3, 2]
    qs = [(0.05, 0.04, 0.03), (0.1, 0.02, 0.03), (0.2, 0.1, 0.05), (0.25, 0.25, 0.1)]
    mats = [F.configs.material_separable_cos(N, device=cuda_device) for N in Ns]
    tuned = F.tune_batch(Ns, mats, qs, F.configs.P_GOLDEN, tolCG=1e-12, reps=1)
    assert sorted(tuned) == [2, 3] and all({"checkEvery", "useGraphs", "passColumns"} <= set(v) for v in tuned.values())
    kw = dict(nev=6, tol=1e-10, tolCG=1e-12)
    lam0, _ = F.solve_batch(Ns, mats, qs, F.configs.P_GOLDEN, **kw)
    forced = {3: dict(checkEvery=16, useGraphs=1, passColumns=4), 2: dict(checkEvery=2, useGraphs=0)}
    for opts in (tuned, forced):
        lam, infos = F.solve_batch(Ns, mats, qs, F.configs.P_GOLDEN, tuned=opts, **kw)
        assert all(i["converged"] for i in infos)
        np.testing.assert_allclose(lam, lam0, rtol=1e-9)


@pytest.mark.parametrize("N,p,nb", [(2, 6, 2), (2, 10, 3), (3, 8, 2), (2, 12, 2), (2, 0, 1), (4, 10, 5)])
def test_taylor_3xtf32_tensor_cores_vs_fp64(cuda_device, N, p, nb):
    """Split-FP32 (3xTF32) tensor-core block moments (operands generated on chip, FP32
    TMEM accumulation over at most 512 modes, FP64 sum of the slices) vs the FP64 form
    (same centers, same evaluation): relative field error below 4e-6 (the tensor cores
    round the FP32 accumulation toward zero; random unit coefficients, up to 2.6e5 modes)."""
    F, S, sg, m = _sys(N, cuda_device)
    Q = F.build_projected_q_modes(sg)
    c = torch.as_tensor(O.start_vector(13, S.NF), device=cuda_device)
    pts, axes, sz = F.build_yee_points(6, 0.0125)
    blocks = F.build_yee_block_partition(sz, nb)
    u64 = F.taylor_on_blocks(c, Q, pts[1], p, blocks).cpu().numpy()
    utc = F.taylor_on_blocks(c, Q, pts[1], p, blocks, tensor_cores=True).cpu().numpy()
    assert rel(utc, u64) < 4e-6, rel(utc, u64)
    utc2 = F.taylor_on_blocks(c, Q, pts[1], p, blocks, tensor_cores=True).cpu().numpy()
    assert np.array_equal(utc, utc2)  # deterministic


def test_taylor_3xtf32_general_centers(cuda_device):
    """Blocks in a permuted order: the centers are no longer a tensor grid in block order, so
    the tensor-core moments take each center's phase by sincosf instead of the per-axis
    factorisation; both give the FP64 form's field (and each other's) to the same bound."""
    F, S, sg, m = _sys(2, cuda_device)
    Q = F.build_projected_q_modes(sg)
    c = torch.as_tensor(O.start_vector(14, S.NF), device=cuda_device)
    pts, axes, sz = F.build_yee_points(6, 0.0125)
    ptr, ids = F.build_yee_block_partition(sz, 3)
    hp, hi = ptr.cpu().numpy(), ids.cpu().numpy()
    perm = np.random.default_rng(3).permutation(len(hp) - 1)
    nptr, nids = [0], []
    for b in perm:
        nids.append(hi[hp[b]:hp[b + 1]])
        nptr.append(nptr[-1] + hp[b + 1] - hp[b])
    pblocks = (torch.as_tensor(np.asarray(nptr, dtype=np.int64), device=cuda_device),
               torch.as_tensor(np.concatenate(nids).astype(np.int64), device=cuda_device))
    for p in (6, 10):
        u64 = F.taylor_on_blocks(c, Q, pts[1], p, pblocks).cpu().numpy()
        ugen = F.taylor_on_blocks(c, Q, pts[1], p, pblocks, tensor_cores=True).cpu().numpy()
        ugrid = F.taylor_on_blocks(c, Q, pts[1], p, (ptr, ids), tensor_cores=True).cpu().numpy()
        assert rel(ugen, u64) < 4e-6 and rel(ugrid, u64) < 4e-6, (rel(ugen, u64), rel(ugrid, u64))
