"""CPU tests: pin the oracle against the reference's known answers and constants."""
import numpy as np
import pytest

import oracle as O


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


P_REF = np.vstack([np.eye(3), np.diag([np.sqrt(2), np.sqrt(3), np.sqrt(5)])])
PHI = (1 + 5 ** 0.5) / 2
P_GOLD = np.vstack([np.eye(3), np.diag([PHI, 1 / PHI, PHI ** 2])])


def test_rank1_plan_constants_n5():
    """exp2/run_experiment2_allgpu_static_check.m:10-11 — M = 24760990, z = 19^(0..5)."""
    p = O.build_radix_exact_rank1_plan_scalar(5)
    assert p["M"] == 24760990
    assert list(p["z"]) == [1, 19, 361, 6859, 130321, 2476099]
    assert len(np.unique(p["inputIdx"])) == p["NF"]
    assert len(np.unique(p["targetIdx"])) == p["NF"]
    assert p["inputIdx"].max() < p["M"]


@pytest.mark.parametrize("N", [1, 2])
def test_rank1_lattice_equals_6d_fft(N):
    """exp1/smoke_test_rank1_lowmem.m:17-23: rank-1 lowmem vs tensor FFT mass < 1e-11."""
    E = O.material_smooth_exp(N)
    plan = O.build_radix_exact_rank1_plan_scalar(N)
    k = O.build_exact_rank1_scalar_kernel_fft(E, plan)
    x = O.start_vector(3, (2 * N) ** 6)
    assert _rel(O.applyMij_rank1_exact(x, k, plan), O.applyMij_fft(x, E, N)) < 1e-11


@pytest.mark.parametrize("N", [2, 3])
def test_stencil_closed_form(N):
    E = O.material_separable_cos(N, 12.0)
    x = O.start_vector(4, (2 * N) ** 6)
    assert _rel(O.mass_stencil_bandlimited(x, N, 12.0), O.applyMij_fft(x, E, N)) < 1e-13


def test_mass_hermitian_positive():
    """exp2/run_experiment3_preflight_n5.m:17-24 (Hermitian defect), at N=2."""
    N = 2
    E = O.material_smooth_exp(N)
    x, y = O.start_vector(1, 4096), O.start_vector(2, 4096)
    Mx, My = O.applyMij_fft(x, E, N), O.applyMij_fft(y, E, N)
    assert abs(np.vdot(y, Mx) - np.conj(np.vdot(x, My))) / abs(np.vdot(y, Mx)) < 1e-10
    assert np.real(np.vdot(x, Mx)) > 0


def test_basis_identities():
    """V V^* equals the curl-curl symbol K on the transverse space; W, invC definitions."""
    N = 1
    S = O.build_q_system(N, P_GOLD, (0.05, 0.04, 0.03), O.material_separable_cos(N))
    n = S.NF
    for j in range(0, n, 7):
        e = np.zeros(3 * n, complex)
        e[j] = 1
        VVe = O.apply_V_blockdiag(O.apply_VH_blockdiag(e, S), S)
        assert _rel(VVe, S.Kop(e)) < 1e-10
    W = O.solveV1H_blockdiag(np.concatenate([np.conj(S.V31), np.conj(S.V32)]),
                             S.V11, S.V12, S.V21, S.V22, S.detV1, n)
    assert _rel(W[:n], S.W1) < 1e-15
    np.testing.assert_allclose(S.invC, 1 / np.sqrt(1 + abs(S.W1) ** 2 + abs(S.W2) ** 2))


def test_gamma_point_raises():
    with pytest.raises(ValueError):
        O.build_q_system(1, P_GOLD, (0.0, 0.0, 0.0), O.material_separable_cos(1))


def test_singular_branch_orthonormal():
    """exp1/assemble_K_and_nullspace_free_basis.m:75-91 — q parallel to (1,1,1)."""
    P = np.vstack([np.eye(3), np.zeros((3, 3))])
    Xi = O.build_fourier_grid_6d(1)
    B = O.assemble_K_and_nullspace_free_basis(P, np.array([0.1, 0.1, 0.1, 0, 0, 0]), Xi)
    assert B["nsingular"] > 0


def test_pcg_semantics():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((30, 30))
    A = A @ A.T + 30 * np.eye(30)
    b = rng.standard_normal(30)
    x, flag, rr, it = O.pcg(lambda v: A @ v, b, 1e-12, 100)
    assert flag == 0 and rr <= 1e-12 and np.linalg.norm(A @ x - b) / np.linalg.norm(b) <= 1e-12
    x, flag, rr, it = O.pcg(lambda v: A @ v, b, 1e-14, 2)
    assert flag == 1 and it == 2
    x, flag, rr, it = O.pcg(lambda v: A @ v, np.zeros(30), 1e-10, 10)
    assert flag == 0 and it == 0 and not x.any()


def test_lanczos_known_diagonal():
    """exp1/smoke_test_rank1_lowmem.m:44-54: diag(linspace(100,1,80)), top-5 rel < 1e-7."""
    d = np.linspace(100, 1, 80)
    v0 = O.start_vector(5, 80)
    U, th, it, info = O.Lanczos(lambda v: d * v, 80, 5, 1e-10, 30, 20, v0)
    assert np.max(np.abs(th - d[:5]) / d[:5]) < 1e-7


def test_dense_eigs_n1():
    """Lanczos on K_r^{-1} reproduces a dense eigensolve of K_r = V^* M^{-1} V at N=1."""
    N = 1
    S = O.build_q_system(N, P_GOLD, (0.05, 0.04, 0.03), O.material_separable_cos(N))
    lam_dense = np.sort(np.linalg.eigvalsh(O.dense_reduced_operator(S)))[:10]
    sol = O.solve_modes(S, nev=10, p=40, tol=1e-10, tolCG=1e-12)
    assert np.max(np.abs(sol["lam"] - lam_dense) / lam_dense) < 1e-10


def test_exact_grid_inverse_and_Kr_n1():
    """M^{-1} as the chain on 1/eps inverts the mass exactly, and the exact K_r matches
    the dense V^* M^{-1} V at N=1."""
    N = 1
    S = O.build_q_system(N, P_GOLD, (0.05, 0.04, 0.03), O.material_separable_cos(N))
    x = O.start_vector(3, S.NF)
    assert _rel(S.mass.inverse_scalar(S.mass.scalar(x)), x) < 1e-14
    K = O.dense_reduced_operator(S)
    y = O.start_vector(4, S.nr)
    assert _rel(O.apply_Kr_exact(y, S), K @ y) < 1e-12


def test_rayleigh_ritz_removes_the_inner_tolerance_error_n2():
    """Ritz vectors of a Lanczos run on a loose K_r^{-1} (tolCG 1e-8: eigenvalues off by
    ~1e-8) refined with the exact K_r agree with a refined tight solve (tolCG 1e-13) to
    1e-10 (the refined error is quadratic in the eigenvector error); at N=1 the refined
    values equal a dense eigensolve of K_r."""
    N = 2
    S = O.build_q_system(N, P_GOLD, (0.05, 0.04, 0.03), O.material_separable_cos(N))
    sol_t = O.solve_modes(S, nev=10, p=40, tol=1e-8, tolCG=1e-13)
    tight = O.rayleigh_ritz_Kr(sol_t["Y"], S)[0]
    sol = O.solve_modes(S, nev=10, p=40, tol=1e-8, tolCG=1e-8)
    raw = np.max(np.abs(np.sort(sol["lam"]) - tight) / tight)
    lam, Yr, relres = O.rayleigh_ritz_Kr(sol["Y"], S)
    assert np.max(np.abs(lam - tight) / tight) < 1e-10 < 1e-9 < raw
    assert np.max(np.abs(np.sort(sol_t["lam"]) - tight) / tight) < 1e-11
    assert np.all(relres < 1e-4)
    S1 = O.build_q_system(1, P_GOLD, (0.05, 0.04, 0.03), O.material_separable_cos(1))
    lam_dense = np.sort(np.linalg.eigvalsh(O.dense_reduced_operator(S1)))[:10]
    lam1 = O.rayleigh_ritz_Kr(O.solve_modes(S1, nev=10, p=40, tol=1e-8, tolCG=1e-10)["Y"], S1)[0]
    assert np.max(np.abs(lam1 - lam_dense) / lam_dense) < 1e-12


def test_explicit_equals_nested_n1():
    """exp1/smoke_test_rank1_lowmem.m:29-39 spirit: two K_r^{-1} realisations agree."""
    N = 1
    S = O.build_q_system(N, P_REF, (0.13, 0.21, 0.17), O.material_smooth_exp(N))
    b = O.start_vector(9, S.nr)
    yc = O.make_explicit_krinv_compact(S, 1e-12, 3000)[0](b)
    yb = O.make_nested_krinv_instrumented(S, 4.0, 1e-12, 1e-13)[0](b)
    assert _rel(yb, yc) < 1e-9


@pytest.mark.slow
def test_reference_kat_n2():
    """exp3/make_config_experiment4.m:38-45 — tracked modes 1, 10 at N=2 (rel 5e-7)."""
    N = 2
    S = O.build_q_system(N, P_REF, (0.13, 0.21, 0.17), O.material_smooth_exp(N, 4.0, 1.2))
    sol = O.solve_modes(S, nev=10, p=40, tol=1e-10, maxRestart=30, tolCG=1e-10)
    ref = np.array([1.201276300237e-02, 4.496454358674e-02])
    assert np.max(np.abs(sol["lam"][[0, 9]] - ref) / ref) < 5e-7


def test_taylor_matches_direct():
    """Taylor (p=10, 8 centers) vs the direct sum at small size (exp2/check_experiment2b_results.m:72-75 e2<=1e-4)."""
    N = 1
    S = O.build_q_system(N, P_GOLD, (0.05, 0.04, 0.03), O.material_separable_cos(N))
    Q = O.build_projected_q_modes(P_GOLD, S.kLift, N)
    c = O.start_vector(11, S.NF)
    r1, r2, r3, sz = O.build_yee_points(6, 0.0125)
    blocks = O.build_yee_block_partition(sz, 2)
    ud = O.reconstruct_field_direct_blocked(c, Q, r1)
    ut = O.reconstruct_field_taylor_multi(c, Q, r1, 10, blocks)
    assert _rel(ut, ud) < 1e-4
    ub = O.reconstruct_component_taylor_batch(c, Q, r1, 10, blocks)[:, 0]
    assert _rel(ub, ut) < 5e-11  # exp3/make_config_experiment4.m:95 streaming vs batched


def test_start_vector_deterministic():
    a = O.start_vector(20260905, 10)
    assert np.array_equal(a, O.start_vector(20260905, 10))
    assert np.all(np.abs(a.real) <= 1) and np.all(np.abs(a.imag) <= 1)


# ---------------------------------------------------------------- LWRQ (a22)
def _yee_rand(n, seed):
    rng = np.random.default_rng(seed)
    m = 2 * n + 3
    return [rng.standard_normal((m, m, m)) + 1j * rng.standard_normal((m, m, m)) for _ in range(3)]


def test_cropped_curlcurl_annihilates_discrete_gradients():
    """The Yee curl-curl of exp3/apply_cropped_A_exp3.m vanishes on forward-difference gradients."""
    n, h = 5, 0.04
    idx = np.arange(-(n + 1), n + 2) * h
    X, Y, Z = np.meshgrid(idx, idx, idx, indexing="ij")
    phi = lambda x, y, z: np.sin(3 * x + 1) * np.cos(2 * y) * np.exp(z)  # noqa: E731
    g = [(phi(X + h, Y, Z) - phi(X, Y, Z)) / h, (phi(X, Y + h, Z) - phi(X, Y, Z)) / h,
         (phi(X, Y, Z + h) - phi(X, Y, Z)) / h]
    A = O.apply_cropped_A(*(c + 0j for c in g), h)
    scale = max(np.abs(c).max() for c in g) / h ** 2
    assert max(np.abs(a).max() for a in A) < 1e-12 * scale


def test_separable_window_matches_direct_convolution():
    from scipy.ndimage import convolve1d
    rng = np.random.default_rng(3)
    X = rng.standard_normal((6, 7, 9))
    k = np.exp(-np.arange(-3, 4) ** 2 / 4.0)
    Y = X
    for ax in range(3):
        Y = convolve1d(Y, k, axis=ax, mode="constant", cval=0.0)
    assert np.abs(Y - O.separable_conv3_same(X, k)).max() < 1e-13


def test_lwrq_partition_of_unity_and_constant_quotient():
    """Column normalisation preserves the totals; a = lambda b gives rho = lambda, V = 0."""
    rng = np.random.default_rng(4)
    b = rng.uniform(0.5, 2.0, (9, 9, 9))
    a = rng.standard_normal((9, 9, 9))
    L = O.compute_lwrq(a, b, 0.05)
    assert L["partitionError"] < 1e-14
    L2 = O.compute_lwrq(0.37 * b, b, 0.05)
    assert abs(L2["lam"] - 0.37) < 1e-15 and L2["V"] < 1e-28


def test_lwrq_metrics_consistency():
    n, h = 4, 0.05
    u = _yee_rand(n, 5)
    P = np.vstack([np.eye(3), np.diag([np.sqrt(2), np.sqrt(3), np.sqrt(5)])])
    met, sp = O.compute_yee_lwrq_metrics(*u, 0.5, P, n, h, ("exp", 4.0, 1.2), save_spatial=True)
    assert met["deltaPart"] < 1e-14 and met["deltaLWRQIdentity"] < 1e-13
    assert met["croppedMass"] > 0 and 0 <= met["eta3D"] <= met["etaUsing6DLambda"] + 1e-15
    assert sp["relativeDeviation_z0"].shape == (2 * n + 1, 2 * n + 1)


def test_method_a_spectrum_equals_null_space_free_n1():
    """Method A (exp1/build_experiment1_q_system_A_only.m) and methods B/C share the
    positive spectrum: the dense original GEVP K x = lambda M x has NF zero eigenvalues
    (gradient fields) and 2NF positive ones equal to those of K_r = V^* M^-1 V
    (exp1/check_fig1bc_results.m:23-25 checks 1e-7 across methods)."""
    N = 1
    S = O.build_q_system(N, P_REF, (0.13, 0.21, 0.17), O.material_smooth_exp(N))
    ev = O.dense_original_gevp(S)
    n = S.NF
    assert np.sum(np.abs(ev) < 1e-10) == n and np.sum(ev > 1e-10) == 2 * n
    kr = np.sort(np.linalg.eigvalsh(O.dense_reduced_operator(S)))
    assert np.max(np.abs(ev[ev > 1e-10] - kr) / kr) < 1e-11


def test_method_a_minres_top_vs_dense_n1():
    """T x = (K - sigma M)^{-1} M x by the restated preconditioned MINRES
    (exp1/make_A_eigs_top_preconditioned.m:61-113, tau = sigma mean(eps)) vs a dense solve."""
    N = 1
    E = O.material_smooth_exp(N)
    S = O.build_q_system(N, P_REF, (0.13, 0.21, 0.17), E)
    sigma = 1e-4
    x = O.start_vector(3, 3 * S.NF)
    y, it, relres = O.osi_top_apply(x, S, sigma, sigma * E.mean(), tol=1e-12)
    K, M3 = O.dense_original_operators(S)
    yd = np.linalg.solve(K - sigma * M3, M3 @ x)
    assert relres < 1e-11 and it < 200
    assert _rel(y, yd) < 1e-10
    # the preconditioner is the exact inverse of K + tau I
    tau = 0.37
    z = O.apply_shift_preconditioner(x, S, tau)
    assert _rel((K + tau * np.eye(3 * S.NF)) @ z, x) < 1e-13


def test_mass_adjoint_matches_finite_differences_n1():
    """The oracle's x^H (dM/dtheta_t) x (the checker of the GPU adjoint, no reference
    function) against central differences of x^H M(theta) x in each of the 7 material
    parameters theta = (delta, a_1..a_6) of eps = 1 + delta prod (1 + a cos)/(1 + a)."""
    N = 1
    theta = np.array([12.0, 0.6, 0.7, 0.8, 0.9, 0.55, 0.95])
    eps, grads = O.material_cos_param(N, theta[0], theta[1:])
    n = (2 * N) ** 6
    X = np.stack([O.start_vector(40 + j, 3 * n) for j in range(2)], 1)
    quad = O.mass_adjoint_quadratic(X, grads, N)

    def xMx(th, x):
        e, _ = O.material_cos_param(N, th[0], th[1:])
        m = O.MassOp(e, N)
        return float(np.real(np.vdot(x, m.full(x))))

    h = 1e-6
    for t in range(7):
        tp, tm = theta.copy(), theta.copy()
        tp[t] += h
        tm[t] -= h
        for j in range(2):
            fd = (xMx(tp, X[:, j]) - xMx(tm, X[:, j])) / (2 * h)
            assert abs(quad[j, t] - fd) <= 1e-6 * max(1.0, abs(fd)), (t, j, quad[j, t], fd)


def test_recovered_eigenvectors_solve_the_original_gevp_n1():
    """exp2/recover_original_eigenvectors_exp2.m: x = M^-1 V y from the null-space-free
    eigenvectors, M-normalised, satisfies the original K x = lambda M x (dense operators)."""
    N = 1
    S = O.build_q_system(N, P_REF, (0.13, 0.21, 0.17), O.material_smooth_exp(N))
    sol = O.solve_modes(S, nev=4, p=20, tol=1e-10, tolCG=1e-12)
    X, MX, _ = O.recover_original_eigenvectors(sol["Y"], S, 1e-12, 3000)
    K, M3 = O.dense_original_operators(S)
    for j, lam in enumerate(sol["lam"]):
        x = X[:, j]
        assert abs(np.vdot(x, M3 @ x) - 1.0) < 1e-10
        r = np.linalg.norm(K @ x - lam * (M3 @ x)) / (np.linalg.norm(K @ x) + lam * np.linalg.norm(M3 @ x))
        assert r < 1e-9, (j, r)


def test_workload_constants_agree_with_the_product():
    """The checker's copy of the benchmark inputs equals the product's (fame_b200.configs)."""
    import fame_b200 as F
    from oracle import workloads as W
    np.testing.assert_array_equal(W.P_GOLDEN, F.configs.P_GOLDEN)
    np.testing.assert_array_equal(W.P_REFERENCE, F.configs.P_REFERENCE)
    assert W.Q_PHYS == F.configs.Q_PHYS and W.Q_TRACKING == F.configs.Q_TRACKING
    assert W.SEED == F.configs.SEED and W.SOLVE == F.configs.SOLVE
