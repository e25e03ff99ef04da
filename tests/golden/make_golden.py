"""Generate the golden fixtures of tests/golden/ from the CPU oracle.

The oracle is pinned to the reference by its known answers (rank-1 lattice
constants, rank-1 == 6D FFT mass, the stored N=2 tracked eigenvalues of
exp3/make_config_experiment4.m:38-45); these fixtures freeze its outputs on
small seeded inputs so the GPU tests can compare against stored vectors.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

PHI = (1 + 5 ** 0.5) / 2
P_GOLDEN = np.vstack([np.eye(3), np.diag([PHI, 1 / PHI, PHI ** 2])])
P_REF = np.vstack([np.eye(3), np.diag([np.sqrt(2), np.sqrt(3), np.sqrt(5)])])
Q_PHYS = (0.05, 0.04, 0.03)
Q_TRACKING = (0.13, 0.21, 0.17)


def main():
    out = {}
    # 6D mass operator, N=2, reference material
    N = 2
    E = O.material_smooth_exp(N)
    x = O.start_vector(7, (2 * N) ** 6)
    out["mass_n2"] = dict(E=E, x=x, y=O.applyMij_fft(x, E, N))
    # basis diagonals, N=2, golden-ratio cut matrix at the benchmark Bloch vector
    S = O.build_q_system(N, P_GOLDEN, Q_PHYS, O.material_separable_cos(N))
    out["basis_n2_golden"] = dict(V11=S.V11, V12=S.V12, V21=S.V21, V22=S.V22, V31=S.V31,
                                  V32=S.V32, detV1=S.detV1, W1=S.W1, W2=S.W2, invC=S.invC,
                                  kLift=S.kLift)
    # explicit K_r^{-1} action, N=2 tracking system, tight inner tolerance
    St = O.build_q_system(N, P_REF, Q_TRACKING, E)
    b = O.start_vector(11, St.nr)
    y = O.make_explicit_krinv_compact(St, 1e-12, 3000)[0](b)
    out["krinv_n2_tracking"] = dict(b=b, y=y)
    # 10 smallest eigenvalues: N=2 tracking system (reference KAT) and N=3 benchmark system
    lam2 = O.solve_modes(St, nev=10, p=40, tol=1e-10, tolCG=1e-12)["lam"]
    S3 = O.build_q_system(3, P_GOLDEN, Q_PHYS, O.material_separable_cos(3))
    lam3 = O.solve_modes(S3, nev=10, p=40, tol=1e-10, tolCG=1e-12)["lam"]
    out["eigs"] = dict(n2_tracking=lam2, n3_golden_cos=lam3,
                       kat_n2=np.array([1.201276300237e-02, 4.496454358674e-02]))
    # Yee-field reconstruction, N=1: direct and multi-center Taylor (p=6, 8 centers)
    S1 = O.build_q_system(1, P_GOLDEN, Q_PHYS, O.material_separable_cos(1))
    Qm = O.build_projected_q_modes(P_GOLDEN, S1.kLift, 1)
    c = O.start_vector(13, S1.NF)
    r1, _, _, sz = O.build_yee_points(4, 0.0125)
    blocks = O.build_yee_block_partition(sz, 2)
    out["recon_n1"] = dict(coeff=c, qModes=Qm, r=r1, direct=O.reconstruct_field_direct_blocked(c, Qm, r1),
                           taylor6=O.reconstruct_field_taylor_multi(c, Qm, r1, 6, blocks))
    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print("wrote", name)


if __name__ == "__main__":
    main()
