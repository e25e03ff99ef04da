"""CPU oracle for the 6D null-space-free eigensolver hot path.

TEST INFRASTRUCTURE ONLY.  This package restates, in NumPy FP64, the
algorithms of the reference MATLAB code (FAME-GPU, "Null-Space Free 6D
Projection Method").  It is used by the tests, by ``smoke()`` and by the
CPU-baseline leg of ``bench.py`` as the checker; nothing in the product
imports it.

Parity pins (see ``tests/test_oracle.py``):
  * the rank-1 lattice constants of the reference's N=5 static check
    (exp2/run_experiment2_allgpu_static_check.m:10-11);
  * rank-1-lattice mass == 6D fftn mass (exp1/smoke_test_rank1_lowmem.m:17-23);
  * the reference's stored tracked eigenvalues at N=2
    (exp3/make_config_experiment4.m:38-45, checked at rel 5e-7 as in
    exp3/solve_tracked_modes_exp4.m:37-42);
  * a dense generalized eigensolve at N=1.
"""
from .fame_oracle import *  # noqa: F401,F403
