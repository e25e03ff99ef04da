"""Pinned inputs of the benchmark workloads, restated for the CPU checker.

TEST INFRASTRUCTURE ONLY (see the package docstring).  The same values are defined
by the product in ``fame_b200.configs``; ``tests/test_oracle.py`` checks that both
agree.  The CPU legs of ``bench.py`` read them from here so that the reference arm
never loads the CUDA library.
"""
import math

import numpy as np

PHI = (1.0 + math.sqrt(5.0)) / 2.0
#: axis-block golden-ratio cut matrix of the benchmark workloads
P_GOLDEN = np.vstack([np.eye(3), np.diag([PHI, 1.0 / PHI, PHI ** 2])])
#: the reference's cut matrix [I3; diag(sqrt2, sqrt3, sqrt5)] (exp1/make_config_exp1bc.m:20-26)
P_REFERENCE = np.vstack([np.eye(3), np.diag([math.sqrt(2.0), math.sqrt(3.0), math.sqrt(5.0)])])
Q_PHYS = (0.05, 0.04, 0.03)        # exp1/make_config_exp1bc.m:34
Q_TRACKING = (0.13, 0.21, 0.17)    # exp3/make_config_experiment4.m:26
SEED = 20260905                    # exp1/make_config_BC_fig1a.m:42
#: 10 smallest eigenpairs: shift 0, Krylov block 40, outer tol 1e-8, inner Mhat PCG tol 1e-10
SOLVE = dict(nev=10, p=40, tol=1e-8, maxRestart=30, tolCG=1e-10, maxitCG=3000)
