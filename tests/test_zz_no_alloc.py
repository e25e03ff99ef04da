"""GPU test of fame_apply_Mhat_C_scalar_compact_noalloc, called through the C ABI.

Some callers of this library cannot let it allocate device memory (a host that
owns every byte of the GPU through its own pool, or a loop that must not pay the
synchronisation of cudaMalloc/cudaFree).  The no-allocation entry point keeps its
scratch in a fixed static device array; here its output is checked against the
allocating entry point on two calls in a row, and sizes beyond the array are
rejected.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _system(N, dev):
    import fame_b200 as F
    m = F.MassBackend(F.configs.material_separable_cos(N, device=dev), N)
    s = F.build_q_system(m, F.configs.P_GOLDEN, F.configs.Q_PHYS)
    return F, m, s


@pytest.mark.parametrize("N,dtype,tol", [(4, torch.complex128, 1e-13), (5, torch.complex64, 1e-6)])
def test_noalloc_matches_allocating_entry_point(cuda_device, N, dtype, tol):
    F, m, s = _system(N, cuda_device)
    lib = F._lib.lib
    prec = 1 if dtype == torch.complex64 else 0
    for seed in (1, 2):  # two calls in a row share the static scratch
        g = torch.Generator(device="cpu").manual_seed(seed)
        x = torch.randn(s.NF, dtype=dtype, generator=g).to(cuda_device)
        y_ref = torch.empty_like(x)
        y = torch.full_like(x, float("nan"))
        s.ctx.bind()
        assert lib.fame_apply_Mhat_C_scalar_compact(s.h, m.h, C.c_void_p(x.data_ptr()),
                                                    C.c_void_p(y_ref.data_ptr()), prec) == 0
        assert lib.fame_apply_Mhat_C_scalar_compact_noalloc(s.h, m.h, C.c_void_p(x.data_ptr()),
                                                            C.c_void_p(y.data_ptr()), prec) == 0
        torch.cuda.synchronize()
        err = float(torch.linalg.norm(y - y_ref) / torch.linalg.norm(y_ref))
        assert np.isfinite(err) and err <= tol, (seed, err)


def test_noalloc_rejects_sizes_beyond_scratch(cuda_device):
    F, m, s = _system(5, cuda_device)  # FP64 N=5 needs 48 MB > 32 MiB
    lib = F._lib.lib
    x = torch.zeros(s.NF, dtype=torch.complex128, device=cuda_device)
    y = torch.zeros_like(x)
    s.ctx.bind()
    st = lib.fame_apply_Mhat_C_scalar_compact_noalloc(s.h, m.h, C.c_void_p(x.data_ptr()),
                                                      C.c_void_p(y.data_ptr()), 0)
    assert st == 1 and b"static scratch" in lib.fame_last_error()
