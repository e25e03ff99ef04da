"""GPU parity of the rank-1 lattice transforms (exp1/rank1_exact_fft_scatter.m:1-13,
exp1/rank1_exact_ifft_gather.m:1-11) against the oracle's NumPy restatement.

``fame_rank1_exact_fft_scatter`` embeds x at the plan's input codes and takes the
length-M DFT (mixed-radix Stockham passes of radix nGrid and B = 2 nGrid - 1);
``fame_rank1_exact_ifft_gather`` inverts a length-M spectrum and reads the target codes.
Composed with the plan's kernel spectrum they must give the 6D mass convolution.
"""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def _rand(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _plans(N):
    """The oracle's plan (0-based codes) and the reference's 1-based index vectors."""
    p0 = O.build_radix_exact_rank1_plan_scalar(N)
    p1 = dict(NF=p0["NF"], M=p0["M"], inputIdx=(p0["inputIdx"] + 1).astype(np.uint32),
              targetIdx=(p0["targetIdx"] + 1).astype(np.uint32))
    return p0, p1


@pytest.mark.parametrize("N", [1, 2, 3])
def test_scatter_matches_oracle(cuda_device, N):
    import fame_b200 as F
    p0, p1 = _plans(N)
    x = _rand((p0["NF"], 2), 40 + N)
    X = F.rank1_exact_fft_scatter(torch.as_tensor(x, device=cuda_device), p1).cpu().numpy()
    assert X.shape == (p0["M"], 2)
    assert _rel(X, O.rank1_exact_fft_scatter(x, p0)) < 1e-13


@pytest.mark.parametrize("N", [1, 2, 3])
def test_gather_matches_oracle(cuda_device, N):
    import fame_b200 as F
    p0, p1 = _plans(N)
    Y = _rand((p0["M"], 2), 50 + N)
    y = F.rank1_exact_ifft_gather(torch.as_tensor(Y, device=cuda_device), p1).cpu().numpy()
    assert y.shape == (p0["NF"], 2)
    assert _rel(y, O.rank1_exact_ifft_gather(Y, p0)) < 1e-13


@pytest.mark.parametrize("N", [1, 2])
def test_scatter_gather_compose_to_the_6d_mass_operator(cuda_device, N):
    """applyMij_rank1_exact = gather(kernelFFT .* scatter(x)) (exp1/applyMij_rank1_exact.m:1-6)
    equals the 6D FFT convolution of the same material (the plan is exact)."""
    import fame_b200 as F
    p0, p1 = _plans(N)
    E = O.material_smooth_exp(N, 4.0, 1.2)
    kf = O.build_exact_rank1_scalar_kernel_fft(E, p0)
    x = _rand(p0["NF"], 60 + N)
    xt = torch.as_tensor(x, device=cuda_device)
    X = F.rank1_exact_fft_scatter(xt, p1)
    y = F.rank1_exact_ifft_gather(torch.as_tensor(kf, device=cuda_device) * X, p1).cpu().numpy()
    assert _rel(y, O.applyMij_fft(x, E, N)) < 1e-12
    m = F.MassBackend(torch.as_tensor(E, device=cuda_device), N)
    assert _rel(y, m.MscalarOp(xt).cpu().numpy()) < 1e-12


def test_round_trip_at_n5(cuda_device):
    """Full size (M = 10 * 19^5 = 24,760,990): gathering the scatter's spectrum at the input
    codes returns x (ifft(fft(embedding)) is the embedding)."""
    import fame_b200 as F
    p0, p1 = _plans(5)
    assert p0["M"] == 24760990
    back = dict(p1, targetIdx=p1["inputIdx"])
    x = torch.as_tensor(_rand(p0["NF"], 70), device=cuda_device)
    X = F.rank1_exact_fft_scatter(x, p1)
    y = F.rank1_exact_ifft_gather(X, back)
    assert float(torch.linalg.norm(y - x) / torch.linalg.norm(x)) < 1e-13
    # the DC coefficient of the spectrum is the plain sum of x
    assert abs(complex(X[0].item()) - complex(x.sum().item())) < 1e-9 * float(torch.linalg.norm(x))


def test_general_lengths_match_numpy(cuda_device):
    """Lengths that are products of other supported radices (16, 27, 13, ...), any codes."""
    import fame_b200 as F
    rng = np.random.default_rng(80)
    for M in (16 * 27, 13 * 12 * 9, 2 * 3 * 5 * 7 * 11, 23 * 8):
        NF = M // 3
        idx = rng.choice(M, NF, replace=False).astype(np.uint32) + 1
        plan = dict(NF=NF, M=M, inputIdx=idx, targetIdx=idx)
        x = _rand(NF, M)
        emb = np.zeros(M, dtype=np.complex128)
        emb[idx.astype(np.int64) - 1] = x
        X = F.rank1_exact_fft_scatter(torch.as_tensor(x, device=cuda_device), plan).cpu().numpy()
        assert _rel(X, np.fft.fft(emb)) < 1e-13, M
        Y = _rand(M, M + 1)
        y = F.rank1_exact_ifft_gather(torch.as_tensor(Y, device=cuda_device), plan).cpu().numpy()
        assert _rel(y, np.fft.ifft(Y)[idx.astype(np.int64) - 1]) < 1e-13, M


def test_errors(cuda_device):
    import fame_b200 as F
    from fame_b200 import _lib as L
    p0, p1 = _plans(1)
    x = torch.as_tensor(_rand(p0["NF"], 90), device=cuda_device)
    with pytest.raises(F.FameError) as e:  # x without plan.NF rows
        F.rank1_exact_fft_scatter(x[:-1], p1)
    assert e.value.status == L.FAME_ERR_INVALID and "BadSize" in str(e.value)
    with pytest.raises(F.FameError) as e:  # Yfft without plan.M rows
        F.rank1_exact_ifft_gather(x, p1)
    assert e.value.status == L.FAME_ERR_INVALID and "BadSize" in str(e.value)
    bad = dict(p1, inputIdx=p1["inputIdx"].copy())
    bad["inputIdx"][3] = p1["M"] + 1  # an index past the embedding: rejected, nothing written there
    with pytest.raises(F.FameError) as e:
        F.rank1_exact_fft_scatter(x, bad)
    assert e.value.status == L.FAME_ERR_INVALID
    odd = dict(p1, M=29 * p1["NF"])  # a prime factor above 27
    with pytest.raises(F.FameError) as e:
        F.rank1_exact_fft_scatter(x, odd)
    assert e.value.status == L.FAME_ERR_UNSUPPORTED
