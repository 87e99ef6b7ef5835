"""traceinv (imate/traceinv/_slq_method.pyx:24) of the headline construction
at n = 8192 against its dense FP64 inverse.

The matrix is the sparse SPD correlation matrix of the headline workload
(points uniform in [0, 1]^2 from seed 1, kernel exp(-r/0.005) cut at 0.05,
diagonal shift 0.1) at n = 8192, where a dense FP64 Cholesky inverse is the
exact answer.  Bars:
- the 1024-probe estimate within 4 standard errors (sample standard
  deviation / sqrt(1024)) of trace(A^-1) from the dense inverse, for the
  default FP32 path, the block tensor-core path and the FP64 engine;
- on identical probes, FP32 samples within 1e-6 relative of the FP64
  engine's (row-group products) and within 1e-5 (block products, FP16
  hi/lo parts with FP32 tensor-core accumulation)."""

import numpy as np
import pytest

import imate_b200 as ib

pytestmark = pytest.mark.gpu

PROBES = 1024
KW = dict(method="slq", gpu=True, return_info=True, min_num_samples=PROBES,
          max_num_samples=PROBES, error_rtol=0.0, lanczos_degree=50,
          orthogonalize=-1, seed=0)


@pytest.fixture(scope="module")
def matrix():
    return ib.correlation_matrix(8192, scale=0.005, threshold=0.05,
                                 shift=0.1, seed=1, dtype="float32")


def _dense_traceinv(A):
    import torch
    D = torch.from_numpy(A.astype(np.float64).toarray()).cuda()
    L = torch.linalg.cholesky(D)
    tr = float(torch.cholesky_inverse(L).diagonal().sum().item())
    del D, L
    torch.cuda.empty_cache()
    return tr


def _run(M, block=256):
    tr, info = ib.traceinv(M, engine=ib.EngineOptions(block_size=block,
                                                      rng="parity"), **KW)
    s = np.asarray(info["convergence"]["samples"][:PROBES], float)
    return float(tr), s


def test_traceinv_matches_dense_inverse(cuda, matrix):
    A = matrix
    exact = _dense_traceinv(A)
    tr64, s64 = _run(ib.Matrix(A.astype(np.float64)))
    tr_r, s_r = _run(ib.Matrix(A))
    Mb = ib.Matrix(A, blocks=True)
    tr_b, s_b = _run(Mb)
    assert Mb.get_device_operator().block_formats
    for tr, s in ((tr64, s64), (tr_r, s_r), (tr_b, s_b)):
        se = np.std(s, ddof=1) / np.sqrt(s.size)
        assert abs(tr - exact) <= 4.0 * se, (tr, exact, se)
        assert se / exact < 5e-3
    assert np.max(np.abs(s_r - s64) / np.abs(s64)) < 1e-6
    assert np.max(np.abs(s_b - s64) / np.abs(s64)) < 1e-5
    print("\ntraceinv n=8192: dense %.6f, FP64 SLQ %.6f, FP32 %.6f, "
          "blocks %.6f, standard error %.2e"
          % (exact, tr64, tr_r, tr_b, np.std(s64, ddof=1) / np.sqrt(PROBES)))
