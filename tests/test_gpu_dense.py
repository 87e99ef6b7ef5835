"""Dense float32 operators: the tensor-core product (three TF32 terms per
product, FP32 accumulation in tensor memory) against FP64 numpy, and SLQ
estimates on dense input against the sparse FP64 path on identical probes.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import imate_b200 as ib

pytestmark = pytest.mark.gpu


def _err(y, ref):
    return float(np.max(np.abs(y - ref)) / np.max(np.abs(ref)))


# products of fewer than 75 row tiles split K over the idle SMs (up to 8
# parts, added by k_dense_epi): (10000, 600) runs unsplit one way and split
# the other; (129, 20000) splits 8 ways
@pytest.mark.parametrize("rows,cols", [(1000, 1000), (300, 700), (129, 33),
                                       (4096, 4096), (10000, 600),
                                       (129, 20000)])
@pytest.mark.parametrize("width", [1, 16, 100, 256, 300])
def test_dense_product_matches_fp64(cuda, rows, cols, width):
    import torch
    rng = np.random.default_rng(rows + cols + width)
    A = rng.standard_normal((rows, cols)).astype(np.float32)
    op = ib.Matrix(A).get_device_operator(need_transpose=True)
    assert getattr(op, "dense", False)
    for transpose in (False, True):
        n_in = rows if transpose else cols
        X = rng.standard_normal((n_in, width)).astype(np.float32)
        Y = op.dot(torch.from_numpy(X).cuda(), transpose=transpose)
        Y = Y.cpu().numpy().astype(np.float64)
        A64 = A.astype(np.float64)
        ref = (A64.T if transpose else A64) @ X.astype(np.float64)
        # three TF32 terms: FP32-level error; the tensor core's FP32
        # accumulation rounds less carefully than an FMA chain (measured
        # 6.7e-6 at K = 1000 against ~2e-6 for FP32 FMAs)
        assert _err(Y, ref) < 5e-5, (transpose, _err(Y, ref))


def test_dense_estimates_match_sparse_fp64(cuda):
    A = ib.correlation_matrix(3000, scale=0.02, shift=0.1, seed=4)
    dense = A.toarray().astype(np.float32)
    kw = dict(min_num_samples=64, max_num_samples=64, error_rtol=1e-8,
              lanczos_degree=30, orthogonalize=-1, seed=2)
    for fn in (ib.logdet, ib.traceinv):
        t32, i32 = fn(dense, method="slq", gpu=True, return_info=True, **kw)
        t64, i64 = fn(A, method="slq", gpu=True, return_info=True, **kw)
        s32 = np.asarray(i32["convergence"]["samples"], float)
        s64 = np.asarray(i64["convergence"]["samples"], float)
        assert np.max(np.abs(s32 - s64) / np.abs(s64)) < 1e-5
        assert abs(t32 - t64) < 1e-5 * abs(t64)


def test_dense_gram_and_shift(cuda):
    rng = np.random.default_rng(9)
    X = rng.standard_normal((600, 200)).astype(np.float32)
    kw = dict(min_num_samples=32, max_num_samples=32, error_rtol=1e-8,
              lanczos_degree=40, orthogonalize=-1, seed=1)
    g32, _ = ib.logdet(X, gram=True, method="slq", gpu=True,
                       return_info=True, **kw)
    g64, _ = ib.logdet(sp.csr_matrix(X.astype(np.float64)), gram=True,
                       method="slq", gpu=True, return_info=True, **kw)
    assert abs(g32 - g64) < 1e-5 * abs(g64)
    S = (X.T @ X / 600.0).astype(np.float32)
    t = [0.1, 1.0]
    a32, _ = ib.logdet(ib.AffineMatrixFunction(S), parameters=t, method="slq",
                       gpu=True, return_info=True, **kw)
    a64, _ = ib.logdet(ib.AffineMatrixFunction(sp.csr_matrix(
        S.astype(np.float64))), parameters=t, method="slq", gpu=True,
        return_info=True, **kw)
    assert np.max(np.abs(a32 - a64) / np.abs(a64)) < 1e-5


def test_dense_operator_refuses_tuning_and_batches(cuda):
    from imate_b200.batch import tune_operator, logdet_batch
    from imate_b200 import _lib
    A = np.eye(64, dtype=np.float32) * 2.0
    op = ib.Matrix(A).get_device_operator()
    with pytest.raises(_lib.SlqError):
        tune_operator(op, 64)
    with pytest.raises(NotImplementedError):
        logdet_batch([A], gpu=True, min_num_samples=4,
                     max_num_samples=4)


def test_dense_wide_block_partials(cuda):
    # a 512-probe block: two 256-probe products per step, whose partial sums
    # (alpha, norms) share one set of partial rows
    A = ib.correlation_matrix(2000, scale=0.03, shift=0.1, seed=6)
    dense = A.toarray().astype(np.float32)
    kw = dict(min_num_samples=300, max_num_samples=300, error_rtol=1e-8,
              lanczos_degree=20, orthogonalize=-1, seed=3)
    eng = ib.EngineOptions(block_size=512)
    t32, i32 = ib.logdet(dense, method="slq", gpu=True, return_info=True,
                         engine=eng, **kw)
    t64, i64 = ib.logdet(A, method="slq", gpu=True, return_info=True,
                         engine=eng, **kw)
    s32 = np.asarray(i32["convergence"]["samples"], float)
    s64 = np.asarray(i64["convergence"]["samples"], float)
    assert np.max(np.abs(s32 - s64) / np.abs(s64)) < 1e-5


def test_dense_split_products_are_deterministic(cuda):
    """A split product adds its K parts in a fixed order: repeated products
    are bitwise equal."""
    import torch
    rng = np.random.default_rng(5)
    A = rng.standard_normal((1500, 5000)).astype(np.float32)
    op = ib.Matrix(A).get_device_operator(need_transpose=True)
    X = torch.from_numpy(rng.standard_normal((5000, 64)).astype(np.float32))
    Y1 = op.dot(X.cuda()).cpu().numpy()
    Y2 = op.dot(X.cuda()).cpu().numpy()
    assert np.array_equal(Y1, Y2)
    ref = A.astype(np.float64) @ X.numpy().astype(np.float64)
    assert _err(Y1.astype(np.float64), ref) < 5e-5
