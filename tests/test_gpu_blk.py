"""Tensor-core block SpMM (k_spmm_blk, tcgen05 kind::tf32 on 128-row blocks
of a float32 operator).

Its products use TF32 hi/lo parts of both operands (three products per K
step, ~2^-22 relative error each) and the tensor core's FP32 accumulation,
whose truncation shrinks |y| by a few 1e-6.  Bar: estimator samples within
RTOL_BLOCK = 1e-5 relative of the FP64 engine and of the CUDA-core FP32
kernels on identical probes."""

import numpy as np
import pytest
import scipy.sparse as sp

import imate_b200 as ib
from imate_b200.batch import tune_operator, set_variant

pytestmark = pytest.mark.gpu

RTOL_BLOCK = 1e-5


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def rel_scaled(a, b):
    """Max |a - b| per probe over that probe's largest |b| (Lanczos
    coefficients of a general matrix can come close to zero)."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    scale = np.nanmax(np.abs(b), axis=1, keepdims=True)
    return float(np.nanmax(np.abs(a - b) / scale))


def _force_block(op, width, transpose=False):
    """Make the block kernel the operator's SpMM at this width (the tuner's
    candidate list, then set_variant)."""
    cands, _ = tune_operator(op, width, transpose=transpose, reps=1)
    idx = [i for i, c in enumerate(cands) if c["kind"] == "block-tc"]
    assert idx, cands
    set_variant(op, width, idx[0], transpose=transpose)


def _run(func, M, block, parameters=None, gram=False, **kw):
    eng = ib.EngineOptions(block_size=block, rng="parity",
                           return_coefficients=True)
    f = {"log": ib.logdet, "inv": ib.traceinv, "id": ib.trace}[func]
    extra = {} if parameters is None else {"parameters": parameters}
    return f(M, method="slq", gpu=True, gram=gram, return_info=True,
             engine=eng, **extra, **kw)


@pytest.mark.parametrize("block", [128, 256])
def test_block_estimator_matches_fp64_and_cuda_core(cuda, block):
    A = ib.correlation_matrix(20000, scale=0.01, threshold=0.05, shift=0.1,
                              seed=2, dtype=np.float32)
    kw = dict(min_num_samples=block, max_num_samples=block, error_rtol=0.0,
              lanczos_degree=24, orthogonalize=-1, seed=3)
    Mb = ib.Matrix(A, blocks=True)
    op = Mb.get_device_operator()
    assert op.block_formats
    # the built-in choice of an operator with blocks is the block kernel;
    # forcing it makes the check independent of that choice
    _force_block(op, block)
    _, ib_ = _run("log", Mb, block, **kw)
    _, i64 = _run("log", ib.Matrix(A.astype(np.float64)), 64, **kw)
    _, i32 = _run("log", ib.Matrix(A), block, **kw)
    sb = ib_["convergence"]["samples"]
    assert rel(sb, i64["convergence"]["samples"]) < RTOL_BLOCK
    assert rel(sb, i32["convergence"]["samples"]) < RTOL_BLOCK
    assert rel_scaled(ib_["engine"]["alpha"],
                      i64["engine"]["alpha"]) < RTOL_BLOCK


def _ragged_matrix():
    """n = 5000 (last block of 8 rows), rows 300-699 empty (rows 384-639 are
    two whole 128-row blocks whose unions are empty: one zero stage each),
    50 explicit zeros; symmetric, unstructured (unions of ~4,700 columns)."""
    rng = np.random.default_rng(7)
    n = 5000
    B = sp.random(n, n, density=0.004, random_state=8, format="coo")
    S = (B + B.T).tocoo()
    keep = ~(((S.row >= 300) & (S.row < 700)) |
             ((S.col >= 300) & (S.col < 700)))
    d = np.r_[0:300, 700:n]
    zr = rng.integers(700, n, 50)  # explicit zeros off the diagonal
    rows = np.concatenate([S.row[keep], d, zr])
    cols = np.concatenate([S.col[keep], d, (zr + 7) % n])
    vals = np.concatenate([S.data[keep], 1.0 + rng.random(d.size),
                           np.zeros(zr.size)])
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n), dtype=np.float32)
    A.sum_duplicates()
    assert np.all(np.diff(A.indptr)[384:640] == 0)
    return A


@pytest.mark.parametrize("width", [128, 256])
@pytest.mark.parametrize("transpose", [False, True])
def test_block_products_match_scipy(cuda, width, transpose):
    # one product through slq_operator_dot, which runs block-wide products
    # of an operator with the block format on the block kernel: error within
    # 1e-5 of |A| |x| per entry, empty rows exactly zero
    import torch
    A = _ragged_matrix()
    n = A.shape[0]
    M = ib.Matrix(A, blocks=True, reorder=False, group_rows=0)
    op = M.get_device_operator(need_transpose=transpose)
    assert len(op.block_formats) == (2 if transpose else 1)
    X = np.random.default_rng(3).standard_normal((n, width)).astype(np.float32)
    Y = op.dot(torch.from_numpy(X).cuda(), transpose=transpose).cpu().numpy()
    At = (A.T if transpose else A).astype(np.float64)
    want = At @ X.astype(np.float64)
    scale = abs(At) @ np.abs(X.astype(np.float64))
    assert np.max(np.abs(Y - want) / np.maximum(scale, 1e-30)) < RTOL_BLOCK
    empty = np.diff(At.tocsr().indptr) == 0
    assert np.all(Y[empty] == 0.0)


@pytest.mark.parametrize("block", [128, 256])
def test_block_kernel_with_empty_rows_and_ragged_last_block(cuda, block):
    # the trace estimator needs no definite matrix; its sample is n alpha_0,
    # and the first Lanczos coefficients are compared before the rounding
    # differences of an unstructured matrix grow with the steps
    A = _ragged_matrix()
    kw = dict(min_num_samples=block, max_num_samples=block, error_rtol=0.0,
              lanczos_degree=16, orthogonalize=-1, seed=11)
    Mb = ib.Matrix(A, blocks=True, reorder=False, group_rows=0)
    _force_block(Mb.get_device_operator(), block)
    _, ib_ = _run("id", Mb, block, **kw)
    _, i64 = _run("id", ib.Matrix(A.astype(np.float64), reorder=False,
                                  group_rows=0), 64, **kw)
    assert rel_scaled(ib_["engine"]["alpha"][:, :4],
                      i64["engine"]["alpha"][:, :4]) < RTOL_BLOCK
    assert rel_scaled(ib_["engine"]["beta"][:, :4],
                      i64["engine"]["beta"][:, :4]) < RTOL_BLOCK
    assert rel(ib_["convergence"]["samples"],
               i64["convergence"]["samples"]) < RTOL_BLOCK


def test_block_kernel_affine_shift(cuda):
    # A + t I: the epilogue adds t s x
    A = ib.correlation_matrix(9000, scale=0.015, threshold=0.05, shift=0.05,
                              seed=4, dtype=np.float32)
    ts = [0.05, 0.5]
    kw = dict(min_num_samples=128, max_num_samples=128, error_rtol=0.0,
              lanczos_degree=20, orthogonalize=-1, seed=2)
    F = ib.AffineMatrixFunction(A, blocks=True)
    _force_block(F.get_device_operator(), 128)
    trb, ib_ = _run("log", F, 128, parameters=ts, **kw)
    tr64, i64 = _run("log", ib.AffineMatrixFunction(A.astype(np.float64)),
                     64, parameters=ts, **kw)
    assert rel(ib_["convergence"]["samples"],
               i64["convergence"]["samples"]) < RTOL_BLOCK


def test_block_kernel_golub_kahn_rectangular(cuda):
    # gram=True on a tall CSC matrix: A and A^T products both on blocks
    rng = np.random.default_rng(5)
    m, n = 3000, 1100
    rows = np.concatenate([rng.choice(m, 12, replace=False) for _ in range(n)])
    cols = np.repeat(np.arange(n), 12)
    X = sp.csc_matrix((rng.standard_normal(rows.size), (rows, cols)),
                      shape=(m, n))
    X = (X + sp.eye(m, n, format="csc") * 2.0).astype(np.float32)
    kw = dict(min_num_samples=128, max_num_samples=128, error_rtol=0.0,
              lanczos_degree=20, orthogonalize=-1, seed=6)
    Mb = ib.Matrix(X, blocks=True)
    op = Mb.get_device_operator(need_transpose=True)
    assert len(op.block_formats) == 2
    _force_block(op, 128)
    _force_block(op, 128, transpose=True)
    _, ib_ = _run("log", Mb, 128, gram=True, **kw)
    _, i64 = _run("log", ib.Matrix(X.astype(np.float64)), 64, gram=True,
                  **kw)
    assert rel(ib_["convergence"]["samples"],
               i64["convergence"]["samples"]) < RTOL_BLOCK


def test_block_kernel_normal_equations(cuda):
    # x -> X^T (X x) + t x: the second product subtracts -t s v (three-term
    # form of the epilogue) and sums (s v) . y
    rng = np.random.default_rng(9)
    m, n = 4000, 1500
    rows = np.concatenate([rng.choice(m, 10, replace=False) for _ in range(n)])
    cols = np.repeat(np.arange(n), 10)
    X = sp.csc_matrix((rng.standard_normal(rows.size), (rows, cols)),
                      shape=(m, n)).astype(np.float32)
    kw = dict(min_num_samples=128, max_num_samples=128, error_rtol=0.0,
              lanczos_degree=20, orthogonalize=-1, seed=8)
    G = ib.GramAffineMatrixFunction(X, blocks=True)
    op = G.get_device_operator(need_transpose=True)
    _force_block(op, 128)
    _force_block(op, 128, transpose=True)
    _, ib_ = _run("log", G, 128, parameters=0.05, **kw)
    _, i64 = _run("log", ib.GramAffineMatrixFunction(X.astype(np.float64)),
                  64, parameters=0.05, **kw)
    assert rel(ib_["convergence"]["samples"],
               i64["convergence"]["samples"]) < RTOL_BLOCK


def test_block_candidate_listed_only_with_the_format(cuda):
    A = ib.correlation_matrix(4096, scale=0.03, threshold=0.05, shift=0.1,
                              seed=1, dtype=np.float32)
    with_b, _ = tune_operator(ib.Matrix(A, blocks=True).get_device_operator(),
                              256, reps=1)
    without, _ = tune_operator(ib.Matrix(A).get_device_operator(), 256,
                               reps=1)
    assert "block-tc" in [c["kind"] for c in with_b]
    assert "block-tc" not in [c["kind"] for c in without]
    # float64 operators never get the block format
    M64 = ib.Matrix(A.astype(np.float64), blocks=True)
    assert not M64.get_device_operator().block_formats


def _wide_matrix():
    """n = 300,000, diagonal plus three entries that make block 0 reach from
    column 0 to column n - 1: a span above the 262,144 columns of a block's
    bitmap, so the build takes the sorted-key path."""
    n = 300000
    i = np.arange(n)
    rows = np.r_[i, 0, 5, 127]
    cols = np.r_[i, n - 1, n - 2, 200000]
    vals = np.r_[1.0 + np.random.default_rng(4).random(n), 0.5, -0.25, 2.0]
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n), dtype=np.float32)


def _corr_matrix():
    return ib.correlation_matrix(20000, scale=0.01, threshold=0.05, shift=0.1,
                                 seed=2, dtype=np.float32)


@pytest.mark.parametrize("case", ["ragged", "wide", "corr"])
def test_block_unions_by_bitmap_equal_sorted_keys(cuda, case):
    # the block format built from per-block column bitmaps (the default) is
    # the one built from sorted (block, column) keys: same blocks and stages,
    # products equal bit for bit in both directions
    import torch
    from imate_b200 import _lib
    lib = _lib.load()
    A = {"ragged": _ragged_matrix, "wide": _wide_matrix,
         "corr": _corr_matrix}[case]()
    opts = {} if case == "corr" else dict(reorder=False, group_rows=0)
    X = torch.from_numpy(np.random.default_rng(5).standard_normal(
        (A.shape[0], 128)).astype(np.float32)).cuda()
    got = []
    for sorted_keys in (1, 0):
        _lib.check(lib.slq_debug_blocks_sorted_keys(sorted_keys))
        try:
            M = ib.Matrix(A, blocks=True, **opts)
            op = M.get_device_operator(need_transpose=True)
        finally:
            _lib.check(lib.slq_debug_blocks_sorted_keys(0))
        assert len(op.block_formats) == 2
        got.append((op.blocks_info(False), op.blocks_info(True),
                    op.dot(X).cpu().numpy(),
                    op.dot(X, transpose=True).cpu().numpy()))
    assert got[0][0] == got[1][0] and got[0][1] == got[1][1]
    assert np.array_equal(got[0][2], got[1][2])
    assert np.array_equal(got[0][3], got[1][3])
    if case == "wide":
        want = A.astype(np.float64) @ X.cpu().numpy().astype(np.float64)
        assert np.max(np.abs(got[1][2] - want)) < 1e-5 * np.max(np.abs(want))


def test_block_unions_hook_rejects_bad_values(cuda):
    from imate_b200 import _lib
    lib = _lib.load()
    assert lib.slq_debug_blocks_sorted_keys(2) == 1  # bad argument
    assert lib.slq_debug_blocks_sorted_keys(0) == 0


def test_block_candidate_order_rejected_for_poor_fill(cuda):
    # an unstructured matrix: the block/group candidate order fills its
    # 16-row groups poorly, so the operator built with it beside the fill
    # check is rebuilt with the row-group statistics' order -- the operator
    # that order gives directly, with products equal to scipy's
    import torch
    from imate_b200.linear_operator import (_fallback_order, _group_fill,
                                            block_group_order, locality_order)
    n = 4096
    B = sp.random(n, n, density=0.006, random_state=12, format="csr")
    A = (B + B.T + sp.identity(n) * 4.0).tocsr().astype(np.float32)
    A.sort_indices()
    assert A.nnz >= 8 * n
    base = locality_order(A)
    cand = block_group_order(A, base, 128, 16)
    assert _group_fill(A, cand, 16) < 0.5
    G, perm = _fallback_order(A, base, "auto", True, True)
    M = ib.Matrix(A, blocks=True)
    op = M.get_device_operator()
    assert op.group_rows == G
    if perm is None:
        assert op.perm is None
    else:
        assert np.array_equal(op.perm.cpu().numpy(), perm)
    X = np.random.default_rng(6).standard_normal((n, 128)).astype(np.float32)
    Y = op.dot(torch.from_numpy(X).cuda()).cpu().numpy()
    want = A.astype(np.float64) @ X.astype(np.float64)
    scale = abs(A.astype(np.float64)) @ np.abs(X.astype(np.float64))
    assert np.max(np.abs(Y - want) / scale) < RTOL_BLOCK
