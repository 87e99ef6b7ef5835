"""Parity of the CUDA engine with the oracle and with the reference's own
golden outputs.  Tolerances: bit-exact for probe bits and sample counts;
1e-10 relative for FP64 Lanczos/Golub-Kahn coefficients, nodes, weights and
per-probe samples (the FP64 parity bar against the reference CPU path);
FP32 operator products within 1e-5 relative of scipy."""

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import imate_b200 as ib
from imate_b200 import _lib
from golden_cases import FUNC_CASES, FUNC_SETTINGS
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-10


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _probes(lib, seed, rng, n, first, count, width, dtype):
    import torch
    tdt = torch.float64 if dtype == _lib.SLQ_F64 else torch.float32
    out = torch.full((n, width), 7.0, dtype=tdt, device="cuda")
    nb = ctypes.c_size_t(0)
    _lib.check(lib.slq_generate_probes_workspace_bytes(n, width,
                                                       ctypes.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    _lib.check(lib.slq_generate_probes(
        seed, rng, n, first, count, width, dtype, out.data_ptr(),
        ws.data_ptr(), ws.numel(),
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("n", [1, 63, 64, 65, 1000, 4097, 70001])
@pytest.mark.parametrize("first,count,width", [(0, 1, 1), (0, 8, 8),
                                               (5, 50, 64)])
def test_parity_probes_bit_exact(cuda, n, first, count, width):
    want = oracle.random_probes(3, n, first + count)[first:]
    for dt in (_lib.SLQ_F32, _lib.SLQ_F64):
        got = _probes(cuda, 3, 0, n, first, count, width, dt)
        assert np.array_equal(got[:, :count].T, want)
        assert np.all(got[:, count:] == 0)


def test_parity_probes_golden(cuda, golden):
    g = golden("rng.npz")
    for seed, n in ((0, 65), (3, 1000), (5, 4097)):
        want = g["probes_seed%d_n%d" % (seed, n)]
        got = _probes(cuda, seed, 0, n, 0, want.shape[0], 8, _lib.SLQ_F64)
        assert np.array_equal((got[:, :want.shape[0]].T > 0).astype(np.int8),
                              want)


def test_fast_probes_are_rademacher(cuda):
    got = _probes(cuda, 11, 1, 100000, 0, 32, 32, _lib.SLQ_F32)
    assert set(np.unique(got)) == {-1.0, 1.0}
    assert abs(got.mean()) < 0.01
    c = np.corrcoef(got.T)
    assert np.max(np.abs(c - np.eye(32))) < 0.02


def _dot(Aop, x, transpose=False, t=0.0):
    import torch
    X = torch.from_numpy(x).cuda()
    return Aop.dot(X, transpose=transpose, t=t).cpu().numpy()


@pytest.mark.parametrize("fmt", ["csr", "csc"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("width", [1, 3, 32, 128])
def test_operator_products(cuda, fmt, dtype, width):
    rng = np.random.default_rng(1)
    A = sp.random(700, 500, density=0.02, format=fmt, random_state=2,
                  dtype=np.float64).astype(dtype)
    M = ib.Matrix(A)
    op = M.get_device_operator(need_transpose=True)
    x = rng.standard_normal((500, width)).astype(dtype)
    z = rng.standard_normal((700, width)).astype(dtype)
    y = _dot(op, x)
    yt = _dot(op, z, transpose=True)
    tol = 1e-12 if dtype == np.float64 else 2e-5
    ref_y = A.astype(np.float64) @ x.astype(np.float64)
    ref_yt = A.T.astype(np.float64) @ z.astype(np.float64)
    assert np.max(np.abs(y - ref_y)) <= tol * np.max(np.abs(ref_y))
    assert np.max(np.abs(yt - ref_yt)) <= tol * np.max(np.abs(ref_yt))


def test_affine_operator_product(cuda, corr_small):
    Aop = ib.AffineMatrixFunction(corr_small)
    op = Aop.get_device_operator()
    x = np.random.default_rng(0).standard_normal((corr_small.shape[0], 4))
    y = _dot(op, x, t=0.75)
    want = corr_small @ x + 0.75 * x
    assert np.max(np.abs(y - want)) < 1e-12 * np.max(np.abs(want))


def _run(func, A, gram=False, block_size=0, coefficients=True, **kw):
    eng = ib.EngineOptions(block_size=block_size,
                           return_coefficients=coefficients)
    f = {"log": ib.logdet, "inv": ib.traceinv, "id": ib.trace}[func]
    tr, info = f(A, gram=gram, method="slq", gpu=True, return_info=True,
                 engine=eng, **kw)
    return tr, info


@pytest.mark.parametrize("orth", [0, -1, 10])
@pytest.mark.parametrize("block_size", [1, 4, 64])
def test_golub_kahn_coefficients_match_reference(cuda, golden, orth,
                                                 block_size):
    g = golden("krylov.npz")
    B = ib.toeplitz(2.0, 1.0, 16384)
    tr, info = _run("log", B, gram=True, block_size=block_size,
                    min_num_samples=4, max_num_samples=4, lanczos_degree=30,
                    orthogonalize=orth, seed=0)
    a = info["engine"]["alpha"]
    b = info["engine"]["beta"]
    for p in range(4):
        key = "c1_orth%d_p%d" % (orth, p)
        assert rel(a[p], g[key + "_alpha"]) < RTOL_FP64
        assert rel(b[p], g[key + "_beta"]) < RTOL_FP64


@pytest.mark.parametrize("orth", [0, -1, 1, 5])
@pytest.mark.parametrize("block_size", [1, 8, 256])
def test_lanczos_coefficients_match_reference(cuda, golden, corr_small, orth,
                                              block_size):
    g = golden("krylov.npz")
    tr, info = _run("log", corr_small, block_size=block_size,
                    min_num_samples=4, max_num_samples=4, lanczos_degree=20,
                    orthogonalize=orth, seed=5)
    a = info["engine"]["alpha"]
    b = info["engine"]["beta"]
    for p in range(4):
        key = "corr_orth%d_p%d" % (orth, p)
        assert rel(a[p], g[key + "_alpha"]) < RTOL_FP64
        assert rel(b[p], g[key + "_beta"]) < RTOL_FP64


def test_nodes_weights_match_lapack(cuda, golden):
    import torch
    g = golden("krylov.npz")
    keys = [("c1_orth-1_p0", 1), ("c1_orth0_p1", 1), ("corr_orth-1_p2", 0),
            ("corr_orth5_p3", 0)]
    for key, gram in keys:
        a = g[key + "_alpha"]
        bb = g[key + "_beta"]
        m = a.size
        A = torch.from_numpy(a.reshape(m, 1).copy()).cuda()
        Bt = torch.from_numpy(bb.reshape(m, 1).copy()).cuda()
        size = torch.tensor([m], dtype=torch.int32, device="cuda")
        th = torch.zeros((m, 1), dtype=torch.float64, device="cuda")
        tau = torch.zeros((m, 1), dtype=torch.float64, device="cuda")
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.check(cuda.slq_nodes_weights(
            A.data_ptr(), Bt.data_ptr(), size.data_ptr(), 1, m, gram,
            th.data_ptr(), tau.data_ptr(), st.data_ptr(),
            torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        t1 = th.cpu().numpy()[:, 0]
        w1 = tau.cpu().numpy()[:, 0] ** 2
        i1 = np.argsort(t1)
        t2 = g[key + "_theta"]
        w2 = g[key + "_tau"] ** 2
        i2 = np.argsort(t2)
        assert rel(t1[i1], t2[i2]) < RTOL_FP64
        assert np.max(np.abs(w1[i1] - w2[i2])) < RTOL_FP64


def _check_estimator(tr, info, g, key):
    used = int(np.atleast_1d(g[key + "_num_samples_used"])[0])
    conv = info["convergence"]
    np.testing.assert_array_equal(np.atleast_1d(conv["num_samples_used"]),
                                  g[key + "_num_samples_used"])
    np.testing.assert_array_equal(np.atleast_1d(conv["num_outliers"]),
                                  g[key + "_num_outliers"])
    order = g[key + "_processed_samples_indices"][:used]
    np.testing.assert_array_equal(conv["samples_processed_order"][:used],
                                  order)
    s = np.asarray(conv["samples"]).reshape(len(conv["samples"]), -1)
    assert rel(s[order], g[key + "_samples"][order]) < RTOL_FP64
    assert rel(np.atleast_1d(tr), g[key + "_trace"]) < RTOL_FP64
    assert rel(np.atleast_1d(info["error"]["absolute_error"]),
               g[key + "_error"]) < 1e-6


@pytest.mark.parametrize("orth", [0, -1])
@pytest.mark.parametrize("block_size", [0, 32])
def test_estimator_toeplitz_matches_reference(cuda, golden, orth, block_size):
    g = golden("estimator.npz")
    B = ib.toeplitz(2.0, 1.0, 16384)
    tr, info = _run("log", B, gram=True, block_size=block_size,
                    coefficients=False, min_num_samples=50,
                    max_num_samples=200, error_rtol=1e-3, lanczos_degree=30,
                    orthogonalize=orth, seed=0)
    _check_estimator(tr, info, g, "c1_log_orth%d" % orth)
    exact = ib.toeplitz_logdet(2.0, 1.0, 16384, gram=True)
    assert abs(tr - exact) / exact < 1e-3


@pytest.mark.parametrize("func", ["log", "inv", "id"])
def test_estimator_functions_match_reference(cuda, golden, corr_small, func):
    g = golden("estimator.npz")
    tr, info = _run(func, corr_small, coefficients=False, min_num_samples=10,
                    max_num_samples=64, error_rtol=1e-2, lanczos_degree=20,
                    orthogonalize=0, seed=3)
    _check_estimator(tr, info, g, "corr_%s" % func)


def test_estimator_gram_affine_exponent_match_reference(cuda, golden,
                                                        corr_small):
    g = golden("estimator.npz")
    tr, info = _run("log", corr_small, gram=True, coefficients=False,
                    min_num_samples=10, max_num_samples=40, error_rtol=1e-2,
                    lanczos_degree=15, orthogonalize=-1, seed=4)
    _check_estimator(tr, info, g, "corr_gram_log")
    Aop = ib.AffineMatrixFunction(corr_small)
    tr, info = _run("inv", Aop, coefficients=False,
                    parameters=[0.1, 1.0, 10.0], min_num_samples=5,
                    max_num_samples=30, error_rtol=1e-3, lanczos_degree=20,
                    orthogonalize=-1, seed=9)
    _check_estimator(tr, info, g, "corr_affine_inv")
    tr, info = ib.logdet(corr_small, p=2.0, method="slq", gpu=True,
                         return_info=True, min_num_samples=5,
                         max_num_samples=20, error_rtol=1e-2,
                         lanczos_degree=10, orthogonalize=3, seed=2)
    _check_estimator(tr, info, g, "corr_log_p2")


def test_estimator_matches_oracle_at_random_sizes(cuda):
    # sizes that exercise partial probe blocks and ragged rows
    rng = np.random.default_rng(8)
    for n, seed in ((37, 1), (301, 2), (1025, 3)):
        M = sp.random(n, n, density=min(1.0, 6.0 / n), random_state=seed,
                      format="csr")
        A = (M @ M.T + sp.eye(n) * 0.5).tocsr()
        for orth, bs in ((0, 4), (-1, 16), (3, 2)):
            kw = dict(min_num_samples=3, max_num_samples=21, error_rtol=1e-8,
                      lanczos_degree=12, orthogonalize=orth, seed=seed)
            tr, info = _run("log", A, block_size=bs, coefficients=False,
                            **kw)
            want = oracle.trace_estimator(A, "log", **kw)
            assert info["convergence"]["num_samples_used"] == \
                want["num_samples_used"][0]
            assert rel(info["convergence"]["samples"],
                       want["samples"][:, 0]) < RTOL_FP64
    assert rng is not None


def test_mixed_precision_toeplitz_accuracy(cuda):
    B = ib.toeplitz(2.0, 1.0, 16384, dtype="float32")
    tr, info = ib.logdet(B, gram=True, method="slq", gpu=True,
                         return_info=True, min_num_samples=50,
                         max_num_samples=200, error_rtol=1e-3,
                         lanczos_degree=30, orthogonalize=-1, seed=0)
    exact = ib.toeplitz_logdet(2.0, 1.0, 16384, gram=True)
    assert info["matrix"]["data_type"] == b"float32"
    assert abs(float(tr) - exact) / exact < 1e-3
    B64 = ib.toeplitz(2.0, 1.0, 16384)
    tr64, info64 = ib.logdet(B64, gram=True, method="slq", gpu=True,
                             return_info=True, min_num_samples=50,
                             max_num_samples=200, error_rtol=1e-3,
                             lanczos_degree=30, orthogonalize=-1, seed=0)
    s32 = info["convergence"]["samples"][:145]
    s64 = info64["convergence"]["samples"][:145]
    assert rel(s32, s64) < 1e-5


def test_bad_csr_is_rejected(cuda):
    A = sp.csr_matrix(np.eye(4))
    A.indices[2] = 9
    with pytest.raises(_lib.SlqError) as e:
        ib.Matrix(A).get_device_operator()
    assert e.value.status == 2


def test_identity_breaks_down_after_one_step(cuda):
    A = sp.eye(500, format="csr")
    tr, info = ib.logdet(A, method="slq", gpu=True, return_info=True,
                         min_num_samples=5, max_num_samples=5,
                         lanczos_degree=10, seed=1)
    assert np.all(info["engine"]["lanczos_size"][:5] == 1)
    assert abs(tr) < 1e-12
    tr, info = ib.traceinv(A, method="slq", gpu=True, return_info=True,
                           min_num_samples=5, max_num_samples=5,
                           lanczos_degree=10, seed=1)
    assert abs(tr - 500.0) < 1e-9


def test_indefinite_matrix_gives_nan_logdet(cuda):
    d = np.r_[np.full(50, 2.0), np.full(50, -1.0)]
    A = sp.diags(d).tocsr()
    tr, info = ib.logdet(A, method="slq", gpu=True, return_info=True,
                         min_num_samples=3, max_num_samples=3,
                         lanczos_degree=8, seed=2)
    assert np.isnan(tr)


def test_reordered_operator_products(cuda):
    A = ib.correlation_matrix(3000, scale=0.02, threshold=0.05, shift=0.1,
                              seed=5)
    M = ib.Matrix(A, reorder=True)
    op = M.get_device_operator(need_transpose=True)
    assert op.perm is not None
    x = np.random.default_rng(0).standard_normal((3000, 8))
    y = _dot(op, x)
    want = A @ x
    assert np.max(np.abs(y - want)) < 1e-12 * np.max(np.abs(want))


def _spread_rows_matrix(n, longest, seed):
    """Symmetric sparse matrix whose row lengths run from a few entries to
    about ``longest`` (every size of the device permutation's per-row
    sorting network)."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(n):
        k = int(rng.integers(1, 40)) if i % 50 else int(rng.integers(40, longest))
        c = rng.choice(n, size=k, replace=False)
        rows.append(np.full(k, i))
        cols.append(c)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    S = sp.csr_matrix((rng.uniform(0.1, 1.0, r.size), (r, c)), shape=(n, n))
    A = (S + S.T + sp.identity(n) * (2.0 * longest)).tocsr()
    A.sort_indices()
    return A


@pytest.mark.parametrize("longest", [900, 1400])
def test_device_permutation_equals_host_permuted_csr(cuda, longest):
    # rows of up to 1,024 entries are sorted one warp per row, longer
    # patterns by one radix sort of (row, column) keys: either way the
    # operator holds A[p][:, p] with sorted rows, so its products equal
    # those of the host-permuted matrix bit for bit
    A = _spread_rows_matrix(3000, longest, 11)
    deg = np.diff(A.indptr)
    assert deg.min() >= 1 and (deg.max() > 1024) == (longest > 1024)
    # rows for every network size: 32, 64, ..., 1,024 keys
    assert {int(np.ceil(np.log2(max(d, 32) / 32))) for d in deg if d <= 1024} \
        == {0, 1, 2, 3, 4, 5}
    M = ib.Matrix(A, reorder=True, group_rows=8)
    op = M.get_device_operator()
    assert op.perm is not None
    p = op.perm.cpu().numpy().astype(np.int64)
    Ap = A[p][:, p].tocsr()
    Ap.sort_indices()
    H = ib.Matrix(Ap, reorder=False, group_rows=8, aggregate=False)
    oph = H.get_device_operator()
    assert oph.perm is None and oph.group_rows == op.group_rows
    x = np.random.default_rng(2).standard_normal((3000, 5))
    y = _dot(op, x)
    yh = _dot(oph, x[p])
    assert np.array_equal(y[p], yh)


@pytest.mark.parametrize("orth", [0, -1])
def test_reordered_lanczos_matches_reference(cuda, golden, corr_small, orth):
    # a symmetric permutation changes only summation order
    g = golden("krylov.npz")
    M = ib.Matrix(corr_small, reorder=True)
    tr, info = _run("log", M, block_size=4, min_num_samples=4,
                    max_num_samples=4, lanczos_degree=20,
                    orthogonalize=orth, seed=5)
    assert M.get_device_operator().perm is not None
    for p in range(4):
        key = "corr_orth%d_p%d" % (orth, p)
        assert rel(info["engine"]["alpha"][p], g[key + "_alpha"]) < RTOL_FP64
        assert rel(info["engine"]["beta"][p], g[key + "_beta"]) < RTOL_FP64


def test_reordered_gram_matches_oracle(cuda, corr_small):
    M = ib.Matrix(corr_small, reorder=True)
    kw = dict(min_num_samples=3, max_num_samples=6, error_rtol=1e-9,
              lanczos_degree=12, orthogonalize=-1, seed=6)
    tr, info = _run("inv", M, gram=True, block_size=2, coefficients=False,
                    **kw)
    want = oracle.trace_estimator(corr_small, "inv", gram=True, **kw)
    assert rel(info["convergence"]["samples"], want["samples"][:, 0]) < \
        RTOL_FP64


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("width", [32, 64, 128, 256])
@pytest.mark.parametrize("group", [4, 8, 16])
def test_row_group_products_bit_identical_to_csr(cuda, dtype, width, group):
    if group == 16 and dtype == np.float64:
        pytest.skip("16-row groups are served by the FP32 kernels only")
    A = ib.correlation_matrix(5000, scale=0.02, threshold=0.05, shift=0.1,
                              seed=7, dtype=dtype)
    x = np.random.default_rng(1).standard_normal((5000, width)).astype(dtype)
    # same row order for both (aggregation would change the summation order)
    plain = ib.Matrix(A, reorder=True, group_rows=0)
    grouped = ib.Matrix(A, reorder=True, group_rows=group, aggregate=False)
    op0 = plain.get_device_operator(need_transpose=True)
    op1 = grouped.get_device_operator(need_transpose=True)
    assert op1.group_rows == group
    y0 = _dot(op0, x)
    y1 = _dot(op1, x)
    assert np.array_equal(y0, y1)
    assert np.array_equal(_dot(op0, x, transpose=True),
                          _dot(op1, x, transpose=True))
    want = A.astype(np.float64) @ x.astype(np.float64)
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert np.max(np.abs(y1 - want)) <= tol * np.max(np.abs(want))


@pytest.mark.parametrize("gram", [False, True])
def test_row_group_estimator_matches_oracle(cuda, gram):
    A = ib.correlation_matrix(3000, scale=0.03, threshold=0.05, shift=0.2,
                              seed=9)
    M = ib.Matrix(A, reorder=True, group_rows=8)
    kw = dict(min_num_samples=5, max_num_samples=40, error_rtol=1e-9,
              lanczos_degree=14, orthogonalize=-1, seed=12)
    tr, info = _run("log", M, gram=gram, block_size=64, coefficients=False,
                    **kw)
    assert M.get_device_operator(need_transpose=gram).group_rows == 8
    want = oracle.trace_estimator(A, "log", gram=gram, **kw)
    assert info["convergence"]["num_samples_used"] == \
        want["num_samples_used"][0]
    assert rel(info["convergence"]["samples"], want["samples"][:, 0]) < \
        RTOL_FP64


@pytest.mark.parametrize("gram", [False, True])
@pytest.mark.parametrize("block_size", [128, 256])
def test_tma_row_group_spmm_bit_identical_in_estimator(cuda, gram, block_size):
    # FP32 row-group operators with 128/256-wide blocks take the TMA
    # gather4 SpMM; its row sums run in the CSR order (bitwise equal
    # products), only the CTA count of the alpha reduction differs, so the
    # runs agree to FP64 rounding
    A = ib.correlation_matrix(6000, scale=0.02, threshold=0.05, shift=0.2,
                              seed=3, dtype=np.float32)
    kw = dict(min_num_samples=block_size, max_num_samples=block_size,
              error_rtol=0.0, lanczos_degree=12, orthogonalize=-1, seed=4)
    out = []
    for g in (0, 8, 16):
        M = ib.Matrix(A, reorder=True, group_rows=g, aggregate=False)
        tr, info = _run("log", M, gram=gram, block_size=block_size,
                        coefficients=True, **kw)
        assert M.get_device_operator(need_transpose=gram).group_rows == g
        out.append(info)
    for o in out[1:]:
        assert rel(o["convergence"]["samples"],
                   out[0]["convergence"]["samples"]) < 1e-9
        assert rel(o["engine"]["alpha"], out[0]["engine"]["alpha"]) < 1e-9
        assert rel(o["engine"]["beta"], out[0]["engine"]["beta"]) < 1e-9


@pytest.mark.parametrize("fmt", ["csr", "csc"])
def test_rectangular_gram_matches_oracle(cuda, fmt):
    # X^T X of a tall X: probes of length ncols, trace scale ncols (the
    # reference uses nrows there, which is only right for square X)
    rng = np.random.default_rng(3)
    X = sp.random(700, 240, density=0.04, random_state=4, format="csr")
    X = (X + sp.eye(700, 240) * 0.7).asformat(fmt)
    kw = dict(min_num_samples=10, max_num_samples=64, error_rtol=1e-3,
              lanczos_degree=20, orthogonalize=-1, seed=5)
    tr, info = ib.logdet(X, gram=True, method="slq", gpu=True,
                         return_info=True, **kw)
    want = oracle.trace_estimator(X, "log", gram=True, **kw)
    used = int(want["num_samples_used"][0])
    assert info["convergence"]["num_samples_used"] == used
    assert rel(info["convergence"]["samples"][:used],
               want["samples"][:used, 0]) < RTOL_FP64
    exact = np.linalg.slogdet((X.T @ X).toarray())[1]
    assert abs(tr - exact) / abs(exact) < 0.02
    assert info["matrix"]["size"] == (700, 240)
    assert rng is not None


def test_distributed_single_rank_nccl_matches_single_process(cuda):
    import os
    import torch.distributed as dist
    from imate_b200.distributed import (distributed_trace_estimator,
                                        engine_block_runner)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29533")
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        A = ib.correlation_matrix(2000, scale=0.03, threshold=0.05,
                                  shift=0.2, seed=8)
        M = ib.Matrix(A)
        kw = dict(lanczos_degree=15, orthogonalize=-1, seed=11)
        run = engine_block_runner(M, "log", **kw)
        res = distributed_trace_estimator(run, q=1, block=16,
                                          min_num_samples=8,
                                          max_num_samples=64,
                                          error_rtol=1e-3)
        tr, info = ib.logdet(M, method="slq", gpu=True, return_info=True,
                             min_num_samples=8, max_num_samples=64,
                             error_rtol=1e-3,
                             engine=ib.EngineOptions(block_size=16), **kw)
        assert int(res["num_samples_used"][0]) == \
            int(info["convergence"]["num_samples_used"])
        assert abs(res["trace"][0] - tr) <= 1e-12 * abs(tr)
    finally:
        dist.destroy_process_group()


def _tall_sparse(m, n, per_col, seed, dtype=np.float64):
    # per_col distinct rows per column, N(0,1) values, CSC (the large
    # Gram-form workload's construction, scaled down)
    rng = np.random.default_rng(seed)
    rows = np.concatenate([rng.choice(m, per_col, replace=False)
                           for _ in range(n)])
    cols = np.repeat(np.arange(n), per_col)
    vals = rng.standard_normal(rows.size)
    return sp.csc_matrix((vals, (rows, cols)), shape=(m, n)).astype(dtype)


@pytest.mark.parametrize("orth", [0, -1])
def test_normal_equations_mode_matches_oracle(cuda, orth):
    X = _tall_sparse(2000, 500, 16, 4)
    lam = 1e-2
    kw = dict(min_num_samples=8, max_num_samples=40, error_rtol=1e-3,
              lanczos_degree=24, orthogonalize=orth, seed=9)
    G = ib.GramAffineMatrixFunction(X)
    tr, info = ib.logdet(G, method="slq", gpu=True, parameters=lam,
                         return_info=True, **kw)
    want = oracle.trace_estimator(X, "log", gram=2, parameters=[lam], **kw)
    used = int(want["num_samples_used"][0])
    assert int(info["convergence"]["num_samples_used"]) == used
    assert rel(info["convergence"]["samples"][:used],
               want["samples"][:used, 0]) < 1e-9
    exact = np.linalg.slogdet((X.T @ X).toarray() + lam * np.eye(500))[1]
    assert abs(tr - exact) / abs(exact) < 0.02


def test_normal_equations_sweep_and_fp32(cuda):
    X = _tall_sparse(3000, 800, 16, 5, dtype=np.float32)
    lams = [1e-2, 1e-1, 1.0]
    G = ib.GramAffineMatrixFunction(X)
    tr, info = ib.logdet(G, method="slq", gpu=True, parameters=lams,
                         return_info=True, min_num_samples=128,
                         max_num_samples=128, error_rtol=0.0,
                         lanczos_degree=40, orthogonalize=0, seed=1,
                         engine=ib.EngineOptions(block_size=128))
    XtX = (X.T @ X).toarray().astype(np.float64)
    for i, lam in enumerate(lams):
        exact = np.linalg.slogdet(XtX + lam * np.eye(800))[1]
        assert abs(tr[i] - exact) / abs(exact) < 0.02


def _consumer_call(A, func, coeff, gram, params, kw):
    # the public wrapper of imate's SLQ consumer that uses this function
    if params is not None:
        A = ib.AffineMatrixFunction(A)
        kw = dict(kw, parameters=params)
    common = dict(method="slq", gpu=True, return_info=True, gram=gram, **kw)
    if func == "exp":
        return ib.trexp(A, coeff=coeff[0], **common)
    if func == "linfrac":
        return ib.trlinfrac(A, coeff=coeff, **common)
    if func == "indicator":
        return ib.eigencount(A, interval=coeff, **common)
    if func == "gaussian":
        return ib.density(A, mu=coeff[0], sigma=coeff[1], **common)
    from imate_b200._trace_estimator import trace_estimator
    d = dict(ib._functions._SLQ_DEFAULTS)
    d.update(kw, gpu=True)
    return trace_estimator(
        A, d["parameters"], func, gram, 1.0, d["min_num_samples"],
        d["max_num_samples"], d["error_atol"], d["error_rtol"],
        d["confidence_level"], d["outlier_significance_level"],
        d["lanczos_degree"], d["lanczos_tol"], d["orthogonalize"], d["seed"],
        d["num_threads"], d["num_gpu_devices"], False, False, True,
        func_coeff=coeff)


@pytest.mark.parametrize("case", FUNC_CASES, ids=[c[0] for c in FUNC_CASES])
def test_other_functions_match_reference(cuda, golden, corr_small, case):
    # trexp / trlinfrac / eigencount / density (and smoothstep) against the
    # reference's own outputs on the same probes
    name, func, coeff, gram, params = case
    g = golden("functions.npz")
    key = "fn_" + name
    tr, info = _consumer_call(corr_small, func, coeff, gram, params,
                              dict(FUNC_SETTINGS))
    conv = info["convergence"]
    used = np.atleast_1d(conv["num_samples_used"])
    assert np.array_equal(used, g[key + "_num_samples_used"])
    order = g[key + "_processed_samples_indices"][:int(used[0])]
    assert np.array_equal(conv["samples_processed_order"][:order.size],
                          order)
    samples = np.asarray(conv["samples"]).reshape(FUNC_SETTINGS[
        "max_num_samples"], -1)
    assert rel(samples[order], g[key + "_samples"][order]) < RTOL_FP64
    assert rel(np.atleast_1d(tr), g[key + "_trace"]) < RTOL_FP64



@pytest.mark.parametrize("group", [8, 16])
def test_aggregated_groups_match_oracle(cuda, group):
    # neighbour-aggregated row order (a symmetric permutation): FP64 samples
    # within 1e-10 of the oracle (8-row groups; 16-row groups are FP32-only,
    # compared with the FP64 run on identical probes)
    A = ib.correlation_matrix(20000, scale=0.01, threshold=0.05, shift=0.2,
                              seed=6)
    kw = dict(min_num_samples=4, max_num_samples=16, error_rtol=1e-9,
              lanczos_degree=12, orthogonalize=-1, seed=8)
    M64 = ib.Matrix(A, reorder=True, group_rows=8, aggregate=True)
    tr64, info64 = _run("log", M64, gram=False, block_size=16,
                        coefficients=False, **kw)
    want = oracle.trace_estimator(A, "log", **kw)
    assert rel(info64["convergence"]["samples"], want["samples"][:, 0]) < \
        RTOL_FP64
    M32 = ib.Matrix(A.astype(np.float32), reorder=True, group_rows=group,
                    aggregate=True)
    op = M32.get_device_operator()
    assert op.group_rows == group and op.perm is not None
    tr32, info32 = _run("log", M32, gram=False, block_size=16,
                        coefficients=False, **kw)
    assert rel(info32["convergence"]["samples"],
               info64["convergence"]["samples"]) < 1e-5


def _device_pattern(A):
    import torch
    A = sp.csr_matrix(A)
    return (torch.from_numpy(A.indptr.astype(np.int32)).cuda(),
            torch.from_numpy(A.indices.astype(np.int32)).cuda())


def test_device_rcm_order_equals_host_order(cuda):
    from imate_b200.linear_operator import rcm_order, rcm_order_device
    R = sp.random(6000, 6000, density=0.0008, random_state=7, format="csr")
    S = sp.random(6000, 6000, density=0.0003, random_state=7, format="csr")
    N = sp.random(3000, 3000, density=0.002, random_state=8, format="csr")
    cases = [ib.correlation_matrix(40000, scale=0.01, shift=0.1, seed=2),
             sp.csr_matrix(R + R.T + sp.eye(6000)),   # connected
             sp.csr_matrix(S + S.T + sp.eye(6000)),   # 176 components
             sp.csr_matrix(S + S.T),                  # 169 empty rows
             sp.csr_matrix(N + sp.eye(3000)),         # not symmetric
             sp.csr_matrix((1, 1))]
    for A in cases:
        A = sp.csr_matrix(A)
        A.sort_indices()
        ip, ind = _device_pattern(A)
        got = rcm_order_device(ip, ind, A.shape[0], A.nnz,
                               max_components=A.shape[0])
        assert got is not None
        assert np.array_equal(got, rcm_order(A))


def test_device_rcm_order_declines_many_components(cuda):
    from imate_b200.linear_operator import rcm_order_device
    A = sp.csr_matrix(sp.block_diag([sp.eye(3) + sp.eye(3, k=1)
                                     for _ in range(100)]))
    ip, ind = _device_pattern(A)
    assert rcm_order_device(ip, ind, A.shape[0], A.nnz,
                            max_components=10) is None


def test_device_rcm_order_rejects_bad_pattern(cuda):
    import torch
    from imate_b200.linear_operator import rcm_order_device
    ip = torch.tensor([0, 1, 2], dtype=torch.int32, device="cuda")
    ind = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.SlqError):
        rcm_order_device(ip, ind, 2, 2)


def _general_b(n, seed):
    rng = np.random.default_rng(seed)
    R = sp.random(n, n, density=2.0 / n, random_state=rng, format="csr")
    return sp.csr_matrix(sp.diags(np.linspace(0.5, 2.0, n)) +
                         0.05 * (R + R.T))


@pytest.mark.parametrize("n,gram", [(500, False), (500, True),
                                    (20000, False)])
def test_affine_general_b_matches_reference(cuda, n, gram):
    # A + t B with B other than I: a Krylov sequence per t on every probe
    # (c_trace_estimator.cpp:496-556), here one device operator per t
    from oracle import ref
    A = ib.correlation_matrix(n, scale=0.05 if n < 1000 else 0.01,
                              shift=0.1, seed=1)
    B = _general_b(n, 7)
    t = [0.1, 1.0, 3.0]
    kw = dict(min_num_samples=6, max_num_samples=6, error_rtol=1e-8,
              lanczos_degree=20, orthogonalize=-1, seed=0)
    want = ref.trace_estimator_b(A, B, "log", t, gram=gram, **kw)
    F = ib.AffineMatrixFunction(A, B=B)
    tr, info = ib.logdet(F, parameters=t, gram=gram, method="slq", gpu=True,
                         return_info=True, **kw)
    got = np.asarray(info["convergence"]["samples"], float)
    assert got.shape == (6, 3)
    assert rel(got, want["samples"]) < 1e-9
    assert rel(tr, want["trace"]) < 1e-9
    assert list(info["convergence"]["num_samples_used"]) == \
        list(want["num_samples_used"])


def test_affine_general_b_float32_close_to_float64(cuda):
    A = ib.correlation_matrix(3000, scale=0.02, shift=0.1, seed=2)
    B = _general_b(3000, 3)
    kw = dict(min_num_samples=32, max_num_samples=32, error_rtol=1e-8,
              lanczos_degree=30, orthogonalize=-1, seed=1)
    t64, _ = ib.traceinv(ib.AffineMatrixFunction(A, B=B),
                         parameters=[0.2, 2.0], method="slq", gpu=True,
                         return_info=True, **kw)
    A32, B32 = A.astype(np.float32), B.astype(np.float32)
    t32, _ = ib.traceinv(ib.AffineMatrixFunction(A32, B=B32),
                         parameters=[0.2, 2.0], method="slq", gpu=True,
                         return_info=True, **kw)
    assert rel(t32, t64) < 1e-4


def test_edge_shapes_match_reference_library(cuda):
    """Shapes at the edges of the estimator against the reference CPU SLQ
    built from its sources, on identical probes: a 1 x 1 matrix, a Krylov
    degree above the order, empty rows and explicit zeros under A + t I (CSR
    and CSC), and a last probe block holding a single probe."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    kw = dict(error_rtol=0.0, seed=5)

    def both(fn, func, A, engine=None, **k):
        extra = {} if engine is None else {"engine": engine}
        tr, info = fn(A if not isinstance(A, tuple) else A[0], method="slq",
                      gpu=True, return_info=True, **dict(kw, **k), **extra)
        B = A if not isinstance(A, tuple) else A[1]
        want = ref.trace_estimator(B, func, **dict(kw, **k))
        return tr, info, want

    one = sp.csr_matrix(np.array([[2.5]]))
    tr, info, want = both(ib.logdet, "log", one, min_num_samples=4,
                          max_num_samples=4, lanczos_degree=10,
                          orthogonalize=0)
    assert rel(info["convergence"]["samples"][:4], want["samples"][:4, 0]) < 1e-12
    assert abs(float(tr) - np.log(2.5)) < 1e-12

    T = sp.diags([np.full(4, -1.0), np.full(5, 4.0), np.full(4, -1.0)],
                 [-1, 0, 1]).tocsr()
    tr, info, want = both(ib.logdet, "log", T, min_num_samples=7,
                          max_num_samples=7, lanczos_degree=20,
                          orthogonalize=-1)
    assert np.all(info["engine"]["lanczos_size"][:7] <= 5)
    assert rel(info["convergence"]["samples"][:7], want["samples"][:7, 0]) < 1e-9

    rng = np.random.default_rng(3)
    M = sp.random(60, 60, density=0.08, random_state=rng, format="csr")
    M = sp.csr_matrix(M @ M.T)
    keep = np.ones(60, bool)
    keep[rng.choice(60, 10, replace=False)] = False
    D = sp.diags(keep.astype(float))
    P = (D @ M @ D).tocoo()                 # 10 empty rows and columns
    # explicit stored zeros at symmetric pairs of empty positions
    dense = P.toarray()
    cand = [(i, j) for i in range(60) for j in range(i + 1, 60)
            if keep[i] and keep[j] and dense[i, j] == 0.0]
    pick = [cand[k] for k in rng.choice(len(cand), 20, replace=False)]
    zi = [i for i, j in pick] + [j for i, j in pick]
    zj = [j for i, j in pick] + [i for i, j in pick]
    P = sp.csr_matrix((np.r_[P.data, np.zeros(40)],
                       (np.r_[P.row, zi], np.r_[P.col, zj])), shape=(60, 60))
    assert P.nnz == np.count_nonzero(P.data) + 40
    assert np.allclose(P.toarray(), P.toarray().T)
    for fmt in ("csr", "csc"):
        Q = P.asformat(fmt)
        tr, info, want = both(ib.traceinv, "inv",
                              (ib.AffineMatrixFunction(Q), Q),
                              engine=ib.EngineOptions(block_size=32),
                              parameters=[0.5, 2.0], min_num_samples=33,
                              max_num_samples=33, lanczos_degree=15,
                              orthogonalize=-1)
        s = np.asarray(info["convergence"]["samples"]).reshape(33, -1)
        assert rel(s, want["samples"][:33]) < 1e-9
