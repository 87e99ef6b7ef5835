"""Batched SLQ plans (every estimate of a batch recorded into one CUDA graph)
and the SpMM autotuner.

Tolerances: a batched estimate runs the same kernels, in the same order, on
the same probes as slq_run on the same operator with the same SpMM choice,
so it must agree bit for bit (samples, estimates, errors, sample counts,
processed order); FP64 batched samples within 1e-10 relative of the oracle
(the reference restatement); the SpMM candidates' operator products are
bitwise equal to each other (their row sums run in one column order)."""

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import imate_b200 as ib
from imate_b200 import _lib
from imate_b200.batch import (BatchPlan, autotune, tune_operator, set_variant,
                              logdet_batch)
from oracle import oracle

pytestmark = pytest.mark.gpu

_FUNCS = {"logdet": ib.logdet, "traceinv": ib.traceinv, "trace": ib.trace}


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _single(est):
    e = dict(est)
    f = _FUNCS[e.pop("func")]
    A = e.pop("A")
    gram = e.pop("gram", False)
    p = e.pop("p", 1.0)
    return f(A, gram=gram, p=p, method="slq", gpu=True, return_info=True,
             **e)


def _same(got, want):
    tr, info = got
    wtr, winfo = want
    assert np.array_equal(np.atleast_1d(tr), np.atleast_1d(wtr))
    c, wc = info["convergence"], winfo["convergence"]
    assert np.array_equal(np.asarray(c["samples"]), np.asarray(wc["samples"]),
                          equal_nan=True)
    assert np.array_equal(np.atleast_1d(c["num_samples_used"]),
                          np.atleast_1d(wc["num_samples_used"]))
    assert np.array_equal(np.atleast_1d(c["num_outliers"]),
                          np.atleast_1d(wc["num_outliers"]))
    assert np.array_equal(np.atleast_1d(c["converged"]),
                          np.atleast_1d(wc["converged"]))
    assert np.array_equal(c["samples_processed_order"],
                          wc["samples_processed_order"])
    assert c["all_converged"] == wc["all_converged"]
    assert np.array_equal(np.atleast_1d(info["error"]["absolute_error"]),
                          np.atleast_1d(winfo["error"]["absolute_error"]))


def _mixed_estimates():
    T = ib.Matrix(ib.toeplitz(2.0, 1.0, 1500))
    C32 = ib.Matrix(ib.correlation_matrix(6000, scale=0.02, shift=0.2,
                                          seed=3, dtype=np.float32),
                    reorder=True, group_rows=8)
    C64 = ib.Matrix(ib.correlation_matrix(2500, scale=0.03, shift=0.2,
                                          seed=5), reorder=True)
    Af = ib.AffineMatrixFunction(ib.correlation_matrix(3000, scale=0.02,
                                                       shift=0.2, seed=8))
    X = sp.random(900, 300, density=0.03, random_state=4, format="csc")
    X = (X + sp.eye(900, 300) * 0.8).tocsc()
    return [
        dict(func="logdet", A=T, gram=True, min_num_samples=10,
             max_num_samples=70, error_rtol=1e-3, lanczos_degree=20,
             orthogonalize=0, seed=0),
        dict(func="logdet", A=C32, min_num_samples=256, max_num_samples=256,
             error_rtol=0.0, lanczos_degree=16, orthogonalize=-1, seed=4),
        dict(func="traceinv", A=C64, min_num_samples=8, max_num_samples=100,
             error_rtol=2e-3, lanczos_degree=18, orthogonalize=-1, seed=2),
        dict(func="logdet", A=Af, parameters=[0.0, 0.5, 2.0],
             min_num_samples=12, max_num_samples=40, error_rtol=1e-2,
             lanczos_degree=15, orthogonalize=4, seed=9),
        dict(func="trace", A=C64, p=2.0, min_num_samples=10,
             max_num_samples=33, error_rtol=1e-2, lanczos_degree=12,
             orthogonalize=0, seed=6),
        dict(func="logdet", A=X, gram=True, min_num_samples=10,
             max_num_samples=48, error_rtol=1e-3, lanczos_degree=20,
             orthogonalize=-1, seed=5),
    ]


def test_batch_equals_single_calls(cuda):
    ests = _mixed_estimates()
    plan = BatchPlan(ests, autotune=False)
    assert plan.graph_kernels > 0
    got = plan.run()
    for est, g in zip(ests, got):
        _same(g, _single(est))
        assert g[1]["engine"]["batch"]["estimates"] == len(ests)
    # a second launch of the same graph gives the same answers
    again = plan.run()
    for g, h in zip(got, again):
        _same(h, g)


def test_batch_of_many_sizes_equals_single_calls(cuda):
    rng = np.random.default_rng(11)
    ests = []
    for i in range(12):
        n = int(rng.integers(300, 5000))
        A = ib.correlation_matrix(n, scale=float(rng.uniform(0.01, 0.05)),
                                  shift=0.2, seed=100 + i,
                                  dtype=np.float32 if i % 2 else np.float64)
        ests.append(dict(func="logdet", A=ib.Matrix(A), min_num_samples=32,
                         max_num_samples=int(rng.integers(32, 160)),
                         error_rtol=1e-3, lanczos_degree=int(rng.integers(8, 30)),
                         orthogonalize=int(rng.choice([0, -1])), seed=i))
    got = BatchPlan(ests, autotune=False).run()
    for est, g in zip(ests, got):
        _same(g, _single(est))


@pytest.mark.parametrize("gram", [False, True])
def test_batch_matches_oracle(cuda, gram):
    A = ib.correlation_matrix(1500, scale=0.03, shift=0.2, seed=21)
    kw = dict(min_num_samples=5, max_num_samples=45, error_rtol=1e-9,
              lanczos_degree=14, orthogonalize=-1, seed=13)
    (tr, info), = BatchPlan([dict(func="logdet", A=A, gram=gram, **kw)],
                            autotune=False).run()
    want = oracle.trace_estimator(A, "log", gram=gram, **kw)
    used = int(want["num_samples_used"][0])
    assert info["convergence"]["num_samples_used"] == used
    assert rel(info["convergence"]["samples"][:used],
               want["samples"][:used, 0]) < 1e-10
    assert rel(tr, want["trace"][0]) < 1e-10


def _dot(op, x, transpose=False):
    import torch
    return op.dot(torch.from_numpy(x).cuda(), transpose=transpose).cpu() \
        .numpy()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tuned_candidates_give_identical_products(cuda, dtype):
    A = ib.correlation_matrix(7000, scale=0.02, shift=0.1, seed=7,
                              dtype=dtype)
    M = ib.Matrix(A, reorder=True, group_rows=8)
    op = M.get_device_operator(need_transpose=True)
    widths = (32, 64) if dtype == np.float64 else (32, 64, 128, 256)
    for w in widths:
        x = np.random.default_rng(w).standard_normal((7000, w)).astype(dtype)
        for tr in (False, True):
            set_variant(op, w, -1, transpose=tr)
            base = _dot(op, x, transpose=tr)
            cands, chosen = tune_operator(op, w, transpose=tr, reps=2)
            assert 0 <= chosen < len(cands)
            assert cands[chosen]["ms"] == min(c["ms"] for c in cands)
            kinds = {c["kind"] for c in cands}
            assert "csr" in kinds and "row-group" in kinds
            if dtype == np.float32 and w in (128, 256):
                assert "row-group-tma" in kinds
            for i, c in enumerate(cands):
                if c["kind"] == "row-group-tma":
                    continue  # runs only with the estimator's tensor maps
                set_variant(op, w, i, transpose=tr)
                assert np.array_equal(_dot(op, x, transpose=tr), base), \
                    (w, tr, c)
            set_variant(op, w, -1, transpose=tr)
            want = (A.T if tr else A).astype(np.float64) @ \
                x.astype(np.float64)
            tol = 1e-12 if dtype == np.float64 else 2e-5
            assert np.max(np.abs(base - want)) <= tol * np.max(np.abs(want))


def test_autotuned_estimator_agrees_with_builtin(cuda):
    A = ib.correlation_matrix(20000, scale=0.01, shift=0.1, seed=3,
                              dtype=np.float32)
    kw = dict(min_num_samples=512, max_num_samples=512, error_rtol=0.0,
              lanczos_degree=20, orthogonalize=0, seed=1)
    M0 = ib.Matrix(A, reorder=True, group_rows=8)
    M1 = ib.Matrix(A, reorder=True, group_rows=8)
    (t0, i0), = BatchPlan([dict(func="logdet", A=M0, **kw)],
                          autotune=False).run()
    plan = BatchPlan([dict(func="logdet", A=M1, **kw)], autotune=True)
    (t1, i1), = plan.run()
    width = plan.tuning[0]["width"]
    assert width in (32, 64, 128, 256, 512)
    assert i1["engine"]["block_size"] == width
    # same probes, different block widths and SpMM tiles: FP32 products
    # and FP64 reductions agree to well below the Monte-Carlo error
    assert rel(i1["convergence"]["samples"], i0["convergence"]["samples"]) \
        < 1e-4
    assert abs(t1 - t0) / abs(t0) < 1e-6


def test_autotune_report(cuda):
    A = ib.correlation_matrix(9000, scale=0.02, shift=0.1, seed=2,
                              dtype=np.float32)
    op = ib.Matrix(A, reorder=True, group_rows=8).get_device_operator()
    width, report = autotune(op, 300, reps=2)
    assert width in report
    assert set(report) == {32, 64, 128, 256, 512}
    costs = {w: r["cost_ms_per_step"] for w, r in report.items()}
    assert costs[width] == min(costs.values())


def test_logdet_batch_convenience(cuda):
    mats = [ib.correlation_matrix(n, scale=0.03, shift=0.2, seed=n)
            for n in (800, 1600, 2400)]
    kw = dict(min_num_samples=20, max_num_samples=20, lanczos_degree=20,
              orthogonalize=-1, seed=3)
    vals = logdet_batch(mats, gpu=True, autotune=False, **kw)
    out = logdet_batch(mats, gpu=True, autotune=False, return_info=True,
                       **kw)
    for A, v, (v2, info) in zip(mats, vals, out):
        assert v == v2
        assert v == ib.logdet(A, method="slq", gpu=True, **kw)
        # Monte-Carlo error: within 4x the estimate's own 95% error bound
        exact = np.linalg.slogdet(A.toarray())[1]
        assert abs(v - exact) < 4.0 * info["error"]["absolute_error"]


def test_batch_argument_errors(cuda):
    import torch
    lib = _lib.load()
    A = ib.Matrix(ib.correlation_matrix(1000, scale=0.03, shift=0.2, seed=1))
    op = A.get_device_operator()
    prm = _lib.SlqParams(func=0, gram=0, exponent=1.0, orthogonalize=0,
                         seed=0, lanczos_degree=10, lanczos_tol=1e-15,
                         min_num_samples=4, max_num_samples=8, error_atol=0,
                         error_rtol=1e-2, confidence_level=0.95,
                         outlier_significance_level=0.001, block_size=0,
                         rng=0, first_probe=0)
    ops = (ctypes.c_void_p * 1)(op.handle.value)
    prms = (_lib.SlqParams * 1)(prm)
    nq = (ctypes.c_int * 1)(1)
    nb = ctypes.c_size_t(0)
    _lib.check(lib.slq_batch_workspace_bytes(1, ops, prms, nq,
                                             ctypes.byref(nb)))
    small = torch.empty(1024, dtype=torch.uint8, device="cuda")
    h = ctypes.c_void_p(None)
    st = lib.slq_batch_create(1, ops, prms, None, nq, small.data_ptr(),
                              small.numel(), None, ctypes.byref(h))
    assert st == 3 and not h.value  # SLQ_ERR_WORKSPACE
    assert lib.slq_operator_set_variant(op.handle, 64, 0, 15) == 1
    assert lib.slq_operator_set_variant(op.handle, 48, 0, 0) == 1


def test_device_built_correlation_matrix(cuda):
    # the device builder gives the host builder's matrix in cell order
    from imate_b200.sample_matrices import (correlation_matrix,
                                            correlation_matrix_device,
                                            correlation_points)
    pts = correlation_points(6000, 2, 17)
    A = correlation_matrix(points=pts, scale=0.03, threshold=0.05, shift=0.1)
    ip, ind, dat, perm = correlation_matrix_device(
        points=pts, scale=0.03, threshold=0.05, shift=0.1, dtype="float64",
        max_candidates=200000)
    B = sp.csr_matrix((dat.cpu().numpy(), ind.cpu().numpy(),
                       ip.cpu().numpy()), shape=A.shape)
    p = perm.cpu().numpy()
    Ap = A[p][:, p].tocsr()
    Ap.sort_indices()
    assert np.array_equal(Ap.indptr, B.indptr)
    assert np.array_equal(Ap.indices, B.indices)
    assert np.max(np.abs(Ap.data - B.data)) < 1e-15
    # an operator over the device arrays equals one uploaded from the host
    D = ib.DeviceMatrix(ip, ind, dat, A.shape, group_rows=8)
    H = ib.Matrix(B, reorder=False, group_rows=8, aggregate=False)
    kw = dict(method="slq", gpu=True, return_info=True, min_num_samples=64,
              max_num_samples=64, error_rtol=0.0, lanczos_degree=20,
              orthogonalize=-1, seed=3)
    td, idv = ib.logdet(D, **kw)
    th, ih = ib.logdet(H, **kw)
    assert np.array_equal(idv["convergence"]["samples"],
                          ih["convergence"]["samples"])
    assert td == th


def test_batch_packed_over_two_logical_devices_equals_one_device(cuda):
    """Estimates packed over two devices (both mapped onto this GPU, one
    host thread per device graph) give the one-graph answers bit for bit."""
    import torch
    ests = _mixed_estimates()
    one = BatchPlan(ests, autotune=False, num_gpu_devices=1)
    assert len(one.plans) == 1
    want = one.run()
    two = BatchPlan(ests, autotune=False, num_gpu_devices=2,
                    device_of=lambda d: torch.cuda.current_device())
    assert sorted(set(two.assignment)) == [0, 1]
    assert len(two.plans) == 2
    got = two.run()
    for g, w in zip(got, want):
        _same(g, w)
    devs = {g[1]["engine"]["batch"]["device"] for g in got}
    assert devs == {torch.cuda.current_device()}
    assert sum(p.graph_kernels for p in two.plans) == two.graph_kernels
    # 0 = every visible device; on one GPU that is one graph
    if torch.cuda.device_count() == 1:
        assert len(BatchPlan(ests[:2], autotune=False,
                             num_gpu_devices=0).plans) == 1
