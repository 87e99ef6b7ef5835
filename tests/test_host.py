"""Host logic that needs no GPU: the C-ABI library loads and exports every
symbol include/slq.h declares, its host-side statistics and probe-stream
jump-ahead agree with the oracle, and the Python host mirrors imate's
argument checks."""

import ctypes
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

import imate_b200 as ib
from imate_b200 import _lib, _build
from imate_b200._trace_estimator import check_arguments, get_operator, \
    find_num_inquiries, get_operator_parameters
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    _build.build()
    return _lib.load()


def header_symbols():
    text = open(os.path.join(ROOT, "include", "slq.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(slq_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lib):
    names = header_symbols()
    assert len(names) >= 16
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTS)
    assert lib.slq_abi_version() == _lib.ABI_VERSION


def test_erfinv_matches_oracle(lib):
    for x in np.linspace(-0.999, 0.999, 41):
        assert abs(lib.slq_erfinv(float(x)) - oracle.erfinv(float(x))) < 1e-15


def _conv_c(lib, samples, order, nproc, min_s, conf, atol, rtol, conv):
    q = samples.shape[1]
    err = np.zeros(q)
    used = np.zeros(q, np.int32)
    conv = conv.astype(np.int32).copy()
    a = lib.slq_check_convergence(
        samples.ctypes.data, q, min_s, order.ctypes.data, nproc, conf, atol,
        rtol, err.ctypes.data, used.ctypes.data, conv.ctypes.data)
    return bool(a), err, used, conv


@pytest.mark.parametrize("q", [1, 3])
def test_convergence_and_average_match_oracle(lib, q):
    rng = np.random.default_rng(4)
    max_s = 60
    samples = np.ascontiguousarray(rng.normal(100, 3, (max_s, q)))
    samples[7, 0] += 80.0  # an outlier
    order = np.arange(max_s, dtype=np.int32)
    conv_c = np.zeros(q, np.int32)
    conv_o = np.zeros(q, np.int32)
    for nproc in range(1, max_s + 1):
        a1, e1, u1, conv_c = _conv_c(lib, samples, order, nproc, 10, 0.95,
                                     0.0, 1e-3, conv_c)
        a2, e2, u2, conv_o = oracle.check_convergence(
            samples, order, nproc, 10, 0.95, 0.0, 1e-3, conv_o)
        assert a1 == a2
        np.testing.assert_array_equal(u1, u2)
        np.testing.assert_array_equal(conv_c, conv_o)
        np.testing.assert_allclose(e1, e2, rtol=1e-14)
    used = np.full(q, max_s, np.int32)
    outl = np.zeros(q, np.int32)
    tr = np.zeros(q)
    er = np.zeros(q)
    lib.slq_average_estimates(0.95, 0.001, q, max_s, used.ctypes.data,
                              order.ctypes.data, samples.ctypes.data,
                              outl.ctypes.data, tr.ctypes.data, er.ctypes.data)
    ol = oracle.load()
    outl2 = np.zeros(q, np.int32)
    tr2 = np.zeros(q)
    er2 = np.zeros(q)
    ol.oracle_average_estimates.argtypes = [ctypes.c_double, ctypes.c_double] \
        + [ctypes.c_int] * 2 + [ctypes.c_void_p] * 6
    ol.oracle_average_estimates(0.95, 0.001, q, max_s, used.ctypes.data,
                                order.ctypes.data, samples.ctypes.data,
                                outl2.ctypes.data, tr2.ctypes.data,
                                er2.ctypes.data)
    np.testing.assert_array_equal(outl, outl2)
    assert outl[0] >= 1
    np.testing.assert_allclose(tr, tr2, rtol=1e-15)
    np.testing.assert_allclose(er, er2, rtol=1e-14)


@pytest.mark.parametrize("k", [1, 100, 511, 512, 4097, 123457])
def test_jump_ahead_matches_sequential_stream(lib, k):
    words = oracle.stream_words(0, k + 2)
    # state after the seeding jump is not exposed by the oracle; compare the
    # engine's jump against stepping its own generator instead
    s = (ctypes.c_uint64 * 4)(0x1234, 0x5678, 0x9abc, 0xdef0)
    t = (ctypes.c_uint64 * 4)(*s)
    lib.slq_xoshiro_jump_ahead(s, k)
    for _ in range(k):
        lib.slq_xoshiro_jump_ahead(t, 1)
    assert list(s) == list(t)
    assert words.size == k + 2


def test_argument_checks_mirror_reference():
    ok = dict(gram=False, exponent=1.0, min_num_samples=10,
              max_num_samples=50, error_atol=None, error_rtol=1e-2,
              confidence_level=0.95, outlier_significance_level=0.001,
              lanczos_degree=20, lanczos_tol=None, orthogonalize=0,
              seed=None, num_threads=0, num_gpu_devices=0, verbose=False,
              plot=False, gpu=True)
    assert check_arguments(**ok) == (0.0, 1e-2)
    bad = [
        (dict(gram=1), TypeError),
        (dict(min_num_samples=0), ValueError),
        (dict(max_num_samples=1.5), TypeError),
        (dict(min_num_samples=60), ValueError),
        (dict(error_rtol=-1.0), ValueError),
        (dict(confidence_level=1.5), ValueError),
        (dict(outlier_significance_level=0.2), ValueError),
        (dict(lanczos_degree=0), ValueError),
        (dict(lanczos_tol=-1.0), ValueError),
        (dict(orthogonalize=21), ValueError),
        (dict(orthogonalize=1.0), TypeError),
        (dict(seed=1.5), TypeError),
        (dict(num_threads=-1), ValueError),
        (dict(gpu="yes"), TypeError),
    ]
    for change, exc in bad:
        kw = dict(ok)
        kw.update(change)
        with pytest.raises(exc):
            check_arguments(**kw)


def test_operator_and_parameter_checks():
    A = sp.random(5, 4, density=0.5, format="csr")
    with pytest.raises(ValueError):
        get_operator(A, gram=False)
    assert get_operator(A, gram=True).get_num_rows() == 5
    with pytest.raises(TypeError):
        get_operator([[1, 2], [3, 4]], gram=False)
    Aop = ib.AffineMatrixFunction(sp.eye(4, format="csr"))
    assert find_num_inquiries(Aop, 3) == 3
    with pytest.raises(ValueError):
        find_num_inquiries(Aop, 0)
    p, k = get_operator_parameters([1.0, 2.0], "float64")
    assert k == 2 and p.dtype == np.float64
    with pytest.raises(ValueError):
        get_operator_parameters(np.ones((2, 2)), "float64")
    F = ib.AffineMatrixFunction(sp.eye(4, format="csr"),
                                B=2 * sp.eye(4, format="csr"))
    assert F.general_B and not F._affine()
    assert find_num_inquiries(F, 2) == 2
    with pytest.raises(ValueError):
        ib.AffineMatrixFunction(sp.eye(4, format="csr"),
                                B=sp.eye(5, format="csr"))
    with pytest.raises(TypeError):
        ib.AffineMatrixFunction(sp.eye(4, format="csr"), B=2.0)


def test_affine_general_b_union_pattern(lib):
    # A + t B with B other than I: one CSR pattern holding both, A's and B's
    # values on it (zeros where a matrix lacks an entry)
    rng = np.random.default_rng(5)
    for n, m in ((50, 50), (300, 300)):
        A = sp.random(n, m, density=0.05, random_state=rng, format="csr")
        B = sp.random(n, m, density=0.03, random_state=rng, format="csc")
        F = ib.AffineMatrixFunction(A, B=B)
        U = F._union_pattern()
        P = sp.csr_matrix((np.ones(U["indices"].size), U["indices"],
                           U["indptr"]), shape=(n, m))
        Au = sp.csr_matrix((U["a"], U["indices"], U["indptr"]), shape=(n, m))
        Bu = sp.csr_matrix((U["b"], U["indices"], U["indptr"]), shape=(n, m))
        assert abs(Au - A).max() == 0 and abs(Bu - B).max() == 0
        assert P.nnz == (abs(A) + abs(B)).nnz
        assert U["G"] in (0, 4, 8, 16)


def test_non_slq_methods_and_cpu_path_are_refused():
    A = ib.toeplitz(2.0, 1.0, 8)
    with pytest.raises(NotImplementedError):
        ib.logdet(A)  # imate's default method is cholesky
    with pytest.raises(ValueError):
        ib.logdet(A, method="slq", gpu=False)


def test_toeplitz_formulas():
    for n in (5, 50, 300):
        A = ib.toeplitz(2.0, 1.0, n, gram=True).toarray()
        assert abs(np.linalg.slogdet(A)[1] - ib.toeplitz_logdet(2, 1, n, True)) < 1e-9
        assert abs(np.trace(A) - ib.toeplitz_trace(2, 1, n, True)) < 1e-9
        ti = np.trace(np.linalg.inv(A))
        assert abs(ti - ib.toeplitz_traceinv(2, 1, n, True)) / ti < (1e-9 if n < 200 else 1e-3)


def test_correlation_matrix_matches_brute_force():
    pts = np.random.default_rng(0).random((300, 2))
    A = ib.correlation_matrix(points=pts, scale=0.05, threshold=0.05,
                              shift=1e-3).toarray()
    r = np.linalg.norm(pts[:, None, :] - pts[None, :, :], axis=2)
    K = np.exp(-r / 0.05)
    K[K < 0.05] = 0.0
    K += 1e-3 * np.eye(300)
    np.testing.assert_allclose(A, K, rtol=1e-14, atol=1e-15)


def test_batch_and_tuner_reject_bad_arguments_without_a_gpu(lib):
    nb = ctypes.c_size_t(0)
    # argument checks come before any CUDA call
    assert lib.slq_batch_workspace_bytes(0, None, None, None,
                                         ctypes.byref(nb)) == 1
    assert lib.slq_batch_create(0, None, None, None, None, None, 0, None,
                                None) == 1
    assert lib.slq_batch_run(None, None, None) == 1
    assert lib.slq_batch_info(None, None, None) == 1
    assert lib.slq_batch_destroy(None) == 0
    assert lib.slq_operator_set_variant(None, 64, 0, 0) == 1
    assert lib.slq_operator_tune_workspace_bytes(None, 64,
                                                 ctypes.byref(nb)) == 1


def test_consumer_argument_checks(corr_small):
    # imate's checks of trlinfrac / eigencount / density arguments
    # (*/_slq_method.pyx check_arguments) run before any device work
    with pytest.raises(ValueError):
        ib.trlinfrac(corr_small, coeff=[1.0, 2.0, 2.0, 4.0], method="slq",
                     gpu=True)
    with pytest.raises(ValueError):
        ib.eigencount(corr_small, interval=[0.0], method="slq", gpu=True)
    with pytest.raises(ValueError):
        ib.density(corr_small, sigma=0.0, method="slq", gpu=True)
    with pytest.raises(NotImplementedError):
        ib.trexp(corr_small, method="eigenvalue")


def test_group_order_is_an_aligned_permutation_that_raises_fill(lib):
    from imate_b200.linear_operator import (group_order, _group_fill,
                                            locality_order)
    A = ib.correlation_matrix(20000, scale=0.01, threshold=0.05, shift=0.1,
                              seed=4)
    base = locality_order(A, True)
    for G in (8, 16):
        order = group_order(A, base, G)
        assert np.array_equal(np.sort(order), np.arange(A.shape[0]))
        # groups are seeds with their neighbours: every group's rows are
        # adjacent to the seed or reached through it
        assert _group_fill(A, order, G) > 1.3 * _group_fill(A, base, G)
        assert np.array_equal(order, group_order(A, base, G))  # deterministic
    # identity base order
    order = group_order(A, None, 8)
    assert np.array_equal(np.sort(order), np.arange(A.shape[0]))


def test_group_order_rejects_bad_input(lib):
    n = 4
    ip = np.array([0, 1, 2, 3, 4], np.int32)
    ind = np.array([0, 1, 2, 5], np.int32)
    out = np.empty(n, np.int32)
    st = lib.slq_group_order(n, ip.ctypes.data, ind.ctypes.data, None, 0, 2,
                             None, out.ctypes.data)
    assert st == 2  # index out of range
    ind = np.array([0, 1, 2, 3], np.int32)
    bad = np.array([0, 0, 1, 2], np.int32)
    st = lib.slq_group_order(n, ip.ctypes.data, ind.ctypes.data, None, 0, 2,
                             bad.ctypes.data, out.ctypes.data)
    assert st == 1  # base order not a permutation
    st = lib.slq_group_order(n, ip.ctypes.data, ind.ctypes.data, None, 0, 2,
                             None, out.ctypes.data)
    assert st == 0 and sorted(out) == [0, 1, 2, 3]


def test_rcm_order_is_a_bandwidth_reducing_permutation(lib):
    from imate_b200.linear_operator import rcm_order
    from scipy.sparse.csgraph import reverse_cuthill_mckee

    def spread(A, perm):
        inv = np.empty(A.shape[0], np.int64)
        inv[perm] = np.arange(A.shape[0])
        ri = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
        return float(np.mean(np.abs(inv[A.indices] - inv[ri])))

    R = sp.random(4000, 4000, density=0.001, random_state=5, format="csr")
    cases = [ib.correlation_matrix(20000, scale=0.01, shift=0.1, seed=2),
             ib.correlation_matrix(3000, scale=0.02, shift=0.1, seed=1),
             sp.csr_matrix(R + R.T + sp.eye(4000))]
    for A in cases:
        perm = rcm_order(A)
        assert np.array_equal(np.sort(perm), np.arange(A.shape[0]))
        ident = np.arange(A.shape[0])
        ours = spread(A, perm)
        assert ours < spread(A, ident)
        ref = spread(A, reverse_cuthill_mckee(A, symmetric_mode=True))
        assert ours <= 1.1 * ref


def _np_group_fill(A, order, G, sample=256):
    """numpy restatement of the sampled group fill (slq_group_fill)."""
    n = A.shape[0]
    ngroups = n // G
    picks = np.unique(np.linspace(0, ngroups - 1,
                                  min(sample, ngroups)).astype(np.int64))
    rows = np.asarray(order)[(picks[:, None] * G +
                              np.arange(G)[None, :]).ravel()]
    S = A[rows]
    grp = np.repeat(np.repeat(np.arange(picks.size), G), np.diff(S.indptr))
    keys = grp.astype(np.int64) * A.shape[1] + S.indices
    union = np.bincount(np.unique(keys) // A.shape[1], minlength=picks.size)
    nnz = np.bincount(grp, minlength=picks.size)
    ok = union > 0
    return float(np.mean(nnz[ok] / (G * union[ok])))


def _np_spread(A, perm=None, sample=20000):
    """numpy restatement of the sampled order spread (slq_order_spread)."""
    n = A.shape[0]
    rows = np.unique(np.linspace(0, n - 1, min(n, sample)).astype(np.int64))
    S = A[rows]
    ri = np.repeat(rows, np.diff(S.indptr))
    cols = S.indices.astype(np.int64)
    if perm is None:
        return float(np.mean(np.abs(cols - ri)))
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    return float(np.mean(np.abs(inv[cols] - inv[ri])))


def test_order_statistics_match_numpy(lib):
    from imate_b200.linear_operator import (_group_fill, order_spread,
                                            rcm_order)
    R = sp.random(5000, 5000, density=0.002, random_state=3, format="csr")
    cases = [ib.correlation_matrix(20000, scale=0.01, shift=0.1, seed=2),
             sp.csr_matrix(R + R.T + sp.eye(5000))]
    for A in cases:
        A = sp.csr_matrix(A)
        perm = rcm_order(A)
        for G in (4, 8, 16):
            for order in (perm, np.arange(A.shape[0], dtype=np.int32)):
                assert abs(_group_fill(A, order, G) -
                           _np_group_fill(A, order, G)) < 1e-12
        assert abs(order_spread(A) - _np_spread(A)) < 1e-9 * _np_spread(A)
        assert abs(order_spread(A, perm) - _np_spread(A, perm)) < \
            1e-9 * _np_spread(A, perm)


def test_group_order_segment_sweeps_keep_groups_compact(lib):
    # large orders: one sweep per segment of n / 8 base positions,
    # each group drawn from one segment; the result does not depend on
    # timing or on the number of threads
    from imate_b200.linear_operator import group_order, rcm_order
    A = sp.csr_matrix(ib.correlation_matrix(262144, scale=0.005, threshold=0.05,
                                            shift=0.1, seed=1, dtype="float32"))
    n, G = A.shape[0], 16
    base = rcm_order(A)
    order = group_order(A, base, G)
    assert np.array_equal(np.sort(order), np.arange(n))
    for _ in range(2):
        assert np.array_equal(order, group_order(A, base, G))
    pos = np.empty(n, np.int64)
    pos[base] = np.arange(n)
    segment = pos[order].reshape(-1, G) // (n // 8)
    # every group but the merged short ones at the end lies in one segment,
    # and the groups follow the base order segment by segment
    assert np.all(segment[:-8] == segment[:-8, :1])
    assert np.all(np.diff(segment[:-8, 0]) >= 0)
    # whole-matrix fill of the 16-row groups, and no group far beyond it
    B = A[order]
    rows = np.repeat(np.arange(n), np.diff(B.indptr))
    union = np.bincount(np.unique((rows // G).astype(np.int64) * n + B.indices)
                        // n, minlength=n // G)
    assert A.nnz / (G * union.sum()) > 0.625
    # the groups filled from scattered leftover rows at a sweep's end are
    # few
    assert np.sum(union > 1.5 * np.median(union)) < 0.01 * union.size


def _block_unions(A, order, rows):
    B = A[order]
    n = A.shape[0]
    r = np.repeat(np.arange(n), np.diff(B.indptr))
    return np.bincount(np.unique((r // rows).astype(np.int64) * n + B.indices)
                       // n, minlength=n // rows)


def test_block_order_keeps_groups_and_shrinks_block_unions(lib):
    # blocks of 8 whole 16-row groups with overlapping column sets: a
    # permutation, every group of group_order kept whole, deterministic, and
    # 128-row blocks with far smaller column unions than 128 consecutive rows
    from imate_b200.linear_operator import (block_order, group_order,
                                            rcm_order)
    A = sp.csr_matrix(ib.correlation_matrix(40000, scale=0.01, threshold=0.05,
                                            shift=0.1, seed=4,
                                            dtype="float32"))
    n, G, B = A.shape[0], 16, 8
    go = group_order(A, rcm_order(A), G)
    bo = block_order(A, go, G, B)
    assert np.array_equal(np.sort(bo), np.arange(n))
    assert np.array_equal(bo, block_order(A, go, G, B))
    groups = {tuple(sorted(go[i * G:(i + 1) * G])) for i in range(n // G)}
    assert {tuple(sorted(bo[i * G:(i + 1) * G])) for i in range(n // G)} \
        == groups
    before = _block_unions(A, go, G * B)[:n // (G * B)]
    after = _block_unions(A, bo, G * B)[:n // (G * B)]
    assert after.mean() < 0.6 * before.mean()


def test_block_order_rejects_bad_input(lib):
    n = 8
    ip = np.arange(n + 1, dtype=np.int32)
    ind = np.arange(n, dtype=np.int32)
    out = np.empty(n, np.int32)
    bad = np.array([0, 0, 1, 2, 3, 4, 5, 6], np.int32)
    assert lib.slq_block_order(n, ip.ctypes.data, ind.ctypes.data,
                               bad.ctypes.data, 2, 2, out.ctypes.data) == 1
    good = np.arange(n, dtype=np.int32)[::-1].copy()
    assert lib.slq_block_order(n, ip.ctypes.data, ind.ctypes.data,
                               good.ctypes.data, 0, 2, out.ctypes.data) == 1
    ind2 = ind.copy()
    ind2[3] = 99
    assert lib.slq_block_order(n, ip.ctypes.data, ind2.ctypes.data,
                               good.ctypes.data, 2, 2, out.ctypes.data) == 2
    # diagonal pattern: no group shares a column, blocks follow the order
    assert lib.slq_block_order(n, ip.ctypes.data, ind.ctypes.data,
                               good.ctypes.data, 2, 2, out.ctypes.data) == 0
    assert np.array_equal(out, good)


def test_block_group_order_nests_groups_in_blocks(lib):
    # 128-row blocks aggregated around seeds, each split into eight 16-row
    # groups from its own rows: a deterministic permutation whose blocks
    # have small column unions and whose groups fill well
    from imate_b200.linear_operator import (block_group_order, rcm_order,
                                            _group_fill)
    A = sp.csr_matrix(ib.correlation_matrix(40000, scale=0.01, threshold=0.05,
                                            shift=0.1, seed=4,
                                            dtype="float32"))
    n = A.shape[0]
    base = rcm_order(A)
    order = block_group_order(A, base, 128, 16)
    assert np.array_equal(np.sort(order), np.arange(n))
    assert np.array_equal(order, block_group_order(A, base, 128, 16))
    whole = (n // 128) * 128
    blk = _block_unions(A, order, 128)[:n // 128]
    consecutive = _block_unions(A, base, 128)[:n // 128]
    assert blk.mean() < 0.5 * consecutive.mean()
    assert _group_fill(A, order, 16) > 1.3 * _group_fill(A, base, 16)
    # rows after the last whole block keep their aggregation order
    assert whole <= n
    with pytest.raises(_lib.SlqError):
        block_group_order(A, base, 100, 16)  # not a multiple


@pytest.mark.parametrize("bad_col", [-1, 40000, 2 ** 31 - 1])
@pytest.mark.parametrize("where", ["first", "middle", "last"])
def test_block_group_order_rejects_out_of_range_columns(lib, bad_col, where):
    # the index check runs beside the aggregation sweeps (2 sweeps for
    # n = 40000 leave the other pool threads to it) or before them; either
    # way one bad column anywhere makes the call fail, and the sweeps never
    # index with it
    A = sp.csr_matrix(ib.correlation_matrix(40000, scale=0.01, threshold=0.05,
                                            shift=0.1, seed=4,
                                            dtype="float32"))
    n = A.shape[0]
    ip = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ind = np.ascontiguousarray(A.indices, dtype=np.int32).copy()
    data = np.ascontiguousarray(A.data)
    k = {"first": 0, "middle": ind.size // 2, "last": ind.size - 1}[where]
    ind[k] = bad_col
    out = np.empty(n, np.int32)
    for fn, args in ((lib.slq_block_group_order, (128, 16)),
                     (lib.slq_group_order, (16,))):
        st = fn(n, ip.ctypes.data, ind.ctypes.data, data.ctypes.data,
                _lib.SLQ_F32, *args, None, out.ctypes.data)
        assert st == 2  # SLQ_ERR_BAD_CSR
        assert b"out of range" in lib.slq_last_error()
