"""The oracle (oracle/slq_oracle.c) pinned against the reference's own
outputs: golden fixtures made by tests/golden/make_golden.py from the
reference's CPU SLQ, and -- where oracle/_ref is built -- the reference
library run side by side."""

import numpy as np
import pytest

from imate_b200.sample_matrices import toeplitz
from golden_cases import FUNC_CASES, FUNC_SETTINGS
from oracle import oracle, ref


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


def test_rng_stream_bits(golden):
    g = golden("rng.npz")
    for seed in (0, 1, 7, 123456789):
        bits = np.unpackbits(g["bits_seed%d" % seed], bitorder="little")
        n = 64 * 299 + 63
        v = oracle.random_probes(seed, n, 1)[0]
        assert np.array_equal((v > 0).astype(np.uint8), bits[:n])


@pytest.mark.parametrize("seed,n", [(0, 1), (0, 63), (0, 64), (0, 65),
                                    (3, 1000), (5, 4097)])
def test_rng_probes(golden, seed, n):
    g = golden("rng.npz")
    want = g["probes_seed%d_n%d" % (seed, n)]
    got = (oracle.random_probes(seed, n, want.shape[0]) > 0).astype(np.int8)
    assert np.array_equal(got, want)


def test_stream_words_consistent_with_probes():
    # word w of the stream gives probe elements 64w .. 64w+63
    w = oracle.stream_words(0, 3)
    v = oracle.random_probes(0, 64 * 3 - 1, 1)[0]
    for k in range(3):
        bits = [(int(w[k]) >> j) & 1 for j in range(64)]
        seg = v[64 * k:64 * k + 64]
        assert [int(x > 0) for x in seg] == bits[:len(seg)]


@pytest.mark.parametrize("orth", [0, -1, 10])
def test_golub_kahn_alpha_beta(golden, orth):
    g = golden("krylov.npz")
    n = 16384
    B = toeplitz(2.0, 1.0, n)
    probes = oracle.random_probes(0, n, 4)
    for p in range(4):
        key = "c1_orth%d_p%d" % (orth, p)
        a, b = oracle.krylov(B, probes[p], 30, gram=True, orthogonalize=orth)
        assert rel(a, g[key + "_alpha"]) < 1e-12
        assert rel(b, g[key + "_beta"]) < 1e-12


@pytest.mark.parametrize("orth", [0, -1, 1, 5])
def test_lanczos_alpha_beta(golden, corr_small, orth):
    g = golden("krylov.npz")
    probes = oracle.random_probes(5, corr_small.shape[0], 4)
    for p in range(4):
        key = "corr_orth%d_p%d" % (orth, p)
        a, b = oracle.krylov(corr_small, probes[p], 20, orthogonalize=orth)
        assert rel(a, g[key + "_alpha"]) < 1e-10
        assert rel(b, g[key + "_beta"]) < 1e-10


def test_affine_lanczos(golden, corr_small):
    g = golden("krylov.npz")
    probes = oracle.random_probes(5, corr_small.shape[0], 2)
    for p in range(2):
        a, b = oracle.krylov(corr_small, probes[p], 20, orthogonalize=-1,
                             t=0.5)
        assert rel(a, g["corr_t0.5_p%d_alpha" % p]) < 1e-10
        assert rel(b, g["corr_t0.5_p%d_beta" % p]) < 1e-10


def _sorted_nodes(theta, tau):
    i = np.argsort(theta)
    return theta[i], tau[i] ** 2


@pytest.mark.parametrize("prefix,gram", [("c1_orth-1_p0", True),
                                         ("c1_orth0_p2", True),
                                         ("corr_orth-1_p1", False),
                                         ("corr_orth0_p3", False)])
def test_nodes_weights_vs_lapack(golden, prefix, gram):
    g = golden("krylov.npz")
    th, tau = oracle.nodes_weights(g[prefix + "_alpha"], g[prefix + "_beta"],
                                   gram=gram)
    t1, w1 = _sorted_nodes(th, tau)
    t2, w2 = _sorted_nodes(g[prefix + "_theta"], g[prefix + "_tau"])
    assert rel(t1, t2) < 1e-10
    assert np.max(np.abs(w1 - w2)) < 1e-10


def _check_estimator(r, g, key, samples_tol=1e-10):
    used = int(g[key + "_num_samples_used"].ravel()[0])
    assert np.array_equal(r["num_samples_used"], g[key + "_num_samples_used"])
    assert np.array_equal(r["num_outliers"], g[key + "_num_outliers"])
    assert np.array_equal(r["converged"], g[key + "_converged"])
    order = g[key + "_processed_samples_indices"][:used]
    assert np.array_equal(r["processed_samples_indices"][:used], order)
    s = r["samples"][order]
    assert rel(s, g[key + "_samples"][order]) < samples_tol
    assert rel(r["trace"], g[key + "_trace"]) < samples_tol
    assert rel(r["error"], g[key + "_error"]) < 1e-6


@pytest.mark.parametrize("orth", [0, -1])
def test_estimator_toeplitz(golden, orth):
    g = golden("estimator.npz")
    B = toeplitz(2.0, 1.0, 16384)
    r = oracle.trace_estimator(B, "log", gram=True, min_num_samples=50,
                               max_num_samples=200, error_rtol=1e-3,
                               lanczos_degree=30, orthogonalize=orth, seed=0)
    _check_estimator(r, g, "c1_log_orth%d" % orth)


@pytest.mark.parametrize("func", ["log", "inv", "id"])
def test_estimator_functions(golden, corr_small, func):
    g = golden("estimator.npz")
    r = oracle.trace_estimator(corr_small, func, min_num_samples=10,
                               max_num_samples=64, error_rtol=1e-2,
                               lanczos_degree=20, orthogonalize=0, seed=3)
    _check_estimator(r, g, "corr_%s" % func)


def test_estimator_gram_affine_exponent(golden, corr_small):
    g = golden("estimator.npz")
    r = oracle.trace_estimator(corr_small, "log", gram=True,
                               min_num_samples=10, max_num_samples=40,
                               error_rtol=1e-2, lanczos_degree=15,
                               orthogonalize=-1, seed=4)
    _check_estimator(r, g, "corr_gram_log")
    r = oracle.trace_estimator(corr_small, "inv", parameters=[0.1, 1.0, 10.0],
                               min_num_samples=5, max_num_samples=30,
                               error_rtol=1e-3, lanczos_degree=20,
                               orthogonalize=-1, seed=9)
    _check_estimator(r, g, "corr_affine_inv")
    r = oracle.trace_estimator(corr_small, "log", exponent=2.0,
                               min_num_samples=5, max_num_samples=20,
                               error_rtol=1e-2, lanczos_degree=10,
                               orthogonalize=3, seed=2)
    _check_estimator(r, g, "corr_log_p2")


@pytest.mark.parametrize("case", FUNC_CASES, ids=[c[0] for c in FUNC_CASES])
def test_estimator_other_functions(golden, corr_small, case):
    # trexp / trlinfrac / eigencount / density functions (and smoothstep)
    # against the reference's own outputs
    name, func, coeff, gram, params = case
    g = golden("functions.npz")
    r = oracle.trace_estimator(corr_small, func, gram=gram, parameters=params,
                               coeff=coeff, **FUNC_SETTINGS)
    _check_estimator(r, g, "fn_" + name)


def test_toeplitz_estimate_vs_exact(golden):
    # the reference's known answer: logdet(B^T B) = 2 n ln 2
    g = golden("estimator.npz")
    exact = 2 * 16384 * np.log(2.0)
    assert abs(g["c1_log_orth-1_trace"][0] - exact) / exact < 1e-3


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_oracle_matches_reference_library(corr_small):
    for kw in (dict(func="log", orthogonalize=0),
               dict(func="inv", orthogonalize=-1),
               dict(func="id", orthogonalize=4, exponent=1.5)):
        a = oracle.trace_estimator(corr_small, min_num_samples=4,
                                   max_num_samples=12, error_rtol=1e-4,
                                   lanczos_degree=12, seed=21, **kw)
        b = ref.trace_estimator(corr_small, min_num_samples=4,
                                max_num_samples=12, error_rtol=1e-4,
                                lanczos_degree=12, seed=21, num_threads=1,
                                **kw)
        assert rel(a["samples"], b["samples"]) < 1e-10
        assert np.array_equal(a["num_samples_used"], b["num_samples_used"])


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_reference_dense_operator_matches_csr():
    """The reference's dense row-major operator (cDenseMatrix,
    cDenseAffineMatrixFunction) gives the CSR operator's samples on the same
    matrix; the oracle matches it on the dense matrix too."""
    import scipy.sparse as sp
    from imate_b200.sample_matrices import dense_correlation_matrix
    A = dense_correlation_matrix(200, scale=0.05, shift=0.1, seed=5)
    kw = dict(min_num_samples=10, max_num_samples=10, error_rtol=0.0,
              lanczos_degree=20, orthogonalize=-1, seed=7)
    d = ref.trace_estimator(A, "log", **kw)
    c = ref.trace_estimator(sp.csr_matrix(A), "log", **kw)
    assert rel(d["samples"], c["samples"]) < 1e-12
    d = ref.trace_estimator(A, "inv", parameters=[0.3, 2.0], **kw)
    c = ref.trace_estimator(sp.csr_matrix(A), "inv", parameters=[0.3, 2.0],
                            **kw)
    assert rel(d["samples"], c["samples"]) < 1e-12
    o = oracle.trace_estimator(sp.csr_matrix(A), func="log", **kw)
    assert rel(o["samples"], ref.trace_estimator(A, "log", **kw)["samples"]) \
        < 1e-10


def test_dense_correlation_matrix_builders_agree():
    """The torch (row-block) and numpy paths of the dense correlation
    builder give the same matrix; it is symmetric with the shifted unit
    diagonal."""
    from imate_b200.sample_matrices import dense_correlation_matrix
    a = dense_correlation_matrix(300, scale=0.03, shift=0.2, seed=2)
    b = dense_correlation_matrix(300, scale=0.03, shift=0.2, seed=2,
                                 device="cpu")
    assert np.max(np.abs(a - b)) < 1e-14
    assert np.array_equal(a, a.T)
    assert np.all(np.diag(a) == 1.2)
    pts = np.random.default_rng(2).random((300, 2))
    r = np.linalg.norm(pts[3] - pts[17])
    assert abs(a[3, 17] - np.exp(-r / 0.03)) < 1e-15


def test_erfinv():
    from math import erf, sqrt
    for x in (0.0, 0.1, 0.5, 0.9, 0.95, 0.99, 0.999, -0.7):
        y = oracle.erfinv(x)
        assert abs(erf(y) - x) < 4e-16
    assert abs(sqrt(2) * oracle.erfinv(0.95) - 1.959963984540054) < 1e-14
