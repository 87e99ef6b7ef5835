"""Loader for the C restatement ``oracle/slq_oracle.c`` -- test infrastructure.

The oracle checks the CUDA engine: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it.  Its
functions follow the reference CPU SLQ (ameli/imate v0.25.2,
``imate/_c_trace_estimator/c_trace_estimator.cpp:192-654`` and callees); see
the header of ``slq_oracle.c`` for the per-function citations.
"""

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "_build", "libslq_oracle.so")
FUNC_IDS = {"log": 0, "inv": 1, "id": 2, "exp": 3, "linfrac": 4,
            "indicator": 5, "gaussian": 6, "smoothstep": 7}

_lib = None


def build():
    """Compile ``slq_oracle.c`` (plain C, gcc)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "all"])


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO):
        build()
    _lib = ctypes.CDLL(ORACLE_SO)
    _lib.oracle_erfinv.restype = ctypes.c_double
    _lib.oracle_erfinv.argtypes = [ctypes.c_double]
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _csr_parts(A):
    import scipy.sparse as sp
    fmt = 1 if getattr(A, "format", "") == "csc" else 0
    A = sp.csc_matrix(A) if fmt else sp.csr_matrix(A)
    A.sort_indices()
    return (A, fmt, np.ascontiguousarray(A.data, dtype=np.float64),
            np.ascontiguousarray(A.indices, dtype=np.int32),
            np.ascontiguousarray(A.indptr, dtype=np.int32))


def erfinv(x):
    return load().oracle_erfinv(float(x))


def random_probes(seed, n, num_probes):
    lib = load()
    out = np.empty((num_probes, n), np.float64)
    lib.oracle_random_probes.restype = None
    lib.oracle_random_probes.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                         ctypes.c_int, ctypes.c_void_p]
    lib.oracle_random_probes(seed, n, num_probes, _p(out))
    return out


def stream_words(seed, count):
    lib = load()
    out = np.empty(count, np.uint64)
    lib.oracle_stream_words.restype = None
    lib.oracle_stream_words.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                        ctypes.c_void_p]
    lib.oracle_stream_words(seed, count, _p(out))
    return out


def krylov(A, v, m, gram=False, orthogonalize=0, tol=None, t=None):
    lib = load()
    A, fmt, data, indices, indptr = _csr_parts(A)
    v = np.ascontiguousarray(v, dtype=np.float64)
    alpha = np.zeros(m, np.float64)
    beta = np.zeros(m, np.float64)
    if tol is None:
        tol = float(np.finfo(np.float64).eps)
    fn = lib.oracle_krylov
    fn.restype = ctypes.c_int
    vp, i32, i64, d = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                       ctypes.c_double)
    fn.argtypes = [vp, vp, vp, i64, i64, i32, i32, d, i32, vp, i32, d, i32,
                   vp, vp]
    size = fn(_p(data), _p(indices), _p(indptr), A.shape[0], A.shape[1], fmt,
              int(t is not None), 0.0 if t is None else float(t), int(gram),
              _p(v), m, tol, orthogonalize, _p(alpha), _p(beta))
    return alpha[:size].copy(), beta[:size].copy()


def nodes_weights(alpha, beta, gram=False):
    lib = load()
    k = len(alpha)
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.zeros(max(k, 1), np.float64)
    b[:k] = beta[:k]
    theta = np.zeros(k, np.float64)
    tau = np.zeros(k, np.float64)
    fn = lib.oracle_nodes_weights
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    if fn(_p(a), _p(b), k, int(gram), _p(theta), _p(tau)) != 0:
        raise RuntimeError("implicit QL did not converge")
    return theta, tau


def check_convergence(samples, order, nproc, min_num_samples, conf, atol,
                      rtol, converged):
    """One call of the reference convergence test; returns (all, error, used,
    converged).  ``samples`` is [max][q]."""
    lib = load()
    samples = np.ascontiguousarray(samples, np.float64)
    q = samples.shape[1]
    order = np.ascontiguousarray(order, np.int32)
    err = np.zeros(q)
    used = np.zeros(q, np.int32)
    conv = np.ascontiguousarray(converged, np.int32).copy()
    fn = lib.oracle_check_convergence
    fn.restype = ctypes.c_int
    vp, i32, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    fn.argtypes = [vp, i32, i32, vp, i32, d, d, d, vp, vp, vp]
    a = fn(_p(samples), q, min_num_samples, _p(order), nproc, conf, atol,
           rtol, _p(err), _p(used), _p(conv))
    return bool(a), err, used, conv


def trace_estimator(A, func, gram=False, exponent=1.0, parameters=None,
                    min_num_samples=10, max_num_samples=50, error_atol=0.0,
                    error_rtol=1e-2, confidence_level=0.95,
                    outlier_significance_level=0.001, lanczos_degree=20,
                    lanczos_tol=None, orthogonalize=0, seed=0, coeff=None):
    """Single-thread restatement of the reference estimator (FP64).
    gram: False/0 Lanczos on A, True/1 Golub-Kahn on A, 2 Lanczos on
    A^T A (+ t I with parameters).  func: 'log', 'inv', 'id', 'exp',
    'linfrac', 'indicator', 'gaussian', 'smoothstep' with coefficients
    ``coeff`` (imate/functions/*.cpp)."""
    lib = load()
    A, fmt, data, indices, indptr = _csr_parts(A)
    affine = parameters is not None
    params = np.atleast_1d(np.asarray(
        parameters if affine else [0.0], dtype=np.float64)).copy()
    q = params.size if affine else 1
    m = lanczos_degree
    if lanczos_tol is None:
        lanczos_tol = float(np.finfo(np.float64).eps)
    trace = np.empty(q)
    error = np.empty(q)
    samples = np.empty((max_num_samples, q))
    order = np.zeros(max_num_samples, np.int32)
    used = np.zeros(q, np.int32)
    outl = np.zeros(q, np.int32)
    conv = np.zeros(q, np.int32)
    sizes = np.zeros(max_num_samples, np.int32)
    alphas = np.zeros((max_num_samples, m))
    betas = np.zeros((max_num_samples, m))
    fid = FUNC_IDS[func]
    fc = np.zeros(4)
    if coeff is not None:
        fc[:len(coeff)] = coeff
    fn = lib.oracle_trace_estimator
    fn.restype = ctypes.c_int
    vp, i32, i64, d = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                       ctypes.c_double)
    fn.argtypes = [vp, vp, vp, i64, i64, i32, i32, vp, i32, i32, vp, i32, d,
                   i32, i64, i32, d, i32, i32, d, d, d, d, vp, vp, vp, vp, vp,
                   vp, vp, vp, vp, vp]
    st = fn(_p(data), _p(indices), _p(indptr), A.shape[0], A.shape[1], fmt,
            int(affine), _p(params), q, fid, _p(fc), int(gram),
            float(exponent),
            orthogonalize, seed, m, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, _p(trace), _p(error), _p(samples),
            _p(order), _p(used), _p(outl), _p(conv), _p(sizes), _p(alphas),
            _p(betas))
    if st < 0:
        raise RuntimeError("oracle eigen-solve failed")
    return dict(all_converged=bool(st), trace=trace, error=error,
                samples=samples, processed_samples_indices=order,
                num_samples_used=used, num_outliers=outl, converged=conv,
                lanczos_sizes=sizes, alphas=alphas, betas=betas)
