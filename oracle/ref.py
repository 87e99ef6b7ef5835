"""Loader for ``oracle/_ref/libimate_ref.so`` -- test infrastructure only.

The library is the reference's own CPU SLQ (ameli/imate v0.25.2,
``imate/_c_trace_estimator/c_trace_estimator.cpp:192-307`` and the sources it
calls), compiled from its own source files by ``oracle/Makefile`` with the
thin entry layer ``oracle/ref_harness.cpp``.  It checks the CUDA
path and the CPU baseline that ``bench.py --impl reference`` times; the
product never imports this module.

``libimate_ref_gpu.so`` is the reference's GPU SLQ
(``imate/_cu_trace_estimator/cu_trace_estimator.cu:197-315`` over
``cuCSRMatrix``: cuSPARSE SpMV and cuBLAS vector operations), compiled from
its sources for sm_100a by the same Makefile (target ``ref_gpu``): a second
reference for the tests and the reference GPU comparator of bench.py's
reference arm.

LAPACK is bound the way the reference binds it
(``imate/_c_trace_estimator/lapack_api.pxi:14``): through
``scipy.linalg.cython_lapack``'s exported function pointers.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(_HERE, "_ref", "libimate_ref.so")
REF_GPU_SO = os.path.join(_HERE, "_ref", "libimate_ref_gpu.so")

_lib = None
_gpu_lib = None


def _capsule_pointer(capsule):
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = ctypes.c_void_p
    get_ptr.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(capsule, get_name(capsule))


def available():
    return os.path.exists(REF_SO)


def _bind_lapack(lib):
    from scipy.linalg import cython_lapack
    capi = cython_lapack.__pyx_capi__
    ptrs = [_capsule_pointer(capi[k])
            for k in ("dstev", "sstev", "dbdsdc", "sbdsdc")]
    lib.ref_set_lapack.restype = ctypes.c_int
    lib.ref_set_lapack.argtypes = [ctypes.c_void_p] * 4
    if lib.ref_set_lapack(*ptrs) != 0:
        raise RuntimeError("could not bind LAPACK for the reference library")


def load():
    """Load the reference library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise FileNotFoundError(
            "reference CPU library not built: run `make -C oracle ref` "
            "where the reference sources are present")
    lib = ctypes.CDLL(REF_SO)
    _bind_lapack(lib)
    _lib = lib
    return lib


def gpu_available():
    return os.path.exists(REF_GPU_SO)


def load_gpu():
    """Load the reference GPU library (``libimate_ref_gpu.so``: the
    reference's cuSPARSE/cuBLAS SLQ, ``cu_trace_estimator.cu:197-315``);
    raises if it was not built."""
    global _gpu_lib
    if _gpu_lib is not None:
        return _gpu_lib
    if not gpu_available():
        raise FileNotFoundError(
            "reference GPU library not built: run `make -C oracle ref_gpu` "
            "where the reference sources are present")
    lib = ctypes.CDLL(REF_GPU_SO)
    _bind_lapack(lib)
    _gpu_lib = lib
    return lib


def gpu_trace_estimator(A, func, gram=False, exponent=1.0, min_num_samples=10,
                        max_num_samples=50, error_atol=0.0, error_rtol=1e-2,
                        confidence_level=0.95,
                        outlier_significance_level=0.001, lanczos_degree=20,
                        lanczos_tol=None, orthogonalize=0, seed=0,
                        num_gpu_devices=1):
    """Run the reference GPU estimator on a CSR matrix, or on a dense
    ndarray (row-major, cuBLAS gemv products), for one inquiry (``func`` in
    {'log', 'inv', 'id'}).  Returns the same dict as ``trace_estimator``."""
    import scipy.sparse as sp
    lib = load_gpu()
    dt = np.float64 if A.dtype == np.float64 else np.float32
    if isinstance(A, np.ndarray):
        # dense row-major operator (cu_dense_matrix.cu)
        data = np.ascontiguousarray(A, dtype=dt)
        indices = indptr = None
    else:
        A = sp.csr_matrix(A)
        A.sort_indices()
        indices = np.ascontiguousarray(A.indices, dtype=np.int32)
        indptr = np.ascontiguousarray(A.indptr, dtype=np.int32)
        data = np.ascontiguousarray(A.data, dtype=dt)
    if lanczos_tol is None:
        lanczos_tol = float(np.finfo(dt).eps)
    trace = np.empty(1, dt)
    error = np.empty(1, dt)
    samples = np.empty(max_num_samples, dt)
    order = np.zeros(max_num_samples, np.int32)
    used = np.zeros(1, np.int32)
    outl = np.zeros(1, np.int32)
    conv = np.zeros(1, np.int32)
    wall = ctypes.c_float(0.0)
    fid = {"log": 0, "inv": 1, "id": 2}[func]
    if dt == np.float64:
        fn, real = lib.ref_gpu_trace_estimator_f64, ctypes.c_double
    else:
        fn, real = lib.ref_gpu_trace_estimator_f32, ctypes.c_float
    fn.restype = ctypes.c_int
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    fn.argtypes = [vp, vp, vp, i64, i64, i32, i32, real, i32, i64, i32, real,
                   i32, i32, real, real, real, real, i32, vp, vp, vp, vp, vp,
                   vp, vp, ctypes.POINTER(ctypes.c_float)]
    allc = fn(_p(data), _p(indices) if indices is not None else None,
              _p(indptr) if indptr is not None else None, A.shape[0],
              A.shape[1], fid,
              int(gram), exponent, orthogonalize, seed, lanczos_degree,
              lanczos_tol, min_num_samples, max_num_samples, error_atol,
              error_rtol, confidence_level, outlier_significance_level,
              num_gpu_devices, _p(trace), _p(error), _p(samples), _p(order),
              _p(used), _p(outl), _p(conv), ctypes.byref(wall))
    return dict(all_converged=bool(allc), trace=trace, error=error,
                samples=samples.reshape(-1, 1),
                processed_samples_indices=order, num_samples_used=used,
                num_outliers=outl, converged=conv,
                alg_wall_time=float(wall.value))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _csr_parts(A):
    """(A, fmt, indices, indptr): fmt 0 = CSR, 1 = CSC, 2 = dense row-major
    ndarray (no index arrays)."""
    import scipy.sparse as sp
    if isinstance(A, np.ndarray):
        empty = np.zeros(1, np.int32)
        return np.ascontiguousarray(A), 2, empty, empty
    fmt = 1 if sp.isspmatrix_csc(A) or getattr(A, "format", "") == "csc" else 0
    if fmt == 0:
        A = sp.csr_matrix(A)
    A.sort_indices()
    return (A, fmt, np.ascontiguousarray(A.indices, dtype=np.int32),
            np.ascontiguousarray(A.indptr, dtype=np.int32))


def trace_estimator(A, func, gram=False, exponent=1.0, parameters=None,
                    min_num_samples=10, max_num_samples=50, error_atol=0.0,
                    error_rtol=1e-2, confidence_level=0.95,
                    outlier_significance_level=0.001, lanczos_degree=20,
                    lanczos_tol=None, orthogonalize=0, seed=0, num_threads=1,
                    coeff=None):
    """Run the reference estimator.  ``func`` in {'log', 'inv', 'id', 'exp',
    'linfrac', 'indicator', 'gaussian', 'smoothstep'} with the function's
    coefficients ``coeff`` (functions/*.cpp).

    ``parameters`` (None or a 1-D array) selects an ``A + t I`` operator as
    ``imate.AffineMatrixFunction(A)`` does.  Returns a dict with the same
    arrays the reference fills.
    """
    lib = load()
    A, fmt, indices, indptr = _csr_parts(A)
    dt = np.float64 if A.dtype == np.float64 else np.float32
    data = np.ascontiguousarray(A if fmt == 2 else A.data, dtype=dt)
    affine = parameters is not None
    params = np.atleast_1d(np.asarray(
        parameters if affine else [0.0], dtype=dt)).copy()
    q = params.size if affine else 1
    if lanczos_tol is None:
        lanczos_tol = float(np.finfo(dt).eps)
    trace = np.empty(q, dt)
    error = np.empty(q, dt)
    samples = np.empty((max_num_samples, q), dt)
    order = np.zeros(max_num_samples, np.int32)
    used = np.zeros(q, np.int32)
    outl = np.zeros(q, np.int32)
    conv = np.zeros(q, np.int32)
    wall = ctypes.c_float(0.0)
    fid = {"log": 0, "inv": 1, "id": 2, "exp": 3, "linfrac": 4,
           "indicator": 5, "gaussian": 6, "smoothstep": 7}[func]
    fc = np.zeros(4)
    if coeff is not None:
        fc[:len(coeff)] = coeff
    if dt == np.float64:
        fn, real = lib.ref_trace_estimator_f64, ctypes.c_double
    else:
        fn, real = lib.ref_trace_estimator_f32, ctypes.c_float
    fn.restype = ctypes.c_int
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    fn.argtypes = [vp, vp, vp, i64, i64, i32, i32, vp, i32, i32, vp, i32,
                   real,
                   i32, i64, i32, real, i32, i32, real, real, real, real, i32,
                   vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_float)]
    allc = fn(_p(data), _p(indices), _p(indptr), A.shape[0], A.shape[1], fmt,
              int(affine), _p(params), q, fid, _p(fc), int(gram), exponent,
              orthogonalize, seed, lanczos_degree, lanczos_tol,
              min_num_samples, max_num_samples, error_atol, error_rtol,
              confidence_level, outlier_significance_level, num_threads,
              _p(trace), _p(error), _p(samples), _p(order), _p(used),
              _p(outl), _p(conv), ctypes.byref(wall))
    return dict(all_converged=bool(allc), trace=trace, error=error,
                samples=samples, processed_samples_indices=order,
                num_samples_used=used, num_outliers=outl, converged=conv,
                alg_wall_time=float(wall.value))


def trace_estimator_b(A, B, func, parameters, gram=False, exponent=1.0,
                      min_num_samples=10, max_num_samples=50, error_atol=0.0,
                      error_rtol=1e-2, confidence_level=0.95,
                      outlier_significance_level=0.001, lanczos_degree=20,
                      lanczos_tol=None, orthogonalize=0, seed=0,
                      num_threads=1, coeff=None):
    """The reference estimator on A + t B for a general (CSR) B, FP64:
    ``imate.AffineMatrixFunction(A, B)``.  Returns the dict of
    ``trace_estimator``."""
    import scipy.sparse as sp
    lib = load()
    A = sp.csr_matrix(A, dtype=np.float64)
    A.sort_indices()
    B = sp.csr_matrix(B, dtype=np.float64)
    B.sort_indices()
    params = np.ascontiguousarray(np.atleast_1d(parameters), dtype=np.float64)
    q = params.size
    if lanczos_tol is None:
        lanczos_tol = float(np.finfo(np.float64).eps)
    arrays = [np.ascontiguousarray(x) for x in (
        A.data, A.indices.astype(np.int32), A.indptr.astype(np.int32),
        B.data, B.indices.astype(np.int32), B.indptr.astype(np.int32))]
    trace = np.empty(q)
    error = np.empty(q)
    samples = np.empty((max_num_samples, q))
    order = np.zeros(max_num_samples, np.int32)
    used = np.zeros(q, np.int32)
    outl = np.zeros(q, np.int32)
    conv = np.zeros(q, np.int32)
    wall = ctypes.c_float(0.0)
    fid = {"log": 0, "inv": 1, "id": 2, "exp": 3, "linfrac": 4,
           "indicator": 5, "gaussian": 6, "smoothstep": 7}[func]
    fc = np.zeros(4)
    if coeff is not None:
        fc[:len(coeff)] = coeff
    fn = lib.ref_trace_estimator_b_f64
    fn.restype = ctypes.c_int
    vp, i32, i64, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, \
        ctypes.c_double
    fn.argtypes = [vp] * 6 + [i64, i64, vp, i32, i32, vp, i32, d, i32, i64,
                              i32, d, i32, i32, d, d, d, d, i32, vp, vp, vp,
                              vp, vp, vp, vp, ctypes.POINTER(ctypes.c_float)]
    allc = fn(*[_p(x) for x in arrays], A.shape[0], A.shape[1], _p(params),
              q, fid, _p(fc), int(gram), exponent, orthogonalize, seed,
              lanczos_degree, lanczos_tol, min_num_samples, max_num_samples,
              error_atol, error_rtol, confidence_level,
              outlier_significance_level, num_threads, _p(trace), _p(error),
              _p(samples), _p(order), _p(used), _p(outl), _p(conv),
              ctypes.byref(wall))
    return dict(all_converged=bool(allc), trace=trace, error=error,
                samples=samples, processed_samples_indices=order,
                num_samples_used=used, num_outliers=outl, converged=conv,
                alg_wall_time=float(wall.value))


def random_probes(seed, n, num_probes):
    """Probe vectors the single-thread reference estimator draws, in order."""
    lib = load()
    out = np.empty((num_probes, n), np.float64)
    lib.ref_random_probes.restype = None
    lib.ref_random_probes.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                      ctypes.c_int, ctypes.c_void_p]
    lib.ref_random_probes(seed, n, num_probes, _p(out))
    return out


def krylov(A, v, m, gram=False, orthogonalize=0, tol=None, t=None):
    """Per-probe alpha/beta of the reference Lanczos / Golub-Kahn (FP64)."""
    lib = load()
    A, fmt, indices, indptr = _csr_parts(A)
    data = np.ascontiguousarray(A if fmt == 2 else A.data, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    alpha = np.zeros(m, np.float64)
    beta = np.zeros(m, np.float64)
    if tol is None:
        tol = float(np.finfo(np.float64).eps)
    fn = lib.ref_krylov_f64
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
    """theta/tau the reference forms from alpha/beta with LAPACK."""
    lib = load()
    k = len(alpha)
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.zeros(max(k, 1), np.float64)
    b[:k] = beta[:k]
    theta = np.zeros(k, np.float64)
    tau = np.zeros(k, np.float64)
    fn = lib.ref_nodes_weights_f64
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    info = fn(_p(a), _p(b), k, int(gram), _p(theta), _p(tau))
    if info != 0:
        raise RuntimeError("LAPACK returned info=%d" % info)
    return theta, tau


def max_threads():
    lib = load()
    lib.ref_max_threads.restype = ctypes.c_int
    return lib.ref_max_threads()
