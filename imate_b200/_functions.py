"""Public SLQ functions: logdet, traceinv, trace, schatten, trexp,
trlinfrac, eigencount, density.

Same signatures and return conventions as imate's public functions
(``imate/logdet/logdet.py:23-394``, ``imate/traceinv/traceinv.py:24``,
``imate/trace/trace.py:23``, ``imate/schatten/schatten.py:24-467``) for
``method='slq'``: f = log for logdet (``functions/logarithm.cpp``),
1/x for traceinv (``functions/inverse.cpp:41``), x for trace
(``functions/identity.cpp:41``), applied as f(theta^p); the other SLQ
consumers differ only in f: exp(c x) for trexp
(``imate/trexp/_slq_method.pyx:814``, ``functions/exponential.cpp``),
(a x + b) / (c x + d) for trlinfrac (``trlinfrac/_slq_method.pyx:823``,
``functions/homographic.cpp``), the indicator of an interval for eigencount
(``eigencount/_slq_method.pyx:824``, ``functions/indicator.cpp``) and a
Gaussian kernel for density (``density/_slq_method.pyx:831``,
``functions/gaussian.cpp``).  The other methods
(cholesky, eigenvalue, exact, hutchinson) are CPU/dense paths outside this
engine and raise NotImplementedError.
"""

import numpy as np

from ._trace_estimator import trace_estimator, EngineOptions

__all__ = ["logdet", "traceinv", "trace", "schatten", "trexp", "trlinfrac",
           "eigencount", "density"]

_SLQ_DEFAULTS = dict(
    parameters=None, min_num_samples=10, max_num_samples=50,
    error_atol=None, error_rtol=1e-2, confidence_level=0.95,
    outlier_significance_level=0.001, lanczos_degree=20, lanczos_tol=None,
    orthogonalize=0, seed=None, num_threads=0, num_gpu_devices=0, gpu=False,
    verbose=False, plot=False)


def _slq(func, A, gram, p, return_info, options, func_coeff=None):
    if not isinstance(return_info, bool):
        raise TypeError('"return_info" should be boolean.')
    kw = dict(_SLQ_DEFAULTS)
    engine = options.pop("engine", None)
    block_size = options.pop("block_size", None)
    rng = options.pop("rng", None)
    unknown = set(options) - set(kw)
    if unknown:
        raise TypeError("unexpected keyword argument(s): %s"
                        % ", ".join(sorted(unknown)))
    kw.update(options)
    if engine is None:
        engine = EngineOptions()
    if block_size is not None:
        engine.block_size = int(block_size)
    if rng is not None:
        engine.rng = rng
    tr, info = trace_estimator(
        A, kw["parameters"], func, gram, p, kw["min_num_samples"],
        kw["max_num_samples"], kw["error_atol"], kw["error_rtol"],
        kw["confidence_level"], kw["outlier_significance_level"],
        kw["lanczos_degree"], kw["lanczos_tol"], kw["orthogonalize"],
        kw["seed"], kw["num_threads"], kw["num_gpu_devices"], kw["verbose"],
        kw["plot"], kw["gpu"], options=engine, func_coeff=func_coeff)
    if return_info:
        return tr, info
    return tr


def _only_slq(name, method):
    if method != "slq":
        raise NotImplementedError(
            '%s(method="%s") is not provided by the B200 engine; it serves '
            'method="slq" only.' % (name, method))


def logdet(A, gram=False, p=1.0, return_info=False, method="cholesky",
           **options):
    """log|det(A^p)| (or of (A^T A)^p with gram) by SLQ on the GPU."""
    _only_slq("logdet", method)
    return _slq("log", A, gram, p, return_info, options)


def traceinv(A, gram=False, p=1, return_info=False, method="cholesky",
             **options):
    """trace(A^-p) (or of (A^T A)^-p with gram) by SLQ on the GPU."""
    _only_slq("traceinv", method)
    return _slq("inv", A, gram, p, return_info, options)


def trace(A, gram=False, p=1.0, return_info=False, method="exact",
          **options):
    """trace(A^p) (or of (A^T A)^p with gram) by SLQ on the GPU."""
    _only_slq("trace", method)
    return _slq("id", A, gram, p, return_info, options)


def schatten(A, gram=False, p=2.0, return_info=False, method="eigenvalue",
             **options):
    """Schatten p-norm as imate defines it (schatten.py:427-462): p = 0 is
    exp(logdet / n), p > 0 (trace(A^p)/n)^(1/p), p < 0
    (traceinv(A^|p|)/n)^(1/p)."""
    if not isinstance(p, (int, np.integer, float)):
        raise ValueError('"p" should be float or integer.')
    n = A.get_num_rows() if hasattr(A, "get_num_rows") else A.shape[0]
    if p == 0:
        out = logdet(A, gram=gram, p=1.0, return_info=return_info,
                     method=method, **options)
        val, info = (out if return_info else (out, None))
        s = np.exp(val / n)
    elif p > 0:
        out = trace(A, gram=gram, p=p, return_info=return_info,
                    method=method, **options)
        val, info = (out if return_info else (out, None))
        s = (val / n) ** (1.0 / p)
    else:
        out = traceinv(A, gram=gram, p=np.abs(p), return_info=return_info,
                       method=method, **options)
        val, info = (out if return_info else (out, None))
        s = (val / n) ** (1.0 / p)
    if return_info:
        return s, info
    return s


def _check_return_info(return_info):
    if not isinstance(return_info, bool):
        raise TypeError('"return_info" should be boolean.')


def trexp(A, gram=False, p=1.0, coeff=1.0, return_info=False,
          method="eigenvalue", **options):
    """trace(exp(coeff A^p)) (or of (A^T A)^p with gram) by SLQ on the GPU
    (``imate/trexp/trexp.py:22``, ``_slq_method.pyx:24-840``)."""
    _only_slq("trexp", method)
    _check_return_info(return_info)
    if not isinstance(coeff, (int, float, np.integer, np.floating)) or \
            isinstance(coeff, bool):
        raise TypeError('"coeff" should be a real scalar.')
    return _slq("exp", A, gram, p, return_info, options,
                func_coeff=[float(coeff)])


def trlinfrac(A, gram=False, p=1.0, coeff=(1.0, 0.0, 1.0, 1.0),
              return_info=False, method="eigenvalue", **options):
    """trace((a A^p + b I)(c A^p + d I)^-1), coeff = (a, b, c, d), by SLQ on
    the GPU (``imate/trlinfrac/trlinfrac.py:22``, argument checks of
    ``_slq_method.pyx``)."""
    _only_slq("trlinfrac", method)
    if not isinstance(coeff, (tuple, list, np.ndarray)):
        raise TypeError('"coeff" should be a tuple, list, or numpy array.')
    if len(coeff) != 4:
        raise ValueError('"coeff" should be an array or list of length 4.')
    if coeff[0] * coeff[3] == coeff[1] * coeff[2]:
        raise ValueError('"coeff" of the linear fractional transformation '
                         'are degenerate.')
    _check_return_info(return_info)
    return _slq("linfrac", A, gram, p, return_info, options,
                func_coeff=[float(c) for c in coeff])


def eigencount(A, gram=False, p=1.0, interval=(0.0, 1.0), return_info=False,
               method="eigenvalue", **options):
    """Number of eigenvalues of A^p (or (A^T A)^p) in the closed interval
    [a, b] by SLQ on the GPU (``imate/eigencount/eigencount.py:22``)."""
    _only_slq("eigencount", method)
    if not isinstance(interval, (tuple, list, np.ndarray)):
        raise TypeError('"interval" should be a tuple,  list, or numpy '
                        'array.')
    if len(interval) != 2:
        raise ValueError('"interval" should be an array or list of length '
                         '2.')
    _check_return_info(return_info)
    return _slq("indicator", A, gram, p, return_info, options,
                func_coeff=[float(interval[0]), float(interval[1])])


def density(A, gram=False, p=1.0, mu=1.0, sigma=1.0, return_info=False,
            method="eigenvalue", **options):
    """Spectral density of A^p (or (A^T A)^p) at mu, smoothed by a Gaussian
    of width sigma: trace(g(A^p)), g(x) = exp(-((x - mu)/sigma)^2/2) /
    (sigma sqrt(2 pi)), by SLQ on the GPU (``imate/density/density.py:22``;
    the reference's Gaussian takes a scalar mu)."""
    _only_slq("density", method)
    if isinstance(mu, (list, tuple, np.ndarray)):
        raise TypeError('"mu" should be a real scalar for method="slq" (one '
                        'Gaussian per call).')
    if not isinstance(mu, (int, float, np.integer, np.floating)) or \
            isinstance(mu, bool):
        raise TypeError('"mu" should be either a real scalar or a real 1D '
                        'array-like, such as list, tuple, or numpy array.')
    if not isinstance(sigma, (int, float, np.integer, np.floating)) or \
            isinstance(sigma, bool):
        raise TypeError('"sigma" should be a scalar real number.')
    if sigma <= 0.0:
        raise ValueError('"sigma" should be positive.')
    _check_return_info(return_info)
    return _slq("gaussian", A, gram, p, return_info, options,
                func_coeff=[float(mu), float(sigma)])
