"""schatten(p) through the drop-in API for p = 0, 2 and -1.

imate defines the norm (schatten.py:427-462) as exp(logdet / n) for p = 0,
(trace(A^p) / n)^(1/p) for p > 0 and (traceinv(A^|p|) / n)^(1/p) for p < 0,
n = A.shape[0].  On the same probes the norm must be that scaling of the
logdet / trace / traceinv estimate bit for bit, and it must match the norm
of the exact eigenvalues within the estimate's own Monte-Carlo error (the
bar: 4 standard errors of the scaled estimate, plus 1e-6 relative)."""

import numpy as np
import pytest

import imate_b200 as ib

pytestmark = pytest.mark.gpu

KW = dict(method="slq", gpu=True, return_info=True, min_num_samples=400,
          max_num_samples=400, error_rtol=0.0, lanczos_degree=40,
          orthogonalize=-1, seed=7)


@pytest.fixture(scope="module")
def spd():
    A = ib.correlation_matrix(1500, scale=0.03, shift=0.2, seed=11)
    return A, np.linalg.eigvalsh(A.toarray())


def _exact(ev, p):
    n = ev.size
    if p == 0:
        return float(np.exp(np.sum(np.log(ev)) / n))
    if p > 0:
        return float((np.sum(ev ** p) / n) ** (1.0 / p))
    return float((np.sum(ev ** p) / n) ** (1.0 / p))


@pytest.mark.parametrize("p", [0, 2, -1])
def test_schatten_is_the_scaled_trace_and_matches_eigenvalues(cuda, spd, p):
    A, ev = spd
    n = A.shape[0]
    s, info = ib.schatten(A, p=p, **KW)
    if p == 0:
        base, binfo = ib.logdet(A, p=1.0, **KW)
        want = np.exp(base / n)
        # d/dx exp(x/n) = exp(x/n) / n
        err = want / n * binfo["error"]["absolute_error"]
    elif p > 0:
        base, binfo = ib.trace(A, p=p, **KW)
        want = (base / n) ** (1.0 / p)
        err = want / (p * base) * binfo["error"]["absolute_error"]
    else:
        base, binfo = ib.traceinv(A, p=abs(p), **KW)
        want = (base / n) ** (1.0 / p)
        err = want / (abs(p) * base) * binfo["error"]["absolute_error"]
    assert s == want
    np.testing.assert_array_equal(info["convergence"]["samples"],
                                  binfo["convergence"]["samples"])
    exact = _exact(ev, p)
    # the confidence-level error is ~1.96 standard errors
    assert abs(s - exact) <= 4.0 / 1.96 * err + 1e-6 * exact
    assert info["precision"]["operator_dtype"] == "float64"
    assert info["precision"]["reductions"] == "float64"


def test_schatten_gram_uses_rows_of_a(cuda):
    """For gram=True the norm is of A^T A, scaled by A.shape[0] as in imate
    (schatten.py:425)."""
    B = ib.toeplitz(2.0, 1.0, 1200)
    s, _ = ib.schatten(B, gram=True, p=2, **KW)
    tr, _ = ib.trace(B, gram=True, p=2, **KW)
    assert s == (tr / B.shape[0]) ** 0.5
