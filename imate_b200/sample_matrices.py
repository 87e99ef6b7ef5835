"""Test matrices with known answers and the synthetic workloads.

``toeplitz`` and its analytic log-determinant / traces follow imate's
sample matrices (``imate/sample_matrices/toeplitz.py:25-540``): the upper
bidiagonal Toeplitz matrix B with a on the diagonal and b above it, whose
Gram matrix B^T B has logdet 2 n ln|a|.

``correlation_matrix`` builds the sparse SPD kernel matrices of the
benchmark workloads: points uniform in the unit square, the exponential
kernel exp(-r / scale) (``imate/sample_matrices/_kernels.pyx:164-180``)
zeroed below a threshold, plus a diagonal shift.  imate's own builder loops
over all point pairs (``_sparse_correlation_matrix.pyx:43-246``, O(n^2));
this one finds the pairs within the cut-off radius with a k-d tree, which
gives the same matrix in O(n log n).
"""

import numpy as np
import scipy.sparse as sp

__all__ = ["toeplitz", "toeplitz_logdet", "toeplitz_traceinv",
           "toeplitz_trace", "correlation_matrix", "correlation_points"]


def toeplitz(a, b, size=20, gram=False, format="csr", dtype="float64"):
    """Upper bidiagonal Toeplitz matrix (or its Gram matrix)."""
    if format not in ("csr", "csc"):
        raise ValueError('format should be "csr" or "csc".')
    diag = np.arange(size)
    rows = np.concatenate([diag, diag[:-1]])
    cols = np.concatenate([diag, diag[1:]])
    vals = np.concatenate([np.full(size, a), np.full(size - 1, b)])
    A = sp.coo_matrix((vals.astype(dtype), (rows, cols)), shape=(size, size))
    if gram:
        A = A.T @ A
    A = A.tocsc() if format == "csc" else A.tocsr()
    A.sort_indices()
    return A.astype(dtype)


def toeplitz_logdet(a, b, size, gram=False):
    """logdet of toeplitz(a, b, size[, gram]) (toeplitz.py:467-540)."""
    v = size * np.log(a)
    return 2.0 * v if gram else v


def toeplitz_trace(a, b, size, gram=False):
    """trace (toeplitz.py:273-348)."""
    if gram:
        return size * a**2 + (size - 1) * b**2
    return size * a


def toeplitz_traceinv(a, b, size, gram=False):
    """trace of the inverse (toeplitz.py:355-460), closed form of the sum."""
    if not gram:
        return size / a
    if a == b:
        return size * (size + 1) / (2.0 * a**2)
    q = b / a
    if size < 200:
        return (1.0 / (a**2 - b**2)) * \
            (size - q**2 * ((q**(2.0 * size) - 1.0) / (q**2 - 1.0)))
    return (1.0 / (a**2 - b**2)) * (size - q**2 / (1.0 - q**2))


def correlation_points(size, dimension=2, seed=1):
    """Points uniform in [0, 1]^dimension from numpy's PCG64 with ``seed``."""
    rng = np.random.default_rng(seed)
    return rng.random((size, dimension))


def correlation_matrix(size=None, dimension=2, scale=0.1, threshold=0.05,
                       shift=1e-3, seed=1, points=None, dtype="float64",
                       format="csr"):
    """Sparse exponential-kernel correlation matrix plus ``shift * I``.

    K_ij = exp(-|x_i - x_j| / scale), kept where K_ij >= threshold (so
    |x_i - x_j| <= -scale ln(threshold)), unit diagonal, plus shift on the
    diagonal.  Entries are computed in float64 and cast to ``dtype``.
    """
    from scipy.spatial import cKDTree
    if points is None:
        points = correlation_points(size, dimension, seed)
    n = points.shape[0]
    radius = -scale * np.log(threshold)
    tree = cKDTree(points)
    pairs = tree.query_pairs(radius, output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    r = np.linalg.norm(points[i] - points[j], axis=1)
    k = np.exp(-r / scale)
    keep = k >= threshold
    i, j, k = i[keep], j[keep], k[keep]
    rows = np.concatenate([i, j, np.arange(n)])
    cols = np.concatenate([j, i, np.arange(n)])
    vals = np.concatenate([k, k, np.full(n, 1.0 + shift)])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n))
    A = A.tocsc() if format == "csc" else A.tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return A.astype(dtype)
