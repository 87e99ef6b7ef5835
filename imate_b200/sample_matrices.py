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
           "toeplitz_trace", "correlation_matrix", "correlation_points",
           "correlation_matrix_device", "batched_correlation_sizes",
           "sparse_gram_design", "dense_correlation_matrix"]


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


def dense_correlation_matrix(size=None, dimension=2, scale=0.1, shift=1e-3,
                             seed=1, points=None, dtype="float64",
                             device=None):
    """Dense exponential-kernel correlation matrix plus ``shift * I``, as
    imate builds it for ``sparse=False``
    (``imate/sample_matrices/_dense_correlation_matrix.pyx:41-150``):
    K_ij = exp(-|x_i - x_j| / scale) for every pair, unit diagonal.

    Returns a C-contiguous numpy array.  Distances and kernel values are
    computed in float64 (on ``device`` with torch when given, in row blocks)
    and cast to ``dtype`` at the end.
    """
    if points is None:
        points = correlation_points(size, dimension, seed)
    n = points.shape[0]
    out = np.empty((n, n), dtype=dtype)
    rows = max(1, (1 << 25) // max(n, 1))
    if device is not None:
        import torch
        P = torch.as_tensor(points, dtype=torch.float64, device=device)
        for r0 in range(0, n, rows):
            D = torch.cdist(P[r0:r0 + rows], P,
                            compute_mode="donot_use_mm_for_euclid_dist")
            K = torch.exp(-D / scale)
            out[r0:r0 + rows] = K.to(getattr(torch, np.dtype(dtype).name)) \
                .cpu().numpy()
    else:
        for r0 in range(0, n, rows):
            d = points[r0:r0 + rows, None, :] - points[None, :, :]
            out[r0:r0 + rows] = np.exp(-np.sqrt(np.sum(d * d, axis=-1)) /
                                       scale)
    idx = np.arange(n)
    out[idx, idx] = 1.0 + shift
    return out


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


def correlation_matrix_device(size=None, scale=0.1, threshold=0.05,
                              shift=1e-3, seed=1, points=None,
                              dtype="float32", device=None,
                              max_candidates=1 << 26):
    """The matrix of ``correlation_matrix`` (dimension 2), built on the GPU.

    Returns (indptr, indices, data, perm) as torch tensors on the device:
    the CSR of P K P^T, where P lists the points cell by cell of a grid of
    cells no smaller than the cut-off radius (row r of the CSR is point
    perm[r]).  A symmetric permutation leaves every trace f(K) unchanged and
    the cell order keeps each row's neighbours close, so the CSR can be used
    as an operator directly (no locality reordering needed).  Pair distances,
    kernel values and the threshold test are computed in float64 as in
    ``correlation_matrix`` and cast to ``dtype`` at the end; rows list their
    columns in increasing order.  Candidate pairs are processed in chunks of
    at most ``max_candidates``.
    """
    import torch
    if points is None:
        points = correlation_points(size, 2, seed)
    dev = torch.device(device) if device is not None else \
        torch.device("cuda", torch.cuda.current_device())
    n = points.shape[0]
    radius = -scale * np.log(threshold)
    nc = max(1, int(np.floor(1.0 / radius)))
    P = torch.from_numpy(np.ascontiguousarray(points, dtype=np.float64)).to(dev)
    cxy = torch.clamp((P * nc).long(), 0, nc - 1)
    cid = cxy[:, 1] * nc + cxy[:, 0]
    cid_sorted, perm = torch.sort(cid, stable=True)
    Ps = P[perm]
    cx = cxy[perm, 0]
    cy = cxy[perm, 1]
    counts = torch.bincount(cid_sorted, minlength=nc * nc)
    cell_start = torch.zeros(nc * nc + 1, dtype=torch.long, device=dev)
    cell_start[1:] = torch.cumsum(counts, 0)
    # the 9 neighbour cells in increasing cell id, so that each row's
    # candidate columns come out sorted
    offs = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    seg_s = []
    seg_e = []
    for dy, dx in offs:
        ny = cy + dy
        nx = cx + dx
        ok = (ny >= 0) & (ny < nc) & (nx >= 0) & (nx < nc)
        c = torch.where(ok, ny * nc + nx, torch.zeros_like(ny))
        s = cell_start[c]
        e = cell_start[c + 1]
        seg_s.append(torch.where(ok, s, torch.zeros_like(s)))
        seg_e.append(torch.where(ok, e, torch.zeros_like(e)))
    seg_s = torch.stack(seg_s, 1)          # [n, 9]
    seg_len = torch.stack(seg_e, 1) - seg_s
    row_cand = seg_len.sum(1)
    cum = torch.cumsum(row_cand, 0)
    r2 = radius * radius
    rows_out, cols_out, vals_out = [], [], []
    r0 = 0
    while r0 < n:
        base = int(cum[r0 - 1]) if r0 > 0 else 0
        r1 = int(torch.searchsorted(cum, base + max_candidates, right=True))
        r1 = max(r1, r0 + 1)
        r1 = min(r1, n)
        L = seg_len[r0:r1].reshape(-1)
        S = seg_s[r0:r1].reshape(-1)
        total = int(L.sum())
        if total:
            seg = torch.repeat_interleave(
                torch.arange(L.numel(), device=dev), L)
            first = torch.cumsum(L, 0) - L
            j = S[seg] + (torch.arange(total, device=dev) - first[seg])
            i = r0 + seg // 9
            d = Ps[i] - Ps[j]
            dist2 = (d * d).sum(1)
            keep = dist2 <= r2
            i, j, dist2 = i[keep], j[keep], dist2[keep]
            k = torch.exp(-torch.sqrt(dist2) / scale)
            keep = (k >= threshold) | (i == j)
            i, j, k = i[keep], j[keep], k[keep]
            k = torch.where(i == j, torch.full_like(k, 1.0 + shift), k)
            rows_out.append(i)
            cols_out.append(j.to(torch.int32))
            vals_out.append(k)
        r0 = r1
    rows = torch.cat(rows_out)
    indices = torch.cat(cols_out)
    tdt = torch.float32 if np.dtype(dtype) == np.float32 else torch.float64
    data = torch.cat(vals_out).to(tdt)
    indptr = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n), 0).to(
        torch.int32)
    return indptr, indices, data, perm.to(torch.int32)


def batched_correlation_sizes(count=64, seed=2, log2_min=10, log2_max=17,
                              scale_min=0.002, scale_max=0.05):
    """Sizes (log-uniform over 2^log2_min..2^log2_max, drawn first) and
    length scales (uniform) of a batch of correlation matrices, from numpy's
    PCG64 with ``seed``."""
    rng = np.random.default_rng(seed)
    sizes = np.round(2.0 ** rng.uniform(log2_min, log2_max, count)).astype(
        np.int64)
    scales = rng.uniform(scale_min, scale_max, count)
    return sizes, scales


def sparse_gram_design(nrows=8388608, ncols=2097152, nnz_per_col=16, seed=4,
                       dtype="float32"):
    """Sparse rectangular X (CSC): each column holds ``nnz_per_col`` distinct
    rows drawn uniformly, with N(0, 1) values (numpy PCG64 ``seed``)."""
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, nrows, size=(ncols, nnz_per_col), dtype=np.int64)
    rows.sort(axis=1)
    while True:
        dup = np.any(rows[:, 1:] == rows[:, :-1], axis=1)
        if not dup.any():
            break
        idx = np.flatnonzero(dup)
        fresh = rng.integers(0, nrows, size=(idx.size, nnz_per_col),
                             dtype=np.int64)
        fresh.sort(axis=1)
        rows[idx] = fresh
    vals = rng.standard_normal(ncols * nnz_per_col).astype(dtype)
    indptr = np.arange(0, ncols * nnz_per_col + 1, nnz_per_col,
                       dtype=np.int64)
    return sp.csc_matrix((vals, rows.reshape(-1).astype(np.int32), indptr),
                         shape=(nrows, ncols))
