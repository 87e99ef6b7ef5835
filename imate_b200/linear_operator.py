"""Linear operators: ``Matrix`` and ``AffineMatrixFunction``.

Mirror of imate's operator classes for the GPU SLQ path
(``imate/linear_operator/matrix.py:286-352``,
``imate/linear_operator/affine_matrix_function.py:278-360``): they hold the
host matrix and lazily create a device operator on first use, reusing it in
later calls.  Device arrays are PyTorch CUDA tensors; the engine
(``libslq_b200.so``) wraps them without copying and derives A^T (for
``gram=True``) or the CSR of A (for CSC input) into a PyTorch-allocated
workspace, with a deterministic device transpose.
"""

import ctypes
import os
from concurrent import futures

import numpy as np
import scipy.sparse as sp

from . import _lib

__all__ = ["LinearOperator", "Matrix", "AffineMatrixFunction",
           "GramAffineMatrixFunction"]


def _dtype_code(dtype):
    if dtype == np.float32:
        return _lib.SLQ_F32
    if dtype == np.float64:
        return _lib.SLQ_F64
    # py_cu_matrix.pyx:136-142 raises TypeError for other types on GPU
    raise TypeError('Data type should be either "float32" or "float64" on '
                    'GPU; got "%s".' % dtype)


class _Stager:
    """Host-to-device copies through a small ring of page-locked buffers
    (4 x 16 MB, allocated on first use and kept for the process): chunk i+1
    is copied into its buffer on the host while chunk i crosses the link, so
    a large array moves at close to the page-locked rate without pinning a
    buffer of its own size.  One copy at a time (a lock); every copy is
    ordered on the device's current stream."""

    CHUNK = 16 << 20
    SLOTS = 4

    def __init__(self):
        import threading
        self.lock = threading.Lock()
        self.bufs = None
        self.events = [None] * self.SLOTS
        self.next = 0

    def upload(self, a, dev):
        import torch
        with self.lock:
            if self.bufs is None:
                self.bufs = [torch.empty(self.CHUNK, dtype=torch.uint8,
                                         pin_memory=True)
                             for _ in range(self.SLOTS)]
            src = torch.from_numpy(a.reshape(-1).view(np.uint8))
            out = torch.empty(a.nbytes, dtype=torch.uint8, device=dev)
            stream = torch.cuda.current_stream(dev)
            for off in range(0, a.nbytes, self.CHUNK):
                slot = self.next % self.SLOTS
                self.next += 1
                if self.events[slot] is not None:
                    self.events[slot].synchronize()  # its last copy is done
                m = min(self.CHUNK, a.nbytes - off)
                buf = self.bufs[slot][:m]
                buf.copy_(src[off:off + m])
                out[off:off + m].copy_(buf, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
                self.events[slot] = ev
            return out.view(torch.from_numpy(np.empty(0, a.dtype)).dtype) \
                .reshape(a.shape)


_STAGER = _Stager()
# arrays of at least this many bytes go through the staging ring
_STAGE_MIN_BYTES = 4 << 20


_SIDE_STREAMS = {}
_UPLOADER = []
# a forked child has none of the parent's threads
os.register_at_fork(after_in_child=_UPLOADER.clear)


def _uploader():
    """The thread that uploads a matrix's values beside its set-up, kept for
    the process: a thread started per matrix spent milliseconds bringing up
    its own team of host copy threads on its first copy."""
    if not _UPLOADER:
        _UPLOADER.append(futures.ThreadPoolExecutor(
            max_workers=1, thread_name_prefix="slq-upload"))
    return _UPLOADER[0]


def _side_stream(dev):
    """One upload stream per device, kept for the process: the caching
    allocator keeps its blocks per stream, so a stream made per call would
    take fresh device memory for every upload."""
    import torch
    s = _SIDE_STREAMS.get(dev.index)
    if s is None:
        s = _SIDE_STREAMS[dev.index] = torch.cuda.Stream(device=dev)
    return s


def to_device(arr, dev, dtype=None):
    """A host array as a tensor on CUDA device ``dev``: small arrays by a
    plain copy, large ones through the page-locked staging ring (about five
    times the pageable rate on a PCIe 5 host link)."""
    import torch
    a = np.ascontiguousarray(arr, dtype=dtype)
    if a.nbytes < _STAGE_MIN_BYTES:
        return torch.from_numpy(a).to(dev)
    return _STAGER.upload(a, dev)


def _pattern(A):
    """int32 indptr / indices of a CSR matrix, as the host orders take them."""
    return (np.ascontiguousarray(A.indptr, dtype=np.int32),
            np.ascontiguousarray(A.indices, dtype=np.int32))


def order_spread(A, perm=None, sample_rows=20000):
    """Mean |position(i) - position(j)| over the nonzeros of sampled rows of
    a square sparse matrix (``slq_order_spread``; positions of ``perm``'s
    inverse, or the identity)."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    ip, ind = _pattern(A)
    p = None if perm is None else np.ascontiguousarray(perm, dtype=np.int32)
    out = ctypes.c_double(0.0)
    _lib.check(_lib.load().slq_order_spread(
        n, ip.ctypes.data, ind.ctypes.data,
        None if p is None else p.ctypes.data, int(sample_rows),
        ctypes.byref(out)))
    return float(out.value)


def locality_order(A, reorder="auto", device_pattern=None, spread=None):
    """Reverse Cuthill-McKee order (``rcm_order``) of a square sparse matrix,
    or None.

    'auto' reorders square matrices of order >= 16384 whose nonzeros lie far
    from the diagonal (mean |i - j| > 256 over sampled rows) when RCM
    shrinks that distance at least fourfold: the SpMM gathers of such
    matrices then stay inside a window that fits L2.  True always reorders a
    square matrix, False never.  ``device_pattern`` = (indptr, indices), A's
    CSR arrays as int32 CUDA tensors, computes the order on the device
    (``rcm_order_device``; the host computes it when that declines).
    ``spread``, if given, is ``order_spread(A, sample_rows=4096)``, already
    computed by the caller.
    """
    if reorder is False or A.shape[0] != A.shape[1]:
        return None
    A = sp.csr_matrix(A)
    n = A.shape[0]
    if reorder == "auto":
        if n < 16384 or A.nnz == 0:
            return None
        if spread is None:
            spread = order_spread(A, sample_rows=4096)
        if spread <= 256.0:
            return None
    perm = None
    if device_pattern is not None:
        perm = rcm_order_device(device_pattern[0], device_pattern[1], n,
                                A.nnz)
    if perm is None:
        perm = rcm_order(A)
    if reorder == "auto" and \
            order_spread(A, perm, sample_rows=4096) * 4.0 > spread:
        return None
    return np.ascontiguousarray(perm, dtype=np.int32)


def rcm_order(A):
    """Reverse Cuthill-McKee order of a square sparse pattern, taken as
    symmetric (``slq_rcm_order``; the order scipy's reverse_cuthill_mckee
    with symmetric_mode=True gives)."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    ip, ind = _pattern(A)
    order = np.empty(n, dtype=np.int32)
    _lib.check(_lib.load().slq_rcm_order(n, ip.ctypes.data, ind.ctypes.data,
                                         order.ctypes.data))
    return order


def rcm_order_device(indptr, indices, n, nnz, max_components=64):
    """``rcm_order`` of a square CSR pattern held on the device (int32 CUDA
    tensors) by ``slq_rcm_order_device``, as a host array; None when the
    pattern has more than ``max_components`` components (the host order is
    then the faster one)."""
    import torch
    lib = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(lib.slq_rcm_order_device_workspace_bytes(int(n),
                                                        ctypes.byref(nbytes)))
    dev = indptr.device
    ws = torch.empty(max(int(nbytes.value), 256), dtype=torch.uint8,
                     device=dev)
    order = torch.empty(max(int(n), 1), dtype=torch.int32, device=dev)
    done = ctypes.c_int(0)
    stream = torch.cuda.current_stream(dev)
    _lib.check(lib.slq_rcm_order_device(
        int(n), int(nnz), indptr.data_ptr(), indices.data_ptr(),
        int(max_components), order.data_ptr(), ctypes.byref(done),
        ws.data_ptr(), ws.numel(), stream.cuda_stream))
    if not done.value:
        return None
    return order[:int(n)].cpu().numpy()


def _group_fill(A, order, G, sample=256):
    """Mean fill of the dense union blocks of sampled groups of G
    consecutive rows of ``order`` (nnz / (G x union size);
    ``slq_group_fill``)."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    ip, ind = _pattern(A)
    o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
    out = ctypes.c_double(0.0)
    _lib.check(_lib.load().slq_group_fill(
        n, ip.ctypes.data, ind.ctypes.data,
        None if o is None else o.ctypes.data, int(G), int(sample),
        ctypes.byref(out)))
    return float(out.value)


def group_order(A, base_perm, G):
    """Row order whose consecutive groups of G rows share many columns
    (``slq_group_order``: each group is a seed row and its strongest
    neighbours, groups following ``base_perm``).  Square matrices only."""
    # the order does not depend on the order of a row's entries
    A = sp.csr_matrix(A)
    n = A.shape[0]
    ip = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ind = np.ascontiguousarray(A.indices, dtype=np.int32)
    data = A.data
    if data.dtype not in (np.float32, np.float64):
        data = data.astype(np.float64)
    data = np.ascontiguousarray(data)
    dt = _lib.SLQ_F64 if data.dtype == np.float64 else _lib.SLQ_F32
    base = None if base_perm is None else \
        np.ascontiguousarray(base_perm, dtype=np.int32)
    order = np.empty(n, dtype=np.int32)
    _lib.check(_lib.load().slq_group_order(
        n, ip.ctypes.data, ind.ctypes.data, data.ctypes.data, dt, int(G),
        None if base is None else base.ctypes.data, order.ctypes.data))
    return order


def block_order(A, group_order, group_rows=16, groups_per_block=8):
    """Row order whose consecutive blocks of ``groups_per_block`` groups of
    ``group_rows`` rows (the groups of ``group_order``, kept whole) have
    overlapping column sets (``slq_block_order``).  Square matrices only."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    ip, ind = _pattern(A)
    go = np.ascontiguousarray(group_order, dtype=np.int32)
    order = np.empty(n, dtype=np.int32)
    _lib.check(_lib.load().slq_block_order(
        n, ip.ctypes.data, ind.ctypes.data, go.ctypes.data, int(group_rows),
        int(groups_per_block), order.ctypes.data))
    return order


def block_group_order(A, base_perm, block_rows=128, group_rows=16):
    """Row order of blocks of ``block_rows`` rows, each of whole groups of
    ``group_rows`` rows, both aggregated around seeds and their strongest
    neighbours (``slq_block_group_order``; groups follow ``base_perm``).
    Serves the tensor-core block format and the row-group format at once.
    Square matrices only."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    ip, ind = _pattern(A)
    data = A.data
    if data.dtype not in (np.float32, np.float64):
        data = data.astype(np.float64)
    data = np.ascontiguousarray(data)
    dt = _lib.SLQ_F64 if data.dtype == np.float64 else _lib.SLQ_F32
    base = None if base_perm is None else \
        np.ascontiguousarray(base_perm, dtype=np.int32)
    order = np.empty(n, dtype=np.int32)
    _lib.check(_lib.load().slq_block_group_order(
        n, ip.ctypes.data, ind.ctypes.data, data.ctypes.data, dt,
        int(block_rows), int(group_rows),
        None if base is None else base.ctypes.data, order.ctypes.data))
    return order


def _fallback_order(A, base, group_rows, aggregate, blocks):
    """(group rows, row order) from the sampled row-group statistics
    (``group_rows_for``), the 16-row groups merged into 128-row blocks
    (``block_order``) when the operator gets the block format."""
    G, perm = group_rows_for(A, base, group_rows, aggregate=aggregate)
    if blocks and G == 16 and perm is not None and A.shape[0] == A.shape[1]:
        # 128-row blocks of eight 16-row groups whose column sets overlap
        # (the groups stay whole, so the row-group format keeps its fill)
        perm = block_order(A, perm, 16, 8)
    return G, perm


# blocks='auto' adds the tensor-core block format to float32 square
# matrices of at least this order
BLOCKS_AUTO_MIN_ROWS = 65536


def blocks_wanted(blocks, A):
    """Whether an operator over host matrix A gets the block format:
    ``blocks`` True (float32 only), False, or 'auto' -- float32 square
    matrices of order at least BLOCKS_AUTO_MIN_ROWS with at least 8 entries
    per row, where the tensor-core products beat the row-group kernels."""
    if blocks == "auto":
        return bool(A.dtype == np.float32 and A.shape[0] == A.shape[1] and
                    A.shape[0] >= BLOCKS_AUTO_MIN_ROWS and
                    A.nnz >= 8 * A.shape[0])
    if blocks not in (True, False):
        raise ValueError("blocks must be True, False or 'auto'")
    return bool(blocks) and A.dtype == np.float32


def group_rows_for(A, perm, group_rows="auto", sample=256, aggregate=True):
    """Row-group width for the device format (0 = CSR only) and the row
    order to store the matrix in: (G, perm).

    'auto' picks 16 (float32) when groups of 16 consecutive rows share
    enough columns that the dense union blocks are at least half filled,
    else 8 when groups of 8 fill at least 35% -- then one gathered probe row
    feeds ~3 useful FMAs or more -- else 0.  With ``aggregate`` (square
    matrices) the groups are formed by ``group_order`` on top of the base
    order ``perm``, which raises the fill of geometric matrices from ~0.45
    to ~0.75 (8 rows) and from ~0.32 to ~0.64 (16 rows); the aggregated
    order is kept only if it fills better.
    """
    A = sp.csr_matrix(A)
    n = A.shape[0]
    square = A.shape[0] == A.shape[1]
    base_perm = perm
    if group_rows is False or group_rows == 0:
        return 0, perm
    if group_rows != "auto" and group_rows not in (4, 8, 16):
        raise ValueError("group_rows must be 'auto', 0, 4, 8 or 16")
    if group_rows == "auto" and (A.nnz < 8 * n or n < 64):
        return 0, perm

    def best_order(G):
        base = perm if perm is not None else np.arange(n, dtype=np.int32)
        fill = _group_fill(A, base, G, sample)
        order = perm
        if aggregate and square and n >= 2 * G:
            agg = group_order(A, perm, G)
            afill = _group_fill(A, agg, G, sample)
            if afill > fill:
                order, fill = agg, afill
        return order, fill

    if group_rows != "auto":
        return int(group_rows), best_order(int(group_rows))[0]
    # 16-row groups (FP32 kernels only) when their blocks are at least half
    # full -- aggregated kernel matrices reach ~0.64 and then beat 8-row
    # groups (fewer gathers per FMA) -- else 8-row groups when at least
    # 35 % full, else CSR only
    if A.dtype == np.float32:
        order, fill = best_order(16)
        if fill >= 0.5:
            return 16, order
    order, fill = best_order(8)
    if fill >= 0.35:
        return 8, order
    return 0, base_perm


class _DeviceOperator:
    """An ``slq_op`` plus the tensors it points into (kept alive here)."""

    def __init__(self, A, affine, need_transpose, check_indices=True,
                 reorder="auto", group_rows="auto", aggregate=True,
                 blocks=False):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device is available for the SLQ "
                               "engine (it has no CPU path)")
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.dense = False
        self.block_formats = []
        if A is None:
            return  # from_device / from_dense fill the fields
        dev = self.device
        early = (A.format == "csr" and A.shape[0] == A.shape[1] and
                 A.has_sorted_indices and A.has_canonical_format and
                 max(A.shape) <= np.iinfo(np.int32).max and
                 A.nnz <= np.iinfo(np.int32).max)
        pattern = None
        upload = None
        pending_fill = None
        spread = None
        if early and reorder == "auto" and A.shape[0] >= 16384 and A.nnz:
            # the natural order's spread, before the uploads below compete
            # with it for the host cores
            spread = order_spread(A, sample_rows=4096)
        if early:
            # canonical CSR goes to the device as it is: upload the pattern
            # first, so that the locality order is computed there, and the
            # values on a helper thread while the host aggregates (both
            # release the GIL)
            # (the small index pointer first: a plain copy waits for the
            # stream's earlier copies)
            self.indptr = to_device(A.indptr, dev, np.int32)
            self.indices = to_device(A.indices, dev, np.int32)
            pattern = (self.indptr, self.indices)
            if A.dtype in (np.float32, np.float64):
                # its own stream, so that the copies run beside the locality
                # order's kernels instead of queueing behind them
                side = _side_stream(dev)

                def _values():
                    with torch.cuda.stream(side):
                        return to_device(A.data, dev)
                upload = _uploader().submit(_values)
        try:
            base = locality_order(A, reorder, device_pattern=pattern,
                                  spread=spread)
            # the values' upload overlaps the locality order (mostly device
            # work); it ends before the host orders below, whose threads it
            # would otherwise compete with
            if upload is not None:
                futures.wait([upload])
                main = torch.cuda.current_stream(dev)
                main.wait_stream(side)
                if upload.exception() is None:
                    upload.result().record_stream(main)
            blocks = blocks_wanted(blocks, A)
            self.group_rows = None
            if blocks and aggregate and group_rows in ("auto", 16) and \
                    A.shape[0] == A.shape[1] and A.shape[0] >= 256 and \
                    A.nnz >= 8 * A.shape[0]:
                # 128-row blocks aggregated around seeds, each split into
                # eight aggregated 16-row groups: one order for the block
                # format and the row-group format
                cand = block_group_order(A, base, 128, 16)
                self.group_rows, perm = 16, cand
                if group_rows != 16:
                    # the check that its 16-row groups fill well (else the
                    # orders of _fallback_order) runs on the upload thread,
                    # idle by now, beside the device build with it
                    pending_fill = _uploader().submit(_group_fill, A, cand, 16)
            if self.group_rows is None:
                self.group_rows, perm = _fallback_order(A, base, group_rows,
                                                        aggregate, blocks)
        finally:
            if upload is not None:
                futures.wait([upload])
        if upload is not None and upload.exception() is not None:
            raise upload.exception()
        if perm is not None and A.format != "csr":
            A = A.tocsr()
        fmt = _lib.SLQ_CSC if A.format == "csc" else _lib.SLQ_CSR
        if A.format not in ("csr", "csc"):
            A = A.tocsr()
            fmt = _lib.SLQ_CSR
        if not (A.has_sorted_indices and A.has_canonical_format):
            A = A.copy()
            A.sort_indices()
            A.sum_duplicates()
        self.dtype_code = _dtype_code(A.dtype)
        self.np_dtype = A.dtype
        self.shape = A.shape
        self.nnz = int(A.nnz)
        if max(A.shape) > np.iinfo(np.int32).max or \
                self.nnz > np.iinfo(np.int32).max:
            raise ValueError("matrix too large for 32-bit indices")
        if upload is not None and A.format == "csr":
            self.data = upload.result()
        else:
            self.data = to_device(A.data, dev)
        if not early:
            self.indices = to_device(A.indices, dev, np.int32)
            self.indptr = to_device(A.indptr, dev, np.int32)
        try:
            self._build(perm, fmt, affine, need_transpose, check_indices,
                        blocks)
        finally:
            if pending_fill is not None:
                futures.wait([pending_fill])
        if pending_fill is not None and pending_fill.result() < 0.5:
            # the candidate's 16-row groups fill poorly: rebuild with the
            # orders the row-group statistics pick
            self._destroy()
            self.group_rows, perm = _fallback_order(A, base, group_rows,
                                                    aggregate, blocks)
            self._build(perm, fmt, affine, need_transpose, check_indices,
                        blocks)

    def _build(self, perm, fmt, affine, need_transpose, check_indices,
               blocks):
        """The device operator over the uploaded arrays in row order
        ``perm`` (None = as stored), with the block format if ``blocks``."""
        import torch
        dev = self.device
        self.perm = None
        self.inv = None
        if perm is not None:
            self.perm = torch.from_numpy(perm).to(dev)
            self.inv = torch.empty_like(self.perm)
            self.inv[self.perm.long()] = torch.arange(
                perm.size, dtype=torch.int32, device=dev)
        self._create(fmt, affine, need_transpose, check_indices)
        if blocks:
            self.add_blocks(need_transpose or fmt == _lib.SLQ_CSC)

    def _destroy(self):
        """Release the engine's operator and the formats built for it."""
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self._lib.slq_operator_destroy(h)
            self.handle = ctypes.c_void_p(None)
        self.block_formats = []
        self.workspace = None

    @classmethod
    def from_device(cls, indptr, indices, data, shape, affine=False,
                    need_transpose=False, group_rows=8, fmt=_lib.SLQ_CSR,
                    check_indices=True, perm=None, blocks=False):
        """Operator over CSR (or CSC) arrays already on the device (torch
        int32 indptr / indices, float32 or float64 data), without copies.
        ``perm`` (a host int32 row order of a square CSR matrix, as
        ``locality_order`` / ``group_rows_for`` give) stores it reordered."""
        import torch
        self = cls(None, affine, need_transpose)
        self.data = data.contiguous()
        self.indices = indices.contiguous()
        self.indptr = indptr.contiguous()
        self.device = self.data.device
        if self.data.dtype == torch.float32:
            self.dtype_code, self.np_dtype = _lib.SLQ_F32, np.dtype(np.float32)
        elif self.data.dtype == torch.float64:
            self.dtype_code, self.np_dtype = _lib.SLQ_F64, np.dtype(np.float64)
        else:
            raise TypeError("data must be float32 or float64")
        self.shape = tuple(int(x) for x in shape)
        self.nnz = int(self.indices.numel())
        self.group_rows = int(group_rows)
        self.perm = None
        self.inv = None
        if perm is not None:
            pm = torch.from_numpy(np.ascontiguousarray(perm, dtype=np.int32))
            self.perm = pm.to(self.device)
            self.inv = torch.empty_like(self.perm)
            self.inv[self.perm.long()] = torch.arange(
                pm.numel(), dtype=torch.int32, device=self.device)
        self._create(fmt, affine, need_transpose, check_indices)
        if blocks and self.dtype_code == _lib.SLQ_F32:
            self.add_blocks(need_transpose or fmt == _lib.SLQ_CSC)
        return self

    def blocks_info(self, transpose=False):
        """(blocks, stages) of the block format of A (or A^T); (0, 0) when
        the operator has none (``slq_operator_blocks_info``)."""
        nb = ctypes.c_int64(0)
        ns = ctypes.c_int64(0)
        _lib.check(self._lib.slq_operator_blocks_info(
            self.handle, int(bool(transpose)), ctypes.byref(nb),
            ctypes.byref(ns)))
        return int(nb.value), int(ns.value)

    def add_blocks(self, with_transpose=False):
        """Attach the tensor-core block format (``slq_operator_add_blocks``:
        128-row blocks of the stored rows, float32) for A and, with
        ``with_transpose``, for A^T; block-wide SpMMs (128 or 256 probes)
        then run on the tensor cores."""
        import torch
        lib = self._lib
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for tr in ((0, 1) if with_transpose else (0,)):
            nb = ctypes.c_size_t(0)
            _lib.check(lib.slq_operator_blocks_scratch_bytes(
                self.handle, tr, ctypes.byref(nb)))
            scratch = torch.empty(max(int(nb.value), 256), dtype=torch.uint8,
                                  device=self.device)
            fb = ctypes.c_size_t(0)
            _lib.check(lib.slq_operator_blocks_bytes(
                self.handle, tr, scratch.data_ptr(), scratch.numel(), stream,
                ctypes.byref(fb)))
            fmt = torch.empty(max(int(fb.value), 256), dtype=torch.uint8,
                              device=self.device)
            _lib.check(lib.slq_operator_add_blocks(
                self.handle, tr, scratch.data_ptr(), scratch.numel(),
                fmt.data_ptr(), fmt.numel(), stream))
            del scratch
            self.block_formats.append(fmt)

    @classmethod
    def from_dense(cls, A, affine=False, need_transpose=False):
        """Dense float32 operator over a host array A (row-major copy on the
        device; ``slq_dense_operator_create``: TF32 parts of A, and of A^T
        with ``need_transpose``, for the tensor-core product)."""
        import torch
        self = cls(None, affine, need_transpose)
        A = np.ascontiguousarray(A, dtype=np.float32)
        self.data = to_device(A, self.device)
        self.indices = None
        self.indptr = None
        self.dtype_code, self.np_dtype = _lib.SLQ_F32, np.dtype(np.float32)
        self.shape = tuple(int(x) for x in A.shape)
        self.nnz = int(A.size)
        self.group_rows = 0
        self.perm = None
        self.inv = None
        self.dense = True
        lib = _lib.load()
        nbytes = ctypes.c_size_t(0)
        _lib.check(lib.slq_dense_operator_workspace_bytes(
            self.shape[0], self.shape[1], _lib.SLQ_F32, int(need_transpose),
            ctypes.byref(nbytes)))
        self.workspace = torch.empty(max(int(nbytes.value), 256),
                                     dtype=torch.uint8, device=self.device)
        self.handle = ctypes.c_void_p(None)
        stream = torch.cuda.current_stream(self.device)
        _lib.check(lib.slq_dense_operator_create(
            self.data.data_ptr(), self.shape[0], self.shape[1], _lib.SLQ_F32,
            int(affine), int(need_transpose), self.workspace.data_ptr(),
            self.workspace.numel(), stream.cuda_stream,
            ctypes.byref(self.handle)))
        self.affine = affine
        self.has_transpose = bool(need_transpose)
        self._lib = lib
        return self

    def _create(self, fmt, affine, need_transpose, check_indices):
        import torch
        lib = _lib.load()
        dev = self.device
        nbytes = ctypes.c_size_t(0)
        _lib.check(lib.slq_operator_workspace_bytes(
            self.shape[0], self.shape[1], self.nnz, self.dtype_code, fmt,
            int(need_transpose), int(self.perm is not None), self.group_rows,
            ctypes.byref(nbytes)))
        self.workspace = torch.empty(max(int(nbytes.value), 256),
                                     dtype=torch.uint8, device=dev)
        self.handle = ctypes.c_void_p(None)
        stream = torch.cuda.current_stream(dev)
        _lib.check(lib.slq_operator_create(
            self.data.data_ptr(), self.indices.data_ptr(),
            self.indptr.data_ptr(), self.shape[0], self.shape[1], self.nnz,
            self.dtype_code, fmt, int(affine), int(need_transpose),
            int(check_indices),
            self.perm.data_ptr() if self.perm is not None else None,
            self.group_rows, self.workspace.data_ptr(),
            self.workspace.numel(), stream.cuda_stream,
            ctypes.byref(self.handle)))
        self.affine = affine
        self.has_transpose = bool(need_transpose) or fmt == _lib.SLQ_CSC
        self._lib = lib

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.slq_operator_destroy(h)
                self.handle = ctypes.c_void_p(None)
            except (AttributeError, TypeError):
                pass  # interpreter shutdown: ctypes is already torn down

    def dot(self, x, transpose=False, t=0.0):
        """y = A x (or A^T x) (+ t x for affine operators) for a torch
        tensor x of shape [len] or [len, width] on the operator's device."""
        import torch
        squeeze = x.dim() == 1
        X = x.reshape(x.shape[0], -1)
        width = X.shape[1]
        wpad = 1
        while wpad < width:
            wpad *= 2
        tdt = torch.float64 if self.dtype_code == _lib.SLQ_F64 else \
            torch.float32
        Xp = torch.zeros((X.shape[0], wpad), dtype=tdt, device=self.device)
        Xp[:, :width] = X if self.perm is None else X[self.perm.long()]
        rows = self.shape[1] if transpose else self.shape[0]
        Y = torch.empty((rows, wpad), dtype=tdt, device=self.device)
        stream = torch.cuda.current_stream(self.device)
        _lib.check(self._lib.slq_operator_dot(
            self.handle, int(transpose), float(t), Xp.data_ptr(),
            Y.data_ptr(), wpad, stream.cuda_stream))
        Y = Y[:, :width]
        if self.perm is not None:
            Y = Y[self.inv.long()]
        return Y.reshape(-1) if squeeze else Y


class LinearOperator:
    """Base class (``imate/linear_operator/linear_operator.py``)."""

    def __init__(self):
        self.A = None
        self.num_parameters = 0
        self._device_ops = {}
        self.data_type_name = None

    def set_data_type_name(self, A):
        self.data_type_name = str(np.dtype(A.dtype).name).encode()

    def get_data_type_name(self):
        return self.data_type_name

    def get_num_rows(self):
        return self.A.shape[0]

    def get_num_columns(self):
        return self.A.shape[1]

    def is_sparse(self):
        return sp.issparse(self.A)

    def get_nnz(self):
        if sp.issparse(self.A):
            return self.A.nnz
        return self.A.shape[0] * self.A.shape[1]

    def get_density(self):
        return self.get_nnz() / (self.A.shape[0] * self.A.shape[1])

    def get_num_parameters(self):
        return self.num_parameters

    def _affine(self):
        return False

    def get_device_operator(self, need_transpose=False):
        """Device operator on the current CUDA device, created on first use
        and reused (``linear_operator.py:114-147``).  Square matrices may be
        stored in a locality order (see ``locality_order``; the ``reorder``
        attribute, default 'auto')."""
        import torch
        dev = torch.cuda.current_device() if torch.cuda.is_available() else -1
        key = (dev, bool(need_transpose))
        op = self._device_ops.get(key)
        if op is None and not need_transpose:
            op = self._device_ops.get((dev, True))
        if op is None and isinstance(self.A, np.ndarray) and \
                self.A.dtype == np.float32 and self.A.ndim == 2:
            # dense float32: tensor-core product (cuDenseMatrix's role)
            op = _DeviceOperator.from_dense(self.A, self._affine(),
                                            need_transpose)
            self._device_ops[key] = op
        if op is None:
            A = self.A if sp.issparse(self.A) else sp.csr_matrix(self.A)
            op = _DeviceOperator(A, self._affine(), need_transpose,
                                 reorder=getattr(self, "reorder", "auto"),
                                 group_rows=getattr(self, "group_rows",
                                                    "auto"),
                                 aggregate=getattr(self, "aggregate", True),
                                 blocks=getattr(self, "blocks", False))
            self._device_ops[key] = op
        return op

    def release(self):
        """Drop the cached device copies."""
        self._device_ops.clear()


class Matrix(LinearOperator):
    """A fixed matrix (``imate/linear_operator/matrix.py``).

    ``reorder`` ('auto', True or False) selects the device storage order of
    square matrices (see ``locality_order``); results do not depend on it
    beyond floating-point summation order.  ``group_rows`` ('auto', 0, 4, 8
    or 16) adds the row-group format and ``aggregate`` lets its groups be
    formed by neighbour aggregation (see ``group_rows_for``); the format
    itself changes no result bit, the aggregated order only the order of
    floating-point sums.  ``blocks`` (float32; 'auto', True or False) stores
    the rows in 128-row blocks of aggregated 16-row groups
    (``block_group_order``) and adds the tensor-core block format, which
    block-wide SpMMs (128 or 256 probes) then use; results change only by
    rounding (FP16 hi/lo parts of scaled values, FP32 accumulation: samples
    within about 1e-5 of FP64).  'auto' adds it to float32 square matrices
    of order at least 65536 (``blocks_wanted``).
    """

    def __init__(self, A, reorder="auto", group_rows="auto", aggregate=True,
                 blocks="auto"):
        super().__init__()
        self.reorder = reorder
        self.group_rows = group_rows
        self.aggregate = aggregate
        self.blocks = blocks
        if not (sp.issparse(A) or isinstance(A, np.ndarray)):
            raise TypeError("A should be a numpy array or a scipy sparse "
                            "matrix.")
        self.A = A
        self.num_parameters = 0
        self.set_data_type_name(A)


def _is_identity(B, n):
    if B is None:
        return True
    if np.isscalar(B):
        return False
    Bs = sp.csr_matrix(B)
    if Bs.shape != (n, n):
        return False
    Bs = Bs.copy()
    Bs.eliminate_zeros()
    d = Bs.diagonal()
    return Bs.nnz == n and np.all(d == 1)


class AffineMatrixFunction(LinearOperator):
    """A + t B (``imate/linear_operator/affine_matrix_function.py:278-360``).

    With B the identity the eigenvalues of A + t I are those of A shifted by
    t, so one Krylov run per probe serves every t
    (``imate/_c_linear_operator/c_affine_matrix_function.cpp:98-113``).  With
    another B no such relation holds and the reference runs a Krylov sequence
    per inquiry on each probe (``imate/_c_trace_estimator/c_trace_estimator.cpp:
    496-556``, ``cu_csr_affine_matrix_function.cu:124-211``); here each t
    gets its own device operator over the union pattern of A and B with the
    values of A + t B (written on the device), in the row order and
    row-group width chosen once for that pattern.
    """

    def __init__(self, A, B=None, reorder="auto", group_rows="auto",
                 blocks=False):
        super().__init__()
        self.reorder = reorder
        self.group_rows = group_rows
        self.blocks = blocks
        self.A = A
        self.B = B
        self.num_parameters = 1
        self.set_data_type_name(A)
        self.general_B = not _is_identity(B, A.shape[0])
        if self.general_B:
            if np.isscalar(B) or not (sp.issparse(B) or
                                      isinstance(B, np.ndarray)):
                raise TypeError("B should be a numpy array or a scipy sparse "
                                "matrix.")
            if B.shape != A.shape:
                raise ValueError("A and B should have the same shape.")
            self._union = None
            self._op_t = None

    def _affine(self):
        return not self.general_B

    def _union_pattern(self):
        """Host CSR pattern of A ∪ B and A's and B's values on it, with the
        row order and row-group width of that pattern (computed once)."""
        if self._union is not None:
            return self._union
        dt = np.dtype(self.get_data_type_name().decode())
        Ac = sp.coo_matrix(self.A)
        Bc = sp.coo_matrix(self.B)
        n, m = self.A.shape
        key = np.concatenate([Ac.row.astype(np.int64) * m + Ac.col,
                              Bc.row.astype(np.int64) * m + Bc.col])
        uk, where = np.unique(key, return_inverse=True)
        a = np.zeros(uk.size, dtype=np.float64)
        b = np.zeros(uk.size, dtype=np.float64)
        np.add.at(a, where[:Ac.nnz], Ac.data)
        np.add.at(b, where[Ac.nnz:], Bc.data)
        rows = uk // m
        indptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
        if max(n, m) > np.iinfo(np.int32).max or \
                uk.size > np.iinfo(np.int32).max:
            raise ValueError("matrix too large for 32-bit indices")
        P = sp.csr_matrix((np.abs(a) + np.abs(b), (uk % m).astype(np.int32),
                           indptr.astype(np.int32)), shape=(n, m))
        base = locality_order(P, self.reorder)
        G, perm = group_rows_for(P, base, self.group_rows)
        self._union = dict(indptr=P.indptr, indices=P.indices,
                           a=a.astype(dt), b=b.astype(dt), G=int(G),
                           perm=perm, shape=(n, m), device=None)
        return self._union

    def device_operator_for(self, t, need_transpose=False):
        """The device operator of A + t B (general B; the previous one is
        released first)."""
        import torch
        U = self._union_pattern()
        dev = torch.device("cuda", torch.cuda.current_device())
        if U["device"] is None or U["device"][0] != dev:
            U["device"] = (dev,
                           torch.from_numpy(U["indptr"]).to(dev),
                           torch.from_numpy(U["indices"]).to(dev),
                           torch.from_numpy(U["a"]).to(dev),
                           torch.from_numpy(U["b"]).to(dev))
        _, ip, ind, a, b = U["device"]
        self._op_t = None
        vals = torch.add(a, b, alpha=float(t))
        self._op_t = _DeviceOperator.from_device(
            ip, ind, vals, U["shape"], affine=False,
            need_transpose=need_transpose, group_rows=U["G"],
            perm=U["perm"])
        return self._op_t

    def get_device_operator(self, need_transpose=False):
        if not self.general_B:
            return super().get_device_operator(need_transpose)
        return self.device_operator_for(0.0, need_transpose)

    def release(self):
        super().release()
        if self.general_B:
            self._op_t = None
            if self._union is not None:
                self._union["device"] = None


class DeviceMatrix(LinearOperator):
    """A sparse matrix whose CSR arrays are already on the GPU (torch
    tensors: int32 indptr and indices, float32 or float64 data), e.g. from
    ``sample_matrices.correlation_matrix_device``.  No host copy is made;
    rows must list their columns in increasing order.  ``group_rows``
    ('auto' = 16 for float32 and 8 for float64, or 0, 4, 8, 16) adds the
    row-group format on the device (the autotuner then picks between its
    kernels and CSR); no reordering is done, so the rows should already be
    in a local order (as the device builder's cell order is)."""

    def __init__(self, indptr, indices, data, shape, group_rows="auto"):
        super().__init__()
        self.indptr, self.indices, self.data = indptr, indices, data
        self.shape = tuple(int(x) for x in shape)
        if group_rows == "auto":
            # 16-row groups (FP32 kernels, including the tensor-core one),
            # else 8
            import torch
            group_rows = 16 if data.dtype == torch.float32 else 8
        self.group_rows = int(group_rows)
        self.num_parameters = 0
        self.data_type_name = str(data.dtype).replace("torch.", "").encode()

    def get_num_rows(self):
        return self.shape[0]

    def get_num_columns(self):
        return self.shape[1]

    def is_sparse(self):
        return True

    def get_nnz(self):
        return int(self.indices.numel())

    def get_density(self):
        return self.get_nnz() / float(self.shape[0] * self.shape[1])

    def get_device_operator(self, need_transpose=False):
        key = (self.data.device.index, bool(need_transpose))
        op = self._device_ops.get(key)
        if op is None and not need_transpose:
            op = self._device_ops.get((self.data.device.index, True))
        if op is None:
            op = _DeviceOperator.from_device(
                self.indptr, self.indices, self.data, self.shape,
                affine=self._affine(), need_transpose=need_transpose,
                group_rows=self.group_rows)
            self._device_ops[key] = op
        return op


class GramAffineMatrixFunction(LinearOperator):
    """A^T A + t I for a sparse (possibly rectangular) A.

    imate can form the Gram matrix of A (``gram=True``) but not shift it:
    its AffineMatrixFunction with ``gram=True`` means (A + t I)^T (A + t I).
    This operator is the shifted Gram matrix itself, an n x n SPD operator
    (n = columns of A) used with ``gram=False``; the engine runs Lanczos on
    it as x -> A^T (A x) + t x (normal-equations mode).  Its eigenvalues
    shift with t, so one Krylov run per probe serves a sweep of t.
    """

    def __init__(self, A, blocks=False):
        super().__init__()
        if not sp.issparse(A):
            A = sp.csr_matrix(A)
        self.A = A
        self.num_parameters = 1
        self.normal_equations = True
        self.reorder = False
        self.group_rows = 0
        self.blocks = blocks
        self.set_data_type_name(A)

    def _affine(self):
        return True

    def get_num_rows(self):
        return self.A.shape[1]

    def get_num_columns(self):
        return self.A.shape[1]

    def get_density(self):
        n = self.A.shape[1]
        return self.A.nnz / float(n * n)
