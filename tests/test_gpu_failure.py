"""Failure paths, exercised without faulting the GPU.

- A bounded device wait that runs out: the test hook
  slq_debug_fail_stream_waits makes the next streaming launch treat its first
  mbarrier wait as timed out.  The kernel takes the path of a real timeout
  (error word set, its issued copies drained with the full bound) and the
  call returns SLQ_ERR_TIMEOUT; the next estimate in the same process must
  match the reference's golden samples to the FP64 parity bar (1e-10).
- Per-probe flags (info['engine']['probe_status']): NaN in the matrix data
  marks every sample non-finite; an indefinite matrix marks the samples with
  a non-positive node under log; both warn.  The reference only warns for a
  vanishing Gram-Schmidt vector (c_orthogonalization.cpp:186-192)."""

import warnings

import numpy as np
import pytest
import scipy.sparse as sp

import imate_b200 as ib
from imate_b200 import _lib

pytestmark = pytest.mark.gpu


def _golden_run(orth=-1):
    B = ib.toeplitz(2.0, 1.0, 16384)
    return ib.logdet(B, gram=True, method="slq", gpu=True, return_info=True,
                     min_num_samples=50, max_num_samples=200, error_rtol=1e-3,
                     lanczos_degree=30, orthogonalize=orth, seed=0)


def test_device_wait_timeout_is_reported_and_the_next_run_is_clean(cuda,
                                                                  golden):
    lib = _lib.load()
    _lib.check(lib.slq_debug_fail_stream_waits(1))
    try:
        with pytest.raises(_lib.SlqError) as e:
            _golden_run()
        assert e.value.status == 8  # SLQ_ERR_TIMEOUT
    finally:
        _lib.check(lib.slq_debug_fail_stream_waits(0))
    tr, info = _golden_run()
    g = golden("estimator.npz")
    key = "c1_log_orth-1"
    used = int(np.atleast_1d(g[key + "_num_samples_used"])[0])
    assert int(info["convergence"]["num_samples_used"]) == used
    order = g[key + "_processed_samples_indices"][:used]
    got = np.asarray(info["convergence"]["samples"], float)[order]
    want = g[key + "_samples"][order].ravel()
    assert np.max(np.abs(got - want) / np.abs(want)) < 1e-10
    assert np.all(info["engine"]["probe_status"][order] == 0)


def test_nan_in_matrix_flags_every_sample(cuda):
    A = ib.toeplitz(2.0, 1.0, 3000).tocsr()
    A = (A.T @ A).tocsr()
    A.data[17] = np.nan
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        tr, info = ib.logdet(A, method="slq", gpu=True, return_info=True,
                             min_num_samples=8, max_num_samples=8,
                             lanczos_degree=10, seed=3)
    st = np.asarray(info["engine"]["probe_status"][:8])
    assert np.all(st & _lib.PROBE_NONFINITE)
    assert np.all(st & _lib.PROBE_SAMPLE)
    assert np.isnan(tr)
    assert any("non-finite" in str(x.message) for x in w)


def test_indefinite_matrix_flags_nonpositive_nodes(cuda):
    d = np.r_[np.full(50, 2.0), np.full(50, -1.0)]
    A = sp.diags(d).tocsr()
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        tr, info = ib.logdet(A, method="slq", gpu=True, return_info=True,
                             min_num_samples=3, max_num_samples=3,
                             lanczos_degree=8, seed=2)
    st = np.asarray(info["engine"]["probe_status"][:3])
    assert np.all(st & _lib.PROBE_NODE)
    assert not np.any(st & _lib.PROBE_NONFINITE)
    assert any("non-positive quadrature node" in str(x.message) for x in w)
    # the same matrix is fine for traceinv (no node is zero): no flags
    tr, info = ib.traceinv(A, method="slq", gpu=True, return_info=True,
                           min_num_samples=3, max_num_samples=3,
                           lanczos_degree=8, seed=2)
    assert np.all(np.asarray(info["engine"]["probe_status"][:3]) == 0)
