"""The reference's own GPU SLQ (cuSPARSE SpMV, cuBLAS vector operations;
``oracle/_ref/libimate_ref_gpu.so``, compiled from its sources for sm_100a)
against this engine and the reference CPU SLQ on identical probes.

With one GPU the reference draws the same xoshiro256** stream as its CPU
path with one thread (``cu_trace_estimator.cu:241``), so every per-probe
sample is comparable.  Its reductions run in plain FP64 (cuBLAS), the CPU
path's in long double, so samples agree to ~1e-10, not bitwise.
"""

import numpy as np
import pytest

import imate_b200 as ib
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_gpu():
    if not ref.gpu_available():
        pytest.skip("reference GPU library not built (make -C oracle ref_gpu)")
    return ref.load_gpu()


def _rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.mark.parametrize("orth", [0, -1])
def test_reference_gpu_gram_toeplitz_matches_engine(cuda, ref_gpu, orth):
    B = ib.toeplitz(2.0, 1.0, 2048)
    kw = dict(min_num_samples=12, max_num_samples=12, error_rtol=1e-8,
              lanczos_degree=20, orthogonalize=orth, seed=0)
    want = ref.gpu_trace_estimator(B, "log", gram=True, **kw)
    cpu = ref.trace_estimator(B, "log", gram=True, **kw)
    tr, info = ib.logdet(B, gram=True, method="slq", gpu=True,
                         return_info=True, **kw)
    got = np.asarray(info["convergence"]["samples"], float)[:12]
    ref_s = want["samples"][:12, 0]
    assert _rel(ref_s, cpu["samples"][:12, 0]) < 1e-9
    assert _rel(got, ref_s) < 1e-9
    assert int(want["num_samples_used"][0]) == 12


def test_reference_gpu_correlation_matches_engine(cuda, ref_gpu):
    A = ib.correlation_matrix(4096, scale=0.02, shift=0.1, seed=1)
    kw = dict(min_num_samples=8, max_num_samples=8, error_rtol=1e-8,
              lanczos_degree=30, orthogonalize=-1, seed=3)
    for func, fn in (("log", ib.logdet), ("inv", ib.traceinv)):
        want = ref.gpu_trace_estimator(A, func, **kw)
        tr, info = fn(A, method="slq", gpu=True, return_info=True, **kw)
        got = np.asarray(info["convergence"]["samples"], float)[:8]
        assert _rel(got, want["samples"][:8, 0]) < 1e-9
        assert abs(float(tr) - float(want["trace"][0])) <= \
            1e-9 * abs(float(want["trace"][0]))


def test_reference_gpu_dense_matches_engine(cuda, ref_gpu):
    """Dense row-major input: the reference's cuDenseMatrix (cuBLAS gemv per
    probe) against this engine on identical probes.  An FP64 array runs this
    engine's FP64 sparse path (1e-9); an FP32 array runs the tensor-core
    dense product (3-term TF32 split, FP32 accumulation, FP64 reductions),
    whose samples stay within 2e-5 of the reference's FP64 samples on the
    same stored values -- closer than the reference's own FP32 path."""
    from imate_b200.sample_matrices import dense_correlation_matrix
    A64 = dense_correlation_matrix(2048, scale=0.03, shift=0.1, seed=4)
    kw = dict(min_num_samples=8, max_num_samples=8, error_rtol=0.0,
              lanczos_degree=30, orthogonalize=-1, seed=2)
    want64 = ref.gpu_trace_estimator(A64, "log", **kw)
    cpu64 = ref.trace_estimator(A64, "log", **kw)
    assert _rel(want64["samples"][:8, 0], cpu64["samples"][:8, 0]) < 1e-9
    tr, info = ib.logdet(A64, method="slq", gpu=True, return_info=True, **kw)
    got = np.asarray(info["convergence"]["samples"], float)[:8]
    assert _rel(got, want64["samples"][:8, 0]) < 1e-9

    A32 = A64.astype(np.float32)
    want = ref.gpu_trace_estimator(A32.astype(np.float64), "log", **kw)
    want32 = ref.gpu_trace_estimator(A32, "log", **kw)
    tr, info = ib.logdet(A32, method="slq", gpu=True, return_info=True, **kw)
    got = np.asarray(info["convergence"]["samples"], float)[:8]
    ref_s = want["samples"][:8, 0]
    assert _rel(got, ref_s) < 2e-5
    assert _rel(got, ref_s) <= _rel(want32["samples"][:8, 0], ref_s)
