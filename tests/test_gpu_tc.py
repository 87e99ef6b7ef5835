"""Tensor-core (tcgen05) building blocks of the tensor-core SpMM, checked on
one tile against numpy.  With small-integer operands every product and sum
is exact in TF32 and FP32, so every mode must reproduce A @ B exactly; with
random FP32 operands the three-term TF32 split must reach FP32-level
accuracy (max error <= 2e-6 of max |D|; the split's stated error is about
2^-21 per product), while one TF32 term alone is ~1e-3 off."""

import numpy as np
import pytest

from imate_b200 import _lib

pytestmark = pytest.mark.gpu


def _tile(lib, a, b, mode):
    import torch
    A = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    B = torch.from_numpy(np.ascontiguousarray(b, np.float32)).cuda()
    D = torch.full((128, 16), np.nan, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.slq_tc_selftest(A.data_ptr(), B.data_ptr(), D.data_ptr(),
                                   int(mode), err.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream))
    return D.cpu().numpy()


def _ints(seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(-8, 9, (128, 8)).astype(np.float32)
    b = rng.integers(-8, 9, (8, 16)).astype(np.float32)
    return a, b


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_tc_tile_exact_on_small_integers(cuda, mode):
    a, b = _ints(mode)
    want = a.astype(np.float64) @ b.astype(np.float64)
    assert np.array_equal(_tile(cuda, a, b, mode), want)


def test_tc_tensor_memory_round_trip(cuda):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((128, 8)).astype(np.float32)
    b = np.zeros((8, 16), np.float32)
    d = _tile(cuda, a, b, 2)
    hi, lo = d[:, :8].astype(np.float64), d[:, 8:].astype(np.float64)
    # hi carries 11 significant bits, hi + lo reproduces a to 2^-21
    assert np.max(np.abs(hi - a) / np.abs(a)) <= 2.0 ** -11
    assert np.max(np.abs(hi + lo - a) / np.abs(a)) <= 2.0 ** -21


def test_tc_tile_three_term_split_reaches_fp32_accuracy(cuda):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((128, 8)).astype(np.float32)
    b = rng.standard_normal((8, 16)).astype(np.float32)
    want = a.astype(np.float64) @ b.astype(np.float64)
    scale = np.max(np.abs(want))
    d3 = _tile(cuda, a, b, 1)
    d1 = _tile(cuda, a, b, 0)
    assert np.max(np.abs(d3 - want)) <= 2e-6 * scale
    assert np.max(np.abs(d1 - want)) > 1e-5 * scale  # one TF32 term is not


def _run(A, gram, width, variant_kind=None, **kw):
    import imate_b200 as ib
    from imate_b200.batch import tune_operator, set_variant
    M = ib.Matrix(A, reorder=True, group_rows=16, aggregate=True)
    op = M.get_device_operator(need_transpose=gram)
    assert op.group_rows == 16
    if variant_kind is not None:
        for tr in ((False, True) if gram else (False,)):
            cands, _ = tune_operator(op, width, transpose=tr, reps=1)
            idx = [i for i, c in enumerate(cands) if c["kind"] == variant_kind]
            assert idx, cands
            set_variant(op, width, idx[0], transpose=tr)
    eng = ib.EngineOptions(block_size=width, return_coefficients=True)
    return ib.logdet(M, gram=gram, method="slq", gpu=True, return_info=True,
                     engine=eng, **kw)


@pytest.mark.parametrize("gram", [False, True])
@pytest.mark.parametrize("width", [128, 256])
def test_tensor_core_spmm_in_estimator(cuda, gram, width):
    # the estimator with the tensor-core SpMM against the same run with the
    # CUDA-core row-group kernel (same operator order, same probes) and
    # against FP64: per-sample agreement to FP32 level (1e-5 relative)
    import imate_b200 as ib
    A = ib.correlation_matrix(8000, scale=0.02, threshold=0.05, shift=0.2,
                              seed=3, dtype=np.float32)
    kw = dict(min_num_samples=width, max_num_samples=width, error_rtol=0.0,
              lanczos_degree=16, orthogonalize=-1, seed=4)
    t_tc, i_tc = _run(A, gram, width, "row-group-tc", **kw)
    t_rg, i_rg = _run(A, gram, width, "row-group", **kw)
    s_tc = np.asarray(i_tc["convergence"]["samples"], float)
    s_rg = np.asarray(i_rg["convergence"]["samples"], float)
    assert np.max(np.abs(s_tc - s_rg) / np.abs(s_rg)) < 1e-5
    a_tc, a_rg = i_tc["engine"]["alpha"], i_rg["engine"]["alpha"]
    assert np.max(np.abs(a_tc - a_rg) / np.abs(a_rg)) < 1e-5
    t64, i64 = ib.logdet(A.astype(np.float64), gram=gram, method="slq",
                         gpu=True, return_info=True, **kw)
    s64 = np.asarray(i64["convergence"]["samples"], float)
    assert np.max(np.abs(s_tc - s64) / np.abs(s64)) < 1e-5


def test_tensor_core_candidate_is_tuned(cuda):
    import imate_b200 as ib
    from imate_b200.batch import tune_operator
    A = ib.correlation_matrix(8000, scale=0.02, threshold=0.05, shift=0.2,
                              seed=3, dtype=np.float32)
    op = ib.Matrix(A, group_rows=16).get_device_operator()
    for w in (128, 256):
        cands, chosen = tune_operator(op, w, reps=2)
        tcs = [c for c in cands if c["kind"] == "row-group-tc"]
        assert len(tcs) == 1 and tcs[0]["ms"] > 0
    cands, _ = tune_operator(op, 64, reps=1)
    assert not [c for c in cands if c["kind"] == "row-group-tc"]


def _tile_mn(lib, a, b, gather):
    import torch
    A = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    B = torch.from_numpy(np.ascontiguousarray(b, np.float32)).cuda()
    D = torch.full((128, 32), np.nan, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.slq_tc_selftest_mn(A.data_ptr(), B.data_ptr(), D.data_ptr(),
                                      int(gather), err.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream))
    return D.cpu().numpy()


@pytest.mark.parametrize("gather", [0, 1])
def test_tc_mn_major_operand_exact_on_small_integers(cuda, gather):
    # B in the 128-byte-swizzled MN-major layout (gather 1: rows brought by
    # TMA tile::gather4 in the order perm), one kind::tf32 MMA
    rng = np.random.default_rng(11 + gather)
    a = rng.integers(-8, 9, (128, 8)).astype(np.float32)
    b = rng.integers(-8, 9, (8, 32)).astype(np.float32)
    perm = [3, 0, 7, 1, 6, 2, 5, 4] if gather else list(range(8))
    want = a.astype(np.float64) @ b[perm].astype(np.float64)
    assert np.array_equal(_tile_mn(cuda, a, b, gather), want)
