"""The headline workload at its full size through the public API: the
sparse SPD correlation matrix with n = 262144 (48.07M nonzeros, diagonal
shift 0.1), FP32 values, 256 probes from the parity stream, 50 Lanczos steps,
full reorthogonalisation.

Both device formats run: the row-group path (locality order, aggregated
16-row groups, TMA row-group SpMM; Matrix(blocks=False)) and the default for
a float32 matrix of this order, the tensor-core block format (128-row
blocks of aggregated 16-row groups, FP16 three-product SpMM).  Bars, on
identical probes:
- row-group path against the FP64 engine: 1e-6 relative per sample (FP32
  products, FP64 reductions);
- block path against the FP64 engine: 1e-5 relative per sample (FP16 hi/lo
  products and the tensor core's FP32 accumulation, which shrinks |y| by a
  few 1e-6);
- the 256-probe estimate against the FP64 sparse-LU logdet of the same
  matrix (tests/golden/c2prime_oracle.json): 1e-3 relative (the Monte-Carlo
  error is ~1e-4)."""

import json
import os

import numpy as np
import pytest

import imate_b200 as ib

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def headline_matrix():
    return ib.correlation_matrix(262144, scale=0.005, threshold=0.05,
                                 shift=0.1, seed=1, dtype="float32")


def _logdet(M, block, probes):
    kw = dict(method="slq", gpu=True, return_info=True,
              min_num_samples=probes, max_num_samples=probes, error_rtol=0.0,
              lanczos_degree=50, orthogonalize=-1, seed=0)
    return ib.logdet(M, engine=ib.EngineOptions(block_size=block,
                                                rng="parity"), **kw)


def test_headline_workload_matches_fp64_and_sparse_lu(cuda, headline_matrix):
    import torch
    A = headline_matrix
    with open(os.path.join(HERE, "golden", "c2prime_oracle.json")) as f:
        oracle = json.load(f)
    assert oracle["n"] == A.shape[0] and oracle["nnz"] == A.nnz

    # FP64 engine on the first 8 probes (the same parity-stream probes)
    _, i64 = _logdet(ib.Matrix(A.astype(np.float64)), 8, 8)
    s64 = np.asarray(i64["convergence"]["samples"][:8], float)
    torch.cuda.empty_cache()

    Mr = ib.Matrix(A, blocks=False)
    tr_r, ir = _logdet(Mr, 256, 256)
    assert Mr.get_device_operator().group_rows == 16
    assert not Mr.get_device_operator().block_formats
    sr = np.asarray(ir["convergence"]["samples"], float)
    del Mr
    torch.cuda.empty_cache()

    Mb = ib.Matrix(A)  # blocks='auto'
    tr_b, ibk = _logdet(Mb, 256, 256)
    assert Mb.get_device_operator().block_formats
    assert Mb.get_device_operator().group_rows == 16
    assert "blocks" in ibk["precision"]["spmm"]
    sb = np.asarray(ibk["convergence"]["samples"], float)
    del Mb
    torch.cuda.empty_cache()

    assert np.all(np.asarray(ir["engine"]["lanczos_size"][:256]) == 50)
    assert np.max(np.abs(sr[:8] - s64) / np.abs(s64)) < 1e-6
    assert np.max(np.abs(sb[:8] - s64) / np.abs(s64)) < 1e-5
    # every sample of the two FP32 paths agrees to the block path's bar
    assert np.max(np.abs(sb - sr) / np.abs(sr)) < 1e-5
    for tr in (tr_r, tr_b):
        assert abs(tr - oracle["logdet"]) / abs(oracle["logdet"]) < 1e-3
