"""Device network kernels against the numpy checker, and the learned sweep
surrogate against SLQ.  Tolerances: FP32 kernels vs FP64 numpy -- forward
within 2e-5 relative, gradients within 1e-3 of the largest component;
surrogate answers within the gate's 1e-3 relative error at all 512 points
of the sweep (trusted intervals within 1e-3, fallback points SLQ itself)."""

import time

import numpy as np
import pytest

import imate_b200 as ib
from imate_b200 import _lib
from imate_b200.surrogate import SweepSurrogate, init_params
from oracle import mlp_oracle

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def test_forward_matches_numpy(cuda):
    p = init_params(3)
    x = np.linspace(-1.2, 1.2, 777).astype(np.float32)
    P, X = _dev(p), _dev(x)
    import torch
    Y = torch.empty_like(X)
    _lib.check(cuda.slq_mlp_forward(P.data_ptr(), X.data_ptr(), x.size,
                                    Y.data_ptr(), _stream()))
    want = mlp_oracle.forward(p.astype(np.float64), x.astype(np.float64))
    got = Y.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 2e-5 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("batch", [1, 17, 32, 64])
def test_gradient_matches_numpy(cuda, batch):
    import torch
    rng = np.random.default_rng(batch)
    p = (init_params(batch) + rng.normal(0, 0.05, mlp_oracle.P)).astype(
        np.float32)
    x = rng.uniform(-1, 1, batch).astype(np.float32)
    t = np.cos(3 * x).astype(np.float32)
    G = torch.empty(mlp_oracle.P, dtype=torch.float32, device="cuda")
    L = torch.empty(1, dtype=torch.float32, device="cuda")
    # keep the device copies alive until the kernel has run
    Pd, Xd, Td = _dev(p), _dev(x), _dev(t)
    _lib.check(cuda.slq_mlp_grad(Pd.data_ptr(), Xd.data_ptr(), Td.data_ptr(),
                                 batch, G.data_ptr(), L.data_ptr(),
                                 _stream()))
    torch.cuda.synchronize()
    loss, g = mlp_oracle.loss_grad(p.astype(np.float64), x, t)
    got = G.cpu().numpy()
    assert np.max(np.abs(got - g)) <= 1e-3 * np.max(np.abs(g))
    assert abs(float(L.item()) - loss) <= 1e-4 * max(loss, 1e-6)


def test_training_follows_numpy_adam(cuda):
    import torch
    x = np.linspace(-1, 1, 32).astype(np.float32)
    t = (np.tanh(2 * x) + 0.3 * x * x).astype(np.float32)
    p0 = init_params(5)
    P = _dev(p0)
    M = torch.zeros_like(P)
    V = torch.zeros_like(P)
    hist = torch.empty(400, dtype=torch.float32, device="cuda")
    Xd, Td = _dev(x), _dev(t)
    _lib.check(cuda.slq_mlp_train(P.data_ptr(), M.data_ptr(), V.data_ptr(),
                                  Xd.data_ptr(), Td.data_ptr(), 32, 400, 0,
                                  np.float32(3e-3), hist.data_ptr(),
                                  _stream()))
    torch.cuda.synchronize()
    losses = hist.cpu().numpy()
    _, _, _, want = mlp_oracle.adam(p0.astype(np.float64), x, t, 400, 3e-3)
    # same trajectory up to FP32 rounding
    assert abs(losses[0] - want[0]) <= 1e-5 * want[0]
    assert losses[-1] < 0.02 * losses[0]
    assert abs(losses[-1] - want[-1]) <= 0.1 * want[-1] + 1e-6


@pytest.mark.parametrize("func", ["log", "inv", "id"])
def test_surrogate_sweep_against_slq(cuda, func):
    import torch
    A = ib.correlation_matrix(20000, scale=0.01, threshold=0.05, shift=0.1,
                              seed=1, dtype="float32")
    opts = dict(min_num_samples=64, max_num_samples=64, lanczos_degree=30,
                orthogonalize=0, seed=2)
    sur = SweepSurrogate(A, func=func, t_min=1e-4, t_max=1e2, steps=20000,
                         **opts).fit()
    t = np.exp(np.linspace(np.log(1e-4), np.log(1e2), 512))
    torch.cuda.synchronize()
    got = sur(t)
    want = sur.slq(t)           # the same probes, shift relation, all t
    trusted = ~sur.last_fallback
    floor = sur.rtol_floor * float(np.mean(np.abs(sur.y_train)))
    err = np.abs(got - want) / np.maximum(np.abs(want), floor)
    # fallback is SLQ itself (same probes; its Krylov run is shifted to the
    # first fallback t, so FP32 rounding differs slightly)
    assert np.all(err[~trusted] < 1e-5)
    assert np.mean(trusted) >= 0.75
    # every one of the 512 answers within the gate's rtol
    assert np.max(err) < 1e-3
    assert np.all(sur.interval_error[sur.interval_trusted] <=
                  sur.margin * sur.rtol)
    # what the network gains: a per-t SLQ run versus the whole sweep from the
    # network (training data and training included, amortised or not)
    f = {"log": ib.logdet, "inv": ib.traceinv, "id": ib.trace}[func]
    M = ib.Matrix(A)
    f(M, method="slq", gpu=True, **opts)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for tv in t[:4]:
        f(ib.AffineMatrixFunction(A), method="slq", gpu=True,
          parameters=float(tv), **opts)
    torch.cuda.synchronize()
    per_t = (time.perf_counter() - t0) / 4
    sweep_per_t = 512 * per_t
    answer = sur.timings["predict"]
    assert sweep_per_t / answer > 50
    print("\n%s: per-t SLQ sweep %.3f s, surrogate answer %.5f s, "
          "fit (SLQ data %.3f s + training %.3f s), trusted %.0f%%, "
          "max held-out err %.2e, max err over the sweep %.2e"
          % (func, sweep_per_t, answer, sur.timings["slq_training_data"],
             sur.timings["train"], 100 * np.mean(trusted),
             np.max(sur.check_error), np.max(err)))
