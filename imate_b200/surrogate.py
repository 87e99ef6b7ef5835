"""Learned surrogate for parameter sweeps of trace f(A + t I).

imate answers sweeps over t either by running SLQ per t or, for A + t I, by
one Krylov run per probe with shifted Ritz values
(imate/_c_trace_estimator/c_trace_estimator.cpp:564-593), and it offers
interpolators of such sweeps (imate/interpolator/,
interpolate_schatten.py:426-492).  This module fits a small network to SLQ
samples of the sweep on the device and answers the sweep from it:

1. SLQ (this engine, one Krylov run per probe thanks to the shift relation)
   evaluates the sweep at ``num_train`` log-spaced training points and at
   ``checks_per_interval`` held-out points inside every interval between
   them (evenly spread in log t; extra points of one Krylov run cost a few
   quadrature evaluations);
2. the network 1 -> 64 -> 64 -> 1 (tanh, FP32; input log t standardised)
   is trained on the device by ``slq_mlp_train`` on the standardised
   residual of a one-parameter base curve with the sweep's limits, tau
   matched to the value at t_min, so the network only carries the shape of
   the spectrum, a small correction: r = f/n - log(t + tau) for logdet,
   r = log(f/n) + log(t + tau) for traceinv (f/n ~ 1/(t + tau); in log space
   an absolute error of the network is a relative error of f), and
   r = f/n - (t + tau) for trace;
3. every held-out point, and every training point, is compared with its
   SLQ value; an interval between training points is trusted only when all
   of its points and both of its ends are within ``margin * rtol`` (relative
   error, judged against a floor of ``rtol_floor`` times the sweep's mean
   magnitude where the values cross zero), the margin covering the error
   between check points; an untrusted interval is answered by SLQ instead
   (the fallback), as is any t outside the trained range.

``SweepSurrogate.timings`` records where the time goes so the sweep can be
compared with per-t SLQ and with the shift relation alone.
"""

import ctypes
import time

import numpy as np

from . import _lib
from ._functions import logdet, traceinv, trace
from ._trace_estimator import EngineOptions
from .linear_operator import AffineMatrixFunction

__all__ = ["SweepSurrogate", "init_params"]

_FUNCS = {"log": logdet, "inv": traceinv, "id": trace}


def init_params(seed=0):
    """Xavier-uniform weights, zero biases, packed as the device expects."""
    rng = np.random.default_rng(seed)
    H = _lib.MLP_WIDTH

    def xavier(fan_in, fan_out, size):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        return rng.uniform(-lim, lim, size)
    W1 = xavier(1, H, H)
    b1 = np.zeros(H)
    W2 = xavier(H, H, H * H)
    b2 = np.zeros(H)
    W3 = xavier(H, 1, H)
    b3 = np.zeros(1)
    return np.concatenate([W1, b1, W2, b2, W3, b3]).astype(np.float32)


class SweepSurrogate:
    """Fitted surrogate of t -> trace f(A + t I) on [t_min, t_max].

    ``slq_options`` are the keyword arguments of the SLQ runs (imate's
    logdet / traceinv / trace options, e.g. lanczos_degree, min/max samples,
    orthogonalize, seed); ``engine`` an EngineOptions.
    """

    def __init__(self, A, func="log", t_min=1e-4, t_max=1e2, num_train=32,
                 checks_per_interval=4, rtol=1e-3, rtol_floor=1e-3,
                 margin=0.5, steps=20000, lr=2e-3, seed=0, engine=None,
                 **slq_options):
        if func not in _FUNCS:
            raise ValueError("func must be 'log', 'inv' or 'id'")
        if not 0 < t_min < t_max:
            raise ValueError("need 0 < t_min < t_max")
        if not 2 <= num_train <= _lib.MLP_MAX_BATCH:
            raise ValueError("num_train is between 2 and %d"
                             % _lib.MLP_MAX_BATCH)
        if checks_per_interval < 1 or not 0 < margin <= 1:
            raise ValueError("need checks_per_interval >= 1 and "
                             "0 < margin <= 1")
        self.A = A
        self.func = func
        self.t_min, self.t_max = float(t_min), float(t_max)
        self.num_train = int(num_train)
        self.checks_per_interval = int(checks_per_interval)
        self.margin = float(margin)
        self.rtol = float(rtol)
        self.rtol_floor = float(rtol_floor)
        self.steps = int(steps)
        self.lr = float(lr)
        self.seed = seed
        self.engine = engine if engine is not None else EngineOptions()
        opts = dict(min_num_samples=64, max_num_samples=64, error_rtol=0.0,
                    lanczos_degree=30, orthogonalize=0, seed=0)
        opts.update(slq_options)
        self.slq_options = opts
        self.n = A.shape[0]
        self.Aop = AffineMatrixFunction(A)
        self.timings = {}
        self.params = None
        self.fitted = False

    # -- SLQ ------------------------------------------------------------------
    def slq(self, t):
        """SLQ values of the sweep at t (one Krylov run per probe)."""
        t = np.atleast_1d(np.asarray(t, dtype=np.float64))
        f = _FUNCS[self.func]
        vals, _ = f(self.Aop, method="slq", gpu=True, parameters=t,
                    return_info=True, engine=self.engine,
                    **self.slq_options)
        return np.atleast_1d(np.asarray(vals, dtype=np.float64))

    # -- fitting --------------------------------------------------------------
    def _x(self, t):
        return ((np.log(t) - self.x_mean) / self.x_scale).astype(np.float32)

    def fit(self):
        import torch
        lib = _lib.load()
        lt0, lt1 = np.log(self.t_min), np.log(self.t_max)
        self.t_train = np.exp(np.linspace(lt0, lt1, self.num_train))
        # held-out points: c evenly spread points (in log t) strictly inside
        # every interval between neighbouring training points
        c = self.checks_per_interval
        frac = (np.arange(c) + 0.5) / c
        lt = np.log(self.t_train)
        lcheck = lt[:-1, None] + (lt[1:] - lt[:-1])[:, None] * frac[None, :]
        self.check_interval = np.repeat(np.arange(lt.size - 1), c)
        self.t_check = np.exp(lcheck.ravel())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        allt = np.concatenate([self.t_train, self.t_check])
        vals = self.slq(allt)
        torch.cuda.synchronize()
        self.timings["slq_training_data"] = time.perf_counter() - t0
        self.y_train = vals[:self.num_train]
        self.y_check = vals[self.num_train:]

        self.x_mean = 0.5 * (lt0 + lt1)
        self.x_scale = 0.5 * (lt1 - lt0)
        yn = self.y_train / self.n
        self._fit_base(yn[0])
        resid = self._to_resid(self.t_train, yn)
        if not np.all(np.isfinite(resid)):
            resid = np.nan_to_num(resid)
            self._usable = False
        else:
            self._usable = True
        self.y_mean = float(np.mean(resid))
        self.y_scale = float(np.std(resid)) or 1.0
        target = ((resid - self.y_mean) / self.y_scale).astype(np.float32)

        dev = torch.device("cuda", torch.cuda.current_device())
        self._p = torch.from_numpy(init_params(self.seed)).to(dev)
        self._m = torch.zeros_like(self._p)
        self._v = torch.zeros_like(self._p)
        xt = torch.from_numpy(self._x(self.t_train)).to(dev)
        tt = torch.from_numpy(target).to(dev)
        hist = torch.empty(max(self.steps, 1), dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.check(lib.slq_mlp_train(
            self._p.data_ptr(), self._m.data_ptr(), self._v.data_ptr(),
            xt.data_ptr(), tt.data_ptr(), self.num_train, self.steps, 0,
            ctypes.c_float(self.lr), hist.data_ptr(), stream))
        torch.cuda.synchronize()
        self.timings["train"] = time.perf_counter() - t0
        self.loss_history = hist.cpu().numpy()[:self.steps]
        self.params = self._p.cpu().numpy()

        pred = self.predict(np.concatenate([self.t_check, self.t_train]))
        floor = self.rtol_floor * float(np.mean(np.abs(self.y_train)))
        ref = np.concatenate([self.y_check, self.y_train])
        err = np.abs(pred - ref) / np.maximum(np.abs(ref), floor)
        self.check_error = err[:self.t_check.size]
        self.train_error = err[self.t_check.size:]
        bound = self.margin * self.rtol
        nint = self.num_train - 1
        worst = np.zeros(nint)
        np.maximum.at(worst, self.check_interval, self.check_error)
        worst = np.maximum(worst, np.maximum(self.train_error[:-1],
                                             self.train_error[1:]))
        self.interval_error = worst
        self.interval_trusted = (worst <= bound) & self._usable
        self.fitted = True
        return self

    def _fit_base(self, y0):
        # base curve through (t_min, y0) with the sweep's large-t behaviour
        t0 = self.t_min
        tiny = 1e-300
        if self.func == "log":
            self.tau = max(float(np.exp(y0)) - t0, tiny)
        elif self.func == "inv":
            self.tau = max(1.0 / y0 - t0, tiny) if y0 > 0 else 1.0
        else:
            self.tau = float(y0) - t0

    def _to_resid(self, t, yn):
        t = np.asarray(t, dtype=np.float64)
        if self.func == "log":
            return yn - np.log(t + self.tau)
        if self.func == "inv":
            with np.errstate(divide="ignore", invalid="ignore"):
                return np.log(yn) + np.log(t + self.tau)
        return yn - (t + self.tau)

    def _from_resid(self, t, r):
        t = np.asarray(t, dtype=np.float64)
        if self.func == "log":
            return r + np.log(t + self.tau)
        if self.func == "inv":
            return np.exp(r) / (t + self.tau)
        return r + t + self.tau

    # -- answering ------------------------------------------------------------
    def predict(self, t):
        """Network values at t (no checks, no fallback)."""
        import torch
        lib = _lib.load()
        t = np.atleast_1d(np.asarray(t, dtype=np.float64))
        dev = self._p.device
        x = torch.from_numpy(self._x(t)).to(dev)
        y = torch.empty_like(x)
        _lib.check(lib.slq_mlp_forward(
            self._p.data_ptr(), x.data_ptr(), t.size, y.data_ptr(),
            torch.cuda.current_stream(dev).cuda_stream))
        z = y.cpu().numpy().astype(np.float64)
        return self._from_resid(t, z * self.y_scale + self.y_mean) * self.n

    def _trusted(self, t):
        """True where t lies in the fitted range inside a trusted interval."""
        t = np.asarray(t, dtype=np.float64)
        inside = (t >= self.t_min * (1 - 1e-12)) & (t <= self.t_max * (1 + 1e-12))
        lt = np.log(np.clip(t, self.t_min, self.t_max))
        edges = np.log(self.t_train)
        interval = np.clip(np.searchsorted(edges, lt, side="right") - 1, 0,
                           edges.size - 2)
        return inside & self.interval_trusted[interval]

    def __call__(self, t):
        """Sweep values at t: the network where trusted, SLQ elsewhere."""
        import torch
        if not self.fitted:
            self.fit()
        t = np.atleast_1d(np.asarray(t, dtype=np.float64))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = self.predict(t)
        torch.cuda.synchronize()
        self.timings["predict"] = time.perf_counter() - t0
        trust = self._trusted(t)
        self.last_fallback = ~trust
        if not np.all(trust):
            t0 = time.perf_counter()
            out[~trust] = self.slq(t[~trust])
            torch.cuda.synchronize()
            self.timings["fallback_slq"] = time.perf_counter() - t0
        else:
            self.timings["fallback_slq"] = 0.0
        return out
