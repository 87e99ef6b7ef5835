"""Batched SLQ: many independent estimates in one CUDA graph launch.

imate estimates one matrix per call (``trace_estimator.pyx:38-390``; its GPU
sample loop ``cu_trace_estimator.cu:197-315`` keeps one matrix per device).
A batch plan records every probe block of every estimate into one CUDA graph
(``slq_batch_create``), each estimate on its own graph branch so that
estimates of small matrices overlap on the device, launches the graph once
and applies imate's stopping rule to each estimate on the host
(``slq_batch_run``).  Each estimate equals what ``logdet`` / ``traceinv`` /
``trace`` return for the same arguments and the same SpMM choice.

``autotune`` picks, per operator, the SpMM storage format and tile (row-group
rows, probes per lane, warps per row group) and the probe block width: every
candidate the operator supports is timed at each width
(``slq_operator_tune``) and the width with the least SpMM time per probe
becomes the estimate's block size.
"""

import ctypes

import numpy as np

from . import _lib
from ._functions import _SLQ_DEFAULTS
from ._trace_estimator import (EngineOptions, prepare, run_outputs, collect,
                               finish, reset_outputs)

__all__ = ["BatchPlan", "autotune", "tune_operator", "logdet_batch",
           "traceinv_batch", "trace_batch", "pack_estimates",
           "estimate_cost"]

_FUNC_OF = {"logdet": "log", "traceinv": "inv", "trace": "id",
            "trexp": "exp", "trlinfrac": "linfrac", "eigencount": "indicator",
            "density": "gaussian"}


def tune_operator(dev_op, width, transpose=False, reps=5):
    """Time every SpMM candidate of a device operator at one block width;
    the fastest becomes the operator's choice at that width.  Returns a list
    of candidate dicts and the chosen index."""
    import torch
    lib = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(lib.slq_operator_tune_workspace_bytes(
        dev_op.handle, int(width), ctypes.byref(nbytes)))
    ws = torch.empty(int(nbytes.value), dtype=torch.uint8,
                     device=dev_op.device)
    res = _lib.SlqTuneResult()
    stream = torch.cuda.current_stream(dev_op.device)
    _lib.check(lib.slq_operator_tune(
        dev_op.handle, int(width), int(bool(transpose)), int(reps),
        ws.data_ptr(), ws.numel(), stream.cuda_stream, ctypes.byref(res)))
    cands = [dict(kind=_lib.SPMM_KINDS[res.kind[i]],
                  group_rows=int(res.group_rows[i]),
                  lanes_vec=int(res.lanes_vec[i]), slices=int(res.slices[i]),
                  ms=float(res.milliseconds[i]))
             for i in range(res.num_candidates)]
    return cands, int(res.chosen)


def set_variant(dev_op, width, candidate, transpose=False):
    """Force SpMM candidate ``candidate`` (index from tune_operator) at this
    width; -1 restores the built-in choice."""
    _lib.check(_lib.load().slq_operator_set_variant(
        dev_op.handle, int(width), int(bool(transpose)), int(candidate)))


def autotune(dev_op, max_num_samples, directions=(False,), widths=None,
             reps=5, per_step_ms=0.01):
    """Tune the operator's SpMM at every candidate block width and return
    the width with the least estimated time per probe-step,

        ceil(S / w) * (sum over directions of the fastest SpMM at w
                       + per_step_ms) / S,

    S = max_num_samples (``per_step_ms`` stands for the launches of a step
    that do not scale with the width).  Returns (width, report) with the
    report listing every width's candidates."""
    bmax = 512 if dev_op.dtype_code == _lib.SLQ_F64 else 1024
    top = min(bmax, 1 << max(0, (int(max_num_samples) - 1).bit_length()))
    if widths is None:
        widths = [w for w in (32, 64, 128, 256, 512, 1024) if w <= top] or \
            [top]
    report = {}
    best = None
    for w in widths:
        t = 0.0
        report[w] = {}
        for tr in directions:
            cands, chosen = tune_operator(dev_op, w, transpose=tr, reps=reps)
            report[w]["transpose" if tr else "direct"] = dict(
                candidates=cands, chosen=chosen)
            t += cands[chosen]["ms"]
        blocks = -(-int(max_num_samples) // w)
        cost = blocks * (t + per_step_ms)
        report[w]["cost_ms_per_step"] = cost
        if best is None or cost < best[1]:
            best = (w, cost)
    return best[0], report


def estimate_cost(A, max_num_samples, lanczos_degree, gram=False,
                  num_runs=1):
    """Work of one estimate in stored-entry visits: (nnz + n) per product
    (the SpMM and the vector updates), one product per Lanczos step (two for
    Golub-Kahn on a Gram estimate), every probe, every run."""
    def nnz_of(M):
        if hasattr(M, "indices") and hasattr(M.indices, "numel"):
            return int(M.indices.numel())
        if hasattr(M, "nnz"):
            return int(M.nnz)
        if isinstance(M, np.ndarray):
            return int(M.size)
        inner = getattr(M, "A", None)
        if inner is not None and inner is not M:
            return nnz_of(inner)
        shape = getattr(M, "shape", (1, 1))
        return int(shape[0]) * int(shape[1])
    n = int(getattr(A, "shape", (0,))[0] or 0)
    per = (nnz_of(A) + n) * (2 if gram else 1)
    return float(per) * int(max_num_samples) * int(lanczos_degree) * \
        max(1, int(num_runs))


def pack_estimates(costs, num_devices, pinned=None):
    """Size-balanced greedy packing (longest processing time first): the
    estimates, in decreasing cost (ties by index), each go to the device
    with the least load so far (ties to the lowest device).  ``pinned`` maps
    an estimate index to a device it must run on (its matrix already lives
    there); those are placed first.  Returns the device of every estimate;
    the result depends only on the costs."""
    D = max(1, int(num_devices))
    pinned = dict(pinned or {})
    load = [0.0] * D
    dev = [0] * len(costs)
    for i, d in pinned.items():
        if not 0 <= d < D:
            raise ValueError("estimate %d is pinned to device %d of %d"
                             % (i, d, D))
        dev[i] = d
        load[d] += float(costs[i])
    free = sorted((i for i in range(len(costs)) if i not in pinned),
                  key=lambda i: (-float(costs[i]), i))
    for i in free:
        d = min(range(D), key=lambda k: (load[k], k))
        dev[i] = d
        load[d] += float(costs[i])
    return dev


class _DevicePlan:
    """The runs of one device recorded into one CUDA graph."""

    def __init__(self, runs, device, lib):
        import torch
        self.runs = runs
        self.device = device
        self._lib = lib
        R = len(runs)
        self._ops = (ctypes.c_void_p * R)(
            *[J.dev_op.handle.value for J, _ in runs])
        self._prms = (_lib.SlqParams * R)(*[J.params[gi] for J, gi in runs])
        self._tps = (ctypes.c_void_p * R)(
            *[J.t_groups[gi].ctypes.data for J, gi in runs])
        self._nq = (ctypes.c_int * R)(*[len(J.groups[gi]) for J, gi in runs])
        nbytes = ctypes.c_size_t(0)
        _lib.check(lib.slq_batch_workspace_bytes(
            R, self._ops, self._prms, self._nq, ctypes.byref(nbytes)))
        with torch.cuda.device(device):
            self.workspace = torch.empty(int(nbytes.value),
                                         dtype=torch.uint8, device=device)
            self.handle = ctypes.c_void_p(None)
            stream = torch.cuda.current_stream(device)
            _lib.check(lib.slq_batch_create(
                R, self._ops, self._prms, self._tps, self._nq,
                self.workspace.data_ptr(), self.workspace.numel(),
                stream.cuda_stream, ctypes.byref(self.handle)))
        k = ctypes.c_int64(0)
        nn = ctypes.c_int64(0)
        _lib.check(lib.slq_batch_info(self.handle, ctypes.byref(k),
                                      ctypes.byref(nn)))
        self.graph_kernels = int(k.value)
        self.graph_nodes = int(nn.value)

    def destroy(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self._lib.slq_batch_destroy(h)
            self.handle = ctypes.c_void_p(None)

    def launch(self):
        import torch
        R = len(self.runs)
        outs = [run_outputs(J, gi) for J, gi in self.runs]
        results = (_lib.SlqResult * R)(*[o[0] for o in outs])
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device)
            status = self._lib.slq_batch_run(self.handle, stream.cuda_stream,
                                             results)
        return results, outs, status


class BatchPlan:
    """Many SLQ estimates recorded into CUDA graphs, one graph per device.

    ``estimates`` is a list of dicts, one per estimate, with keys ``func``
    ('logdet', 'traceinv', 'trace', 'trexp', 'trlinfrac', 'eigencount' or
    'density'), ``A`` (matrix or operator), optional ``gram``, ``p`` and
    ``func_coeff`` (the function's coefficients: trexp [c], trlinfrac
    [a, b, c, d], eigencount [lo, hi], density [mu, sigma]), any of imate's
    SLQ keyword arguments, and optionally ``engine`` (EngineOptions).
    ``autotune=True`` tunes each operator's SpMM and block width first (and
    overrides the estimate's block size); otherwise every operator keeps its
    current choice.  ``gpu=True`` is implied.

    ``num_gpu_devices`` spreads the estimates over that many devices (0:
    every visible device, imate's convention): each estimate runs whole on
    one device, the estimates packed by ``pack_estimates`` on their
    ``estimate_cost``; a ``DeviceMatrix`` stays on the device that holds it.
    The per-device graphs are launched from one host thread each.  An
    estimate's own ``num_gpu_devices`` does not split it inside a batch.
    ``device_of`` maps the packing's device index to a CUDA device (default
    the identity; with it, ``num_gpu_devices`` is taken as given).
    """

    def __init__(self, estimates, autotune=True, tune_reps=5,
                 num_gpu_devices=0, device_of=None):
        import torch
        from ._trace_estimator import resolve_num_devices
        lib = _lib.load()
        self.jobs = []
        self.tuning = []
        tuned = {}
        if device_of is None:
            D = resolve_num_devices(num_gpu_devices)
            home = torch.cuda.current_device()
            devices = [home] + [d for d in range(D) if d != home][:D - 1]
            device_of = devices.__getitem__
        else:
            D = max(1, int(num_gpu_devices))
        parsed = []
        for est in estimates:
            est = dict(est)
            func = _FUNC_OF[est.pop("func")]
            A = est.pop("A")
            gram = bool(est.pop("gram", False))
            p = est.pop("p", 1.0)
            engine = est.pop("engine", None) or EngineOptions()
            coeff = est.pop("func_coeff", None)
            kw = dict(_SLQ_DEFAULTS)
            kw["gpu"] = True
            unknown = set(est) - set(kw)
            if unknown:
                raise TypeError("unexpected keyword argument(s): %s"
                                % ", ".join(sorted(unknown)))
            kw.update(est)
            parsed.append((func, A, gram, p, engine, coeff, kw))
        if not parsed:
            raise ValueError("a batch needs at least one estimate")
        costs = []
        pinned = {}
        phys = [device_of(d) for d in range(D)]
        for i, (func, A, gram, p, engine, coeff, kw) in enumerate(parsed):
            t = kw["parameters"]
            runs = 1 if t is None or np.ndim(t) == 0 else len(np.ravel(t))
            costs.append(estimate_cost(A, kw["max_num_samples"],
                                       kw["lanczos_degree"], gram, runs))
            data = getattr(A, "data", None)
            if hasattr(data, "device") and getattr(data, "is_cuda", False):
                if data.device.index not in phys:
                    raise ValueError(
                        "estimate %d: its matrix is on CUDA device %d, "
                        "outside the batch's devices" % (i, data.device.index))
                pinned[i] = phys.index(data.device.index)
        self.assignment = pack_estimates(costs, D, pinned)
        self.costs = costs
        for i, (func, A, gram, p, engine, coeff, kw) in enumerate(parsed):
            with torch.cuda.device(device_of(self.assignment[i])):
                J = prepare(A, kw["parameters"], func, gram, p,
                            kw["min_num_samples"], kw["max_num_samples"],
                            kw["error_atol"], kw["error_rtol"],
                            kw["confidence_level"],
                            kw["outlier_significance_level"],
                            kw["lanczos_degree"], kw["lanczos_tol"],
                            kw["orthogonalize"], kw["seed"],
                            kw["num_threads"], kw["num_gpu_devices"],
                            kw["verbose"], kw["plot"], kw["gpu"], engine,
                            coeff)
                J.num_devices = 1
                if getattr(J.dev_op, "dense", False):
                    raise NotImplementedError(
                        "batch plans serve sparse operators; a dense "
                        "operator holds the scratch of one product at a "
                        "time (call logdet / traceinv / trace for it)")
                if J.per_group_t is not None:
                    raise NotImplementedError(
                        "batch plans record one device operator per "
                        "estimate; A + t B with B other than the identity "
                        "needs one per t (call logdet / traceinv / trace "
                        "for it)")
                if autotune:
                    key = (id(J.dev_op), J.params[0].gram, J.max_num_samples)
                    if key not in tuned:
                        dirs = (False,) if J.params[0].gram == 0 else \
                            (False, True)
                        tuned[key] = autotune_fn(J.dev_op, J.max_num_samples,
                                                 directions=dirs,
                                                 reps=tune_reps)
                    width, report = tuned[key]
                    for prm in J.params:
                        prm.block_size = width
                    self.tuning.append(dict(width=width, report=report))
                else:
                    self.tuning.append(None)
            self.jobs.append(J)
        self.runs = [(J, gi) for J in self.jobs for gi in range(len(J.params))]
        self.plans = []
        for d in range(D):
            runs = [(J, gi) for i, J in enumerate(self.jobs)
                    if self.assignment[i] == d
                    for gi in range(len(J.params))]
            if runs:
                self.plans.append(_DevicePlan(runs, device_of(d), lib))
        self.num_devices = D
        self.device = self.plans[0].device
        self.graph_kernels = sum(pl.graph_kernels for pl in self.plans)
        self.graph_nodes = sum(pl.graph_nodes for pl in self.plans)
        self._lib = lib

    def __del__(self):
        for pl in getattr(self, "plans", ()):
            pl.destroy()

    def launch(self):
        """One graph launch per device plus the host stopping rule; returns
        the per-run (SlqResult, arrays) pairs in plan order and the worst
        status."""
        if len(self.plans) == 1:
            launched = [self.plans[0].launch()]
        else:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(max_workers=len(self.plans)) as pool:
                launched = list(pool.map(lambda pl: pl.launch(), self.plans))
        by_run = {}
        status = _lib.SLQ_OK
        for pl, (results, outs, st) in zip(self.plans, launched):
            for k, run in enumerate(pl.runs):
                by_run[id(run[0]), run[1]] = (results[k], outs[k], st)
            if st != _lib.SLQ_OK and status in (_lib.SLQ_OK, 6):
                status = st
        order = [by_run[id(J), gi] for J, gi in self.runs]
        return order, status

    def run(self):
        """Run the batch; returns [(trace, info), ...] in estimate order."""
        order, status = self.launch()
        if status not in (_lib.SLQ_OK, 6):
            _lib.check(status)
        for J in self.jobs:
            reset_outputs(J)
        for (J, gi), (res, out, st) in zip(self.runs, order):
            collect(J, gi, res, out[1], st if st == 6 else _lib.SLQ_OK)
        out = []
        for i, J in enumerate(self.jobs):
            tr, info = finish(J)
            pl = next(p for p in self.plans if any(r[0] is J for r in p.runs))
            info["engine"]["batch"] = dict(
                estimates=len(self.jobs), runs=len(self.runs),
                graph_kernels=self.graph_kernels,
                graph_nodes=self.graph_nodes,
                devices=len(self.plans), device=pl.device,
                device_graph_kernels=pl.graph_kernels)
            out.append((tr, info))
        return out


autotune_fn = autotune


def _batch(name, matrices, gram, p, return_info, autotune, options):
    if not isinstance(return_info, bool):
        raise TypeError('"return_info" should be boolean.')
    per = options.pop("per_matrix", None)
    ests = []
    for i, A in enumerate(matrices):
        e = dict(options)
        if per is not None:
            e.update(per[i])
        e.update(func=name, A=A, gram=gram, p=p)
        ests.append(e)
    num_gpu_devices = options.pop("num_gpu_devices", 0)
    plan = BatchPlan(ests, autotune=autotune, num_gpu_devices=num_gpu_devices)
    res = plan.run()
    if return_info:
        return res
    return [tr for tr, _ in res]


def logdet_batch(matrices, gram=False, p=1.0, return_info=False,
                 autotune=True, **options):
    """logdet of every matrix by SLQ in one batched graph launch.  Keyword
    arguments are imate's SLQ options shared by all matrices; ``per_matrix``
    (a list of dicts) overrides them per matrix."""
    return _batch("logdet", matrices, gram, p, return_info, autotune,
                  options)


def traceinv_batch(matrices, gram=False, p=1, return_info=False,
                   autotune=True, **options):
    """trace of the inverse of every matrix, batched (see logdet_batch)."""
    return _batch("traceinv", matrices, gram, p, return_info, autotune,
                  options)


def trace_batch(matrices, gram=False, p=1.0, return_info=False,
                autotune=True, **options):
    """trace of every matrix, batched (see logdet_batch)."""
    return _batch("trace", matrices, gram, p, return_info, autotune,
                  options)
