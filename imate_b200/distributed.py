"""Probe-parallel SLQ over several GPUs (one process per GPU).

The reference runs one host OpenMP thread per GPU, each drawing probes from
its own xoshiro stream and merging samples under a critical section
(imate/_cu_trace_estimator/cu_trace_estimator.cu:229-299); the number of
samples it ends with then depends on thread timing.  Here probes are indexed
globally: in round k every rank r runs the probe block
[k*W*b + r*b, k*W*b + (r+1)*b) of the one parity stream, the ranks exchange
their per-probe samples (an all_gather of b doubles per rank -- the only
collective), and every rank replays the reference's sequential convergence
test over the samples in global probe order.  The result -- samples used,
estimate, error, outliers -- is the one a single process would produce, for
any number of ranks.

The per-rank work is pluggable (``run_block``) so that the host logic can be
exercised on CPU ranks (gloo) without a GPU.
"""

import ctypes

import numpy as np

__all__ = ["shard_block", "replay_convergence", "distributed_trace_estimator",
           "multi_device_trace_estimator"]


def shard_block(round_index, world_size, rank, block):
    """Global probe range (first, count) of ``rank`` in ``round_index``."""
    first = (round_index * world_size + rank) * block
    return first, block


def replay_convergence(samples, q, min_num_samples, confidence_level,
                       error_atol, error_rtol, processed, converged,
                       affine_many=False):
    """Feed new samples (rows of ``samples``, global order) through the
    reference convergence test one at a time.  ``processed`` (list of row
    indices already seen) and ``converged`` (int32[q]) are updated in place.
    Returns (all_converged, error, num_samples_used)."""
    from . import _lib
    lib = _lib.load()
    S = np.ascontiguousarray(samples, dtype=np.float64)
    error = np.zeros(q)
    used = np.zeros(q, dtype=np.int32)
    done = False
    start = len(processed)
    for i in range(start, S.shape[0]):
        if affine_many:
            converged[:] = 0
        processed.append(i)
        order = np.asarray(processed, dtype=np.int32)
        done = bool(lib.slq_check_convergence(
            S.ctypes.data, q, int(min_num_samples), order.ctypes.data,
            len(processed), float(confidence_level), float(error_atol),
            float(error_rtol), error.ctypes.data, used.ctypes.data,
            converged.ctypes.data))
        if done:
            break
    return done, error, used


def _all_gather_rows(rows, group=None):
    """Concatenate [b][q] float64 arrays of all ranks in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.float64)).to(dev)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    return np.concatenate([o.cpu().numpy() for o in out], axis=0)


def distributed_trace_estimator(run_block, q, block, min_num_samples,
                                max_num_samples, confidence_level=0.95,
                                error_atol=0.0, error_rtol=1e-2,
                                outlier_significance_level=0.001,
                                affine_many=False, group=None):
    """Sharded estimate.  ``run_block(first_probe, count)`` returns the
    [count][q] samples of global probes first_probe .. first_probe+count-1
    on this rank's device.  Every rank returns the same dict."""
    import torch.distributed as dist
    from . import _lib
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lib = _lib.load()
    rows = []
    processed = []
    converged = np.zeros(q, dtype=np.int32)
    done = False
    error = np.full(q, np.inf)
    used = np.zeros(q, dtype=np.int32)
    k = 0
    while not done and len(rows) * 1 < max_num_samples:
        first, count = shard_block(k, world, rank, block)
        # every rank takes part in every round (same collectives everywhere)
        mine = np.full((count, q), np.nan)
        lo = max(0, min(count, max_num_samples - first))
        if lo > 0:
            mine[:lo] = run_block(first, lo)
        gathered = _all_gather_rows(mine, group)
        base = k * world * block
        keep = min(gathered.shape[0], max_num_samples - base)
        rows.extend(list(gathered[:keep]))
        S = np.asarray(rows, dtype=np.float64).reshape(len(rows), q)
        done, error, used = replay_convergence(
            S, q, min_num_samples, confidence_level, error_atol, error_rtol,
            processed, converged, affine_many)
        k += 1
        if len(rows) >= max_num_samples:
            break
    S = np.full((max_num_samples, q), np.nan)
    S[:len(rows)] = np.asarray(rows).reshape(len(rows), q)
    order = np.zeros(max_num_samples, dtype=np.int32)
    order[:len(processed)] = processed
    used = np.ascontiguousarray(used, dtype=np.int32)
    outl = np.zeros(q, dtype=np.int32)
    trace = np.zeros(q)
    err = np.zeros(q)
    lib.slq_average_estimates(float(confidence_level),
                              float(outlier_significance_level), q,
                              max_num_samples, used.ctypes.data,
                              order.ctypes.data, S.ctypes.data,
                              outl.ctypes.data, trace.ctypes.data,
                              err.ctypes.data)
    return dict(trace=trace, error=err, samples=S,
                processed_samples_indices=order, num_samples_used=used,
                num_outliers=outl, converged=converged.copy(),
                all_converged=bool(done), rounds=k, world_size=world)


def multi_device_trace_estimator(run_block, num_devices, q, block,
                                 min_num_samples, max_num_samples,
                                 confidence_level=0.95, error_atol=0.0,
                                 error_rtol=1e-2,
                                 outlier_significance_level=0.001,
                                 affine_many=False, first_probe=0):
    """Probe blocks of one estimate dealt over the devices of one process,
    as the reference deals its samples over one OpenMP thread per GPU
    (imate/_cu_trace_estimator/cu_trace_estimator.cu:229-299), but by global
    probe index: in round k device d runs the block of global probes
    [first_probe + (k D + d) b, ... + b) (D devices, b = ``block``), one
    host thread per device, and the host then feeds the round's samples, in
    global order, through the reference's sequential stopping rule.  A round
    is taken only while the rule has not stopped, so every device count gives
    the estimate, samples used, error and outliers of one device (it may
    compute up to D - 1 blocks past the stopping point).

    ``run_block(device, first, count)`` returns a dict with 'samples'
    ([count][q]) and optionally 'lanczos_size', 'probe_status' ([count]),
    'alpha', 'beta' ([count][m]) for global probes first .. first+count-1
    (``first`` counted from ``first_probe``).  Returns the merged outputs."""
    from concurrent.futures import ThreadPoolExecutor
    from . import _lib
    lib = _lib.load()
    D = max(1, int(num_devices))
    rows = []
    extra = {}
    processed = []
    converged = np.zeros(q, dtype=np.int32)
    done = False
    used = np.zeros(q, dtype=np.int32)
    k = 0
    with ThreadPoolExecutor(max_workers=D) as pool:
        while not done and len(rows) < max_num_samples:
            jobs = []
            for d in range(D):
                first = (k * D + d) * block
                count = min(block, max_num_samples - first)
                if count > 0:
                    jobs.append((first, pool.submit(run_block, d, first, count)))
            for first, fut in jobs:
                out = fut.result()
                s = np.asarray(out["samples"], dtype=np.float64)
                rows.extend(list(s.reshape(s.shape[0], q)))
                for key in ("lanczos_size", "probe_status", "alpha", "beta"):
                    if out.get(key) is not None:
                        extra.setdefault(key, []).extend(list(out[key]))
            S = np.asarray(rows, dtype=np.float64).reshape(len(rows), q)
            done, _, used = replay_convergence(
                S, q, min_num_samples, confidence_level, error_atol,
                error_rtol, processed, converged, affine_many)
            k += 1
    # as one device reports them: samples past the stopping point NaN,
    # Krylov sizes only for the samples the rule took
    nproc = len(processed)
    S = np.full((max_num_samples, q), np.nan)
    S[:nproc] = np.asarray(rows[:nproc]).reshape(nproc, q)
    order = np.zeros(max_num_samples, dtype=np.int32)
    order[:nproc] = processed
    used = np.ascontiguousarray(used, dtype=np.int32)
    outl = np.zeros(q, dtype=np.int32)
    trace = np.zeros(q)
    err = np.zeros(q)
    lib.slq_average_estimates(float(confidence_level),
                              float(outlier_significance_level), q,
                              max_num_samples, used.ctypes.data,
                              order.ctypes.data, S.ctypes.data,
                              outl.ctypes.data, trace.ctypes.data,
                              err.ctypes.data)
    if "lanczos_size" in extra:
        extra["lanczos_size"] = list(extra["lanczos_size"][:nproc])
    res = dict(trace=trace, error=err, samples=S,
               processed_samples_indices=order, num_samples_used=used,
               num_outliers=outl, converged=converged.copy(),
               all_converged=bool(done), rounds=k, num_devices=D,
               num_probes_computed=len(rows))
    for key, vals in extra.items():
        res[key] = np.asarray(vals)
    return res


def engine_block_runner(Aop, func, gram=False, exponent=1.0, parameters=None,
                        lanczos_degree=20, lanczos_tol=None, orthogonalize=0,
                        seed=0, rng="parity"):
    """``run_block`` for distributed_trace_estimator backed by the GPU
    engine on this rank's current device."""
    from . import _lib
    from ._trace_estimator import EngineOptions, trace_estimator

    def run(first, count):
        eng = EngineOptions(block_size=count, rng=rng, first_probe=first)
        _, info = trace_estimator(
            Aop, parameters, func, gram, exponent, count, count, None, 0.0,
            0.95, 0.001, lanczos_degree, lanczos_tol, orthogonalize, seed, 0,
            0, False, False, True, options=eng)
        s = np.asarray(info["convergence"]["samples"], dtype=np.float64)
        return s.reshape(count, -1)
    assert _lib is not None
    return run
