"""Host side of the SLQ estimator.

Mirrors imate's dispatcher for ``method='slq'``
(``imate/_trace_estimator/trace_estimator.pyx:38-390`` with
``trace_estimator_utilities.py:24-373``): the same argument checks and
defaults, the same outputs and the same ``info`` dictionary, with the sample
loop, Krylov recurrences, eigen-solves and quadrature running in
``libslq_b200.so`` on the GPU.  Only ``gpu=True`` is served; there is no CPU
path.
"""

import ctypes
import numbers
import time

import numpy as np
import scipy.sparse as sp

from . import _lib
from .__version__ import __version__
from .linear_operator import LinearOperator, Matrix

__all__ = ["trace_estimator", "EngineOptions"]


class EngineOptions:
    """Engine settings beyond imate's keyword arguments.

    block_size : probes advanced together on the device (power of two,
        <= 1024 for float32, <= 512 for float64); 0 picks
        min(256, next power of two >= max_num_samples).
    rng : 'parity' reproduces the reference's xoshiro256** Rademacher stream
        bit for bit; 'fast' uses a counter-based hash (no host set-up).
    first_probe : global index of the first probe (sample i uses probe
        first_probe + i of the stream), so that shards of one estimate can
        run on different devices without sharing probes.
    return_coefficients : put the per-sample Lanczos coefficients in
        info['engine']['alpha'] / ['beta'].
    """

    def __init__(self, block_size=0, rng="parity", return_coefficients=False,
                 first_probe=0):
        self.block_size = int(block_size)
        self.rng = rng
        self.return_coefficients = bool(return_coefficients)
        self.first_probe = int(first_probe)


def _is_int(x):
    return isinstance(x, (int, np.integer)) and not isinstance(x, bool)


def _is_float(x):
    return isinstance(x, (int, float, np.integer, np.floating)) and \
        not isinstance(x, bool)


def get_operator(A, gram):
    """Wrap the input as an operator (trace_estimator_utilities.py:24-55)."""
    if isinstance(A, np.ndarray) or sp.issparse(A):
        if A.ndim != 2:
            raise ValueError("Input matrix should be a 2-dimensional array.")
        if not gram and A.shape[0] != A.shape[1]:
            raise ValueError("Input matrix should be a square matrix.")
        return Matrix(A)
    if isinstance(A, LinearOperator):
        if not gram and A.get_num_rows() != A.get_num_columns():
            raise ValueError("Input operator should have the same number of "
                             "rows and columns.")
        return A
    raise TypeError('The linear operator "A" should be either a '
                    'numpy.ndarray, a scipy.sparse array, or an instance of '
                    'a class derived from the "LinearOperator" class.')


def get_operator_parameters(parameters, data_type_name):
    """Normalise ``parameters`` (trace_estimator_utilities.py:62-101)."""
    if parameters is None:
        return None, 0
    if np.isscalar(parameters):
        return parameters, 1
    if isinstance(parameters, (list, np.ndarray)):
        arr = np.asarray(parameters, dtype=data_type_name)
        if arr.ndim != 1:
            raise ValueError('"parameters", if given as an array, should be a '
                             'one-dimensional array. Current dimension of '
                             'parameters is %d.' % arr.ndim)
        return arr, arr.size
    raise TypeError('"parameters" type should be either "None", a scalar, a '
                    'flat list, or one-dimensional "numpy.ndarray.')


def find_num_inquiries(Aop, parameters_size):
    """Number of parameter sets (trace_estimator_utilities.py:338-373)."""
    k = Aop.get_num_parameters()
    if k == 0:
        return 1
    if parameters_size < k:
        raise ValueError("Not enough parameters are provided. The given "
                         "parameter size is %d, which should be larger than "
                         "%d, the number of parameters of the linear "
                         "operator." % (parameters_size, k))
    if parameters_size % k != 0:
        raise ValueError("Parameters size (given %d) is not an integer-"
                         "multiple of %d, the number of the parameters of the "
                         "linear operator." % (parameters_size, k))
    return parameters_size // k


def check_arguments(gram, exponent, min_num_samples, max_num_samples,
                    error_atol, error_rtol, confidence_level,
                    outlier_significance_level, lanczos_degree, lanczos_tol,
                    orthogonalize, seed, num_threads, num_gpu_devices,
                    verbose, plot, gpu):
    """Type and range checks of imate's SLQ keyword arguments
    (trace_estimator_utilities.py:108-305).  Returns (error_atol,
    error_rtol) with None mapped to 0."""

    def flag(name, v):
        if v is None:
            raise TypeError('"%s" cannot be None.' % name)
        if not np.isscalar(v):
            raise TypeError('"%s" should be a scalar value.' % name)
        if not isinstance(v, bool):
            raise TypeError('"%s" should be boolean.' % name)

    def count(name, v, minimum, none_error=ValueError):
        if v is None:
            raise none_error('"%s" cannot be None.' % name)
        if not np.isscalar(v):
            raise TypeError('"%s" should be a scalar value.' % name)
        if not _is_int(v):
            raise TypeError('"%s" should be an integer.' % name)
        if v < minimum:
            raise ValueError('"%s" should be at least %d.' % (name, minimum))

    flag("gram", gram)
    if exponent is None:
        raise TypeError('"exponent" cannot be None.')
    if not np.isscalar(exponent):
        raise TypeError('"exponent" should be a scalar value.')
    if isinstance(exponent, complex):
        raise TypeError('"exponent" cannot be a complex number.')
    count("min_num_samples", min_num_samples, 1)
    count("max_num_samples", max_num_samples, 1)
    if min_num_samples > max_num_samples:
        raise ValueError('"min_num_samples" cannot be greater than '
                         '"max_num_samples".')

    def tolerance(name, v):
        if v is None:
            return 0.0
        if not np.isscalar(v):
            raise TypeError('"%s" should be a scalar value.' % name)
        if not isinstance(v, (int, float)) or isinstance(v, bool):
            raise TypeError('"%s" should be a float number.' % name)
        if v < 0.0:
            raise ValueError('"%s" cannot be negative.' % name)
        return v

    error_atol = tolerance("error_atol", error_atol)
    error_rtol = tolerance("error_rtol", error_rtol)

    if confidence_level is None:
        raise TypeError('"confidence_level" cannot be None.')
    if not np.isscalar(confidence_level):
        raise TypeError('"confidence_level" should be a scalar.')
    if not isinstance(confidence_level, (int, float)) or \
            isinstance(confidence_level, bool):
        raise TypeError('"confidence_level" should be a float number.')
    if not 0.0 <= confidence_level <= 1.0:
        raise ValueError('"confidence_level" should be between 0 and 1.')

    osl = outlier_significance_level
    if osl is None:
        raise TypeError('"outlier_significance_level" cannot be None.')
    if not np.isscalar(osl):
        raise TypeError('"outlier_significance_level" should be a scalar.')
    if not _is_float(osl):
        raise TypeError('"outlier_significance_level" must be a float number.')
    if not 0.0 <= osl <= 1.0:
        raise ValueError('"outlier_significance_level" must be in [0, 1] '
                         'interval.')
    if osl > 1.0 - confidence_level:
        raise ValueError('The sum of "confidence_level" and '
                         '"outlier_significance_level" should be less than 1.')

    count("lanczos_degree", lanczos_degree, 1, none_error=TypeError)
    if lanczos_tol is not None:
        if not np.isscalar(lanczos_tol):
            raise TypeError('"lanczos_tol" should be a scalar value.')
        if not _is_float(lanczos_tol):
            raise TypeError('"lanczos_tol" should be a float number.')
        if lanczos_tol < 0.0:
            raise ValueError('"lancozs_tol" cannot be negative.')

    if orthogonalize is None:
        raise TypeError('"orthogonalize" cannot be None.')
    if not np.isscalar(orthogonalize):
        raise TypeError('"orthogonalize" should be a scalar value.')
    if not _is_int(orthogonalize):
        raise TypeError('"orthogonalize" should be an integer.')
    if orthogonalize > lanczos_degree:
        raise ValueError('"orthogonalize", if positive, should be at most '
                         'equal to "lanczos_degree".')

    if seed is not None:
        if not np.isscalar(seed):
            raise TypeError('"seed" should be a None or a scalar value.')
        if not _is_int(seed):
            raise TypeError('"seed" should be None or an integer.')

    for name, v in (("num_threads", num_threads),
                    ("num_gpu_devices", num_gpu_devices)):
        if v is None:
            raise TypeError('"%s" cannot be None.' % name)
        if not np.isscalar(v):
            raise TypeError('"%s" should be a scalar value.' % name)
        if not _is_int(v):
            raise TypeError('"%s" should be an integer.' % name)
        if v < 0:
            raise ValueError('"%s" should be a non-negative integer.' % name)

    flag("verbose", verbose)
    flag("plot", plot)
    flag("gpu", gpu)
    return error_atol, error_rtol


def _clock_seed():
    # a non-negative seed from the high-resolution clock (the reference maps
    # seed=None to -1, which seeds SplitMix64 from the clock,
    # split_mix_64.cpp:33-41)
    return int(time.perf_counter_ns() & 0x7FFFFFFF)


class _Job:
    """One estimator call prepared for the engine: the checked arguments,
    the device operator, one ``SlqParams`` per run and the output arrays the
    runs fill in."""


def prepare(A, parameters, func, gram, exponent, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, lanczos_degree, lanczos_tol,
            orthogonalize, seed, num_threads, num_gpu_devices, verbose, plot,
            gpu, options=None, func_coeff=None):
    """Argument checks and set-up of one estimate (the part of
    ``trace_estimator.pyx:38-260`` before the sample loop).  Returns a job
    whose ``runs`` (one per group of inquiries) are executed by ``slq_run``
    or by a batch plan, then ``collect``-ed and ``finish``-ed."""
    import torch

    if options is None:
        options = EngineOptions()
    if not gpu:
        raise ValueError('This engine runs SLQ on the GPU only: call with '
                         '"gpu=True" (imate\'s CPU path serves gpu=False).')
    if func not in _lib.FUNC_IDS:
        raise ValueError("unknown matrix function %r" % (func,))
    if options.rng not in _lib.RNG_IDS:
        raise ValueError('rng must be "parity" or "fast"')

    Aop = get_operator(A, gram)
    data_type_name = Aop.get_data_type_name()
    dtype_str = data_type_name.decode()
    parameters, parameters_size = get_operator_parameters(parameters,
                                                          dtype_str)
    num_inquiries = find_num_inquiries(Aop, parameters_size)
    error_atol, error_rtol = check_arguments(
        gram, exponent, min_num_samples, max_num_samples, error_atol,
        error_rtol, confidence_level, outlier_significance_level,
        lanczos_degree, lanczos_tol, orthogonalize, seed, num_threads,
        num_gpu_devices, verbose, plot, gpu)
    if lanczos_degree > _lib.MAX_DEGREE:
        raise ValueError('"lanczos_degree" is at most %d on this engine.'
                         % _lib.MAX_DEGREE)
    if seed is None:
        seed_used = _clock_seed()
    else:
        seed_used = int(seed)
        if seed_used < 0:
            seed_used = _clock_seed()
    if lanczos_tol is None:
        lanczos_tol = float(np.finfo(dtype_str).eps)
    if num_threads < 1:
        import os
        num_threads = os.cpu_count() or 1

    _lib.load()
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device is available for the SLQ engine")

    J = _Job()
    J.init_wall = time.perf_counter()
    J.init_proc = time.process_time()

    affine = Aop.get_num_parameters() > 0
    normal = bool(getattr(Aop, "normal_equations", False))
    if normal and gram:
        raise ValueError('GramAffineMatrixFunction is already a Gram '
                         'operator: call with "gram=False".')
    if affine:
        t_values = np.atleast_1d(np.asarray(parameters, dtype=np.float64))
    else:
        t_values = np.zeros(1)

    # gram with several shifts: the shift relation does not hold for
    # (A + tI)^T (A + tI), so each t gets its own Krylov runs; nor for
    # A + t B with B other than I, where each t also gets its own operator
    general_b = bool(getattr(Aop, "general_B", False))
    if general_b or (gram and affine and num_inquiries > 1):
        groups = [[j] for j in range(num_inquiries)]
    else:
        groups = [list(range(num_inquiries))]

    m = int(lanczos_degree)
    coeff = [0.0] * 4
    if func_coeff is not None:
        coeff[:len(func_coeff)] = [float(c) for c in func_coeff]
    J.Aop = Aop
    J.per_group_t = t_values if general_b else None
    J.need_transpose = bool(gram) or normal
    J.dev_op = (Aop.device_operator_for(t_values[0], J.need_transpose)
                if general_b else
                Aop.get_device_operator(need_transpose=J.need_transpose))
    gram_mode = 2 if normal else int(bool(gram))
    J.groups = groups
    J.params = []
    J.t_groups = []
    for group in groups:
        J.params.append(_lib.SlqParams(
            func=_lib.FUNC_IDS[func], gram=gram_mode,
            exponent=float(exponent), orthogonalize=int(orthogonalize),
            seed=seed_used, lanczos_degree=m, lanczos_tol=float(lanczos_tol),
            min_num_samples=int(min_num_samples),
            max_num_samples=int(max_num_samples),
            error_atol=float(error_atol), error_rtol=float(error_rtol),
            confidence_level=float(confidence_level),
            outlier_significance_level=float(outlier_significance_level),
            block_size=options.block_size, rng=_lib.RNG_IDS[options.rng],
            first_probe=options.first_probe,
            func_coeff=(ctypes.c_double * 4)(*coeff)))
        # a per-t operator holds A + t B itself: no shift on top
        J.t_groups.append(np.zeros(len(group)) if general_b else
                          np.ascontiguousarray(t_values[group],
                                               dtype=np.float64))
    J.options = options
    J.dtype_str = dtype_str
    J.data_type_name = data_type_name
    J.gram = gram
    J.exponent = exponent
    J.parameters = parameters
    J.num_inquiries = num_inquiries
    J.error_atol, J.error_rtol = error_atol, error_rtol
    J.confidence_level = confidence_level
    J.outlier_significance_level = outlier_significance_level
    J.min_num_samples, J.max_num_samples = min_num_samples, max_num_samples
    J.lanczos_degree, J.lanczos_tol = lanczos_degree, lanczos_tol
    J.orthogonalize, J.seed, J.seed_used = orthogonalize, seed, seed_used
    J.num_threads = num_threads
    J.verbose, J.plot = verbose, plot
    J.num_devices = resolve_num_devices(num_gpu_devices)
    reset_outputs(J)
    return J


def reset_outputs(J):
    """Fresh output arrays and counters for job J (before its runs)."""
    q = J.num_inquiries
    mx = J.max_num_samples
    m = int(J.lanczos_degree)
    ng = len(J.groups)
    J.trace = np.full(q, np.nan)
    J.error = np.full(q, np.nan)
    J.samples = np.full((mx, q), np.nan)
    J.processed = np.zeros(mx, dtype=np.int32)
    J.num_samples_used = np.zeros(q, dtype=np.int32)
    J.num_outliers = np.zeros(q, dtype=np.int32)
    J.converged = np.zeros(q, dtype=np.int32)
    J.lanczos_size = np.zeros((mx, ng), dtype=np.int32)
    J.probe_status = np.full((mx, ng), -1, dtype=np.int32)
    J.alphas = J.betas = None
    if J.options.return_coefficients:
        J.alphas = np.full((ng, mx, m), np.nan)
        J.betas = np.full((ng, mx, m), np.nan)
    J.all_converged = True
    J.alg_wall_time = 0.0
    J.engine = dict(block_size=None, rng=J.options.rng, num_blocks=0,
                    num_probes_computed=0, gpu_launches=0)


def run_outputs(J, gi):
    """Host arrays for run ``gi`` of job J and the SlqResult pointing at
    them."""
    gq = len(J.groups[gi])
    mx = J.max_num_samples
    m = int(J.lanczos_degree)
    a = dict(
        trace=np.zeros(gq), error=np.zeros(gq), samples=np.zeros((mx, gq)),
        order=np.zeros(mx, dtype=np.int32),
        used=np.zeros(gq, dtype=np.int32), out=np.zeros(gq, dtype=np.int32),
        conv=np.zeros(gq, dtype=np.int32), size=np.zeros(mx, dtype=np.int32),
        status=np.full(mx, -1, dtype=np.int32),
        alpha=np.zeros((mx, m)) if J.alphas is not None else None,
        beta=np.zeros((mx, m)) if J.betas is not None else None)

    def ptr(x):
        return x.ctypes.data if x is not None else None
    res = _lib.SlqResult(
        trace=ptr(a["trace"]), error=ptr(a["error"]),
        samples=ptr(a["samples"]), processed_samples_indices=ptr(a["order"]),
        num_samples_used=ptr(a["used"]), num_outliers=ptr(a["out"]),
        converged=ptr(a["conv"]), lanczos_size=ptr(a["size"]),
        alpha=ptr(a["alpha"]), beta=ptr(a["beta"]),
        probe_status=ptr(a["status"]))
    return res, a


def collect(J, gi, res, a, status):
    """Put run ``gi``'s outputs into the job (raising on engine errors; an
    eigen-solve failure is reported as a warning, as the samples it affects
    are NaN)."""
    lib = _lib.load()
    if status == 6:
        import warnings
        warnings.warn("SLQ: " + lib.slq_last_error().decode())
    elif status != _lib.SLQ_OK:
        _lib.check(status)
    for k, j in enumerate(J.groups[gi]):
        J.trace[j] = a["trace"][k]
        J.error[j] = a["error"][k]
        J.samples[:, j] = a["samples"][:, k]
        J.num_samples_used[j] = a["used"][k]
        J.num_outliers[j] = a["out"][k]
        J.converged[j] = a["conv"][k]
    if gi == 0:
        J.processed = a["order"]
    J.lanczos_size[:, gi] = a["size"]
    J.probe_status[:, gi] = a["status"]
    if J.alphas is not None:
        J.alphas[gi] = a["alpha"]
        J.betas[gi] = a["beta"]
    J.all_converged = J.all_converged and bool(res.all_converged)
    J.alg_wall_time += float(res.alg_wall_time)
    J.engine["num_blocks"] += int(res.num_blocks)
    J.engine["num_probes_computed"] += int(res.num_probes_computed)
    J.engine["gpu_launches"] += int(res.gpu_launches)


def resolve_num_devices(num_gpu_devices):
    """Devices an estimate runs on: all visible devices for 0 (the
    reference's convention, trace_estimator.pyx:215-216), else at most the
    number asked for."""
    import torch
    avail = max(1, torch.cuda.device_count())
    n = int(num_gpu_devices)
    return avail if n == 0 else max(1, min(n, avail))


def _block_on_device(J, device, first, count):
    """Samples of global probes ``first`` .. ``first+count-1`` of job J's
    single run on CUDA device ``device`` (run by the calling host thread):
    a replica of the operator on that device and one block of slq_run."""
    import torch
    lib = _lib.load()
    torch.cuda.set_device(device)
    op = J.Aop.get_device_operator(need_transpose=J.need_transpose)
    base = J.params[0]
    prm = _lib.SlqParams.from_buffer_copy(base)
    prm.first_probe = base.first_probe + first
    prm.min_num_samples = count
    prm.max_num_samples = count
    prm.error_rtol = 0.0
    prm.error_atol = 0.0
    gq = J.num_inquiries
    m = int(J.lanczos_degree)
    ws_bytes = ctypes.c_size_t(0)
    _lib.check(lib.slq_run_workspace_bytes(op.handle, ctypes.byref(prm), gq,
                                           ctypes.byref(ws_bytes)))
    workspace = torch.empty(int(ws_bytes.value), dtype=torch.uint8,
                            device=op.device)
    a = dict(trace=np.zeros(gq), error=np.zeros(gq),
             samples=np.zeros((count, gq)),
             order=np.zeros(count, dtype=np.int32),
             used=np.zeros(gq, dtype=np.int32), out=np.zeros(gq, dtype=np.int32),
             conv=np.zeros(gq, dtype=np.int32),
             size=np.zeros(count, dtype=np.int32),
             status=np.full(count, -1, dtype=np.int32),
             alpha=np.zeros((count, m)) if J.alphas is not None else None,
             beta=np.zeros((count, m)) if J.betas is not None else None)

    def ptr(x):
        return x.ctypes.data if x is not None else None
    res = _lib.SlqResult(
        trace=ptr(a["trace"]), error=ptr(a["error"]),
        samples=ptr(a["samples"]), processed_samples_indices=ptr(a["order"]),
        num_samples_used=ptr(a["used"]), num_outliers=ptr(a["out"]),
        converged=ptr(a["conv"]), lanczos_size=ptr(a["size"]),
        alpha=ptr(a["alpha"]), beta=ptr(a["beta"]),
        probe_status=ptr(a["status"]))
    t_g = J.t_groups[0]
    stream = torch.cuda.current_stream(op.device)
    status = lib.slq_run(op.handle, ctypes.byref(prm), t_g.ctypes.data, gq,
                         workspace.data_ptr(), workspace.numel(),
                         stream.cuda_stream, ctypes.byref(res))
    if status not in (_lib.SLQ_OK, 6):
        _lib.check(status)
    return dict(samples=a["samples"], lanczos_size=a["size"],
                probe_status=a["status"], alpha=a["alpha"], beta=a["beta"],
                launches=int(res.gpu_launches))


def run_job_multi(J, num_devices, device_of=None):
    """Job J (one run) with its probe blocks dealt over ``num_devices``
    devices, one host thread each (multi_device_trace_estimator); the result
    equals that of one device.  ``device_of`` maps the dealing index to a
    CUDA device (default: the identity)."""
    from .distributed import multi_device_trace_estimator
    import torch
    b = block_width(J.max_num_samples, J.params[0].block_size, J.dtype_str)
    q = J.num_inquiries
    affine_many = bool(J.Aop.get_num_parameters() > 0 and q > 1)
    launches = []
    if device_of is None:
        def device_of(d):
            return d
    home = torch.cuda.current_device()
    # the operator replicas first, one device after the other (their host
    # orders run on the process's thread pool)
    for d in range(num_devices):
        torch.cuda.set_device(device_of(d))
        J.Aop.get_device_operator(need_transpose=J.need_transpose)
    torch.cuda.set_device(home)

    def run_block(device, first, count):
        out = _block_on_device(J, device_of(device), first, count)
        launches.append(out.pop("launches"))
        return out
    t0 = time.perf_counter()
    r = multi_device_trace_estimator(
        run_block, num_devices, q, b, J.min_num_samples, J.max_num_samples,
        confidence_level=J.confidence_level, error_atol=J.error_atol,
        error_rtol=J.error_rtol,
        outlier_significance_level=J.outlier_significance_level,
        affine_many=affine_many)
    torch.cuda.set_device(home)
    J.trace[:] = r["trace"]
    J.error[:] = r["error"]
    J.samples[:] = r["samples"]
    J.processed = r["processed_samples_indices"]
    J.num_samples_used[:] = r["num_samples_used"]
    J.num_outliers[:] = r["num_outliers"]
    J.converged[:] = r["converged"]
    n = len(r.get("lanczos_size", []))
    J.lanczos_size[:n, 0] = r["lanczos_size"][:n]
    st = r.get("probe_status")
    if st is not None:
        J.probe_status[:len(st), 0] = st
    if J.alphas is not None and r.get("alpha") is not None:
        k = min(J.max_num_samples, len(r["alpha"]))
        J.alphas[0][:k] = r["alpha"][:k]
        J.betas[0][:k] = r["beta"][:k]
    J.all_converged = bool(r["all_converged"])
    J.alg_wall_time += time.perf_counter() - t0
    J.engine["num_blocks"] += (r["num_probes_computed"] + b - 1) // b
    J.engine["num_probes_computed"] += int(r["num_probes_computed"])
    J.engine["gpu_launches"] += int(sum(launches))


def run_job(J):
    """Run every group of J with slq_run on the current stream (on several
    devices when the job asks for them and has one run)."""
    import torch
    D = getattr(J, "num_devices", 1)
    if D > 1 and len(J.params) == 1:
        run_job_multi(J, D)
        return
    J.num_devices = 1
    lib = _lib.load()
    dev_op = J.dev_op
    stream = torch.cuda.current_stream(dev_op.device)
    for gi, prm in enumerate(J.params):
        gq = len(J.groups[gi])
        if J.per_group_t is not None and gi > 0:
            J.dev_op = None
            J.dev_op = J.Aop.device_operator_for(
                J.per_group_t[J.groups[gi][0]], J.need_transpose)
            dev_op = J.dev_op
        ws_bytes = ctypes.c_size_t(0)
        _lib.check(lib.slq_run_workspace_bytes(dev_op.handle,
                                               ctypes.byref(prm), gq,
                                               ctypes.byref(ws_bytes)))
        workspace = torch.empty(int(ws_bytes.value), dtype=torch.uint8,
                                device=dev_op.device)
        res, a = run_outputs(J, gi)
        t_g = J.t_groups[gi]
        status = lib.slq_run(dev_op.handle, ctypes.byref(prm),
                             t_g.ctypes.data, gq, workspace.data_ptr(),
                             workspace.numel(), stream.cuda_stream,
                             ctypes.byref(res))
        del workspace
        collect(J, gi, res, a, status)


PROBE_FLAG_NAMES = (
    (_lib.PROBE_NONFINITE, "non-finite Lanczos coefficients"),
    (_lib.PROBE_EIGEN, "tridiagonal eigen-solve did not converge"),
    (_lib.PROBE_NODE, "non-positive quadrature node under log (or zero "
                      "node under 1/x): is the matrix positive definite?"),
    (_lib.PROBE_SAMPLE, "non-finite sample"),
)


def _warn_probe_status(J):
    """One warning naming the flags the engine set on the samples the
    estimate used (the reference warns only for a vanishing vector in its
    Gram-Schmidt step, c_orthogonalization.cpp:186-192)."""
    used = J.processed[:int(np.max(J.num_samples_used))] \
        if J.num_samples_used.size else J.processed[:0]
    st = J.probe_status[used]
    st = st[st > 0]
    if st.size == 0:
        return
    import warnings
    names = [name for bit, name in PROBE_FLAG_NAMES
             if np.any(st & bit)]
    warnings.warn("SLQ: %d of %d samples flagged: %s (per-sample flags in "
                  "info['engine']['probe_status'])"
                  % (st.size, used.size, "; ".join(names)))


def _precision_info(J):
    """The arithmetic of the run: operator dtype, where each part of the
    computation runs in which precision, and the SpMM format the operator
    holds."""
    op = J.dev_op
    b = J.engine.get("block_size") or 0
    fp64 = J.dtype_str == "float64"
    # bar: largest relative difference of a sample from the FP64 engine's on
    # the same probes that the test suite holds this format to (None where
    # no such bar is tested)
    if getattr(op, "dense", False):
        spmm = "dense, tensor cores (TF32 three-term products, FP32 sums)"
        bar = None
    elif getattr(op, "block_formats", None) and b in (128, 256):
        spmm = ("128-row blocks, tensor cores (FP16 three-product split of "
                "scaled FP32 values, FP32 accumulation)")
        bar = 1e-5
    elif getattr(op, "group_rows", 0):
        spmm = "row groups of %d rows, CUDA cores" % op.group_rows
        bar = 1e-6
    else:
        spmm = "CSR, CUDA cores"
        bar = 1e-6
    return {
        "operator_dtype": J.dtype_str,
        "mode": "fp64" if fp64 else "mixed",
        "spmm": spmm,
        "vector_storage": J.dtype_str,
        "reductions": "float64",
        "eigensolve_quadrature": "float64",
        "sample_rel_diff_vs_fp64_tested": 0.0 if fp64 else bar,
    }


def block_width(max_num_samples, block_size, dtype_str):
    """The engine's block width for these settings (make_plan's rule)."""
    b = block_size
    if b <= 0:
        b = min(256, 1 << max(0, (max_num_samples - 1).bit_length()))
    bmax = 512 if dtype_str == "float64" else 1024
    return min(1 << max(0, (b - 1).bit_length()), bmax,
               1 << max(0, (max_num_samples - 1).bit_length()))


def finish(J):
    """(trace, info) of a completed job, as ``trace_estimator.pyx:260-390``
    returns them."""
    import torch
    J.engine["block_size"] = block_width(J.max_num_samples,
                                         J.params[0].block_size, J.dtype_str)
    tot_wall_time = time.perf_counter() - J.init_wall
    cpu_proc_time = time.process_time() - J.init_proc
    Aop = J.Aop
    props = torch.cuda.get_device_properties(J.dev_op.device)
    out_dtype = np.dtype(J.dtype_str)
    trace_out = J.trace.astype(out_dtype)
    error_out = J.error.astype(out_dtype)
    samples_out = J.samples.astype(out_dtype)
    ngroups = len(J.groups)
    info = {
        "matrix": {
            "data_type": J.data_type_name,
            "gram": J.gram,
            "exponent": J.exponent,
            "size": (Aop.get_num_rows(), Aop.get_num_columns()),
            "sparse": Aop.is_sparse(),
            "nnz": Aop.get_nnz(),
            "density": Aop.get_density(),
            "num_inquiries": J.num_inquiries,
            "num_operator_parameters": Aop.get_num_parameters(),
            "parameters": J.parameters,
        },
        "error": {
            "absolute_error": None,
            "relative_error": None,
            "error_atol": J.error_atol,
            "error_rtol": J.error_rtol,
            "confidence_level": J.confidence_level,
            "outlier_significance_level": J.outlier_significance_level,
        },
        "convergence": {
            "converged": None,
            "all_converged": bool(J.all_converged),
            "min_num_samples": J.min_num_samples,
            "max_num_samples": J.max_num_samples,
            "num_samples_used": None,
            "num_outliers": None,
            "samples": None,
            "samples_mean": None,
            "samples_processed_order": J.processed,
        },
        "time": {
            "tot_wall_time": tot_wall_time,
            "alg_wall_time": J.alg_wall_time,
            "cpu_proc_time": cpu_proc_time,
        },
        "device": {
            "num_cpu_threads": J.num_threads,
            "num_gpu_devices": getattr(J, "num_devices", 1),
            "num_gpu_multiprocessors": props.multi_processor_count,
            "num_gpu_threads_per_multiprocessor":
                props.max_threads_per_multi_processor,
        },
        "solver": {
            "version": __version__,
            "lanczos_degree": J.lanczos_degree,
            "lanczos_tol": J.lanczos_tol,
            "orthogonalize": J.orthogonalize,
            "seed": J.seed_used if J.seed is not None and J.seed >= 0
            else -1,
            "method": "slq",
        },
        "engine": dict(J.engine, lanczos_size=J.lanczos_size[:, 0]
                       if ngroups == 1 else J.lanczos_size,
                       probe_status=J.probe_status[:, 0]
                       if ngroups == 1 else J.probe_status),
        "precision": _precision_info(J),
    }
    _warn_probe_status(J)
    if J.alphas is not None:
        info["engine"]["alpha"] = J.alphas[0] if ngroups == 1 else J.alphas
        info["engine"]["beta"] = J.betas[0] if ngroups == 1 else J.betas

    output_is_array = not (J.parameters is None or np.isscalar(J.parameters))
    eps = np.finfo(float).eps
    if output_is_array:
        info["error"]["absolute_error"] = error_out
        info["error"]["relative_error"] = error_out / (np.abs(trace_out) + eps)
        info["convergence"]["converged"] = J.converged.astype(bool)
        info["convergence"]["num_samples_used"] = J.num_samples_used
        info["convergence"]["num_outliers"] = J.num_outliers
        info["convergence"]["samples"] = samples_out
        info["convergence"]["samples_mean"] = trace_out
    else:
        info["error"]["absolute_error"] = error_out[0]
        info["error"]["relative_error"] = \
            error_out[0] / (np.abs(trace_out[0]) + eps)
        info["convergence"]["converged"] = bool(J.converged[0])
        info["convergence"]["num_samples_used"] = J.num_samples_used[0]
        info["convergence"]["num_outliers"] = J.num_outliers[0]
        info["convergence"]["samples"] = samples_out[:, 0]
        info["convergence"]["samples_mean"] = trace_out[0]

    if J.verbose:
        print_summary(info)
    if J.plot:
        import warnings
        warnings.warn("plot=True: convergence plots are not produced by the "
                      "B200 engine (no plotting stack)")

    if output_is_array:
        return trace_out, info
    return trace_out[0], info


def trace_estimator(A, parameters, func, gram, exponent, min_num_samples,
                    max_num_samples, error_atol, error_rtol,
                    confidence_level, outlier_significance_level,
                    lanczos_degree, lanczos_tol, orthogonalize, seed,
                    num_threads, num_gpu_devices, verbose, plot, gpu,
                    options=None, func_coeff=None):
    """SLQ estimate of trace(f(A^p)) (or of f((A^T A)^p) with gram) on the
    GPU.  ``func`` is a key of ``_lib.FUNC_IDS`` ('log', 'inv', 'id', 'exp',
    'linfrac', 'indicator', 'gaussian', 'smoothstep') with its coefficients
    in ``func_coeff``.  Returns (trace, info) like ``trace_estimator.pyx``."""
    J = prepare(A, parameters, func, gram, exponent, min_num_samples,
                max_num_samples, error_atol, error_rtol, confidence_level,
                outlier_significance_level, lanczos_degree, lanczos_tol,
                orthogonalize, seed, num_threads, num_gpu_devices, verbose,
                plot, gpu, options, func_coeff)
    run_job(J)
    return finish(J)


def print_summary(info):
    """Results table in the spirit of imate's verbose output
    (trace_estimator_utilities.py:380)."""
    conv = info["convergence"]
    err = info["error"]
    q = info["matrix"]["num_inquiries"]
    tr = np.atleast_1d(conv["samples_mean"])
    ae = np.atleast_1d(err["absolute_error"])
    re = np.atleast_1d(err["relative_error"]) * 100.0
    used = np.atleast_1d(conv["num_samples_used"])
    outl = np.atleast_1d(conv["num_outliers"])
    cv = np.atleast_1d(conv["converged"])
    params = info["matrix"]["parameters"]
    print("=" * 78)
    print("i   parameter        trace      abs. error   rel. error   "
          "num  out  converged")
    print("=" * 78)
    for i in range(q):
        pv = "none" if params is None else "%.4e" % np.atleast_1d(params)[i]
        print("%-3d %-12s %+12.5e  %10.3e  %9.3f%%  %4d %4d  %s"
              % (i + 1, pv, tr[i], ae[i], re[i], used[i], outl[i],
                 bool(cv[i])))
    t = info["time"]
    d = info["device"]
    print("-" * 78)
    print("alg wall time %.4f s   total wall time %.4f s   GPU: %d SMs"
          % (t["alg_wall_time"], t["tot_wall_time"],
             d["num_gpu_multiprocessors"]))
    s = info["solver"]
    e = info["engine"]
    print("lanczos degree %d   orthogonalize %s   block %s   rng %s   "
          "kernels %d" % (s["lanczos_degree"], s["orthogonalize"],
                          e["block_size"], e["rng"], e["gpu_launches"]))
    print("=" * 78)
