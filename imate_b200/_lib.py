"""ctypes binding of ``libslq_b200.so`` (declarations in ``include/slq.h``).

Replaces imate's runtime loader of the CUDA libraries
(``imate/_cuda_dynamic_loading/dynamic_loading.h:97-110``): the engine is one
in-tree shared library, linked against the CUDA runtime only, and loading it
fails loudly when it is missing -- there is no CPU fallback.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libslq_b200.so")

SLQ_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "BAD_ARG", 2: "BAD_CSR", 3: "WORKSPACE", 4: "CUDA",
    5: "NAN", 6: "EIGEN", 7: "UNSUPPORTED", 8: "TIMEOUT",
}
SLQ_F32, SLQ_F64 = 0, 1
ABI_VERSION = 5
# per-probe status bits (slq_result.probe_status)
PROBE_NONFINITE, PROBE_EIGEN, PROBE_NODE, PROBE_SAMPLE = 1, 2, 4, 8
SLQ_CSR, SLQ_CSC = 0, 1
FUNC_IDS = {"log": 0, "inv": 1, "id": 2, "exp": 3, "linfrac": 4,
            "indicator": 5, "gaussian": 6, "smoothstep": 7}
RNG_IDS = {"parity": 0, "fast": 1}
MAX_DEGREE = 256

# every symbol include/slq.h declares
EXPORTS = (
    "slq_operator_workspace_bytes", "slq_operator_create",
    "slq_operator_destroy", "slq_operator_dot", "slq_run_workspace_bytes",
    "slq_run", "slq_generate_probes", "slq_generate_probes_workspace_bytes",
    "slq_nodes_weights", "slq_check_convergence", "slq_average_estimates",
    "slq_erfinv", "slq_xoshiro_jump_ahead", "slq_device_info",
    "slq_last_error", "slq_abi_version", "slq_profile_begin",
    "slq_profile_end", "slq_generate_probes_noalloc", "slq_mlp_forward",
    "slq_mlp_grad", "slq_mlp_train", "slq_operator_tune_workspace_bytes",
    "slq_operator_tune", "slq_operator_set_variant",
    "slq_batch_workspace_bytes", "slq_batch_create", "slq_batch_run",
    "slq_batch_info", "slq_batch_destroy", "slq_group_order",
    "slq_rcm_order", "slq_tc_selftest", "slq_tc_selftest_mn",
    "slq_order_spread", "slq_group_fill", "slq_block_order",
    "slq_block_group_order", "slq_operator_blocks_info",
    "slq_rcm_order_device_workspace_bytes", "slq_rcm_order_device",
    "slq_dense_operator_workspace_bytes", "slq_dense_operator_create",
    "slq_operator_blocks_scratch_bytes", "slq_operator_blocks_bytes",
    "slq_operator_add_blocks", "slq_debug_fail_stream_waits",
    "slq_debug_blocks_sorted_keys",
)
TUNE_MAX_CANDIDATES = 16
SPMM_KINDS = ("csr", "row-group", "row-group-tma", "row-group-tc", "block-tc")
MLP_WIDTH = 64
MLP_PARAMS = 64 + 64 + 64 * 64 + 64 + 64 + 1
MLP_MAX_BATCH = 64


class SlqError(RuntimeError):
    """A status other than SLQ_OK returned by the engine."""

    def __init__(self, status, message):
        self.status = status
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status),
                                     message))


class SlqParams(ctypes.Structure):
    _fields_ = [
        ("func", ctypes.c_int),
        ("gram", ctypes.c_int),
        ("exponent", ctypes.c_double),
        ("orthogonalize", ctypes.c_int),
        ("seed", ctypes.c_int64),
        ("lanczos_degree", ctypes.c_int),
        ("lanczos_tol", ctypes.c_double),
        ("min_num_samples", ctypes.c_int),
        ("max_num_samples", ctypes.c_int),
        ("error_atol", ctypes.c_double),
        ("error_rtol", ctypes.c_double),
        ("confidence_level", ctypes.c_double),
        ("outlier_significance_level", ctypes.c_double),
        ("block_size", ctypes.c_int),
        ("rng", ctypes.c_int),
        ("first_probe", ctypes.c_int64),
        ("func_coeff", ctypes.c_double * 4),
    ]


KERNEL_KINDS = ("spmm", "dots", "reorth", "finalize", "eig", "probe", "other",
                "split")


class SlqKernelStat(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_int64),
        ("milliseconds", ctypes.c_double),
        ("bytes", ctypes.c_double),
    ]


class SlqResult(ctypes.Structure):
    _fields_ = [
        ("trace", ctypes.c_void_p),
        ("error", ctypes.c_void_p),
        ("samples", ctypes.c_void_p),
        ("processed_samples_indices", ctypes.c_void_p),
        ("num_samples_used", ctypes.c_void_p),
        ("num_outliers", ctypes.c_void_p),
        ("converged", ctypes.c_void_p),
        ("lanczos_size", ctypes.c_void_p),
        ("alpha", ctypes.c_void_p),
        ("beta", ctypes.c_void_p),
        ("probe_status", ctypes.c_void_p),
        ("all_converged", ctypes.c_int32),
        ("num_blocks", ctypes.c_int32),
        ("num_probes_computed", ctypes.c_int64),
        ("gpu_launches", ctypes.c_int64),
        ("alg_wall_time", ctypes.c_float),
    ]


class SlqTuneResult(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32),
        ("transpose", ctypes.c_int32),
        ("num_candidates", ctypes.c_int32),
        ("chosen", ctypes.c_int32),
        ("kind", ctypes.c_int32 * 16),
        ("group_rows", ctypes.c_int32 * 16),
        ("lanes_vec", ctypes.c_int32 * 16),
        ("slices", ctypes.c_int32 * 16),
        ("milliseconds", ctypes.c_double * 16),
    ]


_lib = None


def _declare(lib):
    vp, sz, i32, i64, d = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                           ctypes.c_int64, ctypes.c_double)
    psz = ctypes.POINTER(ctypes.c_size_t)
    sig = {
        "slq_operator_workspace_bytes": (i32, [i64, i64, i64, i32, i32, i32,
                                               i32, i32, psz]),
        "slq_operator_create": (i32, [vp, vp, vp, i64, i64, i64, i32, i32,
                                      i32, i32, i32, vp, i32, vp, sz, vp,
                                      ctypes.POINTER(vp)]),
        "slq_operator_destroy": (i32, [vp]),
        "slq_operator_dot": (i32, [vp, i32, d, vp, vp, i32, vp]),
        "slq_run_workspace_bytes": (i32, [vp, ctypes.POINTER(SlqParams), i32,
                                          psz]),
        "slq_run": (i32, [vp, ctypes.POINTER(SlqParams), vp, i32, vp, sz, vp,
                          ctypes.POINTER(SlqResult)]),
        "slq_generate_probes": (i32, [i64, i32, i64, i64, i32, i32, i32, vp,
                                      vp, sz, vp]),
        "slq_generate_probes_workspace_bytes": (i32, [i64, i32, psz]),
        "slq_generate_probes_noalloc": (i32, [i64, i32, i64, i64, i32, i32,
                                              i32, vp, vp]),
        "slq_nodes_weights": (i32, [vp, vp, vp, i32, i32, i32, vp, vp, vp,
                                    vp]),
        "slq_check_convergence": (i32, [vp, i32, i32, vp, i32, d, d, d, vp,
                                        vp, vp]),
        "slq_average_estimates": (None, [d, d, i32, i32, vp, vp, vp, vp, vp,
                                         vp]),
        "slq_erfinv": (d, [d]),
        "slq_xoshiro_jump_ahead": (None, [vp, ctypes.c_uint64]),
        "slq_device_info": (i32, [vp, vp, vp]),
        "slq_last_error": (ctypes.c_char_p, []),
        "slq_profile_begin": (i32, []),
        "slq_profile_end": (i32, [ctypes.POINTER(SlqKernelStat)]),
        "slq_abi_version": (i32, []),
        "slq_mlp_forward": (i32, [vp, vp, i32, vp, vp]),
        "slq_mlp_grad": (i32, [vp, vp, vp, i32, vp, vp, vp]),
        "slq_mlp_train": (i32, [vp, vp, vp, vp, vp, i32, i32, i32,
                                ctypes.c_float, vp, vp]),
        "slq_operator_tune_workspace_bytes": (i32, [vp, i32, psz]),
        "slq_operator_tune": (i32, [vp, i32, i32, i32, vp, sz, vp,
                                    ctypes.POINTER(SlqTuneResult)]),
        "slq_operator_set_variant": (i32, [vp, i32, i32, i32]),
        "slq_batch_workspace_bytes": (i32, [i32, vp, vp, vp, psz]),
        "slq_batch_create": (i32, [i32, vp, vp, vp, vp, vp, sz, vp,
                                   ctypes.POINTER(vp)]),
        "slq_batch_run": (i32, [vp, vp, vp]),
        "slq_batch_info": (i32, [vp, ctypes.POINTER(i64),
                                 ctypes.POINTER(i64)]),
        "slq_batch_destroy": (i32, [vp]),
        "slq_group_order": (i32, [i64, vp, vp, vp, i32, i32, vp, vp]),
        "slq_rcm_order": (i32, [i64, vp, vp, vp]),
        "slq_block_order": (i32, [i64, vp, vp, vp, i32, i32, vp]),
        "slq_block_group_order": (i32, [i64, vp, vp, vp, i32, i32, i32, vp,
                                        vp]),
        "slq_operator_blocks_info": (i32, [vp, i32, ctypes.POINTER(i64),
                                           ctypes.POINTER(i64)]),
        "slq_order_spread": (i32, [i64, vp, vp, vp, i64, vp]),
        "slq_group_fill": (i32, [i64, vp, vp, vp, i32, i64, vp]),
        "slq_rcm_order_device_workspace_bytes": (i32, [i64, vp]),
        "slq_dense_operator_workspace_bytes": (i32, [i64, i64, i32, i32, psz]),
        "slq_dense_operator_create": (i32, [vp, i64, i64, i32, i32, i32, vp, sz,
                                            vp, ctypes.POINTER(vp)]),
        "slq_rcm_order_device": (i32, [i64, i64, vp, vp, i32, vp, vp, vp, sz,
                                        vp]),
        "slq_tc_selftest": (i32, [vp, vp, vp, i32, vp, vp]),
        "slq_operator_blocks_scratch_bytes": (i32, [vp, i32, psz]),
        "slq_operator_blocks_bytes": (i32, [vp, i32, vp, sz, vp, psz]),
        "slq_operator_add_blocks": (i32, [vp, i32, vp, sz, vp, sz, vp]),
        "slq_debug_fail_stream_waits": (i32, [i32]),
        "slq_debug_blocks_sorted_keys": (i32, [i32]),
        "slq_tc_selftest_mn": (i32, [vp, vp, vp, i32, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def load():
    """Load the engine library; raises ImportError if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libslq_b200.so is missing: build it with "
            "`python -m imate_b200._build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    _declare(lib)
    _lib = lib
    return lib


def profile_begin():
    check(load().slq_profile_begin())


def profile_end():
    """Per-kernel-class stats since profile_begin():
    {kind: (launches, milliseconds, bytes)}."""
    stats = (SlqKernelStat * len(KERNEL_KINDS))()
    check(load().slq_profile_end(stats))
    return {k: (int(s.launches), float(s.milliseconds), float(s.bytes))
            for k, s in zip(KERNEL_KINDS, stats)}


def check(status):
    if status != SLQ_OK:
        msg = load().slq_last_error()
        raise SlqError(status, msg.decode() if msg else "")
