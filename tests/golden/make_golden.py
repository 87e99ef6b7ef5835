"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own CPU SLQ (ameli/imate v0.25.2), compiled from its
sources by ``make -C oracle ref`` into ``oracle/_ref/libimate_ref.so``, on
seeded inputs and stores what it returns:

  rng.npz        xoshiro256** stream words and Rademacher probes
                 (random_array_generator.cpp:63-165) for several seeds / n
  krylov.npz     per-probe alpha/beta of Lanczos and Golub-Kahn
                 (c_lanczos_tridiagonalization.cpp, c_golub_kahn_
                 bidiagonalization.cpp) and LAPACK nodes/weights
                 (diagonalization.cpp) on the Toeplitz workload and a small
                 correlation matrix
  estimator.npz  full estimator outputs (c_trace_estimator.cpp:192-307,
                 num_threads=1): samples, processed order, num_samples_used,
                 outliers, trace, error
  functions.npz  the same for the other matrix functions of imate's SLQ
                 consumers (functions/exponential.cpp, homographic.cpp,
                 indicator.cpp, gaussian.cpp, smoothstep.cpp) with their
                 coefficients, settings in FUNC_SETTINGS

Usage (needs the reference tree and oracle/_ref built):
    python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import ref  # noqa: E402
from golden_cases import FUNC_CASES, FUNC_SETTINGS  # noqa: E402
from imate_b200.sample_matrices import toeplitz, correlation_matrix  # noqa


def small_correlation(dtype="float64"):
    # n = 400 points, scale 0.1, threshold 0.05, shift 0.1 (SPD)
    return correlation_matrix(400, scale=0.1, threshold=0.05, shift=0.1,
                              seed=11, dtype=dtype)


def make_rng():
    out = {}
    for seed in (0, 1, 7, 123456789):
        # words 0..299 of the stream = probes of n=64*k-1.. via one stream
        v = ref.random_probes(seed, 64 * 299 + 63, 1)[0]
        bits = (v > 0).astype(np.uint8)
        out["bits_seed%d" % seed] = np.packbits(bits, bitorder="little")
    for seed, n in ((0, 1), (0, 63), (0, 64), (0, 65), (3, 1000), (5, 4097)):
        v = ref.random_probes(seed, n, 5)
        out["probes_seed%d_n%d" % (seed, n)] = (v > 0).astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "rng.npz"), **out)


def make_krylov():
    out = {}
    n = 16384
    B = toeplitz(2.0, 1.0, n)
    probes = ref.random_probes(0, n, 4)
    for orth in (0, -1, 10):
        for p in range(4):
            a, b = ref.krylov(B, probes[p], 30, gram=True, orthogonalize=orth)
            th, tau = ref.nodes_weights(a, b, gram=True)
            key = "c1_orth%d_p%d" % (orth, p)
            out[key + "_alpha"] = a
            out[key + "_beta"] = b
            out[key + "_theta"] = th
            out[key + "_tau"] = tau
    C = small_correlation()
    out["corr_data"] = C.data
    out["corr_indices"] = C.indices.astype(np.int32)
    out["corr_indptr"] = C.indptr.astype(np.int32)
    probes = ref.random_probes(5, C.shape[0], 4)
    for orth in (0, -1, 1, 5):
        for p in range(4):
            a, b = ref.krylov(C, probes[p], 20, gram=False,
                              orthogonalize=orth)
            th, tau = ref.nodes_weights(a, b, gram=False)
            key = "corr_orth%d_p%d" % (orth, p)
            out[key + "_alpha"] = a
            out[key + "_beta"] = b
            out[key + "_theta"] = th
            out[key + "_tau"] = tau
    # affine A + t I at t = 0.5
    for p in range(2):
        a, b = ref.krylov(C, probes[p], 20, gram=False, orthogonalize=-1,
                          t=0.5)
        out["corr_t0.5_p%d_alpha" % p] = a
        out["corr_t0.5_p%d_beta" % p] = b
    np.savez_compressed(os.path.join(HERE, "krylov.npz"), **out)


def _store(out, key, r):
    for k in ("trace", "error", "samples", "processed_samples_indices",
              "num_samples_used", "num_outliers", "converged"):
        out[key + "_" + k] = np.asarray(r[k])
    out[key + "_all_converged"] = np.asarray(r["all_converged"])


def make_estimator():
    out = {}
    n = 16384
    B = toeplitz(2.0, 1.0, n)
    for orth in (0, -1):
        r = ref.trace_estimator(B, "log", gram=True, min_num_samples=50,
                                max_num_samples=200, error_rtol=1e-3,
                                lanczos_degree=30, orthogonalize=orth,
                                seed=0, num_threads=1)
        _store(out, "c1_log_orth%d" % orth, r)
    C = small_correlation()
    for func in ("log", "inv", "id"):
        r = ref.trace_estimator(C, func, gram=False, min_num_samples=10,
                                max_num_samples=64, error_rtol=1e-2,
                                lanczos_degree=20, orthogonalize=0, seed=3,
                                num_threads=1)
        _store(out, "corr_%s" % func, r)
    r = ref.trace_estimator(C, "log", gram=True, min_num_samples=10,
                            max_num_samples=40, error_rtol=1e-2,
                            lanczos_degree=15, orthogonalize=-1, seed=4,
                            num_threads=1)
    _store(out, "corr_gram_log", r)
    r = ref.trace_estimator(C, "inv", parameters=[0.1, 1.0, 10.0],
                            min_num_samples=5, max_num_samples=30,
                            error_rtol=1e-3, lanczos_degree=20,
                            orthogonalize=-1, seed=9, num_threads=1)
    _store(out, "corr_affine_inv", r)
    r = ref.trace_estimator(C, "log", exponent=2.0, min_num_samples=5,
                            max_num_samples=20, error_rtol=1e-2,
                            lanczos_degree=10, orthogonalize=3, seed=2,
                            num_threads=1)
    _store(out, "corr_log_p2", r)
    np.savez_compressed(os.path.join(HERE, "estimator.npz"), **out)


def make_functions():
    out = {}
    C = small_correlation()
    for name, func, coeff, gram, params in FUNC_CASES:
        r = ref.trace_estimator(C, func, gram=gram, parameters=params,
                                coeff=coeff, num_threads=1, **FUNC_SETTINGS)
        _store(out, "fn_" + name, r)
    np.savez_compressed(os.path.join(HERE, "functions.npz"), **out)


if __name__ == "__main__":
    make_rng()
    make_krylov()
    make_estimator()
    make_functions()
    for f in ("rng.npz", "krylov.npz", "estimator.npz", "functions.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
