"""imate_b200 -- B200-native stochastic Lanczos quadrature.

A drop-in for imate's GPU SLQ path: ``logdet``, ``traceinv``, ``trace`` and
``schatten`` with ``method='slq', gpu=True`` on scipy CSR/CSC matrices (or
``Matrix`` / ``AffineMatrixFunction`` operators), keeping imate's keyword
arguments, return values and ``info`` dictionary.  The work runs in
hand-written sm_100a CUDA kernels in ``libslq_b200.so`` (C ABI in
``include/slq.h``), called through ctypes with PyTorch tensors as device
buffers.
"""

from .__version__ import __version__
from ._functions import (logdet, traceinv, trace, schatten, trexp,
                         trlinfrac, eigencount, density)
from ._trace_estimator import EngineOptions
from .linear_operator import (LinearOperator, Matrix, AffineMatrixFunction,
                              GramAffineMatrixFunction, DeviceMatrix)
from .sample_matrices import (toeplitz, toeplitz_logdet, toeplitz_trace,
                              toeplitz_traceinv, correlation_matrix)

__all__ = ["__version__", "logdet", "traceinv", "trace", "schatten",
           "trexp", "trlinfrac", "eigencount", "density",
           "EngineOptions", "LinearOperator", "Matrix",
           "AffineMatrixFunction", "GramAffineMatrixFunction", "DeviceMatrix",
           "toeplitz", "toeplitz_logdet", "toeplitz_trace",
           "toeplitz_traceinv", "correlation_matrix"]
