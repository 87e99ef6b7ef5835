"""num_gpu_devices in the drop-in API.

The reference runs one host OpenMP thread per GPU
(imate/_cu_trace_estimator/cu_trace_estimator.cu:229-299), 0 meaning every
device (trace_estimator.pyx:215-216).  Here the probe blocks of an estimate
are dealt over the devices by global probe index and the host replays the
stopping rule, so any device count gives the one-device result exactly.  A
box with one GPU checks that 0 (all devices) and 1 agree and that the dealing
itself -- two host threads, two logical devices mapped onto the one GPU --
reproduces the one-device estimate bit for bit."""

import numpy as np
import pytest

import imate_b200 as ib
from imate_b200 import _trace_estimator as te

pytestmark = pytest.mark.gpu

KW = dict(min_num_samples=50, max_num_samples=200, error_rtol=1e-3,
          lanczos_degree=30, orthogonalize=-1, seed=0)


def test_num_gpu_devices_zero_means_every_device(cuda):
    import torch
    B = ib.toeplitz(2.0, 1.0, 16384)
    tr1, i1 = ib.logdet(B, gram=True, method="slq", gpu=True,
                        return_info=True, num_gpu_devices=1, **KW)
    tr0, i0 = ib.logdet(B, gram=True, method="slq", gpu=True,
                        return_info=True, num_gpu_devices=0, **KW)
    assert i0["device"]["num_gpu_devices"] == torch.cuda.device_count()
    assert i1["device"]["num_gpu_devices"] == 1
    assert tr0 == tr1
    np.testing.assert_array_equal(i0["convergence"]["samples"],
                                  i1["convergence"]["samples"])


def test_blocks_dealt_over_two_devices_equal_one_device(cuda):
    B = ib.toeplitz(2.0, 1.0, 16384)
    args = (B, None, "log", True, 1.0, KW["min_num_samples"],
            KW["max_num_samples"], None, KW["error_rtol"], 0.95, 0.001,
            KW["lanczos_degree"], None, KW["orthogonalize"], KW["seed"], 0,
            1, False, False, True)
    J1 = te.prepare(*args, options=ib.EngineOptions(block_size=32))
    te.run_job(J1)
    tr1, i1 = te.finish(J1)
    J2 = te.prepare(*args, options=ib.EngineOptions(block_size=32))
    te.run_job_multi(J2, 2, device_of=lambda d: 0)
    tr2, i2 = te.finish(J2)
    c1, c2 = i1["convergence"], i2["convergence"]
    assert c1["num_samples_used"] == c2["num_samples_used"]
    used = int(c1["num_samples_used"])
    np.testing.assert_array_equal(c1["samples_processed_order"][:used],
                                  c2["samples_processed_order"][:used])
    np.testing.assert_array_equal(c1["samples"], c2["samples"])
    assert tr1 == tr2
    assert i1["error"]["absolute_error"] == i2["error"]["absolute_error"]
    assert c1["num_outliers"] == c2["num_outliers"]
    np.testing.assert_array_equal(i1["engine"]["lanczos_size"][:used],
                                  i2["engine"]["lanczos_size"][:used])
