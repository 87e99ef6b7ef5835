"""Probe sharding across ranks (imate_b200.distributed) on CPU gloo ranks.

Each rank computes the samples of its global probe indices with the oracle
(standing in for its GPU), the ranks all_gather them, and every rank replays
the reference's stopping rule.  The result must equal the single-process
estimate for any world size."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from imate_b200.distributed import shard_block

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _matrix():
    import imate_b200 as ib
    return ib.correlation_matrix(300, scale=0.1, threshold=0.05, shift=0.2,
                                 seed=2)


KW = dict(lanczos_degree=12, orthogonalize=-1, seed=7)


def _oracle_block(A, first, count):
    from oracle import oracle
    r = oracle.trace_estimator(A, "log", min_num_samples=first + count,
                               max_num_samples=first + count, error_rtol=0.0,
                               **KW)
    return r["samples"][first:first + count]


def _worker(rank, world, port, block, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    from imate_b200.distributed import distributed_trace_estimator
    A = _matrix()
    res = distributed_trace_estimator(
        lambda first, count: _oracle_block(A, first, count), q=1,
        block=block, min_num_samples=6, max_num_samples=40,
        error_rtol=2e-3)
    np.savez(os.path.join(out_dir, "rank%d.npz" % rank),
             **{k: np.asarray(v) for k, v in res.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_shard_block_covers_probes_disjointly():
    seen = []
    for k in range(3):
        for r in range(4):
            first, count = shard_block(k, 4, r, 8)
            seen.extend(range(first, first + count))
    assert seen == list(range(96))


@pytest.mark.parametrize("world,block", [(2, 4), (2, 16), (3, 5)])
def test_sharded_estimate_equals_single_process(tmp_path, world, block):
    from oracle import oracle
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker,
                         args=(r, world, port, block, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    want = oracle.trace_estimator(_matrix(), "log", min_num_samples=6,
                                  max_num_samples=40, error_rtol=2e-3, **KW)
    res = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(world)]
    for r in res:
        # every rank ends with the same, single-process answer
        assert int(r["num_samples_used"][0]) == int(want["num_samples_used"][0])
        used = int(want["num_samples_used"][0])
        np.testing.assert_array_equal(r["samples"][:used, 0],
                                      want["samples"][:used, 0])
        assert abs(r["trace"][0] - want["trace"][0]) <= \
            1e-13 * abs(want["trace"][0])
        np.testing.assert_array_equal(r["num_outliers"], want["num_outliers"])
    assert int(res[0]["rounds"]) >= 1


@pytest.mark.parametrize("devices,block", [(1, 4), (2, 4), (3, 5), (4, 16)])
def test_multi_device_estimate_equals_single_device(devices, block):
    # the probe blocks of one estimate dealt over the devices of one process
    # (one host thread each, here a stand-in that serves the oracle's
    # samples): every device count gives the single-device answer, and
    # device d gets the blocks d, d + D, ... of the global probe order
    from oracle import oracle
    from imate_b200.distributed import multi_device_trace_estimator
    A = _matrix()
    want = oracle.trace_estimator(A, "log", min_num_samples=6,
                                  max_num_samples=40, error_rtol=2e-3, **KW)
    every = oracle.trace_estimator(A, "log", min_num_samples=40,
                                   max_num_samples=40, error_rtol=0.0,
                                   **KW)["samples"]
    calls = []

    def run_block(device, first, count):
        calls.append((device, first, count))
        return {"samples": every[first:first + count],
                "lanczos_size": np.full(count, 12, dtype=np.int32),
                "probe_status": np.zeros(count, dtype=np.int32)}
    res = multi_device_trace_estimator(run_block, devices, 1, block, 6, 40,
                                       error_rtol=2e-3)
    used = int(want["num_samples_used"][0])
    assert int(res["num_samples_used"][0]) == used
    np.testing.assert_array_equal(res["samples"][:used, 0],
                                  want["samples"][:used, 0])
    assert np.all(np.isnan(res["samples"][used:, 0]))
    np.testing.assert_array_equal(res["processed_samples_indices"][:used],
                                  want["processed_samples_indices"][:used])
    assert abs(res["trace"][0] - want["trace"][0]) <= \
        1e-13 * abs(want["trace"][0])
    np.testing.assert_array_equal(res["num_outliers"], want["num_outliers"])
    assert len(res["lanczos_size"]) == used
    for device, first, count in calls:
        assert (first // block) % devices == device
    # no round is started once the rule has stopped
    assert res["num_probes_computed"] < used + devices * block
