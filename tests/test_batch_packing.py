"""Packing of batch estimates over devices (host logic, no GPU).

Every estimate of a batch runs whole on one device; the estimates are packed
by decreasing cost onto the least-loaded device.  The packing depends only on
the costs, so every process and every run place the same estimate on the
same device."""

import numpy as np
import pytest
import scipy.sparse as sp

from imate_b200.batch import pack_estimates, estimate_cost


def test_one_device_takes_everything():
    assert pack_estimates([5.0, 1.0, 3.0], 1) == [0, 0, 0]


def test_longest_first_onto_least_loaded():
    # 8 -> d0, 7 -> d1, 6 -> d1 (7 < 8), 5 -> d0 (8 < 13), 4 -> d0 (13 = 13,
    # lowest index), ...
    costs = [5.0, 8.0, 4.0, 7.0, 6.0]
    dev = pack_estimates(costs, 2)
    assert dev == [0, 0, 0, 1, 1]
    loads = [sum(c for c, d in zip(costs, dev) if d == k) for k in range(2)]
    assert loads == [17.0, 13.0]


def test_ties_broken_by_index_and_device():
    assert pack_estimates([1.0] * 6, 3) == [0, 1, 2, 0, 1, 2]


def test_pinned_estimates_stay_and_count_as_load():
    costs = [10.0, 3.0, 3.0, 3.0]
    dev = pack_estimates(costs, 2, pinned={0: 1})
    assert dev[0] == 1
    # device 0 is empty, so the free estimates fill it first
    assert dev[1:] == [0, 0, 0]
    with pytest.raises(ValueError):
        pack_estimates(costs, 2, pinned={0: 2})


def test_balance_within_the_largest_cost():
    rng = np.random.default_rng(3)
    for D in (2, 3, 4, 8):
        costs = list(rng.lognormal(0.0, 1.5, size=64))
        dev = pack_estimates(costs, D)
        loads = np.bincount(dev, weights=costs, minlength=D)
        # greedy list scheduling: the spread is at most the largest job
        assert loads.max() - loads.min() <= max(costs) + 1e-9
        # deterministic
        assert pack_estimates(costs, D) == dev


def test_estimate_cost_counts_products():
    A = sp.random(1000, 1000, density=0.01, random_state=0, format="csr")
    c = estimate_cost(A, 64, 30)
    assert c == (A.nnz + 1000) * 64 * 30
    assert estimate_cost(A, 64, 30, gram=True) == 2 * c
    assert estimate_cost(A, 64, 30, num_runs=3) == 3 * c
    D = np.ones((50, 50))
    assert estimate_cost(D, 1, 1) == 2500 + 50
