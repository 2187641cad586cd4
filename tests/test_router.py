"""Placement across GPUs without a GPU: the router's rule (pa_route_pick) and
the batch partition (pa_batch_partition) are host arithmetic."""
import numpy as np
import pytest


def test_route_pick_smallest_fraction_of_budget(pa):
    assert pa.route_pick([0, 0], [100, 100], 10) == 0                 # tie: lowest index
    assert pa.route_pick([50, 10], [100, 100], 10) == 1
    assert pa.route_pick([50, 60], [100, 200], 10) == 1               # 70/200 < 60/100
    assert pa.route_pick([0], [1], 1 << 40) == 0
    # exact comparison where floating point would round: huge budgets
    big = 1 << 62
    assert pa.route_pick([big - 2, big - 3], [big, big], 1) == 1


def test_route_pick_spreads_equal_requests(pa):
    load, budget = [0, 0, 0, 0], [1000, 1000, 2000, 1000]
    picks = []
    for _ in range(50):
        i = pa.route_pick(load, budget, 10)
        load[i] += 10
        picks.append(i)
    counts = np.bincount(picks, minlength=4)
    assert counts[2] == 20 and (counts[[0, 1, 3]] == 10).all()        # by budget share


@pytest.mark.parametrize("k", [1, 2, 3, 8])
def test_batch_partition_is_balanced_and_complete(pa, k):
    rng = np.random.default_rng(3)
    prms = []
    for i in range(300):
        d = int(rng.integers(1, 33))
        n = max(d + 1, int(round(10 ** rng.uniform(2, 6))))
        prms.append(pa.make_params(n, d, 0.5, seed=i))
    part = pa.batch_partition(prms, k)
    assert len(part) == 300 and set(part) <= set(range(k))
    w = np.array([pa.sizes(q)[0] for q in prms], dtype=np.float64)
    loads = np.bincount(part, weights=w, minlength=k)
    # LPT bound: no part above the mean by more than the largest item
    assert loads.max() <= w.sum() / k + w.max()
    assert part == pa.batch_partition(prms, k)                        # deterministic


def test_batch_partition_rejects_bad_arguments(pa):
    import ctypes
    out = (ctypes.c_uint32 * 1)()
    prm = (pa.PaParams * 1)(pa.make_params(100, 4, 0.5))
    assert pa.lib().pa_batch_partition(prm, 1, 0, out) == pa.PA_ERR_INVALID
    bad = (pa.PaParams * 1)(pa.make_params(100, 4, 0.5))
    bad[0].d = 0
    assert pa.lib().pa_batch_partition(bad, 1, 2, out) == pa.PA_ERR_INVALID
    assert pa.batch_partition([], 4) == []
