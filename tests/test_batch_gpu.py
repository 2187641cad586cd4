"""Batched generation: many uneven graphs in one persistent launch must give,
graph by graph, exactly what the single-graph generator gives (and hence the
oracle)."""
import numpy as np
import pytest
import torch

import _oracle as orc

pytestmark = pytest.mark.gpu


def _mixed(pa, count, rng, max_n=200_000, bits=32, mixed_start=False):
    """Random instances; with mixed_start each instance's start region is, at
    random, the default (the whole graph), none, or 1500 nodes (so the tail
    launch runs too)."""
    prms = []
    for i in range(count):
        n = int(round(10 ** rng.uniform(1.2, np.log10(max_n))))
        d = int(rng.integers(1, 33))
        n = max(n, d + 1)
        p = float(rng.uniform(0.1, 0.9))
        mode = int(rng.integers(0, 2))
        sn = [0, pa.PA_START_NONE, 1500][int(rng.integers(0, 3))] if mixed_start else 0
        prms.append(pa.make_params(n, d, p, seed=1000 + i, id_bits=bits, seed_mode=mode,
                                   start_nodes=sn))
    prms.sort(key=lambda q: -q.n * q.d)   # large graphs first
    return prms


@pytest.mark.parametrize("mixed_start", [False, True])
@pytest.mark.parametrize("bits", [32, 64])
def test_batch_equals_single_graph_runs(pa, cuda_ok, bits, mixed_start):
    rng = np.random.default_rng(5)
    prms = _mixed(pa, 60, rng, bits=bits, mixed_start=mixed_start)
    batch = pa.Batch(prms)
    batch.generate()
    st = batch.finish()
    assert st.status == 0
    for i, prm in enumerate(prms):
        want, _ = pa.generate(prm)
        assert torch.equal(batch.graph(i), want), f"instance {i}: n={prm.n} d={prm.d}"


def test_batch_against_oracle_and_seed_only_graphs(pa, cuda_ok):
    prms = [pa.make_params(50_000, 4, 0.5, seed=1, seed_mode=1),
            pa.make_params(7, 6, 0.5, seed=2, seed_mode=1),        # seed graph only
            pa.make_params(3000, 32, 0.2, seed=3, seed_mode=0),
            pa.make_params(2, 1, 0.5, seed=4, seed_mode=0),        # seed graph only
            pa.make_params(20_000, 1, 0.9, seed=5, seed_mode=1)]
    batch = pa.Batch(prms)
    batch.generate()
    assert batch.finish().status == 0
    for i, prm in enumerate(prms):
        G = orc.generate(prm.n, prm.d, prm.p, prm.seed, prm.seed_mode)
        want = orc.pairs_slot_order(G, prm.seed_mode)
        assert (batch.graph(i).cpu().numpy().astype(np.int64) == want).all()


def test_batch_repeatable(pa, cuda_ok):
    rng = np.random.default_rng(9)
    prms = _mixed(pa, 200, rng, max_n=50_000)
    b = pa.Batch(prms)
    b.generate()
    first = [g.clone() for g in (b.graph(i) for i in range(len(prms)))]
    b.generate()
    assert b.finish().status == 0
    assert all(torch.equal(first[i], b.graph(i)) for i in range(len(prms)))
