"""Captured generations (pa_plan_*) and the autotuner on the GPU: a replayed
plan writes what pa_generate writes, and every launch shape the tuner tries
generates the same graph."""
import numpy as np
import pytest
import torch

from cuppa_b200 import autotune as at

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,d,bits", [(100_000, 4, 32), (30_000, 16, 64), (7, 6, 32)])
def test_plan_replay_equals_generate(pa, cuda_ok, n, d, bits):
    prm = pa.make_params(n, d, 0.5, seed=11, id_bits=bits)
    want, _ = pa.generate(prm)
    edges, scratch = pa.alloc_buffers(prm)
    plan = pa.Plan(prm, edges, scratch)
    s = torch.cuda.Stream()
    for _ in range(2):
        edges.zero_()
        torch.cuda.synchronize()
        plan.launch(s)
        assert pa.finish(scratch, s).status == 0
        assert torch.equal(edges[: pa.edge_count(prm)], want)
    plan.close()


def test_every_tuned_shape_gives_the_same_graph(pa, cuda_ok):
    n, d = 40_000, 4
    want, _ = pa.generate(pa.make_params(n, d, 0.5, seed=1, id_bits=32))
    for shape in at.candidates(torch.cuda.get_device_properties(0).multi_processor_count):
        got, st = pa.generate(at.apply(pa.make_params(n, d, 0.5, seed=1, id_bits=32), shape))
        assert st.status == 0 and torch.equal(got, want), shape
    best, times = at.tune(n, d, 0.5, 32, reps=2, path=None, table={})
    assert best in at.candidates(torch.cuda.get_device_properties(0).multi_processor_count)
    assert len(times) == len(at.candidates())
