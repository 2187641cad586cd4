"""pa_fill + PA_FLAG_PREFILLED: a generation into a buffer filled beforehand
(on another stream, as a back-to-back caller does with two buffers) writes
exactly the graph of an ordinary generation -- every layout and kernel path."""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,d,bits,layout", [(200_000, 4, 64, 0), (50_001, 7, 32, 0),
                                             (30_000, 5, 32, 1), (5_000, 40, 64, 0),
                                             (3_001, 33, 32, 1)])
def test_prefilled_generation_equals_plain(pa, cuda_ok, n, d, bits, layout):
    prm = pa.make_params(n, d, 0.5, seed=17, id_bits=bits, layout=layout)
    want, _ = pa.generate(prm)
    edges, scratch = pa.alloc_buffers(prm)
    edges.fill_(123)                       # a previous graph's leftovers
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        pa.fill(prm, edges, side)
    torch.cuda.current_stream().wait_stream(side)
    q = pa.make_params(n, d, 0.5, seed=17, id_bits=bits, layout=layout,
                       flags=pa.PA_FLAG_PREFILLED)
    pa.generate_into(q, edges, scratch)
    assert pa.finish(scratch).status == 0
    got = edges[: want.shape[0]]
    assert torch.equal(got, want)


def test_fill_of_a_seed_only_graph_is_empty(pa, cuda_ok):
    """n = d + 1 has no generated slots: the fill writes nothing and the
    prefilled generation still writes the seed edges."""
    prm = pa.make_params(5, 4, 0.5, seed=1, id_bits=64)
    edges, scratch = pa.alloc_buffers(prm)
    edges.fill_(7)
    pa.fill(prm, edges)
    torch.cuda.synchronize()
    assert bool((edges == 7).all())
    q = pa.make_params(5, 4, 0.5, seed=1, id_bits=64, flags=pa.PA_FLAG_PREFILLED)
    pa.generate_into(q, edges, scratch)
    assert pa.finish(scratch).status == 0
    want, _ = pa.generate(prm)
    assert torch.equal(edges[: want.shape[0]], want)
