"""GPU generator vs the oracle, through the C ABI.

Bar: bit-exact.  The generator's PAIRS layout (seed edges, then each node's d
pairs in slot order) is compared with the oracle's identical layout, so every
slot value and its order are checked, not just the edge set."""
import json
import os

import numpy as np
import pytest

import _oracle as orc

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gpu_pairs(pa, n, d, p, seed, mode, bits, **kw):
    prm = pa.make_params(n, d, p, seed=seed, id_bits=bits, seed_mode=mode, **kw)
    edges, st = pa.generate(prm)
    return prm, edges, st


def assert_bit_exact(pa, n, d, p, seed, mode, bits, **kw):
    prm, edges, st = gpu_pairs(pa, n, d, p, seed, mode, bits, **kw)
    assert st.status == 0
    G, retries = orc.generate(n, d, p, seed, mode, with_retries=True)
    want = orc.pairs_slot_order(G, mode)
    got = edges.cpu().numpy().astype(np.int64)
    assert got.shape == want.shape
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, f"first mismatch at pair {bad[:5]}: got {got[bad[:3]]} want {want[bad[:3]]}"
    assert st.retries == retries
    return prm, edges


SWEEP = []
for d in (1, 2, 3, 4, 5, 7, 8, 16, 31, 32):
    for p in (0.0, 0.1, 0.5, 0.9, 1.0):
        SWEEP.append((20000, d, p, 100 + d, 1, 32))
for n in (2, 3, 6, 7, 40, 333, 4097):
    SWEEP.append((n, 1 if n < 6 else 5, 0.5, 7, 0, 32))
for d in (4, 16):
    for mode in (0, 1):
        for bits in (32, 64):
            SWEEP.append((50000, d, 0.5, 2 ** 33 + d, mode, bits))


# How the nodes are split between the start kernel (slot-granular waits) and the
# persistent kernel (tile flags and the watermark): the default (every node of
# these small graphs in the start kernel), none in it, and a boundary inside the
# graph (2000 nodes, rounded up to whole superblocks).
START = {"start": 0, "persistent": None, "split": 2000}


def start_nodes(pa, which):
    v = START[which]
    return pa.PA_START_NONE if v is None else v


@pytest.mark.parametrize("start", list(START))
@pytest.mark.parametrize("n,d,p,seed,mode,bits", SWEEP)
def test_bit_exact_sweep(pa, cuda_ok, n, d, p, seed, mode, bits, start):
    if n < d + 1:
        pytest.skip("fewer than d+1 nodes")
    assert_bit_exact(pa, n, d, p, seed, mode, bits, start_nodes=start_nodes(pa, start))


@pytest.mark.parametrize("start", ["persistent", "split"])
@pytest.mark.parametrize("passes", [1, 2, 4, 8])
@pytest.mark.parametrize("d", [3, 4, 16])
def test_bit_exact_every_tile_shape(pa, cuda_ok, passes, d, start):
    sn = start_nodes(pa, start)
    assert_bit_exact(pa, 30000, d, 0.4, 9, 1, 32, tile_passes=passes, start_nodes=sn)
    assert_bit_exact(pa, 30000, d, 0.0, 9, 0, 64, tile_passes=passes, start_nodes=sn)


@pytest.mark.parametrize("start", list(START))
@pytest.mark.parametrize("blocks", [1, 2, 3, 7, 4000])
def test_any_grid_size_is_deadlock_free_and_exact(pa, cuda_ok, blocks, start):
    """Work is claimed in order by running warps, so a single CTA, or far more
    CTAs than fit at once, still finish with the same bits."""
    assert_bit_exact(pa, 20000, 4, 0.3, 5, 1, 32, blocks=blocks,
                     start_nodes=start_nodes(pa, start))


def test_benchmark_cpu_config_matches_golden(pa, cuda_ok):
    """n = 100,000, d = 4, p = 0.5, int32, clique seed, Philox seed 42."""
    prm, edges, st = gpu_pairs(pa, 100000, 4, 0.5, 42, 1, 32)
    assert edges.shape[0] == 399990
    pa.canonicalize(prm, edges)
    got = edges.cpu().numpy()
    case = [c for c in json.load(open(os.path.join(GOLD, "philox_digests.json")))["cases"]
            if (c["n"], c["d"], c["seed"], c["seed_mode"]) == (100000, 4, 42, 1)][0]
    assert f"{orc.fnv1a64(got.astype(np.int32)):016x}" == case["fnv_canonical_i32"]


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLD, "philox_digests.json")))["cases"],
                         ids=lambda c: f"n{c['n']}_d{c['d']}_p{c['p']}_m{c['seed_mode']}")
def test_golden_digests(pa, cuda_ok, case):
    prm, edges, st = gpu_pairs(pa, case["n"], case["d"], case["p"], case["seed"],
                               case["seed_mode"], 64)
    got = edges.cpu().numpy()
    assert f"{orc.fnv1a64(got):016x}" == case["fnv_slot_i64"]
    pa.canonicalize(prm, edges)
    assert f"{orc.fnv1a64(edges.cpu().numpy()):016x}" == case["fnv_canonical_i64"]


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("d", [1, 4, 16, 32])
def test_canonicalize_and_degrees(pa, cuda_ok, bits, d):
    n, p, seed, mode = 30000, 0.35, 3, 1
    prm, edges, st = gpu_pairs(pa, n, d, p, seed, mode, bits)
    G = orc.generate(n, d, p, seed, mode)
    deg = pa.degrees(prm, edges).cpu().numpy()
    assert (deg == orc.degrees(G, mode)).all()
    out = edges.clone()
    pa.canonicalize(prm, edges, out)
    assert (out.cpu().numpy() == orc.pairs_canonical(G, mode)).all()
    pa.canonicalize(prm, edges)   # in place
    assert (edges.cpu().numpy() == orc.pairs_canonical(G, mode)).all()


@pytest.mark.parametrize("start", [0, 100_000])
def test_million_node_bit_exact(pa, cuda_ok, start):
    assert_bit_exact(pa, 1_000_000, 4, 0.5, 1234, 1, 64, start_nodes=start)
    assert_bit_exact(pa, 1_000_000, 4, 0.0, 1234, 1, 64, start_nodes=start)


def test_repeatable_and_stream_ordered(pa, cuda_ok):
    import torch
    prm = pa.make_params(200000, 8, 0.5, seed=5, id_bits=32)
    e1, s1 = pa.generate(prm)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        e2, s2 = pa.generate(prm, stream=s)
    s.synchronize()
    assert torch.equal(e1, e2)
    assert s1.retries == s2.retries


@pytest.mark.parametrize("start", list(START))
def test_wait_limit_reports_error_and_context_survives(pa, cuda_ok, start):
    """The first tile (or, in the start kernel, the first warp pass) is never
    published: every wait on it ends at the 20 ms limit, the call returns
    PA_ERR_SPIN_TIMEOUT, and the context stays usable for the next generation."""
    prm = pa.make_params(200000, 4, 0.2, seed=1, flags=pa.PA_FLAG_TEST_WITHHOLD_FIRST_TILE,
                         spin_limit_ns=20_000_000, start_nodes=start_nodes(pa, start))
    edges, st = pa.generate(prm, raise_on_error=False)
    assert st.status == pa.PA_ERR_SPIN_TIMEOUT
    with pytest.raises(pa.CuppaError):
        pa.generate(prm)
    assert_bit_exact(pa, 20000, 4, 0.2, 1, 1, 32)
