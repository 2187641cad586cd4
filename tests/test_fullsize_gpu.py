"""The benchmark configurations at their full sizes, on the GPU.

Whole-graph parity: the device digest (pa_digest) of the entire edge list --
and, where the configuration builds one, of the CSR's rowptr and col -- must
equal the oracle's digest of the same configuration
(tests/golden/fullsize_digests.json, written by tests/golden/make_golden.py
from orc_graph_digests, which generates the whole graph on the CPU).  The
digest is position-keyed, so a single wrong id or two ids in swapped slots
anywhere in the 4.3e9 edges changes it.

Besides that, each test checks (1) a prefix of millions of nodes element by
element against the oracle (a node depends only on earlier nodes, so the first
N nodes are the graph of N nodes; this localises a failure that the digest only
detects), (2) properties over the whole graph that hold for every correct
output -- row sources, targets below their source, distinct targets per row,
the closure of p = 0 -- (3) a second generation gives the same digest, and, for
n = 2^30, (4) the degree distribution against the reference's own `-A scm`
run (KS statistic and tail exponent; the exponent does not drift with n: the
oracle gives 2.8395 at 10^6 and 2.8374 at 2^25 nodes).  The CSR of n = 10^8,
d = 16 is also checked by its invariants: every row strictly ascending (own
targets below the row id, then in-neighbours above it), no self entry, row
lengths equal to the degrees, and both directions of every edge present (hash
sums)."""
import json
import os

import numpy as np
import pytest
import torch

import _oracle as orc
from test_statistics import ALPHA_TOL, KS_BOUND, _hist, ks_statistic, tail_alpha

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CHUNK = 1 << 26     # rows per property pass (bounded temporaries)


def _mix(x):
    """A 64-bit mixing function in wrapping int64 arithmetic (equality checks only)."""
    x = x * -7046029254386353131          # 0x9E3779B97F4A7C15 as int64
    x = x ^ (x >> 29)
    x = x * -4658895280553007687          # 0xBF58476D1CE4E5B9 as int64
    return x ^ (x >> 32)


def _wrap(x):
    """x reduced to a signed 64-bit value (sums of wrapped per-chunk sums)."""
    return (x + 2 ** 63) % 2 ** 64 - 2 ** 63


def _pair_hash(u, v):
    return _mix(u * 1000003 + _mix(v))


def check_rows(E, n, d, seed_edges, closure=None):
    """Row sources, targets below the source, distinct targets; returns a
    checksum of the whole edge list."""
    rows = n - d - 1
    body = E[seed_edges:].view(rows, d, 2)
    h = torch.zeros((), dtype=torch.int64, device=E.device)
    for r0 in range(0, rows, CHUNK):
        blk = body[r0:r0 + CHUNK].to(torch.int64)
        u = torch.arange(d + 1 + r0, d + 1 + r0 + blk.shape[0], device=E.device)
        assert bool((blk[:, :, 0] == u[:, None]).all()), f"row source wrong near row {r0}"
        v = blk[:, :, 1]
        assert bool((v >= 0).all()) and bool((v < u[:, None]).all()), f"target range near {r0}"
        if d > 1:
            s, _ = torch.sort(v, dim=1)
            assert bool((s[:, 1:] > s[:, :-1]).all()), f"duplicate target near row {r0}"
        if closure is not None:
            assert bool((v <= closure).all())
        h += _pair_hash(u[:, None].expand_as(v), v).sum()
        del blk, v
    return int(h.item())


def check_prefix(E, d, p, seed, mode, nodes):
    G = orc.generate(nodes, d, p, seed, mode)
    want = orc.pairs_slot_order(G, mode)
    got = E[: want.shape[0]].cpu().numpy().astype(np.int64)
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, f"prefix mismatch at pair {bad[:5]}"


def fixture(name):
    """The oracle's whole-graph digests of one configuration."""
    with open(os.path.join(GOLD, "fullsize_digests.json")) as f:
        cases = {c["name"]: c for c in json.load(f)["cases"]}
    c = cases[name]
    return {k: tuple(int(x, 16) for x in c[k]) for k in ("pairs", "rowptr", "col") if k in c}


def free():
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("p", [0.5, 0.0])
def test_c3_full_size(pa, cuda_ok, p):
    """n = 2^30, d = 4, int64, clique seed, Philox seed 1234: ~4.3e9 edges, 68.7 GB."""
    n, d, seed, mode = 2 ** 30, 4, 1234, pa.PA_SEED_CLIQUE
    want = fixture("c3_p0.5" if p else "c3_p0")
    prm = pa.make_params(n, d, p, seed=seed, id_bits=64, seed_mode=mode)
    edges, scratch = pa.alloc_buffers(prm)
    E = edges[: pa.edge_count(prm)]
    pa.generate_into(prm, edges, scratch)
    st = pa.finish(scratch)
    assert st.status == 0
    seed_edges = orc.seed_edge_count(d, orc.SEED_CLIQUE)
    # whole graph against the oracle
    assert pa.digest(E.reshape(-1)) == want["pairs"], "whole-graph digest differs from the oracle"
    # (1) the first 2^22 nodes (2^20 at p = 0, where every node retries more)
    check_prefix(E, d, p, seed, orc.SEED_CLIQUE, 2 ** 22 if p else 2 ** 20)
    # (2) every row; at p = 0 every target stays in the seed clique 0..d
    check_rows(E, n, d, seed_edges, closure=d if p == 0 else None)
    # (3) the same bits again
    pa.generate_into(prm, edges, scratch)
    assert pa.finish(scratch).status == 0
    assert pa.digest(E.reshape(-1)) == want["pairs"]
    del scratch
    if p == 0.5:
        # (4) degrees against the reference's own n = 10^6 run of the same model
        deg = pa.degrees(prm, E)
        counts = torch.bincount(deg).cpu().numpy()
        ks = np.nonzero(counts)[0]
        ks = ks[ks > 0]
        mine = (ks, counts[ks])
        with open(os.path.join(GOLD, "scm_dd", "scm_n1000000_m4_p0.5.csv")) as f:
            ref = _hist(f.read())
        assert ks_statistic(mine, ref) < KS_BOUND
        assert abs(tail_alpha(mine) - tail_alpha(ref)) < ALPHA_TOL
        assert int(deg.sum().item()) == 2 * E.shape[0]
        del deg
        free()
        # the whole CSR (rowptr and col) against the oracle's
        rowptr, col = pa.build_csr(prm, E)
        assert pa.digest(rowptr) == want["rowptr"]
        assert pa.digest(col) == want["col"]
        del rowptr, col
    del edges, E
    free()


def test_c3_full_size_int32(pa, cuda_ok):
    """The same graph with 32-bit ids (34 GB): the digest takes ids sign-extended,
    so the 64-bit configuration's fixture applies."""
    prm = pa.make_params(2 ** 30, 4, 0.5, seed=1234, id_bits=32, seed_mode=pa.PA_SEED_CLIQUE)
    E, st = pa.generate(prm)
    assert st.status == 0
    assert pa.digest(E.reshape(-1)) == fixture("c3_p0.5")["pairs"]
    del E
    free()


def test_sba_full_size(pa, cuda_ok):
    """The BA model (-A sba) at n = 2^30, d = 4, int64, star seed, Philox seed 1234."""
    n, d, seed = 2 ** 30, 4, 1234
    want = fixture("sba_n2^30")
    prm = pa.make_params(n, d, 0.0, seed=seed, id_bits=64, seed_mode=pa.PA_SEED_STAR_REF,
                         model=pa.PA_MODEL_BA)
    E, st = pa.generate(prm)
    assert st.status == 0
    assert pa.digest(E.reshape(-1)) == want["pairs"], "whole-graph digest differs from the oracle"
    del E
    free()


def test_c2_full_size_with_csr(pa, cuda_ok):
    """n = 10^8, d = 16, int64, clique seed, Philox seed 7: ~1.6e9 edges, then CSR."""
    n, d, p, seed = 10 ** 8, 16, 0.5, 7
    prm = pa.make_params(n, d, p, seed=seed, id_bits=64, seed_mode=pa.PA_SEED_CLIQUE)
    want = fixture("c2")
    E, st = pa.generate(prm)
    assert st.status == 0
    m = E.shape[0]
    seed_edges = orc.seed_edge_count(d, orc.SEED_CLIQUE)
    assert pa.digest(E.reshape(-1)) == want["pairs"], "whole-graph digest differs from the oracle"
    check_prefix(E, d, p, seed, orc.SEED_CLIQUE, 2 ** 20)
    edge_hash = check_rows(E, n, d, seed_edges)
    # seed edges are part of the graph too
    su, sv = E[:seed_edges, 0].to(torch.int64), E[:seed_edges, 1].to(torch.int64)
    edge_hash += int(_pair_hash(su, sv).sum().item())

    deg = pa.degrees(prm, E)
    rowptr, col = pa.build_csr(prm, E)
    del E
    free()
    assert col.shape[0] == 2 * m
    assert pa.digest(rowptr) == want["rowptr"] and pa.digest(col) == want["col"]
    assert int(rowptr[0].item()) == 0 and int(rowptr[-1].item()) == 2 * m
    assert torch.equal(rowptr[1:] - rowptr[:-1], deg)
    del deg
    out_hash = in_hash = 0
    step = 1 << 28
    for a in range(0, 2 * m, step):
        b = min(2 * m, a + step)
        pos = torch.arange(a, b, device=col.device)
        row = torch.searchsorted(rowptr, pos, right=True) - 1
        c = col[a:b].to(torch.int64)
        assert bool((c != row).all()), "self entry"
        # strictly ascending inside a row (out part < row < in part)
        same_row = row[1:] == row[:-1]
        assert bool(((c[1:] > c[:-1]) | ~same_row).all()), f"row not ascending near {a}"
        if a > 0:
            prev_row = int(torch.searchsorted(rowptr, torch.tensor([a - 1], device=col.device),
                                              right=True).item()) - 1
            if prev_row == int(row[0].item()):
                assert int(col[a].item()) > int(col[a - 1].item())
        lo = c < row
        out_hash += int(_pair_hash(row[lo], c[lo]).sum().item())     # (u, v) with v < u
        in_hash += int(_pair_hash(c[~lo], row[~lo]).sum().item())    # (u, v) seen from v
        del pos, row, c, same_row, lo
    assert _wrap(out_hash) == _wrap(edge_hash) and _wrap(in_hash) == _wrap(edge_hash)
    del rowptr, col
    free()
