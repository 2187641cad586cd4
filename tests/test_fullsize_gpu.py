"""The benchmark configurations at their full sizes, on the GPU.

The oracle cannot run 4.3e9 edges in a test, but it does not have to for the
first nodes: a node's slots depend only on its own draws and on earlier nodes,
so the first N nodes of any graph are the whole graph of N nodes.  Each test
therefore checks (1) a prefix of millions of nodes bit-exact against the
oracle, (2) properties over the whole graph that hold for every correct output
-- row sources, targets below their source, distinct targets per row, the
closure of p = 0 -- (3) a second generation gives the same checksum, and, for
n = 2^30, (4) the degree distribution against the reference's own `-A scm`
run (KS statistic and tail exponent; the exponent does not drift with n: the
oracle gives 2.8395 at 10^6 and 2.8374 at 2^25 nodes).  The CSR of n = 10^8,
d = 16 is checked by its invariants: every row strictly ascending (own targets
below the row id, then in-neighbours above it), no self entry, row lengths
equal to the degrees, and both directions of every edge present (hash sums)."""
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


def free():
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("p", [0.5, 0.0])
def test_c3_full_size(pa, cuda_ok, p):
    """n = 2^30, d = 4, int64, clique seed, Philox seed 1234: ~4.3e9 edges, 68.7 GB."""
    n, d, seed, mode = 2 ** 30, 4, 1234, pa.PA_SEED_CLIQUE
    prm = pa.make_params(n, d, p, seed=seed, id_bits=64, seed_mode=mode)
    edges, scratch = pa.alloc_buffers(prm)
    E = edges[: pa.edge_count(prm)]
    pa.generate_into(prm, edges, scratch)
    st = pa.finish(scratch)
    assert st.status == 0
    seed_edges = orc.seed_edge_count(d, orc.SEED_CLIQUE)
    # (1) the first 2^22 nodes (2^20 at p = 0, where every node retries more)
    check_prefix(E, d, p, seed, orc.SEED_CLIQUE, 2 ** 22 if p else 2 ** 20)
    # (2) every row; at p = 0 every target stays in the seed clique 0..d
    h1 = check_rows(E, n, d, seed_edges, closure=d if p == 0 else None)
    # (3) the same bits again
    pa.generate_into(prm, edges, scratch)
    assert pa.finish(scratch).status == 0
    assert check_rows(E, n, d, seed_edges) == h1
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
    del edges, scratch, E
    free()


def test_c2_full_size_with_csr(pa, cuda_ok):
    """n = 10^8, d = 16, int64, clique seed, Philox seed 7: ~1.6e9 edges, then CSR."""
    n, d, p, seed = 10 ** 8, 16, 0.5, 7
    prm = pa.make_params(n, d, p, seed=seed, id_bits=64, seed_mode=pa.PA_SEED_CLIQUE)
    E, st = pa.generate(prm)
    assert st.status == 0
    m = E.shape[0]
    seed_edges = orc.seed_edge_count(d, orc.SEED_CLIQUE)
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
