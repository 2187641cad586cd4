"""Device CSR build vs the oracle's CSR (bit-exact: rowptr and every row's
sorted column list).  Shapes cover the three sorting paths of the in parts:
warp (<= 32 entries), shared memory (<= 8192) and the bitmap pass for hub rows
(> 8192 entries: the seed nodes at p = 0, the hubs at p = 0.2)."""
import numpy as np
import pytest

import _oracle as orc

pytestmark = pytest.mark.gpu

CASES = [
    (30000, 4, 0.5, 1, orc.SEED_CLIQUE, 32),
    (30000, 4, 0.5, 2, orc.SEED_STAR_REF, 64),
    (50000, 4, 0.0, 3, orc.SEED_CLIQUE, 32),       # seed hubs of ~40k in-edges
    (1_000_000, 4, 0.2, 4, orc.SEED_STAR_REF, 32), # heavy tail, hubs > 8192
    (40000, 16, 0.5, 5, orc.SEED_CLIQUE, 64),
    (20000, 1, 0.5, 6, orc.SEED_CLIQUE, 32),
    (5000, 32, 0.3, 7, orc.SEED_STAR_REF, 32),
    (6, 5, 0.5, 8, orc.SEED_CLIQUE, 32),             # seed graph only
]


@pytest.mark.parametrize("n,d,p,seed,mode,bits", CASES)
def test_csr_matches_oracle(pa, cuda_ok, n, d, p, seed, mode, bits):
    prm = pa.make_params(n, d, p, seed=seed, id_bits=bits, seed_mode=mode)
    edges, st = pa.generate(prm)
    rowptr, col = pa.build_csr(prm, edges)
    G = orc.generate(n, d, p, seed, mode)
    want_rp, want_col = orc.csr(G, mode)
    assert (rowptr.cpu().numpy() == want_rp).all()
    assert (col.cpu().numpy().astype(np.int64) == want_col).all()


def test_csr_from_canonical_order_is_the_same(pa, cuda_ok):
    prm = pa.make_params(100000, 8, 0.4, seed=9, id_bits=32)
    edges, st = pa.generate(prm)
    rp1, c1 = pa.build_csr(prm, edges)
    pa.canonicalize(prm, edges)
    rp2, c2 = pa.build_csr(prm, edges)
    assert (rp1 == rp2).all() and (c1 == c2).all()
