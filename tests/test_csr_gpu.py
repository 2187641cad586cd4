"""Device CSR build vs the oracle's CSR (bit-exact: rowptr and every row's
sorted column list).  Shapes cover both ways a row's in part is copied: by the
warp that writes the row (<= 512 entries), and in 512-entry pieces spread over
all warps for longer ones -- the hubs at p = 0.2 and d = 16, and the seed nodes
at p = 0 and n = 2 * 10^6 (~1.6e6 entries each, thousands of pieces)."""
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
    (2_000_000, 4, 0.0, 10, orc.SEED_CLIQUE, 64),    # five rows of ~1.6e6 in-edges
    (300_000, 16, 0.5, 11, orc.SEED_STAR_REF, 32),   # hubs of 512 .. 4600 in-edges
    (200_000, 8, 0.5, 12, orc.SEED_CLIQUE, 64),      # two 9-bit passes
    # d not dividing 32: idle lanes in every out-part pass of the row writer
    (40000, 3, 0.5, 13, orc.SEED_CLIQUE, 32),
    (30000, 7, 0.3, 14, orc.SEED_STAR_REF, 64),
    (20000, 20, 0.6, 15, orc.SEED_CLIQUE, 32),
    (10000, 31, 0.5, 16, orc.SEED_STAR_REF, 64),
    (50000, 2, 0.1, 17, orc.SEED_CLIQUE, 32),
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
