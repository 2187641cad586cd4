"""pa_digest on the GPU against the oracle's digest (orc_digest_ids).

The digest is the position-keyed fingerprint the full-size tests and bench.py
use to compare whole graphs with the oracle without copying them out, so it is
pinned here first on graphs small enough to compare element by element: both
id widths, aligned (16-byte vector) and unaligned (scalar) starts, pieces with
index bases, and the CSR arrays."""
import numpy as np
import pytest
import torch

import _oracle as orc

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("n,d,p,mode", [(50_000, 4, 0.5, 1), (20_000, 16, 0.3, 0),
                                        (7_001, 3, 0.0, 1), (5_000, 1, 0.5, 1)])
def test_edge_list_digest_matches_oracle(pa, cuda_ok, bits, n, d, p, mode):
    prm = pa.make_params(n, d, p, seed=77, id_bits=bits, seed_mode=mode)
    E, st = pa.generate(prm)
    G = orc.generate(n, d, p, 77, mode)
    want = orc.digest_ids(orc.pairs_slot_order(G, mode))
    assert pa.digest(E) == want
    assert orc.graph_digests(n, d, p, 77, mode)["pairs"] == want


@pytest.mark.parametrize("bits", [32, 64])
def test_digest_in_pieces_and_unaligned(pa, cuda_ok, bits):
    dt = torch.int64 if bits == 64 else torch.int32
    x = torch.randint(-5, 2 ** 31 - 1, (100_003,), dtype=dt, device="cuda")
    want = orc.digest_ids(x.cpu().numpy().astype(np.int64))
    assert pa.digest(x) == want
    # pieces at odd offsets: the unaligned ones take the scalar path
    total_s, total_x, a = 0, 0, 0
    for b in (1, 7, 4096, 4097, 50_000, 100_003):
        s, xx = pa.digest(x[a:b], index_base=a)
        total_s, total_x, a = (total_s + s) & M64, total_x ^ xx, b
    assert (total_s, total_x) == want


def test_csr_digest_matches_oracle(pa, cuda_ok):
    n, d, p, mode = 30_000, 8, 0.5, 1
    prm = pa.make_params(n, d, p, seed=5, id_bits=64, seed_mode=mode)
    E, _ = pa.generate(prm)
    rowptr, col = pa.build_csr(prm, E)
    dg = orc.graph_digests(n, d, p, 5, mode, with_csr=True)
    assert pa.digest(rowptr) == dg["rowptr"]
    assert pa.digest(col) == dg["col"]
