"""The repeated-nodes Barabasi-Albert model (-A sba) on the GPU, through the C ABI.

Bar: bit-exact against the oracle's BA model (tests/_oracle.py generate_ba,
itself pinned to the reference SerialBA's degree distributions in
test_oracle.py), slot by slot in the PAIRS layout, on every kernel path: the
start kernel, the persistent kernel, a split between them, batches mixing both
models, the request server and CSR.  At n = 10^6 the Philox stream is compared
with the reference's own MT19937-64 run by its degree distribution."""
import json
import os
import subprocess

import numpy as np
import pytest
import torch

import _oracle as orc
from test_statistics import KS_BOUND, ALPHA_TOL, _hist, ks_statistic, tail_alpha

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STAR = orc.SEED_STAR_REF


def ba_params(pa, n, d, seed, bits=32, **kw):
    return pa.make_params(n, d, 0.0, seed=seed, id_bits=bits, seed_mode=pa.PA_SEED_STAR_REF,
                          model=pa.PA_MODEL_BA, **kw)


def assert_ba_exact(pa, n, d, seed, bits=32, **kw):
    prm = ba_params(pa, n, d, seed, bits, **kw)
    edges, st = pa.generate(prm)
    assert st.status == 0
    G, retries = orc.generate_ba(n, d, seed, with_retries=True)
    want = orc.pairs_slot_order(G, STAR)
    got = edges.cpu().numpy().astype(np.int64)
    assert got.shape == want.shape
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, f"first mismatch at pair {bad[:5]}: got {got[bad[:3]]} want {want[bad[:3]]}"
    assert st.retries == retries
    return prm, edges, G


START = {"start": 0, "persistent": None, "split": 2000}


def start_nodes(pa, which):
    v = START[which]
    return pa.PA_START_NONE if v is None else v


@pytest.mark.parametrize("start", list(START))
@pytest.mark.parametrize("d", [1, 2, 3, 4, 5, 7, 8, 16, 31, 32])
def test_ba_bit_exact_sweep(pa, cuda_ok, d, start):
    assert_ba_exact(pa, 20000, d, 300 + d, start_nodes=start_nodes(pa, start))


@pytest.mark.parametrize("start", list(START))
@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("d", [4, 16])
def test_ba_bit_exact_wide_ids_and_seed(pa, cuda_ok, d, bits, start):
    assert_ba_exact(pa, 50000, d, 2 ** 33 + d, bits, start_nodes=start_nodes(pa, start))


@pytest.mark.parametrize("n,d", [(2, 1), (3, 2), (6, 5), (7, 5), (40, 3), (333, 5), (4097, 5)])
def test_ba_small_and_seed_only_graphs(pa, cuda_ok, n, d):
    assert_ba_exact(pa, n, d, 7)


@pytest.mark.parametrize("start", ["persistent", "split"])
@pytest.mark.parametrize("passes", [1, 2, 4, 8])
def test_ba_every_tile_shape(pa, cuda_ok, passes, start):
    assert_ba_exact(pa, 30000, 3, 9, tile_passes=passes, start_nodes=start_nodes(pa, start))
    assert_ba_exact(pa, 30000, 16, 9, 64, tile_passes=passes, start_nodes=start_nodes(pa, start))


@pytest.mark.parametrize("blocks", [1, 3, 4000])
def test_ba_any_grid_size(pa, cuda_ok, blocks):
    assert_ba_exact(pa, 20000, 4, 5, blocks=blocks, start_nodes=pa.PA_START_NONE)


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLD, "ba_philox_digests.json")))["cases"],
                         ids=lambda c: f"n{c['n']}_d{c['d']}_s{c['seed']}")
def test_ba_golden_digests(pa, cuda_ok, case):
    prm = ba_params(pa, case["n"], case["d"], case["seed"], 64)
    edges, st = pa.generate(prm)
    assert st.retries == case["retries"]
    assert f"{orc.fnv1a64(edges.cpu().numpy()):016x}" == case["fnv_slot_i64"]


def test_ba_degree_distribution_is_the_reference_format(pa, cuda_ok, tmp_path):
    """pa_write_degree_distribution of a BA graph counts what the reference's
    outputSBADegreeDistribution counts (every edge of nodes M..N-1)."""
    prm, edges, G = assert_ba_exact(pa, 100000, 4, 11)
    path = str(tmp_path / "dd.csv")
    pa.write_degree_distribution(prm, edges, path)
    with open(path) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, STAR))


@pytest.mark.parametrize("bits", [32, 64])
def test_ba_csr(pa, cuda_ok, bits):
    prm, edges, G = assert_ba_exact(pa, 60000, 8, 21, bits)
    rowptr, col = pa.build_csr(prm, edges)
    want_rp, want_col = orc.csr(G, STAR)
    assert (rowptr.cpu().numpy() == want_rp).all()
    assert (col.cpu().numpy().astype(np.int64) == want_col).all()


def test_ba_batch_mixed_with_copy_model(pa, cuda_ok):
    rng = np.random.default_rng(17)
    prms = []
    for i in range(40):
        d = int(rng.integers(1, 33))
        n = max(d + 1, int(round(10 ** rng.uniform(1.2, 5.3))))
        sn = [0, pa.PA_START_NONE, 1500][i % 3]
        if i % 2:
            prms.append(ba_params(pa, n, d, 900 + i, start_nodes=sn))
        else:
            prms.append(pa.make_params(n, d, float(rng.uniform(0.1, 0.9)), seed=900 + i,
                                       seed_mode=int(rng.integers(0, 2)), start_nodes=sn))
    prms.sort(key=lambda q: -q.n * q.d)
    batch = pa.Batch(prms)
    batch.generate()
    assert batch.finish().status == 0
    for i, prm in enumerate(prms):
        if prm.model == pa.PA_MODEL_BA:
            G = orc.generate_ba(prm.n, prm.d, prm.seed)
        else:
            G = orc.generate(prm.n, prm.d, prm.p, prm.seed, prm.seed_mode)
        want = orc.pairs_slot_order(G, prm.seed_mode)
        assert (batch.graph(i).cpu().numpy().astype(np.int64) == want).all(), f"instance {i}"


def test_ba_served(pa, cuda_ok):
    prms = [ba_params(pa, 10 ** 5, 4, 1), ba_params(pa, 3000, 32, 2, 64),
            pa.make_params(10 ** 5, 4, 0.5, seed=3)]
    with pa.Server() as srv:
        tickets = [srv.submit(p) for p in prms]
        for t, prm in zip(tickets, prms):
            rc, res = srv.wait(t, 30_000_000_000)
            assert rc == 0 and res.status == 0
            want, _ = pa.generate(prm)
            assert torch.equal(pa.Server.edges_view(res, prm.id_bits), want)
            srv.release(t)


def test_ba_class_mirror(pa, cuda_ok, tmp_path):
    """SerialBA(n, m).generateGraph(conf), the reference's -A sba entry."""
    conf = pa.ExperimentConfiguration(_algorithm="sba", _n1=50000, _x1=4,
                                      _FLAG_SHOW_DEGREE_DISTRIBUTION=True, _distfile1="dd.csv",
                                      _outputDir=str(tmp_path), seed=5)
    g = pa.SerialBA(conf._n1, conf._x1)
    edges = g.generateGraph(conf)
    G = orc.generate_ba(50000, 4, 5)
    assert (edges.cpu().numpy().astype(np.int64) == orc.pairs_slot_order(G, STAR)).all()
    with open(os.path.join(str(tmp_path), "dd.csv")) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, STAR))


def test_runner_sba(cuda_ok, tmp_path):
    runner = os.path.join(ROOT, "cuppa-public_b200", "bin", "cuppa_runner")
    out = subprocess.run([runner, "-A", "sba", "-n", "20000", "-x", "4", "--seed", "8",
                          "--show-dd", "1", "--dd-filename", "dd.csv", "-o", str(tmp_path)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    G = orc.generate_ba(20000, 4, 8)
    with open(os.path.join(str(tmp_path), "dd.csv")) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, STAR))


def test_ba_matches_reference_distribution(pa, cuda_ok):
    """Philox BA at n = 10^6, M = 4 against the reference -A sba's own run."""
    prm = ba_params(pa, 10 ** 6, 4, 99)
    edges, st = pa.generate(prm)
    mine = _hist(pa.degree_distribution_csv(pa.degrees(prm, edges)))
    with open(os.path.join(GOLD, "sba_dd", "sba_n1000000_m4.csv")) as f:
        ref = _hist(f.read())
    assert ks_statistic(mine, ref) < KS_BOUND
    assert abs(tail_alpha(mine) - tail_alpha(ref)) < ALPHA_TOL
