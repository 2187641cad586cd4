"""File outputs through the C ABI: the edge text of PAHelper::writeGraphToDisk
and the "Degree,Count" CSV of cuPPA::printDegreeDistribution, compared with the
oracle (exact bytes)."""
import os

import numpy as np
import pytest

import _oracle as orc

pytestmark = pytest.mark.gpu


def reference_edge_text(G, d):
    """writeGraphToDisk (src/PA/SPA/PAHelper.hpp:163-177): rows u = M..N-1 in
    slot order, "u G[u][j]" per line (reference seed graph)."""
    n = G.shape[0]
    u = np.repeat(np.arange(d, n), d)
    v = G[d:].reshape(-1)
    return "".join(f"{a} {b}\n" for a, b in zip(u.tolist(), v.tolist()))


@pytest.mark.parametrize("bits", [32, 64])
def test_edge_text_is_the_reference_format_and_order(pa, cuda_ok, tmp_path, bits):
    n, d, p, seed = 20000, 4, 0.5, 17
    prm = pa.make_params(n, d, p, seed=seed, id_bits=bits, seed_mode=pa.PA_SEED_STAR_REF)
    edges, _ = pa.generate(prm)
    path = str(tmp_path / "g.edges")
    pa.write_edges(prm, edges, path)
    G = orc.generate(n, d, p, seed, orc.SEED_STAR_REF)
    with open(path) as f:
        assert f.read() == reference_edge_text(G, d)


def test_edge_binary_round_trip(pa, cuda_ok, tmp_path):
    prm = pa.make_params(50000, 8, 0.3, seed=5, id_bits=64)
    edges, _ = pa.generate(prm)
    path = str(tmp_path / "g.bin")
    pa.write_edges(prm, edges, path, binary=True)
    got = np.fromfile(path, dtype=np.int64).reshape(-1, 2)
    assert (got == edges.cpu().numpy()).all()


@pytest.mark.parametrize("n,d,p,mode", [(100000, 4, 0.5, 1), (200000, 4, 0.2, 0),
                                        (50000, 4, 0.0, 1), (30000, 16, 0.5, 0)])
def test_degree_distribution_csv(pa, cuda_ok, tmp_path, n, d, p, mode):
    prm = pa.make_params(n, d, p, seed=23, id_bits=32, seed_mode=mode)
    edges, _ = pa.generate(prm)
    path = str(tmp_path / "dd.csv")
    pa.write_degree_distribution(prm, edges, path)
    G = orc.generate(n, d, p, 23, mode)
    with open(path) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, mode))


def test_cuppa_class_mirror(pa, cuda_ok, tmp_path):
    """The reference-shaped host interface: cuPPA(n, m, p).generateGraph(conf)."""
    conf = pa.ExperimentConfiguration(_n1=100000, _x1=4, _alpha=0.5,
                                      _FLAG_SHOW_DEGREE_DISTRIBUTION=True,
                                      _distfile1="dd.csv", _outputDir=str(tmp_path),
                                      seed=42, id_bits=32, seed_mode=pa.PA_SEED_CLIQUE)
    g = pa.cuPPA(conf._n1, conf._x1, conf._alpha)
    edges = g.generateGraph(conf)
    assert edges.shape[0] == 399990
    G = orc.generate(100000, 4, 0.5, 42, orc.SEED_CLIQUE)
    assert (edges.cpu().numpy() == orc.pairs_slot_order(G, orc.SEED_CLIQUE)).all()
    with open(os.path.join(str(tmp_path), "dd.csv")) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, orc.SEED_CLIQUE))
    assert (g.generateGraphAdaptive(conf) == edges).all()


def test_serial_copy_model_mirror(pa, cuda_ok, tmp_path):
    """SerialCopyModel(n, m, p).generateGraph(conf), the reference's -A scm entry:
    the copy model on the reference's star seed."""
    conf = pa.ExperimentConfiguration(_algorithm="scm", _n1=50000, _x1=4, _alpha=0.3,
                                      _FLAG_SHOW_DEGREE_DISTRIBUTION=True, _distfile1="dd.csv",
                                      _outputDir=str(tmp_path), seed=13)
    g = pa.SerialCopyModel(conf._n1, conf._x1, conf._alpha)
    edges = g.generateGraph(conf)
    G = orc.generate(50000, 4, 0.3, 13, orc.SEED_STAR_REF)
    assert (edges.cpu().numpy().astype(np.int64) == orc.pairs_slot_order(G, orc.SEED_STAR_REF)).all()
    with open(os.path.join(str(tmp_path), "dd.csv")) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, orc.SEED_STAR_REF))
