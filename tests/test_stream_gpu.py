"""The targets-only layout and the streaming edge writer, against the oracle.

Bar: bit-exact / byte-exact.  SLOTS must hold exactly the oracle's slot rows
d+1..n-1; the streamed text must be byte for byte the reference format ("u v"
per line, PAHelper.hpp:163-177) of the oracle's PAIRS order, and the binary
output its (src, dst) pairs -- for both layouts, both id widths, and chunk
sizes small enough that tiles and chunks split rows at many places."""
import os

import numpy as np
import pytest
import torch

import _oracle as orc

pytestmark = pytest.mark.gpu


def oracle_pairs(n, d, p, seed, mode, model=0):
    G = orc.generate_ba(n, d, seed) if model else orc.generate(n, d, p, seed, mode)
    return G, orc.pairs_slot_order(G, mode)


def text_of(pairs):
    return "".join(f"{u} {v}\n" for u, v in pairs.tolist()).encode()


def collect(pa, prm, edges, binary=False, chunk_edges=0):
    parts = []
    total = pa.stream_edges(prm, edges, parts.append, binary=binary, chunk_edges=chunk_edges)
    out = b"".join(parts)
    assert total == len(out)
    return out


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("d,mode", [(1, 1), (3, 0), (4, 1), (7, 1), (16, 0), (32, 1)])
def test_slots_layout_bit_exact(pa, cuda_ok, d, mode, bits):
    n, p, seed = 30000, 0.4, 77 + d
    prm = pa.make_params(n, d, p, seed=seed, id_bits=bits, seed_mode=mode,
                         layout=pa.PA_LAYOUT_SLOTS)
    S, st = pa.generate(prm)
    assert st.status == 0
    G, retries = orc.generate(n, d, p, seed, mode, with_retries=True)
    assert S.shape == (n - d - 1, d)
    assert (S.cpu().numpy().astype(np.int64) == G[d + 1:]).all()
    assert st.retries == retries


def test_slots_layout_ba_and_seed_only(pa, cuda_ok):
    prm = pa.make_params(20000, 5, 0.0, seed=3, seed_mode=pa.PA_SEED_STAR_REF,
                         model=pa.PA_MODEL_BA, layout=pa.PA_LAYOUT_SLOTS)
    S, st = pa.generate(prm)
    assert (S.cpu().numpy().astype(np.int64) == orc.generate_ba(20000, 5, 3)[6:]).all()
    prm = pa.make_params(6, 5, 0.5, seed=3, layout=pa.PA_LAYOUT_SLOTS)   # seed graph only
    S, st = pa.generate(prm)
    assert st.status == 0 and S.shape[0] == 0
    want = text_of(orc.pairs_slot_order(orc.generate(6, 5, 0.5, 3, 1), 1))
    assert collect(pa, prm, S) == want


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("chunk", [0, 1, 700, 5000])
def test_stream_text_is_the_reference_format(pa, cuda_ok, layout, bits, chunk):
    n, d, p, seed, mode = 20000, 3, 0.5, 11, 0
    prm = pa.make_params(n, d, p, seed=seed, id_bits=bits, seed_mode=mode, layout=layout)
    E, _ = pa.generate(prm)
    _, pairs = oracle_pairs(n, d, p, seed, mode)
    assert collect(pa, prm, E, chunk_edges=chunk) == text_of(pairs)


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("chunk", [0, 999])
def test_stream_binary_pairs(pa, cuda_ok, layout, bits, chunk):
    n, d, p, seed, mode = 50000, 8, 0.3, 5, 1
    prm = pa.make_params(n, d, p, seed=seed, id_bits=bits, seed_mode=mode, layout=layout)
    E, _ = pa.generate(prm)
    _, pairs = oracle_pairs(n, d, p, seed, mode)
    got = np.frombuffer(collect(pa, prm, E, binary=True, chunk_edges=chunk),
                        dtype=np.int64 if bits == 64 else np.int32).reshape(-1, 2)
    assert (got.astype(np.int64) == pairs).all()


@pytest.mark.parametrize("d", [1, 2, 5, 31, 32])
def test_stream_text_every_row_width(pa, cuda_ok, d):
    """Tiles hold 2048 // d whole rows: every d splits chunks differently."""
    n, p, seed, mode = 9000, 0.7, 40 + d, 1
    prm = pa.make_params(n, d, p, seed=seed, seed_mode=mode, layout=pa.PA_LAYOUT_SLOTS)
    E, _ = pa.generate(prm)
    _, pairs = oracle_pairs(n, d, p, seed, mode)
    assert collect(pa, prm, E, chunk_edges=3 * d + 1) == text_of(pairs)


def test_write_edges_and_generate_to_file(pa, cuda_ok, tmp_path):
    n, d, p, seed, mode = 100000, 4, 0.5, 42, 1
    _, pairs = oracle_pairs(n, d, p, seed, mode)
    want = text_of(pairs)
    for layout in (0, 1):
        prm = pa.make_params(n, d, p, seed=seed, seed_mode=mode, layout=layout)
        path = str(tmp_path / f"g{layout}.txt")
        st, nbytes = pa.generate_to_file(prm, path)
        assert st.status == 0 and nbytes == len(want)
        with open(path, "rb") as f:
            assert f.read() == want
        E, _ = pa.generate(prm)
        path2 = str(tmp_path / f"w{layout}.bin")
        pa.write_edges(prm, E, path2, binary=True)
        got = np.fromfile(path2, dtype=np.int32).reshape(-1, 2)
        assert (got.astype(np.int64) == pairs).all()


def test_stream_text_across_digit_counts(pa, cuda_ok):
    """Ids of 1 to 7 digits: line widths change inside tiles and chunks."""
    n, d = 2 ** 21, 2
    prm = pa.make_params(n, d, 0.5, seed=9, id_bits=64, layout=pa.PA_LAYOUT_SLOTS)
    E, _ = pa.generate(prm)
    G = orc.generate(n, d, 0.5, 9, orc.SEED_CLIQUE)
    out = collect(pa, prm, E, chunk_edges=1 << 20)
    assert out == text_of(orc.pairs_slot_order(G, orc.SEED_CLIQUE))


def test_sink_failure_stops_the_stream(pa, cuda_ok):
    prm = pa.make_params(200000, 4, 0.5, layout=pa.PA_LAYOUT_SLOTS)
    E, _ = pa.generate(prm)
    calls = []

    def sink(b):
        calls.append(len(b))
        return len(calls) >= 2     # stop at the second chunk
    with pytest.raises(pa.CuppaError) as ei:
        pa.stream_edges(prm, E, sink, chunk_edges=10000)
    assert ei.value.status == pa.PA_ERR_IO
    assert len(calls) == 2
    # the library is still usable afterwards
    assert len(collect(pa, prm, E)) > 0


def test_slots_degrees_and_dd(pa, cuda_ok, tmp_path):
    n, d, p, seed, mode = 60000, 6, 0.25, 8, 0
    prm = pa.make_params(n, d, p, seed=seed, seed_mode=mode, layout=pa.PA_LAYOUT_SLOTS)
    S, _ = pa.generate(prm)
    G = orc.generate(n, d, p, seed, mode)
    assert (pa.degrees(prm, S).cpu().numpy() == orc.degrees(G, mode)).all()
    path = str(tmp_path / "dd.csv")
    pa.write_degree_distribution(prm, S, path)
    with open(path) as f:
        assert f.read() == orc.dd_csv_from_degrees(orc.degrees(G, mode))


def test_staging_cache_grows_and_trims(pa, cuda_ok):
    """A small stream, a larger one (the cached buffers grow), then trim; the
    outputs are unaffected by what the cache held before."""
    small = pa.make_params(3000, 4, 0.5, seed=1, layout=pa.PA_LAYOUT_SLOTS)
    big = pa.make_params(300000, 8, 0.5, seed=2, layout=pa.PA_LAYOUT_SLOTS)
    Es, _ = pa.generate(small)
    Eb, _ = pa.generate(big)
    want_s = text_of(oracle_pairs(3000, 4, 0.5, 1, 1)[1])
    assert collect(pa, small, Es) == want_s
    out_b = collect(pa, big, Eb, chunk_edges=1 << 18)
    assert out_b == text_of(oracle_pairs(300000, 8, 0.5, 2, 1)[1])
    assert collect(pa, small, Es) == want_s
    pa.stream_trim()
    assert collect(pa, small, Es, binary=True) == collect(pa, small, Es, binary=True)
    pa.stream_trim()


def test_runner_writes_slots_graph(cuda_ok, tmp_path):
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    runner = os.path.join(root, "cuppa-public_b200", "bin", "cuppa_runner")
    out = str(tmp_path / "g.txt")
    r = subprocess.run([runner, "-A", "scm", "-n", "30000", "-x", "4", "-a", "0.5", "--seed", "5",
                        "--layout", "slots", "--out", out], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    G = orc.generate(30000, 4, 0.5, 5, orc.SEED_STAR_REF)
    with open(out, "rb") as f:
        assert f.read() == text_of(orc.pairs_slot_order(G, orc.SEED_STAR_REF))


def test_unwritable_paths_report_io_errors(pa, cuda_ok, tmp_path):
    prm = pa.make_params(1000, 4, 0.5)
    E, _ = pa.generate(prm)
    bad = str(tmp_path / "no-such-dir" / "x.txt")
    with pytest.raises(pa.CuppaError) as ei:
        pa.write_edges(prm, E, bad)
    assert ei.value.status == pa.PA_ERR_IO
    with pytest.raises(pa.CuppaError) as ei:
        pa.write_degree_distribution(prm, E, bad)
    assert ei.value.status == pa.PA_ERR_IO
    with pytest.raises(pa.CuppaError) as ei:
        pa.generate_to_file(prm, bad)
    assert ei.value.status == pa.PA_ERR_IO
