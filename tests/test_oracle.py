"""The CPU oracle, pinned before it is trusted.

* Philox4x32-10 against the published known-answer vectors of the Random123
  distribution (Salmon et al., SC'11);
* MT19937-64 against the value the C++ standard fixes for the 10000th output of
  a default-seeded std::mt19937_64 ([rand.predef]);
* MT_REF mode (the reference's own RNG and draw order) against the degree
  distributions written by the reference `-A scm` itself (tests/golden/scm_dd,
  made by tests/golden/make_golden.py) -- byte-for-byte;
* the model's hand-checkable cases: p = 1, p = 0,
  seed shapes, duplicate retries, id-width boundaries;
* the oracle's own Philox-mode digests (regression pin);
* the repeated-nodes BA model (-A sba): MT_REF mode against the reference
  `-A sba` degree distributions, and a literal replay on the endpoint array.
"""
import json
import os

import numpy as np
import pytest

import _oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# Random123 kat_vectors, philox4x32 with 10 rounds: (ctr, key, expected)
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    assert orc.philox(ctr, key) == want


def test_mt19937_64_standard_value():
    out = orc.mt19937_64(5489, 10000)
    assert int(out[-1]) == 9981545732273789042


def _scm_runs():
    with open(os.path.join(GOLD, "scm_dd.json")) as f:
        return json.load(f)["runs"]


@pytest.mark.parametrize("run", [r for r in _scm_runs() if r["n"] <= 100000],
                         ids=lambda r: f"n{r['n']}_m{r['m']}_p{r['p']}")
def test_mt_ref_mode_reproduces_reference_scm(run):
    """The oracle's copy-model loop, driven by the reference's RNG, gives the
    reference's exact degree distribution: the model semantics shared with the
    Philox mode are the reference's."""
    G = orc.generate(run["n"], run["m"], run["p"], 5489, orc.SEED_STAR_REF, orc.RNG_MT_REF)
    mine = orc.dd_csv_from_degrees(orc.degrees(G, orc.SEED_STAR_REF))
    with open(os.path.join(GOLD, run["file"])) as f:
        ref = f.read()
    assert mine == ref


@pytest.mark.slow
@pytest.mark.parametrize("run", [r for r in _scm_runs() if r["n"] > 100000],
                         ids=lambda r: f"n{r['n']}_m{r['m']}_p{r['p']}")
def test_mt_ref_mode_reproduces_reference_scm_large(run):
    G = orc.generate(run["n"], run["m"], run["p"], 5489, orc.SEED_STAR_REF, orc.RNG_MT_REF)
    mine = orc.dd_csv_from_degrees(orc.degrees(G, orc.SEED_STAR_REF))
    with open(os.path.join(GOLD, run["file"])) as f:
        assert mine == f.read()


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLD, "philox_digests.json")))["cases"],
                         ids=lambda c: f"n{c['n']}_d{c['d']}_p{c['p']}_s{c['seed']}_m{c['seed_mode']}")
def test_philox_mode_digests(case):
    G, retries = orc.generate(case["n"], case["d"], case["p"], case["seed"], case["seed_mode"],
                              orc.RNG_PHILOX, with_retries=True)
    slot = orc.pairs_slot_order(G, case["seed_mode"])
    can = orc.pairs_canonical(G, case["seed_mode"])
    assert slot.shape[0] == case["edges"]
    assert retries == case["retries"]
    assert f"{orc.fnv1a64(slot):016x}" == case["fnv_slot_i64"]
    assert f"{orc.fnv1a64(can):016x}" == case["fnv_canonical_i64"]
    assert f"{orc.fnv1a64(can.astype(np.int32)):016x}" == case["fnv_canonical_i32"]


def test_tiny_text_fixture():
    G = orc.generate(40, 3, 0.5, 42, orc.SEED_CLIQUE)
    can = orc.pairs_canonical(G, orc.SEED_CLIQUE)
    text = "".join(f"{u} {v}\n" for u, v in can.tolist())
    with open(os.path.join(GOLD, "tiny_n40_d3_p0.5_s42_clique.txt")) as f:
        assert text == f.read()


# ---- model properties -------------------------------------------------------

def _check_simple_graph(G, d, seed_mode):
    n = G.shape[0]
    gen = G[d + 1:]
    u = np.arange(d + 1, n)[:, None]
    assert (gen >= 0).all() and (gen < u).all(), "targets in [0, u)"
    s = np.sort(gen, axis=1)
    assert (np.diff(s, axis=1) > 0).all(), "no multi-edges within a node"
    can = orc.pairs_canonical(G, seed_mode)
    assert (can[:, 0] > can[:, 1]).all(), "no self loops; u > v"
    key = can[:, 0] * n + can[:, 1]
    assert (np.diff(key) > 0).all(), "canonical list strictly sorted"


@pytest.mark.parametrize("d", [1, 2, 3, 4, 8, 16, 32])
@pytest.mark.parametrize("p", [0.0, 0.1, 0.5, 0.9, 1.0])
@pytest.mark.parametrize("mode", [orc.SEED_STAR_REF, orc.SEED_CLIQUE])
def test_simple_graph_properties(d, p, mode):
    n = 3000
    G = orc.generate(n, d, p, 1000 + d, mode)
    _check_simple_graph(G, d, mode)
    assert orc.pairs_slot_order(G, mode).shape[0] == orc.edge_count(n, d, mode)


def test_seed_shapes():
    d = 5
    G = orc.generate(d + 1, d, 0.5, 1, orc.SEED_CLIQUE)
    can = orc.pairs_canonical(G, orc.SEED_CLIQUE)
    want = [(v, w) for v in range(d + 1) for w in range(v)]
    assert [tuple(x) for x in can.tolist()] == want
    G = orc.generate(d + 1, d, 0.5, 1, orc.SEED_STAR_REF)
    assert G[:d].tolist() == [[i] * d for i in range(d)]
    assert G[d].tolist() == list(range(d))
    can = orc.pairs_canonical(G, orc.SEED_STAR_REF)
    assert [tuple(x) for x in can.tolist()] == [(d, j) for j in range(d)]
    assert orc.seed_edge_count(d, orc.SEED_CLIQUE) == 15
    assert orc.seed_edge_count(d, orc.SEED_STAR_REF) == 5


def test_p0_star_ref_is_complete_bipartite():
    """p = 0 with the reference seed: every node copies a seed target, so every
    new node links to exactly {0..d-1} -- K_{d,n-d}, no power law."""
    n, d = 5000, 4
    G = orc.generate(n, d, 0.0, 99, orc.SEED_STAR_REF)
    assert (np.sort(G[d + 1:], axis=1) == np.arange(d)).all()


def test_p0_clique_closure():
    n, d = 5000, 4
    G = orc.generate(n, d, 0.0, 99, orc.SEED_CLIQUE)
    assert G[d + 1:].max() <= d


def test_p1_uniform_distinct():
    """p = 1: direct picks only, so every slot is a uniform earlier node."""
    n, d = 200000, 4
    G = orc.generate(n, d, 1.0, 5, orc.SEED_CLIQUE)
    u = np.arange(d + 1, n)
    frac = G[d + 1:, 0] / u   # first slot never retries: uniform on [0, 1)
    hist, _ = np.histogram(frac, bins=10, range=(0, 1))
    expect = len(frac) / 10
    assert (np.abs(hist - expect) < 5 * np.sqrt(expect)).all()


def test_duplicate_retry_path():
    """Retries happen and the accepted draw is the first non-duplicate: replay
    node u slot by slot with the raw Philox draws."""
    n, d, p, seed = 300, 8, 0.0, 77
    G, retries = orc.generate(n, d, p, seed, orc.SEED_CLIQUE, with_retries=True)
    assert retries > 0
    pth = orc.p_threshold(p)
    replay_retries = 0
    for u in range(d + 1, n):
        row = []
        for i in range(d):
            r = 0
            while True:
                w = orc.philox((u & 0xFFFFFFFF, u >> 32, i, r), (seed & 0xFFFFFFFF, seed >> 32))
                v = ((((w[1] << 32) | w[0]) * u) >> 64)
                k = (w[3] * d) >> 32
                cand = v if w[2] < pth else int(G[v, k])
                if cand not in row:
                    row.append(cand)
                    break
                r += 1
                replay_retries += 1
        assert row == G[u].tolist()
    assert replay_retries == retries


def test_p_threshold():
    assert orc.p_threshold(0.0) == 0
    assert orc.p_threshold(1.0) == 1 << 32
    assert orc.p_threshold(0.5) == 1 << 31
    assert orc.p_threshold(0.25) == 1 << 30


def test_id_width_boundaries():
    """Large node ids: the Philox counter carries u's high word, and the
    multiply-shift keeps v < u.  A tiny graph cannot reach 2^32 nodes, so check
    the draw arithmetic directly at the boundary."""
    for u in (2 ** 31 - 1, 2 ** 31, 2 ** 32 - 1, 2 ** 32, 2 ** 33 + 5):
        for i in range(4):
            w = orc.philox((u & 0xFFFFFFFF, u >> 32, i, 0), (7, 0))
            v = ((((w[1] << 32) | w[0]) * u) >> 64)
            assert 0 <= v < u
    # the counter's high word matters
    a = orc.philox((5, 0, 0, 0), (1, 2))
    b = orc.philox((5, 1, 0, 0), (1, 2))
    assert a != b


def test_csr_sorted_and_symmetric():
    n, d = 4000, 4
    for mode in (orc.SEED_STAR_REF, orc.SEED_CLIQUE):
        G = orc.generate(n, d, 0.3, 3, mode)
        rowptr, col = orc.csr(G, mode)
        deg = orc.degrees(G, mode)
        assert (np.diff(rowptr) == deg).all()
        for x in range(n):
            row = col[rowptr[x]:rowptr[x + 1]]
            assert (np.diff(row) > 0).all()
        can = orc.pairs_canonical(G, mode)
        und = np.concatenate([can, can[:, ::-1]])
        order = np.lexsort((und[:, 1], und[:, 0]))
        assert (und[order, 1] == col).all()


# ---- repeated-nodes BA (-A sba) ---------------------------------------------

def _sba_runs():
    with open(os.path.join(GOLD, "sba_dd.json")) as f:
        return json.load(f)["runs"]


@pytest.mark.parametrize("run", [r for r in _sba_runs() if r["n"] <= 100000],
                         ids=lambda r: f"n{r['n']}_m{r['m']}")
def test_ba_mt_ref_mode_reproduces_reference_sba(run):
    """The oracle's BA model driven by the reference's RNG gives the exact
    degree distribution the reference -A sba writes."""
    G = orc.generate_ba(run["n"], run["m"], 5489, orc.RNG_MT_REF)
    mine = orc.dd_csv_from_degrees(orc.degrees(G, orc.SEED_STAR_REF))
    with open(os.path.join(GOLD, run["file"])) as f:
        assert mine == f.read()


@pytest.mark.slow
@pytest.mark.parametrize("run", [r for r in _sba_runs() if r["n"] > 100000],
                         ids=lambda r: f"n{r['n']}_m{r['m']}")
def test_ba_mt_ref_mode_reproduces_reference_sba_large(run):
    G = orc.generate_ba(run["n"], run["m"], 5489, orc.RNG_MT_REF)
    mine = orc.dd_csv_from_degrees(orc.degrees(G, orc.SEED_STAR_REF))
    with open(os.path.join(GOLD, run["file"])) as f:
        assert mine == f.read()


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLD, "ba_philox_digests.json")))["cases"],
                         ids=lambda c: f"n{c['n']}_d{c['d']}_s{c['seed']}")
def test_ba_philox_digests(case):
    G, retries = orc.generate_ba(case["n"], case["d"], case["seed"], orc.RNG_PHILOX,
                                 with_retries=True)
    slot = orc.pairs_slot_order(G, orc.SEED_STAR_REF)
    assert slot.shape[0] == case["edges"]
    assert retries == case["retries"]
    assert f"{orc.fnv1a64(slot):016x}" == case["fnv_slot_i64"]


@pytest.mark.parametrize("d", [1, 2, 5])
@pytest.mark.parametrize("rng", [orc.RNG_PHILOX, orc.RNG_MT_REF])
def test_ba_replay_on_endpoint_array(d, rng):
    """Replay the reference loop literally (src/PA/SPA/SerialBA.cpp:93-161):
    keep the endpoint array -- node i < d repeated 2d times, then per node w
    its pairs (target, w) -- and index it with each draw.  The oracle's closed
    form decode must pick the same endpoints."""
    n, seed = 400, 2024
    G, retries = orc.generate_ba(n, d, seed, rng, with_retries=True)
    mt = orc.mt19937_64(seed, 200000) if rng == orc.RNG_MT_REF else None
    mt_pos = 0
    ends = [i for i in range(d) for _ in range(2 * d)]
    targets = list(range(d))          # node d's targets
    replay_retries = 0
    for u in range(d, n):
        for t in targets:
            ends += [t, u]
        if u + 1 == n:
            break
        Z = len(ends)
        assert Z == 2 * d * d + 2 * d * (u + 1 - d)
        targets = []
        for i in range(d):
            r = 0
            while True:
                if rng == orc.RNG_PHILOX:
                    v = u + 1
                    w = orc.philox((v & 0xFFFFFFFF, v >> 32, i, r), (seed & 0xFFFFFFFF, seed >> 32))
                    R = ((((w[1] << 32) | w[0]) * Z) >> 64)
                else:
                    R = int(mt[mt_pos]) % Z
                    mt_pos += 1
                cand = ends[R]
                if cand not in targets:
                    targets.append(cand)
                    break
                r += 1
                replay_retries += 1
        assert targets == G[u + 1].tolist()
    assert replay_retries == retries


@pytest.mark.parametrize("d", [1, 3, 8, 32])
def test_ba_simple_graph_properties(d):
    n = 3000
    G = orc.generate_ba(n, d, 500 + d)
    _check_simple_graph(G, d, orc.SEED_STAR_REF)
    assert G[d].tolist() == list(range(d))


def test_ba_rejects_bad_shapes():
    with pytest.raises(ValueError):
        orc.generate_ba(4, 4, 1)
    with pytest.raises(ValueError):
        orc.generate_ba(10, 0, 1)


def test_text_format_is_the_reference_writers():
    """The reference's PAHelper::writeGraphToDisk, run on the oracle's MT_REF
    graph (tests/golden/ref_write_*.txt), writes exactly the "u v" lines of the
    PAIRS order with the reference seed: node M's star row, then rows M+1..N-1."""
    n, m, p = 2000, 3, 0.5
    G = orc.generate(n, m, p, 5489, orc.SEED_STAR_REF, orc.RNG_MT_REF)
    text = "".join(f"{u} {v}\n" for u, v in orc.pairs_slot_order(G, orc.SEED_STAR_REF).tolist())
    with open(os.path.join(GOLD, f"ref_write_n{n}_m{m}_p{p}.txt")) as f:
        assert text == f.read()


# ---------------------------------------------------------------------------
# Whole-graph digests (orc_digest_ids, orc_graph_digests)

_M64 = (1 << 64) - 1


def _fmix64_py(k):
    k ^= k >> 33
    k = (k * 0xFF51AFD7ED558CCD) & _M64
    k ^= k >> 33
    k = (k * 0xC4CEB9FE1A85EC53) & _M64
    return k ^ (k >> 33)


def _digest_py(ids, base=0):
    """The digest's definition, restated in plain Python integers."""
    s = x = 0
    for i, v in enumerate(ids):
        h = _fmix64_py(_fmix64_py(((base + i) * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) & _M64)
                       ^ (int(v) & _M64))
        s = (s + h) & _M64
        x ^= h
    return s, x


def test_digest_definition():
    ids = np.array([0, 1, 2, 7, -1, 2 ** 40 + 3, 5, 5, 123456789], dtype=np.int64)
    assert orc.digest_ids(ids) == _digest_py(ids.tolist())
    assert orc.digest_ids(ids, 1000) == _digest_py(ids.tolist(), 1000)
    # position-keyed: swapping two elements changes it
    sw = ids.copy()
    sw[[1, 2]] = sw[[2, 1]]
    assert orc.digest_ids(sw) != orc.digest_ids(ids)
    # pieces with their index bases add up to the whole
    a = orc.digest_ids(ids[:4])
    b = orc.digest_ids(ids[4:], 4)
    assert ((a[0] + b[0]) & _M64, a[1] ^ b[1]) == orc.digest_ids(ids)


@pytest.mark.parametrize("n,d,p,seed,mode,model", [
    (3000, 4, 0.5, 42, orc.SEED_CLIQUE, orc.MODEL_COPY),
    (3000, 4, 0.5, 42, orc.SEED_STAR_REF, orc.MODEL_COPY),
    (2000, 7, 0.2, 5, orc.SEED_CLIQUE, orc.MODEL_COPY),
    (2000, 1, 0.5, 3, orc.SEED_CLIQUE, orc.MODEL_COPY),
    (1500, 4, 0.0, 1234, orc.SEED_CLIQUE, orc.MODEL_COPY),
    (500, 32, 0.9, 2, orc.SEED_CLIQUE, orc.MODEL_COPY),
    (3000, 4, 0.0, 9, orc.SEED_STAR_REF, orc.MODEL_BA),
])
def test_graph_digests_equal_the_materialised_outputs(n, d, p, seed, mode, model):
    """The streaming whole-graph digests (int32 slots, no edge list in memory)
    equal the digests of the int64 oracle's edge list and CSR."""
    dg = orc.graph_digests(n, d, p, seed, mode, model, with_csr=True)
    if model == orc.MODEL_BA:
        G, r = orc.generate_ba(n, d, seed, with_retries=True)
    else:
        G, r = orc.generate(n, d, p, seed, mode, with_retries=True)
    pairs = orc.pairs_slot_order(G, mode)
    rowptr, col = orc.csr(G, mode)
    assert dg["pairs"] == orc.digest_ids(pairs)
    assert dg["rowptr"] == orc.digest_ids(rowptr)
    assert dg["col"] == orc.digest_ids(col)
    assert dg["retries"] == r


def test_fullsize_digest_fixture_is_complete():
    """The committed whole-graph digests of the benchmark configurations."""
    with open(os.path.join(GOLD, "fullsize_digests.json")) as f:
        cases = {c["name"]: c for c in json.load(f)["cases"]}
    for name in ("c3_p0.5", "c3_p0", "c2", "sba_n2^30", "c1", "c3s", "c3m"):
        c = cases[name]
        assert c["edges"] == orc.edge_count(c["n"], c["d"], c["seed_mode"])
        assert len(c["pairs"]) == 2 and all(len(h) == 16 for h in c["pairs"])
    for name in ("c3_p0.5", "c2", "c1", "c3s", "c3m"):
        assert "rowptr" in cases[name] and "col" in cases[name]
    # the smallest one recomputed here: the fixture is the oracle's output
    c = cases["c1"]
    dg = orc.graph_digests(c["n"], c["d"], c["p"], c["seed"], c["seed_mode"], c["model"], True)
    for k in ("pairs", "rowptr", "col"):
        assert [f"{x:016x}" for x in dg[k]] == c[k]
