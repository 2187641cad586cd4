"""Regenerate the committed golden fixtures under tests/golden/.

    python tests/golden/make_golden.py

Two kinds of fixture:

1. Reference outputs.  oracle/_ref/scm_ref is the reference's own sequential
   copy model (src/PA/SPA/SerialCopyModel3.cpp, built by `make -C oracle ref`
   from the cuPPA-Public sources).  For each (n, M, p) below it writes the
   "Degree,Count" CSV of src/PA/SPA/PAHelper.hpp:15-67.  The reference seeds its
   MT19937-64 with the default 5489 and its seed graph is the star seed, so these
   runs are deterministic.  They pin the oracle's MT_REF mode exactly and are the
   samples for the statistical comparison of the Philox generator.
   oracle/_ref/sba_ref is the reference's repeated-nodes BA (-A sba,
   src/PA/SPA/SerialBA.cpp, same seed 5489); its "Degree,Count" CSVs
   (src/PA/SPA/PAHelper.hpp:69-147) pin the oracle's BA model in MT_REF mode.
   oracle/_ref/write_ref runs the reference's edge-list writer
   (PAHelper::writeGraphToDisk, src/PA/SPA/PAHelper.hpp:163-177) on the
   oracle's MT_REF star-seed graph; its file pins the text format and row order.
2. Oracle digests.  FNV-1a 64 of the oracle's Philox-mode edge lists (slot
   order and canonical, int64 little-endian) for a fixed list of shapes, plus one
   tiny full edge list.  They pin the oracle itself across edits.
3. Whole-graph digests of the benchmark configurations at full size
   (`python tests/golden/make_golden.py fullsize`, about half an hour on one
   core per configuration, up to 26 GB of host memory each): the oracle's
   position-keyed digests (orc_graph_digests) of the PAIRS edge list and, where
   listed, of the CSR's rowptr and col.  The GPU tests and bench.py compare the
   device's digest of its own output against these.

Needs the reference tree only for part 1 (scm_ref and sba_ref must already be
built).  With arguments, only the named parts run (scm, sba, write, digest,
ba_digest, fullsize).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import _oracle as orc  # noqa: E402

# (n, M, p) runs of the reference scm.  Small ones pin MT_REF exactly; the n=10^6
# d=4 runs are the statistical samples (tail exponent, KS on degrees).
SCM_RUNS = [
    (100000, 4, 0.5), (20000, 4, 0.2), (20000, 4, 0.8), (10000, 4, 0.0),
    (20000, 8, 0.5), (5000, 1, 0.5), (30000, 16, 0.3), (10000, 32, 0.5),
    (3000, 2, 1.0), (1000000, 4, 0.2), (1000000, 4, 0.5), (1000000, 4, 0.8),
]

# (n, M) runs of the reference sba.
SBA_RUNS = [
    (20000, 4), (5000, 1), (10000, 8), (3000, 32), (50000, 2), (20000, 16),
    (1000000, 4),
]

# Philox-mode BA digests: (n, d, seed).
BA_DIGEST_CASES = [(100000, 4, 42), (20000, 16, 7), (5000, 1, 3), (5000, 32, 5),
                   (4000, 7, 2 ** 40 + 17)]

# Philox-mode digests: (n, d, p, seed, seed_mode).
DIGEST_CASES = [
    (100000, 4, 0.5, 42, orc.SEED_CLIQUE),      # the CPU-runnable benchmark configuration
    (100000, 4, 0.5, 42, orc.SEED_STAR_REF),
    (20000, 16, 0.5, 7, orc.SEED_CLIQUE),
    (20000, 4, 0.0, 1234, orc.SEED_CLIQUE),
    (20000, 4, 0.0, 1234, orc.SEED_STAR_REF),
    (5000, 1, 0.3, 3, orc.SEED_CLIQUE),
    (5000, 32, 0.9, 5, orc.SEED_CLIQUE),
    (4000, 3, 1.0, 11, orc.SEED_CLIQUE),
    (4000, 7, 0.1, 2 ** 40 + 17, orc.SEED_STAR_REF),
]


def scm_fixtures():
    if not os.path.exists(orc.REF_SCM):
        raise SystemExit(f"{orc.REF_SCM} missing: run `make -C oracle ref` first")
    outdir = os.path.join(HERE, "scm_dd")
    os.makedirs(outdir, exist_ok=True)
    index = []
    for n, m, p in SCM_RUNS:
        name = f"scm_n{n}_m{m}_p{p}.csv"
        with tempfile.TemporaryDirectory() as td:
            subprocess.run([orc.REF_SCM, str(n), str(m), str(p), td, name], check=True,
                           cwd=td, stdout=subprocess.DEVNULL)
            with open(os.path.join(td, name)) as f:
                text = f.read()
        with open(os.path.join(outdir, name), "w") as f:
            f.write(text)
        index.append({"n": n, "m": m, "p": p, "file": f"scm_dd/{name}"})
    with open(os.path.join(HERE, "scm_dd.json"), "w") as f:
        json.dump({"generator": "reference -A scm (SerialCopyModel3.cpp), MT19937-64 seed 5489, "
                                "star seed", "runs": index}, f, indent=1)


def sba_fixtures():
    if not os.path.exists(orc.REF_SBA):
        raise SystemExit(f"{orc.REF_SBA} missing: run `make -C oracle ref` first")
    outdir = os.path.join(HERE, "sba_dd")
    os.makedirs(outdir, exist_ok=True)
    index = []
    for n, m in SBA_RUNS:
        name = f"sba_n{n}_m{m}.csv"
        with tempfile.TemporaryDirectory() as td:
            subprocess.run([orc.REF_SBA, str(n), str(m), td, name], check=True, cwd=td,
                           stdout=subprocess.DEVNULL)
            with open(os.path.join(td, name)) as f:
                text = f.read()
        with open(os.path.join(outdir, name), "w") as f:
            f.write(text)
        index.append({"n": n, "m": m, "file": f"sba_dd/{name}"})
    with open(os.path.join(HERE, "sba_dd.json"), "w") as f:
        json.dump({"generator": "reference -A sba (SerialBA.cpp), MT19937-64 seed 5489",
                   "runs": index}, f, indent=1)


def ba_digest_fixtures():
    cases = []
    for n, d, seed in BA_DIGEST_CASES:
        G, retries = orc.generate_ba(n, d, seed, orc.RNG_PHILOX, with_retries=True)
        slot = orc.pairs_slot_order(G, orc.SEED_STAR_REF)
        cases.append({"n": n, "d": d, "seed": seed, "edges": int(slot.shape[0]),
                      "retries": retries, "fnv_slot_i64": f"{orc.fnv1a64(slot):016x}"})
    with open(os.path.join(HERE, "ba_philox_digests.json"), "w") as f:
        json.dump({"digest": "FNV-1a 64 over little-endian (src, dst) pairs, slot order",
                   "cases": cases}, f, indent=1)


WRITE_RUN = (2000, 3, 0.5)


def write_fixture():
    ref = os.path.join(orc.ORACLE_DIR, "_ref", "write_ref")
    if not os.path.exists(ref):
        raise SystemExit(f"{ref} missing: run `make -C oracle ref` first")
    n, m, p = WRITE_RUN
    out = os.path.join(HERE, f"ref_write_n{n}_m{m}_p{p}.txt")
    subprocess.run([ref, str(n), str(m), str(p), out], check=True, stdout=subprocess.DEVNULL)


def digest_fixtures():
    cases = []
    for n, d, p, seed, mode in DIGEST_CASES:
        G, retries = orc.generate(n, d, p, seed, mode, orc.RNG_PHILOX, with_retries=True)
        slot = orc.pairs_slot_order(G, mode)
        can = orc.pairs_canonical(G, mode)
        cases.append({
            "n": n, "d": d, "p": p, "seed": seed, "seed_mode": mode,
            "edges": int(slot.shape[0]), "retries": retries,
            "fnv_slot_i64": f"{orc.fnv1a64(slot):016x}",
            "fnv_canonical_i64": f"{orc.fnv1a64(can):016x}",
            "fnv_canonical_i32": f"{orc.fnv1a64(can.astype(np.int32)):016x}",
        })
    with open(os.path.join(HERE, "philox_digests.json"), "w") as f:
        json.dump({"digest": "FNV-1a 64 over little-endian (src, dst) pairs", "cases": cases},
                  f, indent=1)
    # one tiny full edge list in the reference's text format ("u v" per line)
    G = orc.generate(40, 3, 0.5, 42, orc.SEED_CLIQUE)
    can = orc.pairs_canonical(G, orc.SEED_CLIQUE)
    with open(os.path.join(HERE, "tiny_n40_d3_p0.5_s42_clique.txt"), "w") as f:
        f.writelines(f"{u} {v}\n" for u, v in can.tolist())


# Full-size configurations: (name, n, d, p, seed, seed_mode, model, with_csr).
# The longest runs first: the pool works through the list in order.
FULLSIZE_CASES = [
    ("c3_p0.5", 2 ** 30, 4, 0.5, 1234, orc.SEED_CLIQUE, orc.MODEL_COPY, True),
    ("c3_p0", 2 ** 30, 4, 0.0, 1234, orc.SEED_CLIQUE, orc.MODEL_COPY, False),
    ("c2", 10 ** 8, 16, 0.5, 7, orc.SEED_CLIQUE, orc.MODEL_COPY, True),
    ("sba_n2^30", 2 ** 30, 4, 0.0, 1234, orc.SEED_STAR_REF, orc.MODEL_BA, False),
    # the benchmark's smaller workloads (CPU-runnable case and profiling sizes)
    ("c1", 10 ** 5, 4, 0.5, 42, orc.SEED_CLIQUE, orc.MODEL_COPY, True),
    ("c3s", 2 ** 25, 4, 0.5, 1234, orc.SEED_CLIQUE, orc.MODEL_COPY, True),
    ("c3m", 2 ** 26, 4, 0.5, 1234, orc.SEED_CLIQUE, orc.MODEL_COPY, True),
]


def _fullsize_one(case):
    import time
    name, n, d, p, seed, mode, model, with_csr = case
    t0 = time.time()
    dg = orc.graph_digests(n, d, p, seed, mode, model, with_csr)
    rec = {"name": name, "n": n, "d": d, "p": p, "seed": seed, "seed_mode": mode,
           "model": model, "edges": orc.edge_count(n, d, mode if model == orc.MODEL_COPY
                                                     else orc.SEED_STAR_REF),
           "retries": dg["retries"], "pairs": [f"{x:016x}" for x in dg["pairs"]],
           "oracle_seconds": round(time.time() - t0, 1)}
    if with_csr:
        rec["rowptr"] = [f"{x:016x}" for x in dg["rowptr"]]
        rec["col"] = [f"{x:016x}" for x in dg["col"]]
    return rec


def fullsize_fixtures(workers: int = 2):
    """Runs the cases in `workers` spawned processes (host memory bounds it)."""
    import multiprocessing as mp
    path = os.path.join(HERE, "fullsize_digests.json")
    done = {}
    if os.path.exists(path):
        with open(path) as f:
            done = {c["name"]: c for c in json.load(f)["cases"]}
    todo = [c for c in FULLSIZE_CASES if c[0] not in done]
    with mp.get_context("spawn").Pool(workers) as pool:
        for rec in pool.imap_unordered(_fullsize_one, todo):
            done[rec["name"]] = rec
            order = [c[0] for c in FULLSIZE_CASES]
            with open(path, "w") as f:
                json.dump({"digest": "orc_digest_ids: sum and xor (hex) of "
                                     "fmix64(fmix64(pos*0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) ^ id) "
                                     "over a flat id array (PAIRS: src at 2e, dst at 2e+1; "
                                     "CSR rowptr[0..n], col[0..2E)); Philox mode",
                           "cases": [done[k] for k in order if k in done]}, f, indent=1)
            print("fullsize", rec["name"], rec["oracle_seconds"], "s", flush=True)


PARTS = {"scm": scm_fixtures, "sba": sba_fixtures, "write": write_fixture,
         "digest": digest_fixtures, "ba_digest": ba_digest_fixtures,
         "fullsize": fullsize_fixtures}

if __name__ == "__main__":
    names = sys.argv[1:] or ["scm", "sba", "write", "digest", "ba_digest"]
    for name in names:
        PARTS[name]()
    print("fixtures written to", HERE)
