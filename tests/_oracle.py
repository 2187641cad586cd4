"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) for the tests.

Test infrastructure: the product never imports this module.  The oracle is the
sequential restatement of src/PA/SPA/SerialCopyModel3.cpp:38-78 (see
oracle/pa_oracle.h for what each entry point follows).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SCM = os.path.join(ORACLE_DIR, "_ref", "scm_ref")
REF_SBA = os.path.join(ORACLE_DIR, "_ref", "sba_ref")

SEED_STAR_REF = 0
SEED_CLIQUE = 1
RNG_PHILOX = 0
RNG_MT_REF = 1

_u64, _u32, _i, _vp = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p
_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        L = ctypes.CDLL(LIB)
        L.orc_philox4x32_10.argtypes = [_vp, _vp, _vp]
        L.orc_mt19937_64.argtypes = [_u64, _u64, _vp]
        L.orc_p_threshold.argtypes = [ctypes.c_double]
        L.orc_p_threshold.restype = _u64
        L.orc_seed_edge_count.argtypes = [_u32, _i]
        L.orc_seed_edge_count.restype = _u64
        L.orc_edge_count.argtypes = [_u64, _u32, _i]
        L.orc_edge_count.restype = _u64
        L.orc_generate.argtypes = [_u64, _u32, ctypes.c_double, _u64, _i, _i, _vp, _vp]
        L.orc_generate.restype = _i
        L.orc_generate_ba.argtypes = [_u64, _u32, _u64, _i, _vp, _vp]
        L.orc_generate_ba.restype = _i
        for f in ("orc_pairs_slot_order", "orc_pairs_canonical", "orc_degrees"):
            getattr(L, f).argtypes = [_u64, _u32, _i, _vp, _vp]
        L.orc_csr.argtypes = [_u64, _u32, _i, _vp, _vp, _vp]
        L.orc_digest_ids.argtypes = [_vp, _u64, _u64, _vp]
        L.orc_graph_digests.argtypes = [_u64, _u32, ctypes.c_double, _u64, _i, _i, _i, _vp]
        L.orc_graph_digests.restype = _i
        L.orc_fnv1a64.argtypes = [_vp, _u64]
        L.orc_fnv1a64.restype = _u64
        _lib = L
    return _lib


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return tuple(o)


def mt19937_64(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint64)
    lib().orc_mt19937_64(seed, count, out.ctypes.data)
    return out


def p_threshold(p: float) -> int:
    return int(lib().orc_p_threshold(p))


def edge_count(n: int, d: int, seed_mode: int) -> int:
    return int(lib().orc_edge_count(n, d, seed_mode))


def seed_edge_count(d: int, seed_mode: int) -> int:
    return int(lib().orc_seed_edge_count(d, seed_mode))


def generate(n: int, d: int, p: float, seed: int, seed_mode: int = SEED_CLIQUE,
             rng: int = RNG_PHILOX, with_retries: bool = False):
    """Slot array G[n][d] (int64) of the sequential copy model."""
    G = np.empty(n * d, dtype=np.int64)
    r = ctypes.c_uint64()
    rc = lib().orc_generate(n, d, p, seed, seed_mode, rng, G.ctypes.data, ctypes.byref(r))
    if rc != 0:
        raise ValueError(f"oracle rejected n={n} d={d} p={p}")
    G = G.reshape(n, d)
    return (G, int(r.value)) if with_retries else G


def generate_ba(n: int, d: int, seed: int, rng: int = RNG_PHILOX, with_retries: bool = False):
    """Slot array G[n][d] (int64) of the repeated-nodes BA model (STAR_REF seed)."""
    G = np.empty(n * d, dtype=np.int64)
    r = ctypes.c_uint64()
    rc = lib().orc_generate_ba(n, d, seed, rng, G.ctypes.data, ctypes.byref(r))
    if rc != 0:
        raise ValueError(f"oracle rejected BA n={n} d={d}")
    G = G.reshape(n, d)
    return (G, int(r.value)) if with_retries else G


def _pairs(fn: str, G: np.ndarray, seed_mode: int) -> np.ndarray:
    n, d = G.shape
    E = edge_count(n, d, seed_mode)
    out = np.empty((E, 2), dtype=np.int64)
    getattr(lib(), fn)(n, d, seed_mode, np.ascontiguousarray(G).ctypes.data, out.ctypes.data)
    return out


def pairs_slot_order(G: np.ndarray, seed_mode: int) -> np.ndarray:
    """The GPU PAIRS layout: seed edges, then rows d+1.. in slot order."""
    return _pairs("orc_pairs_slot_order", G, seed_mode)


def pairs_canonical(G: np.ndarray, seed_mode: int) -> np.ndarray:
    return _pairs("orc_pairs_canonical", G, seed_mode)


def degrees(G: np.ndarray, seed_mode: int) -> np.ndarray:
    n, d = G.shape
    deg = np.empty(n, dtype=np.int64)
    lib().orc_degrees(n, d, seed_mode, np.ascontiguousarray(G).ctypes.data, deg.ctypes.data)
    return deg


def csr(G: np.ndarray, seed_mode: int):
    n, d = G.shape
    E = edge_count(n, d, seed_mode)
    rowptr = np.empty(n + 1, dtype=np.int64)
    col = np.empty(2 * E, dtype=np.int64)
    lib().orc_csr(n, d, seed_mode, np.ascontiguousarray(G).ctypes.data, rowptr.ctypes.data,
                  col.ctypes.data)
    return rowptr, col


def fnv1a64(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a)
    return int(lib().orc_fnv1a64(a.ctypes.data, a.nbytes))


MODEL_COPY = 0
MODEL_BA = 1


def digest_ids(a: np.ndarray, index_base: int = 0, acc=(0, 0)) -> tuple[int, int]:
    """Position-keyed (sum, xor) digest of a flat id array (orc_digest_ids)."""
    a = np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=np.int64)
    out = (ctypes.c_uint64 * 2)(*acc)
    lib().orc_digest_ids(a.ctypes.data, a.size, index_base, out)
    return int(out[0]), int(out[1])


def graph_digests(n: int, d: int, p: float, seed: int, seed_mode: int = SEED_CLIQUE,
                  model: int = MODEL_COPY, with_csr: bool = False) -> dict:
    """Whole-graph digests without materialising the edge list (orc_graph_digests)."""
    out = (ctypes.c_uint64 * 7)()
    rc = lib().orc_graph_digests(n, d, p, seed, seed_mode, model, int(with_csr), out)
    if rc != 0:
        raise ValueError(f"oracle digest failed ({rc}) for n={n} d={d} p={p}")
    return {"pairs": (int(out[0]), int(out[1])), "rowptr": (int(out[2]), int(out[3])),
            "col": (int(out[4]), int(out[5])), "retries": int(out[6])}


def dd_csv_from_degrees(deg: np.ndarray) -> str:
    """'Degree,Count' rows of src/PA/SPA/PAHelper.hpp:57-62 (count > 0 only)."""
    vals, cnts = np.unique(deg, return_counts=True)
    rows = ["Degree,Count"] + [f"{v},{c}" for v, c in zip(vals.tolist(), cnts.tolist()) if v > 0]
    return "\n".join(rows) + "\n"


def hist_from_dd_csv(text: str) -> dict[int, int]:
    out = {}
    for line in text.strip().splitlines()[1:]:
        a, b = line.split(",")
        out[int(a)] = int(b)
    return out
