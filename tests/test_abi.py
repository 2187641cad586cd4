"""The C ABI without a GPU: the library loads, exports every function that
include/*.h declares, and its host-side checks and size arithmetic agree with
the oracle.  No compute call is made here."""
import ctypes
import glob
import os
import re

import pytest

import _oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(pa_\w+)\s*\([^;{]*\)\s*;", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("pa_generate", "pa_generate_finish", "pa_edges_bytes", "pa_scratch_bytes",
                 "pa_canonicalize", "pa_degrees", "pa_strerror", "pa_graph_create"):
        assert must in names


def test_library_exports_every_declared_symbol(pa):
    L = ctypes.CDLL(pa.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version_and_strerror(pa):
    assert pa.lib().pa_abi_version() == 1
    for s in range(0, 10):
        assert pa.strerror(s) != "unknown status"
    assert pa.strerror(0) == "ok"


@pytest.mark.parametrize("n,d,mode", [(100000, 4, 1), (100000, 4, 0), (10 ** 8, 16, 1),
                                      (2 ** 30, 4, 1), (34, 32, 0), (2, 1, 1)])
def test_edge_count_matches_oracle(pa, n, d, mode):
    bits = 64 if n > 2 ** 31 - 1 else 32
    prm = pa.make_params(n, d, 0.5, id_bits=bits, seed_mode=mode)
    assert pa.edge_count(prm) == orc.edge_count(n, d, mode)
    eb, sb = pa.sizes(prm)
    assert eb == orc.edge_count(n, d, mode) * 2 * bits // 8
    assert sb >= 256


def test_param_checks(pa):
    def rc(**kw):
        base = dict(n=1000, d=4, p=0.5)
        base.update(kw)
        prm = pa.PaParams()
        pa.lib().pa_params_init(ctypes.byref(prm))
        for k, v in base.items():
            setattr(prm, k, v)
        return pa.lib().pa_params_check(ctypes.byref(prm))

    assert rc() == pa.PA_OK
    assert rc(d=0) == pa.PA_ERR_INVALID
    assert rc(d=33) == pa.PA_OK                        # the wide kernel (d > 32)
    assert rc(d=32767, n=40000) == pa.PA_OK            # the reference's int16 EdgeIndexType
    assert rc(d=32768, n=40000) == pa.PA_ERR_NOT_SUPPORTED
    assert rc(d=33, n=2 ** 31 + 1, id_bits=64) == pa.PA_ERR_NOT_SUPPORTED   # 31-bit node ids
    assert rc(n=4, d=4) == pa.PA_ERR_INVALID          # fewer than d+1 nodes
    assert rc(n=5, d=4) == pa.PA_OK                   # the seed graph alone
    assert rc(p=-0.1) == pa.PA_ERR_INVALID
    assert rc(p=1.5) == pa.PA_ERR_INVALID
    assert rc(p=float("nan")) == pa.PA_ERR_INVALID
    assert rc(id_bits=16) == pa.PA_ERR_INVALID
    assert rc(id_bits=32, n=2 ** 31) == pa.PA_ERR_INVALID
    assert rc(id_bits=64, n=2 ** 31) == pa.PA_OK
    assert rc(seed_mode=7) == pa.PA_ERR_INVALID
    assert rc(tile_passes=3) == pa.PA_ERR_INVALID
    assert rc(flags=2) == pa.PA_ERR_INVALID
    assert rc(flags=pa.PA_FLAG_TEST_WITHHOLD_FIRST_TILE) == pa.PA_OK


def test_generate_rejects_bad_buffers_without_touching_the_device(pa):
    prm = pa.make_params(1000, 4, 0.5)
    eb, sb = pa.sizes(prm)
    L = pa.lib()
    # NULL buffers
    assert L.pa_generate(ctypes.byref(prm), None, eb, None, sb, None) == pa.PA_ERR_INVALID
    # too-small buffers (pointers are never dereferenced on this path)
    fake = ctypes.c_void_p(0x10000)
    assert L.pa_generate(ctypes.byref(prm), fake, eb - 1, fake, sb, None) == pa.PA_ERR_CAPACITY
    assert L.pa_generate(ctypes.byref(prm), fake, eb, fake, sb - 1, None) == pa.PA_ERR_CAPACITY
    # misaligned
    bad = ctypes.c_void_p(0x10004)
    assert L.pa_generate(ctypes.byref(prm), bad, eb, fake, sb, None) == pa.PA_ERR_INVALID


def test_start_split(pa):
    """Nodes below the split are the start kernel's: all of a graph below 2^31
    nodes by default, none with PA_START_NONE, otherwise whole superblocks of
    the persistent launch (64 tiles of 32/d * 2 nodes)."""
    def split(n, d, sn, bits=64):
        return pa.start_split(pa.make_params(n, d, 0.5, id_bits=bits, start_nodes=sn))
    assert split(2 ** 30, 4, 0) == 2 ** 30
    assert split(2 ** 30, 4, pa.PA_START_NONE) == 5
    assert split(10 ** 6, 4, 100_000) == 5 + 98 * 1024
    assert split(2 ** 33, 4, 0) == 5 + 2 ** 31
    assert split(100, 4, 10 ** 9) == 100


def test_claim_tiles_and_model_checked(pa):
    prm = pa.make_params(1000, 4, 0.5, claim_tiles=65)
    assert pa.lib().pa_params_check(ctypes.byref(prm)) == pa.PA_ERR_INVALID
    prm = pa.make_params(1000, 4, 0.5, claim_tiles=64)
    assert pa.lib().pa_params_check(ctypes.byref(prm)) == pa.PA_OK
    prm.model = 2
    assert pa.lib().pa_params_check(ctypes.byref(prm)) == pa.PA_ERR_INVALID
    # BA runs on the reference's star seed only
    prm = pa.make_params(1000, 4, 0.5, model=pa.PA_MODEL_BA, seed_mode=pa.PA_SEED_CLIQUE)
    assert pa.lib().pa_params_check(ctypes.byref(prm)) == pa.PA_ERR_INVALID
    prm = pa.make_params(1000, 4, 0.5, model=pa.PA_MODEL_BA, seed_mode=pa.PA_SEED_STAR_REF)
    assert pa.lib().pa_params_check(ctypes.byref(prm)) == pa.PA_OK


@pytest.mark.parametrize("n,d,bits", [(100000, 4, 32), (10 ** 6, 32, 64), (6, 5, 32), (2 ** 31 + 5, 4, 64)])
def test_slots_layout_sizes(pa, n, d, bits):
    """SLOTS holds the targets alone: (n - d - 1) * d ids, half of PAIRS less the
    seed rows; the edge count is the same graph's."""
    prm = pa.make_params(n, d, 0.5, id_bits=bits, layout=pa.PA_LAYOUT_SLOTS)
    eb, _ = pa.sizes(prm)
    assert eb == (n - d - 1) * d * bits // 8
    assert pa.edge_count(prm) == orc.edge_count(n, d, orc.SEED_CLIQUE)


def test_slots_layout_limits(pa):
    chk = pa.lib().pa_params_check
    # the whole graph must fit the start kernel (n - d - 1 <= 2^31)
    prm = pa.make_params(2 ** 31 + 6, 4, 0.5, id_bits=64, layout=pa.PA_LAYOUT_SLOTS)
    assert chk(ctypes.byref(prm)) == pa.PA_ERR_NOT_SUPPORTED
    prm = pa.make_params(10 ** 6, 4, 0.5, layout=pa.PA_LAYOUT_SLOTS, start_nodes=1000)
    assert chk(ctypes.byref(prm)) == pa.PA_ERR_NOT_SUPPORTED
    prm = pa.make_params(10 ** 6, 4, 0.5, layout=2)
    assert chk(ctypes.byref(prm)) == pa.PA_ERR_NOT_SUPPORTED
    # edge-list consumers refuse it without touching the device
    prm = pa.make_params(10 ** 6, 4, 0.5, layout=pa.PA_LAYOUT_SLOTS)
    rb, cb, sb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    assert pa.lib().pa_csr_bytes(ctypes.byref(prm), ctypes.byref(rb), ctypes.byref(cb),
                                 ctypes.byref(sb)) == pa.PA_ERR_NOT_SUPPORTED
    arr = (pa.PaParams * 1)(prm)
    assert pa.lib().pa_batch_scratch_bytes(arr, 1, ctypes.byref(sb)) == pa.PA_ERR_NOT_SUPPORTED


def test_stream_edges_rejects_bad_arguments(pa):
    prm = pa.make_params(1000, 4, 0.5)
    sink = pa._SINK(lambda ctx, data, n: 0)
    total = ctypes.c_uint64()
    L = pa.lib()
    assert L.pa_stream_edges(ctypes.byref(prm), None, 0, 0, ctypes.cast(sink, ctypes.c_void_p),
                             None, None, ctypes.byref(total)) == pa.PA_ERR_INVALID
    assert L.pa_stream_edges(ctypes.byref(prm), ctypes.c_void_p(16), 7, 0,
                             ctypes.cast(sink, ctypes.c_void_p), None, None,
                             ctypes.byref(total)) == pa.PA_ERR_INVALID
    assert L.pa_stream_edges(ctypes.byref(prm), ctypes.c_void_p(16), 0, 0, None, None, None,
                             ctypes.byref(total)) == pa.PA_ERR_INVALID


def test_binding_fails_loudly_without_the_library(pa, monkeypatch, tmp_path):
    """No silent fallback: a missing native library is an error, not a CPU path."""
    monkeypatch.setattr(pa, "LIB_PATH", str(tmp_path / "libcuppa_pa.so"))
    monkeypatch.setattr(pa, "_lib", None)
    with pytest.raises(FileNotFoundError):
        pa.lib()


def test_digest_rejects_bad_arguments_without_touching_the_device(pa):
    L = pa.lib()
    acc = ctypes.c_void_p(4096)          # never dereferenced: every call below is refused
    assert L.pa_digest(ctypes.c_void_p(4096), 10, 64, 0, None, None) == pa.PA_ERR_INVALID
    assert L.pa_digest(ctypes.c_void_p(4096), 10, 16, 0, acc, None) == pa.PA_ERR_INVALID
    assert L.pa_digest(None, 10, 64, 0, acc, None) == pa.PA_ERR_INVALID
    assert L.pa_digest(ctypes.c_void_p(4096), 10, 64, 0, ctypes.c_void_p(4100), None) == \
        pa.PA_ERR_INVALID
    assert L.pa_digest(None, 0, 32, 0, acc, None) == pa.PA_OK     # nothing to do


def test_fill_checks_and_prefilled_flag(pa):
    L = pa.lib()
    prm = pa.make_params(1000, 4, 0.5)
    assert L.pa_fill(ctypes.byref(prm), None, 1 << 20, None) == pa.PA_ERR_INVALID
    assert L.pa_fill(ctypes.byref(prm), ctypes.c_void_p(4104), 1 << 20, None) == pa.PA_ERR_INVALID
    assert L.pa_fill(ctypes.byref(prm), ctypes.c_void_p(4096), 16, None) == pa.PA_ERR_CAPACITY
    prm.flags = pa.PA_FLAG_PREFILLED
    assert L.pa_params_check(ctypes.byref(prm)) == pa.PA_OK
