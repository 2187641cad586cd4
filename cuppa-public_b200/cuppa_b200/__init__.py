"""Python binding of the B200 copy-model preferential-attachment generator.

The product is the C ABI in ``include/cuppa_pa.h`` (``lib/libcuppa_pa.so``);
this module binds it with ctypes and uses torch only for device memory and
streams.  There is no CPU fallback: if the shared library is missing or no CUDA
device is present, calls fail with an exception.

The host-side interface mirrors the reference's (paths relative to the
cuPPA-Public tree):

* ``cuPPA(nNodes, mEdgesPerNode, p)`` with ``generateGraph(conf)``,
  ``generateGraphAdaptive(conf)`` and ``printDegreeDistribution(conf)``
  -- ``src/PA/cuPPA/cuPPA.cuh:84-105``;
* ``ExperimentConfiguration`` with the reference field names
  (``_n1``, ``_x1``, ``_alpha``, ``_blockSize``, ``_threadsPerBlock``,
  ``_stages``, ``_FLAG_SHOW_DEGREE_DISTRIBUTION``, ``_distfile1``,
  ``_outputDir``) -- ``src/Utility/ExperimentConfiguration.hpp:51-96``,
  plus the new ``seed``, ``id_bits`` and ``seed_mode``.

Where the reference exits the process on a CUDA error
(``src/Common/CommonHelper.cuh:148-157``) this binding raises ``CuppaError``.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libcuppa_pa.so")

PA_OK = 0
PA_ERR_INVALID = 1
PA_ERR_OOM = 2
PA_ERR_SPIN_TIMEOUT = 3
PA_ERR_CUDA = 4
PA_ERR_CAPACITY = 5
PA_ERR_NOT_SUPPORTED = 6
PA_ERR_BUSY = 7
PA_ERR_NOT_FOUND = 8
PA_ERR_IO = 9

PA_SEED_STAR_REF = 0
PA_SEED_CLIQUE = 1
PA_MODEL_COPY = 0   # copy model (-A cuppa, -A scm)
PA_MODEL_BA = 1     # repeated-nodes Barabasi-Albert (-A sba); STAR_REF seed only
PA_LAYOUT_PAIRS = 0
PA_LAYOUT_SLOTS = 1   # targets only: half the bytes; read out with write_edges / stream_edges
PA_FORMAT_TEXT = 0
PA_FORMAT_BINARY = 1

# Test-only: the generator never publishes its first tile, so every wait on it
# runs into the wait limit (a flag that nothing sets).
PA_FLAG_TEST_WITHHOLD_FIRST_TILE = 1 << 31
# the edge buffer's generation region was set to all-ones by fill(): skip the fill
PA_FLAG_PREFILLED = 1
# start_nodes: no start kernel (every node in the persistent launch)
PA_START_NONE = (1 << 64) - 1
# request server outputs (a mask)
PA_OUT_PAIRS = 1
PA_OUT_CSR = 2


class CuppaError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {strerror(status)} (status {status})")


class PaParams(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint64),
        ("d", ctypes.c_uint32),
        ("id_bits", ctypes.c_uint32),
        ("p", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("seed_mode", ctypes.c_uint32),
        ("layout", ctypes.c_uint32),
        ("blocks", ctypes.c_uint32),
        ("threads", ctypes.c_uint32),
        ("tile_passes", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("spin_limit_ns", ctypes.c_uint64),
        ("start_nodes", ctypes.c_uint64),
        ("claim_tiles", ctypes.c_uint32),
        ("model", ctypes.c_uint32),
    ]


class PaStats(ctypes.Structure):
    _fields_ = [
        ("retries", ctypes.c_uint64),
        ("waits", ctypes.c_uint64),
        ("tiles", ctypes.c_uint64),
        ("pending_reads", ctypes.c_uint64),
        ("pending_polls", ctypes.c_uint64),
        ("status", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class PaGraph(ctypes.Structure):
    _fields_ = [
        ("params", PaParams),
        ("edges", ctypes.c_void_p),
        ("n_edges", ctypes.c_uint64),
        ("edges_bytes", ctypes.c_uint64),
        ("scratch", ctypes.c_void_p),
        ("scratch_bytes", ctypes.c_uint64),
    ]


class PaServerConfig(ctypes.Structure):
    _fields_ = [
        ("budget_bytes", ctypes.c_uint64),
        ("max_batch", ctypes.c_uint32),
        ("max_inflight", ctypes.c_uint32),
        ("max_queue", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("ttl_ns", ctypes.c_uint64),
        ("aging_ns", ctypes.c_uint64),
        ("outputs", ctypes.c_uint32),
        ("express_edges", ctypes.c_uint32),
    ]


class PaResult(ctypes.Structure):
    _fields_ = [
        ("edges", ctypes.c_void_p),
        ("n_edges", ctypes.c_uint64),
        ("edges_bytes", ctypes.c_uint64),
        ("status", ctypes.c_int32),
        ("batch_size", ctypes.c_uint32),
        ("t_submit_ns", ctypes.c_uint64),
        ("t_start_ns", ctypes.c_uint64),
        ("t_done_ns", ctypes.c_uint64),
        ("rowptr", ctypes.c_void_p),
        ("col", ctypes.c_void_p),
        ("col_bytes", ctypes.c_uint64),
    ]


class PaServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in (
        "submitted", "completed", "released", "expired", "failed", "batches", "queued",
        "running", "bytes_in_use", "budget_bytes", "edges_done")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib: Optional[ctypes.CDLL] = None

_P = ctypes.POINTER
_SIGS = {
    "pa_abi_version": (ctypes.c_int, []),
    "pa_last_cuda_error": (ctypes.c_int, []),
    "pa_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "pa_params_init": (ctypes.c_int, [_P(PaParams)]),
    "pa_params_check": (ctypes.c_int, [_P(PaParams)]),
    "pa_seed_edge_count": (ctypes.c_uint64, [ctypes.c_uint32, ctypes.c_uint32]),
    "pa_edge_count": (ctypes.c_uint64, [_P(PaParams)]),
    "pa_edges_bytes": (ctypes.c_int, [_P(PaParams), _P(ctypes.c_uint64)]),
    "pa_scratch_bytes": (ctypes.c_int, [_P(PaParams), _P(ctypes.c_uint64)]),
    "pa_generate": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_uint64,
                                   ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "pa_generate_finish": (ctypes.c_int, [ctypes.c_void_p, _P(PaStats), ctypes.c_void_p]),
    "pa_fill": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "pa_start_split": (ctypes.c_int, [_P(PaParams), _P(ctypes.c_uint64)]),
    "pa_generate_timed": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_uint64,
                                         ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                         _P(ctypes.c_void_p)]),
    "pa_generate_trace": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_uint32, _P(ctypes.c_uint32), ctypes.c_void_p]),
    "pa_canonicalize": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]),
    "pa_degrees": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p]),
    "pa_digest": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                 ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]),
    "pa_csr_bytes": (ctypes.c_int, [_P(PaParams), _P(ctypes.c_uint64), _P(ctypes.c_uint64),
                                    _P(ctypes.c_uint64)]),
    "pa_build_csr": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                    ctypes.c_void_p]),
    "pa_write_edges": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_char_p,
                                      ctypes.c_int, ctypes.c_void_p]),
    "pa_stream_edges": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, _P(ctypes.c_uint64)]),
    "pa_stream_trim": (ctypes.c_int, []),
    "pa_generate_to_file": (ctypes.c_int, [_P(PaParams), ctypes.c_char_p, ctypes.c_int,
                                           _P(PaStats), _P(ctypes.c_uint64)]),
    "pa_write_degree_distribution": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p,
                                                    ctypes.c_char_p, ctypes.c_void_p]),
    "pa_batch_scratch_bytes": (ctypes.c_int, [_P(PaParams), ctypes.c_uint32,
                                              _P(ctypes.c_uint64)]),
    "pa_batch_generate": (ctypes.c_int, [_P(PaParams), ctypes.c_uint32, _P(ctypes.c_void_p),
                                         _P(ctypes.c_uint64), ctypes.c_void_p, ctypes.c_uint64,
                                         ctypes.c_void_p]),
    "pa_graph_create": (ctypes.c_int, [_P(PaParams), _P(PaGraph)]),
    "pa_graph_generate": (ctypes.c_int, [_P(PaGraph), ctypes.c_void_p, _P(PaStats)]),
    "pa_graph_destroy": (ctypes.c_int, [_P(PaGraph)]),
    "pa_server_config_init": (ctypes.c_int, [_P(PaServerConfig)]),
    "pa_server_create": (ctypes.c_int, [_P(PaServerConfig), _P(ctypes.c_void_p)]),
    "pa_server_submit": (ctypes.c_int, [ctypes.c_void_p, _P(PaParams), _P(ctypes.c_uint64)]),
    "pa_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _P(PaResult)]),
    "pa_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                      _P(PaResult)]),
    "pa_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "pa_server_stats_get": (ctypes.c_int, [ctypes.c_void_p, _P(PaServerStats)]),
    "pa_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "pa_plan_create": (ctypes.c_int, [_P(PaParams), ctypes.c_void_p, ctypes.c_uint64,
                                      ctypes.c_void_p, ctypes.c_uint64, _P(ctypes.c_void_p)]),
    "pa_plan_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "pa_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "pa_router_create": (ctypes.c_int, [_P(PaServerConfig), _P(ctypes.c_int32), ctypes.c_uint32,
                                        _P(ctypes.c_void_p)]),
    "pa_router_submit": (ctypes.c_int, [ctypes.c_void_p, _P(PaParams), _P(ctypes.c_uint64)]),
    "pa_router_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _P(PaResult)]),
    "pa_router_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                      _P(PaResult)]),
    "pa_router_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "pa_router_device_of": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _P(ctypes.c_int32)]),
    "pa_router_stats_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _P(PaServerStats)]),
    "pa_router_size": (ctypes.c_uint32, [ctypes.c_void_p]),
    "pa_router_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "pa_route_pick": (ctypes.c_uint32, [_P(ctypes.c_uint64), _P(ctypes.c_uint64), ctypes.c_uint32,
                                        ctypes.c_uint64]),
    "pa_batch_partition": (ctypes.c_int, [_P(PaParams), ctypes.c_uint32, ctypes.c_uint32,
                                          _P(ctypes.c_uint32)]),
    "pa_sched_create": (ctypes.c_void_p, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32]),
    "pa_sched_destroy": (None, [ctypes.c_void_p]),
    "pa_sched_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_uint64]),
    "pa_sched_admit": (ctypes.c_uint32, [ctypes.c_void_p, ctypes.c_uint64, _P(ctypes.c_uint64),
                                         ctypes.c_uint32]),
    "pa_sched_submit_lane": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                            ctypes.c_uint64, ctypes.c_uint32]),
    "pa_sched_admit_lanes": (ctypes.c_uint32, [ctypes.c_void_p, ctypes.c_uint64,
                                               _P(ctypes.c_uint64), ctypes.c_uint32,
                                               ctypes.c_uint32]),
    "pa_sched_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]),
    "pa_sched_in_use": (ctypes.c_uint64, [ctypes.c_void_p]),
    "pa_sched_queued": (ctypes.c_uint64, [ctypes.c_void_p]),
}


def lib() -> ctypes.CDLL:
    """Load libcuppa_pa.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C cuppa-public_b200`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def strerror(status: int) -> str:
    try:
        return lib().pa_strerror(status).decode()
    except Exception:  # pragma: no cover - only when the library is absent
        return f"status {status}"


def check(status: int, where: str) -> None:
    if status != PA_OK:
        raise CuppaError(status, where)


def make_params(n: int, d: int, p: float, seed: int = 42, id_bits: int = 32,
                seed_mode: int = PA_SEED_CLIQUE, blocks: int = 0, threads: int = 0,
                tile_passes: int = 0, flags: int = 0, spin_limit_ns: int = 0,
                start_nodes: int = 0, claim_tiles: int = 0,
                model: int = 0, layout: int = 0) -> PaParams:
    prm = PaParams()
    check(lib().pa_params_init(ctypes.byref(prm)), "pa_params_init")
    prm.n, prm.d, prm.p, prm.seed = n, d, float(p), seed
    prm.id_bits, prm.seed_mode = id_bits, seed_mode
    prm.blocks, prm.threads, prm.tile_passes = blocks, threads, tile_passes
    prm.flags, prm.spin_limit_ns, prm.start_nodes = flags, spin_limit_ns, start_nodes
    prm.claim_tiles, prm.model, prm.layout = claim_tiles, model, layout
    return prm


def edge_count(prm: PaParams) -> int:
    return int(lib().pa_edge_count(ctypes.byref(prm)))


def sizes(prm: PaParams) -> tuple[int, int]:
    """(edge buffer bytes, scratch bytes) for prm."""
    eb, sb = ctypes.c_uint64(), ctypes.c_uint64()
    check(lib().pa_edges_bytes(ctypes.byref(prm), ctypes.byref(eb)), "pa_edges_bytes")
    check(lib().pa_scratch_bytes(ctypes.byref(prm), ctypes.byref(sb)), "pa_scratch_bytes")
    return int(eb.value), int(sb.value)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("cuppa_b200 needs a CUDA device; there is no CPU fallback")
    return torch


def _stream_ptr(stream) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def alloc_buffers(prm: PaParams, device=None):
    """Device tensors for the edges (E x 2 ids; SLOTS: (n-d-1) x d targets) and
    the generation scratch."""
    torch = _torch()
    eb, sb = sizes(prm)
    dt = torch.int64 if prm.id_bits == 64 else torch.int32
    if prm.layout == PA_LAYOUT_SLOTS:
        rows = prm.n - prm.d - 1
        edges = torch.empty((max(rows, 1), prm.d), dtype=dt, device=device or "cuda")
        scratch = torch.empty(max(sb, 256), dtype=torch.uint8, device=device or "cuda")
        return edges, scratch
    E = edge_count(prm)
    edges = torch.empty((max(E, 1), 2), dtype=dt, device=device or "cuda")
    scratch = torch.empty(max(sb, 256), dtype=torch.uint8, device=device or "cuda")
    return edges, scratch


def generate_into(prm: PaParams, edges, scratch, stream=None) -> None:
    """Stream-ordered pa_generate into the given device tensors."""
    rc = lib().pa_generate(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                           edges.numel() * edges.element_size(),
                           ctypes.c_void_p(scratch.data_ptr()), scratch.numel(),
                           ctypes.c_void_p(_stream_ptr(stream)))
    check(rc, "pa_generate")


def fill(prm: PaParams, edges, stream=None) -> None:
    """pa_fill: all-ones over the generation region of `edges`, on a small grid
    that can run beside a generation on another stream (for a later generation
    with PA_FLAG_PREFILLED)."""
    check(lib().pa_fill(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                        edges.numel() * edges.element_size(),
                        ctypes.c_void_p(_stream_ptr(stream))), "pa_fill")


def generate_timed(prm: PaParams, edges, scratch, events, stream=None) -> None:
    """pa_generate_timed: `events` are four torch.cuda.Event(enable_timing=True)
    recorded before the first launch, before the start kernel, before the
    persistent launch and after the last launch."""
    for ev in events:
        if not ev.cuda_event:
            ev.record(stream)      # the CUDA event is created on first record
    arr = (ctypes.c_void_p * 4)(*[ev.cuda_event for ev in events])
    rc = lib().pa_generate_timed(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                                 edges.numel() * edges.element_size(),
                                 ctypes.c_void_p(scratch.data_ptr()), scratch.numel(),
                                 ctypes.c_void_p(_stream_ptr(stream)), arr)
    check(rc, "pa_generate_timed")


def start_split(prm: PaParams) -> int:
    """First node left to the persistent launch (pa_start_split)."""
    u = ctypes.c_uint64()
    check(lib().pa_start_split(ctypes.byref(prm), ctypes.byref(u)), "pa_start_split")
    return int(u.value)


def finish(scratch, stream=None) -> PaStats:
    st = PaStats()
    lib().pa_generate_finish(ctypes.c_void_p(scratch.data_ptr()), ctypes.byref(st),
                             ctypes.c_void_p(_stream_ptr(stream)))
    return st


def trace(prm: PaParams, scratch, stream=None, max_samples: int = 2048):
    """Progress samples of the last generation into `scratch`: list of
    (elapsed ns, nodes complete)."""
    import numpy as np
    buf = np.zeros(2 * max_samples, dtype=np.uint64)
    cnt = ctypes.c_uint32()
    check(lib().pa_generate_trace(ctypes.byref(prm), ctypes.c_void_p(scratch.data_ptr()),
                                  buf.ctypes.data_as(ctypes.c_void_p), max_samples,
                                  ctypes.byref(cnt), ctypes.c_void_p(_stream_ptr(stream))),
          "pa_generate_trace")
    return [(int(buf[2 * i]), int(buf[2 * i + 1])) for i in range(cnt.value)]


def generate(prm: PaParams, stream=None, raise_on_error: bool = True):
    """Generate one graph; returns (edges tensor [E, 2] on the device, PaStats)
    -- for PA_LAYOUT_SLOTS the targets [n-d-1, d] instead."""
    edges, scratch = alloc_buffers(prm)
    generate_into(prm, edges, scratch, stream)
    st = finish(scratch, stream)
    if raise_on_error:
        check(st.status, "pa_generate (device)")
    if prm.layout == PA_LAYOUT_SLOTS:
        return edges[: prm.n - prm.d - 1], st
    return edges[: edge_count(prm)], st


class Batch:
    """Device buffers for a batch of graphs generated by one persistent launch."""

    def __init__(self, prms, device=None):
        torch = _torch()
        self.prms = list(prms)
        k = len(self.prms)
        self._arr = (PaParams * k)(*self.prms)
        sb = ctypes.c_uint64()
        check(lib().pa_batch_scratch_bytes(self._arr, k, ctypes.byref(sb)), "pa_batch_scratch_bytes")
        self.scratch = torch.empty(sb.value, dtype=torch.uint8, device=device or "cuda")
        self.edges = []
        for prm in self.prms:
            dt = torch.int64 if prm.id_bits == 64 else torch.int32
            self.edges.append(torch.empty((max(edge_count(prm), 1), 2), dtype=dt,
                                          device=device or "cuda"))
        self._ptrs = (ctypes.c_void_p * k)(*[e.data_ptr() for e in self.edges])
        self._bytes = (ctypes.c_uint64 * k)(*[e.numel() * e.element_size() for e in self.edges])

    def generate(self, stream=None) -> None:
        check(lib().pa_batch_generate(self._arr, len(self.prms), self._ptrs, self._bytes,
                                      ctypes.c_void_p(self.scratch.data_ptr()),
                                      self.scratch.numel(), ctypes.c_void_p(_stream_ptr(stream))),
              "pa_batch_generate")

    def finish(self, stream=None) -> PaStats:
        return finish(self.scratch, stream)

    def graph(self, i: int):
        return self.edges[i][: edge_count(self.prms[i])]


def canonicalize(prm: PaParams, edges, out=None, stream=None):
    out = edges if out is None else out
    check(lib().pa_canonicalize(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                                ctypes.c_void_p(out.data_ptr()),
                                ctypes.c_void_p(_stream_ptr(stream))), "pa_canonicalize")
    return out


def degrees(prm: PaParams, edges, stream=None):
    torch = _torch()
    deg = torch.empty(prm.n, dtype=torch.int64, device=edges.device)
    check(lib().pa_degrees(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                           ctypes.c_void_p(deg.data_ptr()),
                           ctypes.c_void_p(_stream_ptr(stream))), "pa_degrees")
    return deg


def digest(ids, index_base: int = 0, stream=None) -> tuple[int, int]:
    """pa_digest of a device tensor of int32/int64 ids taken as one flat array:
    (sum, xor) of the position-keyed terms, as unsigned 64-bit integers."""
    torch = _torch()
    if ids.dtype not in (torch.int32, torch.int64) or not ids.is_contiguous():
        raise ValueError("digest needs a contiguous int32 or int64 tensor")
    s = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(s):            # the accumulator is cleared on the launch stream
        acc = torch.zeros(2, dtype=torch.int64, device=ids.device)
    check(lib().pa_digest(ctypes.c_void_p(ids.data_ptr()), ids.numel(),
                          32 if ids.dtype == torch.int32 else 64, index_base,
                          ctypes.c_void_p(acc.data_ptr()), ctypes.c_void_p(int(s.cuda_stream))),
          "pa_digest")
    s.synchronize()
    a, b = acc.tolist()
    return a & (2 ** 64 - 1), b & (2 ** 64 - 1)


def build_csr(prm: PaParams, edges, stream=None):
    """Undirected CSR (rowptr int64[n+1], col ids[2E]) with sorted rows."""
    torch = _torch()
    rb, cb, sb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    check(lib().pa_csr_bytes(ctypes.byref(prm), ctypes.byref(rb), ctypes.byref(cb),
                             ctypes.byref(sb)), "pa_csr_bytes")
    rowptr = torch.empty(prm.n + 1, dtype=torch.int64, device=edges.device)
    dt = torch.int64 if prm.id_bits == 64 else torch.int32
    col = torch.empty(max(cb.value // (prm.id_bits // 8), 1), dtype=dt, device=edges.device)
    scratch = torch.empty(sb.value, dtype=torch.uint8, device=edges.device)
    check(lib().pa_build_csr(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                             ctypes.c_void_p(rowptr.data_ptr()), ctypes.c_void_p(col.data_ptr()),
                             ctypes.c_void_p(scratch.data_ptr()), sb.value,
                             ctypes.c_void_p(_stream_ptr(stream))), "pa_build_csr")
    return rowptr, col[: cb.value // (prm.id_bits // 8)]


def write_edges(prm: PaParams, edges, path: str, binary: bool = False, stream=None) -> None:
    """PAHelper::writeGraphToDisk's "u v" text (or raw pairs), formatted on the
    device and streamed to the file (either layout)."""
    check(lib().pa_write_edges(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                               path.encode(), PA_FORMAT_BINARY if binary else PA_FORMAT_TEXT,
                               ctypes.c_void_p(_stream_ptr(stream))), "pa_write_edges")


_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64)


def stream_edges(prm: PaParams, edges, sink, binary: bool = False, chunk_edges: int = 0,
                 stream=None) -> int:
    """pa_stream_edges: sink(bytes) receives the output in order (called from a
    library thread); returns the byte count.  A sink that raises or returns a
    true value stops the stream (PaError PA_ERR_IO)."""
    def _cb(ctx, data, nbytes):
        try:
            return 1 if sink(ctypes.string_at(data, nbytes)) else 0
        except Exception:
            return 1
    cb = _SINK(_cb)
    total = ctypes.c_uint64()
    check(lib().pa_stream_edges(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                                PA_FORMAT_BINARY if binary else PA_FORMAT_TEXT, chunk_edges,
                                ctypes.cast(cb, ctypes.c_void_p), None,
                                ctypes.c_void_p(_stream_ptr(stream)), ctypes.byref(total)),
          "pa_stream_edges")
    return int(total.value)


def stream_trim() -> None:
    """Free the staging memory pa_stream_edges keeps between calls."""
    check(lib().pa_stream_trim(), "pa_stream_trim")


def generate_to_file(prm: PaParams, path: str, binary: bool = False):
    """pa_generate_to_file: generate into library memory and write; returns
    (PaStats, bytes written)."""
    st, total = PaStats(), ctypes.c_uint64()
    check(lib().pa_generate_to_file(ctypes.byref(prm), path.encode(),
                                    PA_FORMAT_BINARY if binary else PA_FORMAT_TEXT,
                                    ctypes.byref(st), ctypes.byref(total)), "pa_generate_to_file")
    return st, int(total.value)


def write_degree_distribution(prm: PaParams, edges, path: str, stream=None) -> None:
    """cuPPA::printDegreeDistribution's "Degree,Count" CSV, computed on the device."""
    check(lib().pa_write_degree_distribution(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                                             path.encode(), ctypes.c_void_p(_stream_ptr(stream))),
          "pa_write_degree_distribution")


def degree_distribution_csv(deg) -> str:
    """'Degree,Count' CSV of src/PA/cuPPA/cuPPA.cu:150-157 (degree-0 nodes skipped)."""
    torch = _torch()
    vals, cnts = torch.unique(deg[deg > 0], return_counts=True)
    rows = ["Degree,Count"] + [f"{int(v)},{int(c)}" for v, c in zip(vals.tolist(), cnts.tolist())]
    return "\n".join(rows) + "\n"


# ---------------------------------------------------------------------------
# Mirror of the reference's host interface
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class ExperimentConfiguration:
    """Reference field names (src/Utility/ExperimentConfiguration.hpp:51-96)
    with the runner defaults of src/main.cu:130-174, plus seed/id width/seed mode."""
    _algorithm: str = "cuppa"
    _n1: int = 1000
    _x1: int = 4
    _alpha: float = 0.5
    _stages: int = 1000
    _blockSize: int = 0          # -b: 0 = one full wave of the GPU
    _threadsPerBlock: int = 0    # -t: 0 = auto
    _warpSize: int = 32
    _FLAG_SHOW_DEGREE_DISTRIBUTION: bool = False
    _distfile1: str = "degreeDistribution.txt"
    _outputDir: str = "./"
    seed: int = 42
    id_bits: int = 32
    seed_mode: int = PA_SEED_CLIQUE


class cuPPA:  # noqa: N801 - reference class name
    """cuPPA(nNodes, mEdgesPerNode, p) -- src/PA/cuPPA/cuPPA.cuh:84-105.

    Unlike the reference, the generated graph is kept (``self.edges``, a device
    tensor of (u, v) pairs) instead of being freed before return
    (src/PA/cuPPA/cuPPA_1.cu:247-250)."""

    def __init__(self, nNodes: int, mEdgesPerNode: int, p: float):
        self._N, self._M, self._p = int(nNodes), int(mEdgesPerNode), float(p)
        self.edges = None
        self.stats: Optional[PaStats] = None
        self._prm: Optional[PaParams] = None

    def _params(self, conf: ExperimentConfiguration) -> PaParams:
        self._N, self._M, self._p = int(conf._n1), int(conf._x1), float(conf._alpha)
        threads = conf._threadsPerBlock if conf._threadsPerBlock in (0, 256) else 0
        return make_params(self._N, self._M, self._p, seed=conf.seed, id_bits=conf.id_bits,
                           seed_mode=conf.seed_mode, blocks=conf._blockSize, threads=threads)

    def generateGraph(self, conf: ExperimentConfiguration):
        """cuPPA_1.cu:9 -- one persistent launch replaces the staged loop."""
        self._prm = self._params(conf)
        self.edges, self.stats = generate(self._prm)
        if conf._FLAG_SHOW_DEGREE_DISTRIBUTION:
            self.printDegreeDistribution(conf)
        return self.edges

    def generateGraphAdaptive(self, conf: ExperimentConfiguration):
        """cuPPA_2.cu:9 -- the adaptive stage tuner has nothing to tune here."""
        return self.generateGraph(conf)

    def printDegreeDistribution(self, conf: ExperimentConfiguration) -> str:
        """cuPPA.cu:103-165 -- degrees on the device, 'Degree,Count' CSV to
        outputDir/distfile1."""
        if self.edges is None:
            raise RuntimeError("generateGraph first")
        path = os.path.join(conf._outputDir, conf._distfile1)
        write_degree_distribution(self._prm, self.edges, path)
        with open(path) as f:
            return f.read()


class SerialCopyModel:  # noqa: N801 - reference class name
    """SerialCopyModel(nNodes, mEdgesPerNode, p) -- src/PA/SPA/SerialCopyModel.h,
    the sequential copy model of -A scm (src/main.cu:93-98, SerialCopyModel.h:26-45),
    run on the device:
    the same model as cuPPA on the reference's star seed graph
    (SerialCopyModel3.cpp:38-49).  generateGraph keeps the edges; the degree
    distribution is the "Degree,Count" CSV of src/PA/SPA/PAHelper.hpp:15-67."""

    def __init__(self, nNodes: int, mEdgesPerNode: int, p: float):
        self._N, self._M, self._p = int(nNodes), int(mEdgesPerNode), float(p)
        self.edges = None
        self.stats: Optional[PaStats] = None
        self._prm: Optional[PaParams] = None

    def generateGraph(self, conf: ExperimentConfiguration):
        self._N, self._M, self._p = int(conf._n1), int(conf._x1), float(conf._alpha)
        self._prm = make_params(self._N, self._M, self._p, seed=conf.seed, id_bits=conf.id_bits,
                                seed_mode=PA_SEED_STAR_REF, blocks=conf._blockSize)
        self.edges, self.stats = generate(self._prm)
        if conf._FLAG_SHOW_DEGREE_DISTRIBUTION:
            self.printDegreeDistribution(conf)
        return self.edges

    def printDegreeDistribution(self, conf: ExperimentConfiguration) -> str:
        if self.edges is None:
            raise RuntimeError("generateGraph first")
        path = os.path.join(conf._outputDir, conf._distfile1)
        write_degree_distribution(self._prm, self.edges, path)
        with open(path) as f:
            return f.read()


class SerialBA:  # noqa: N801 - reference class name
    """SerialBA(nNodes, mEdgesPerNode) -- src/PA/SPA/SerialBA.h:17-37, the
    repeated-nodes Barabasi-Albert generator of -A sba, run on the device
    (model PA_MODEL_BA, the reference's star seed).  generateGraph keeps the
    edges (``self.edges``: node M's edges to 0..M-1, then each later node's M
    edges in draw order); printDegreeDistribution writes the "Degree,Count" CSV
    of src/PA/SPA/PAHelper.hpp:69-147."""

    def __init__(self, nNodes: int, mEdgesPerNode: int):
        self._N, self._M = int(nNodes), int(mEdgesPerNode)
        self.edges = None
        self.stats: Optional[PaStats] = None
        self._prm: Optional[PaParams] = None

    def generateGraph(self, conf: ExperimentConfiguration):
        self._N, self._M = int(conf._n1), int(conf._x1)
        self._prm = make_params(self._N, self._M, 0.0, seed=conf.seed, id_bits=conf.id_bits,
                                seed_mode=PA_SEED_STAR_REF, blocks=conf._blockSize,
                                model=PA_MODEL_BA)
        self.edges, self.stats = generate(self._prm)
        if conf._FLAG_SHOW_DEGREE_DISTRIBUTION:
            self.printDegreeDistribution(conf)
        return self.edges

    def printDegreeDistribution(self, conf: ExperimentConfiguration) -> str:
        if self.edges is None:
            raise RuntimeError("generateGraph first")
        path = os.path.join(conf._outputDir, conf._distfile1)
        write_degree_distribution(self._prm, self.edges, path)
        with open(path) as f:
            return f.read()


# ---------------------------------------------------------------------------
# Request server and its admission queue
# ---------------------------------------------------------------------------
class _DeviceArray:
    """A device buffer the server owns, exposed through __cuda_array_interface__
    so torch.as_tensor can view it without a copy."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (ptr, False), "version": 2, "strides": None}


class Plan:
    """A generation captured into a CUDA graph (pa_plan_*), for fixed parameters
    and device buffers; launch() replays it."""

    def __init__(self, prm: PaParams, edges, scratch):
        h = ctypes.c_void_p()
        check(lib().pa_plan_create(ctypes.byref(prm), ctypes.c_void_p(edges.data_ptr()),
                                   edges.numel() * edges.element_size(),
                                   ctypes.c_void_p(scratch.data_ptr()), scratch.numel(),
                                   ctypes.byref(h)), "pa_plan_create")
        self._h, self.edges, self.scratch = h, edges, scratch

    def launch(self, stream=None) -> None:
        check(lib().pa_plan_launch(self._h, ctypes.c_void_p(_stream_ptr(stream))),
              "pa_plan_launch")

    def close(self):
        if getattr(self, "_h", None):
            lib().pa_plan_destroy(self._h)
            self._h = None

    __del__ = close


class Sched:
    """The server's admission queue alone (host logic; no GPU needed)."""

    def __init__(self, budget_bytes: int, aging_ns: int = 100_000_000, max_queue: int = 0):
        self._h = lib().pa_sched_create(budget_bytes, aging_ns, max_queue)
        if not self._h:
            raise MemoryError("pa_sched_create")

    def close(self):
        if getattr(self, "_h", None):
            lib().pa_sched_destroy(self._h)
            self._h = None

    __del__ = close

    def submit(self, ticket: int, nbytes: int, now_ns: int, lane: int = 0) -> int:
        if lane == 0:
            return lib().pa_sched_submit(self._h, ticket, nbytes, now_ns)
        return lib().pa_sched_submit_lane(self._h, ticket, nbytes, now_ns, lane)

    def admit(self, now_ns: int, cap: int = 4096, lanes: int = 0xFFFFFFFF) -> list:
        out = (ctypes.c_uint64 * cap)()
        if lanes == 0xFFFFFFFF:
            n = lib().pa_sched_admit(self._h, now_ns, out, cap)
        else:
            n = lib().pa_sched_admit_lanes(self._h, now_ns, out, cap, lanes)
        return [int(out[i]) for i in range(n)]

    def release(self, ticket: int, nbytes: int = (1 << 64) - 1) -> int:
        return lib().pa_sched_release(self._h, ticket, nbytes)

    @property
    def in_use(self) -> int:
        return int(lib().pa_sched_in_use(self._h))

    @property
    def queued(self) -> int:
        return int(lib().pa_sched_queued(self._h))


class Server:
    """Continuous-batching generation server (pa_server_*)."""

    def __init__(self, budget_bytes: int = 0, max_batch: int = 0, max_inflight: int = 0,
                 max_queue: int = 0, device: int = -1, ttl_ns: int = 0, aging_ns: int = 0,
                 outputs: int = 0, express_edges: int = 0):
        cfg = PaServerConfig()
        check(lib().pa_server_config_init(ctypes.byref(cfg)), "pa_server_config_init")
        cfg.budget_bytes, cfg.max_batch, cfg.max_inflight = budget_bytes, max_batch, max_inflight
        cfg.max_queue, cfg.device, cfg.ttl_ns, cfg.aging_ns = max_queue, device, ttl_ns, aging_ns
        cfg.outputs, cfg.express_edges = outputs, express_edges
        h = ctypes.c_void_p()
        check(lib().pa_server_create(ctypes.byref(cfg), ctypes.byref(h)), "pa_server_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().pa_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, prm: PaParams) -> int:
        t = ctypes.c_uint64()
        check(lib().pa_server_submit(self._h, ctypes.byref(prm), ctypes.byref(t)),
              "pa_server_submit")
        return int(t.value)

    def try_submit(self, prm: PaParams):
        """(status, ticket) without raising."""
        t = ctypes.c_uint64()
        rc = lib().pa_server_submit(self._h, ctypes.byref(prm), ctypes.byref(t))
        return rc, int(t.value)

    def poll(self, ticket: int):
        """(status, PaResult): PA_OK when finished, PA_ERR_BUSY while pending."""
        r = PaResult()
        rc = lib().pa_server_poll(self._h, ticket, ctypes.byref(r))
        return rc, r

    def wait(self, ticket: int, timeout_ns: int = 0):
        r = PaResult()
        rc = lib().pa_server_wait(self._h, ticket, timeout_ns, ctypes.byref(r))
        return rc, r

    def release(self, ticket: int) -> int:
        return lib().pa_server_release(self._h, ticket)

    def stats(self) -> PaServerStats:
        st = PaServerStats()
        check(lib().pa_server_stats_get(self._h, ctypes.byref(st)), "pa_server_stats_get")
        return st

    @staticmethod
    def edges_view(result: PaResult, id_bits: int):
        """A torch tensor [n_edges, 2] viewing a finished result's device buffer
        (valid until the ticket is released)."""
        torch = _torch()
        ts = "<i8" if id_bits == 64 else "<i4"
        arr = _DeviceArray(int(result.edges), (int(result.n_edges), 2), ts)
        return torch.as_tensor(arr, device="cuda")

    @staticmethod
    def csr_view(result: PaResult, n: int, id_bits: int):
        """(rowptr int64 [n + 1], col [2 * n_edges]) tensors viewing a finished
        result's CSR (server with PA_OUT_CSR; valid until the ticket is released)."""
        torch = _torch()
        rp = torch.as_tensor(_DeviceArray(int(result.rowptr), (n + 1,), "<i8"), device="cuda")
        ts = "<i8" if id_bits == 64 else "<i4"
        col = torch.as_tensor(_DeviceArray(int(result.col), (2 * int(result.n_edges),), ts),
                              device="cuda")
        return rp, col



# ---------------------------------------------------------------------------
# Several GPUs: request router and batch partition
# ---------------------------------------------------------------------------
def route_pick(load_bytes, budget_bytes, request_bytes: int) -> int:
    """pa_route_pick: the server index a request of request_bytes goes to."""
    n = len(load_bytes)
    lo = (ctypes.c_uint64 * n)(*load_bytes)
    bu = (ctypes.c_uint64 * n)(*budget_bytes)
    return int(lib().pa_route_pick(lo, bu, n, request_bytes))


def batch_partition(prms, k: int) -> list:
    """pa_batch_partition: part index (0..k-1) of every instance, LPT by edge bytes."""
    arr = (PaParams * len(prms))(*prms)
    out = (ctypes.c_uint32 * max(len(prms), 1))()
    check(lib().pa_batch_partition(arr, len(prms), k, out), "pa_batch_partition")
    return list(out)[: len(prms)]


class Router:
    """One request server per device behind one ticket space (pa_router_*)."""

    def __init__(self, devices, budget_bytes: int = 0, max_batch: int = 0,
                 max_inflight: int = 0, max_queue: int = 0, ttl_ns: int = 0,
                 aging_ns: int = 0, outputs: int = 0):
        cfg = PaServerConfig()
        check(lib().pa_server_config_init(ctypes.byref(cfg)), "pa_server_config_init")
        cfg.budget_bytes, cfg.max_batch, cfg.max_inflight = budget_bytes, max_batch, max_inflight
        cfg.max_queue, cfg.ttl_ns, cfg.aging_ns, cfg.outputs = max_queue, ttl_ns, aging_ns, outputs
        devs = (ctypes.c_int32 * len(devices))(*devices)
        h = ctypes.c_void_p()
        check(lib().pa_router_create(ctypes.byref(cfg), devs, len(devices), ctypes.byref(h)),
              "pa_router_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().pa_router_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return int(lib().pa_router_size(self._h))

    def submit(self, prm: PaParams) -> int:
        t = ctypes.c_uint64()
        check(lib().pa_router_submit(self._h, ctypes.byref(prm), ctypes.byref(t)),
              "pa_router_submit")
        return int(t.value)

    def poll(self, ticket: int):
        r = PaResult()
        return lib().pa_router_poll(self._h, ticket, ctypes.byref(r)), r

    def wait(self, ticket: int, timeout_ns: int = 0):
        r = PaResult()
        return lib().pa_router_wait(self._h, ticket, timeout_ns, ctypes.byref(r)), r

    def release(self, ticket: int) -> int:
        return lib().pa_router_release(self._h, ticket)

    def device_of(self, ticket: int) -> int:
        d = ctypes.c_int32()
        check(lib().pa_router_device_of(self._h, ticket, ctypes.byref(d)), "pa_router_device_of")
        return int(d.value)

    def server_of(self, ticket: int) -> int:
        return ticket & 0xFF

    def stats(self, index=None) -> PaServerStats:
        st = PaServerStats()
        i = len(self) if index is None else index
        check(lib().pa_router_stats_get(self._h, i, ctypes.byref(st)), "pa_router_stats_get")
        return st
