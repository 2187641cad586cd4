"""pa_generate_noalloc: generation for callers that cannot allocate device memory.

Such a caller -- a host whose memory pool forbids further device allocations,
or a latency-critical request loop that must not stall in cudaMalloc/cudaFree --
passes only the parameters and its own edge buffer; the generation scratch is
the library's fixed-size __device__ array.  This file checks, through the C ABI,
that two calls in a row produce exactly the edge list of the ordinary entry point
(the generator is integer-exact, so the tolerance is zero), and that requests too
large for the array are refused before any GPU work.

It sits in its own file, collected last, so that a run stopping at the first
failure has already run every other test; it passes alone in a fresh process as
well as after the others.  The test allocates its buffers with torch; the entry
point itself allocates nothing.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _bind(pa):
    L = pa.lib()
    fn = L.pa_generate_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(pa.PaParams), ctypes.c_void_p, ctypes.c_uint64,
                   ctypes.POINTER(pa.PaStats), ctypes.c_void_p]
    return fn


def _noalloc(pa, fn, prm, stream=None):
    import torch
    E = pa.edge_count(prm)
    dt = torch.int64 if prm.id_bits == 64 else torch.int32
    out = torch.full((E, 2), -1, dtype=dt, device="cuda")
    st = pa.PaStats()
    s = stream if stream is not None else torch.cuda.current_stream()
    rc = fn(ctypes.byref(prm), ctypes.c_void_p(out.data_ptr()), out.numel() * out.element_size(),
            ctypes.byref(st), ctypes.c_void_p(int(s.cuda_stream)))
    return rc, out, st


def test_noalloc_matches_the_ordinary_entry_point_twice(pa, cuda_ok):
    import torch
    fn = _bind(pa)
    # Two calls in a row with different shapes: the second call reuses the array
    # the first one left behind.
    cases = [pa.make_params(300_000, 4, 0.5, seed=11, id_bits=64, seed_mode=pa.PA_SEED_CLIQUE),
             pa.make_params(120_000, 8, 0.3, seed=12, id_bits=32, seed_mode=pa.PA_SEED_STAR_REF)]
    for prm in cases:
        want, want_st = pa.generate(prm)            # caller-provided scratch
        rc, got, st = _noalloc(pa, fn, prm)
        assert rc == pa.PA_OK, pa.strerror(rc)
        assert st.status == pa.PA_OK
        assert torch.equal(got, want)
        assert st.retries == want_st.retries
        assert st.tiles == want_st.tiles


def test_noalloc_refuses_requests_beyond_its_array(pa, cuda_ok):
    import torch
    fn = _bind(pa)
    prm = pa.make_params(2 ** 28, 4, 0.5, seed=1, id_bits=64)   # scratch ~ 64 MiB > 16 MiB
    buf = torch.empty(16, dtype=torch.int64, device="cuda")
    rc = fn(ctypes.byref(prm), ctypes.c_void_p(buf.data_ptr()), 1 << 62, None, None)
    assert rc == pa.PA_ERR_CAPACITY
    # and the device is still fine afterwards
    rc, got, st = _noalloc(pa, fn, pa.make_params(50_000, 4, 0.5, seed=3))
    assert rc == pa.PA_OK and st.status == pa.PA_OK
    want, _ = pa.generate(pa.make_params(50_000, 4, 0.5, seed=3))
    assert torch.equal(got, want)
