"""The request server: every result equals the same request generated alone
(pa_generate), whatever batch it was served in; the budget is never exceeded;
release, TTL expiry and admission errors behave as documented."""
import threading
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests(pa, count, rng, max_exp=6.0, bits=None):
    out = []
    for i in range(count):
        n = int(round(10 ** rng.uniform(2, max_exp)))
        d = int(rng.integers(1, 33))
        n = max(n, d + 1)
        b = bits or (32 if rng.random() < 0.7 else 64)
        out.append(pa.make_params(n, d, float(rng.uniform(0.1, 0.9)), seed=5000 + i, id_bits=b,
                                  seed_mode=int(rng.integers(0, 2))))
    return out


def _check_alone(pa, prm, res):
    assert res.status == 0
    got = pa.Server.edges_view(res, prm.id_bits)
    want, _ = pa.generate(prm)
    assert torch.equal(got, want), f"n={prm.n} d={prm.d} p={prm.p} seed={prm.seed}"


def _drain(srv, timeout=5.0):
    deadline = time.time() + timeout
    while srv.stats().bytes_in_use and time.time() < deadline:
        time.sleep(0.01)


def test_results_equal_alone_in_the_mix(pa, cuda_ok):
    rng = np.random.default_rng(1)
    prms = _requests(pa, 120, rng)
    with pa.Server(budget_bytes=8 << 30) as srv:
        tickets = [srv.submit(q) for q in prms]
        sizes = []
        for t, q in zip(tickets, prms):
            rc, res = srv.wait(t)
            assert rc == 0
            sizes.append(res.batch_size)
            _check_alone(pa, q, res)
            assert srv.release(t) == 0
        assert max(sizes) > 1          # requests really were served together
        st = srv.stats()
        assert st.completed == len(prms) and st.failed == 0
        _drain(srv)
        assert srv.stats().bytes_in_use == 0


def test_concurrent_clients_and_budget(pa, cuda_ok):
    """Four client threads submit while results are consumed and released; the
    memory held never exceeds the budget."""
    budget = 256 << 20
    rng = np.random.default_rng(2)
    prms = _requests(pa, 160, rng, max_exp=5.5, bits=32)
    peak = [0]
    errors = []
    with pa.Server(budget_bytes=budget, max_batch=64) as srv:
        stop = threading.Event()

        def watch():
            while not stop.is_set():
                peak[0] = max(peak[0], srv.stats().bytes_in_use)
                time.sleep(0.0005)

        def client(part):
            try:
                for q in part:
                    t = srv.submit(q)
                    rc, res = srv.wait(t)
                    assert rc == 0
                    _check_alone(pa, q, res)
                    assert srv.release(t) == 0
            except Exception as e:  # surfaced below
                errors.append(e)

        w = threading.Thread(target=watch)
        w.start()
        th = [threading.Thread(target=client, args=(prms[i::4],)) for i in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        stop.set()
        w.join()
        assert not errors, errors[0]
        _drain(srv)
        st = srv.stats()
        assert st.bytes_in_use == 0 and st.completed == len(prms)
    assert 0 < peak[0] <= budget


def test_capacity_ttl_and_release(pa, cuda_ok):
    with pa.Server(budget_bytes=64 << 20, ttl_ns=50_000_000) as srv:
        big = pa.make_params(10_000_000, 8, 0.5, seed=1)           # 640 MB of pairs
        rc, _ = srv.try_submit(big)
        assert rc == pa.PA_ERR_CAPACITY
        small = [pa.make_params(20_000, 4, 0.5, seed=s) for s in range(5)]
        ts = [srv.submit(q) for q in small]
        for t in ts:
            rc, _ = srv.wait(t)
            assert rc == 0
        assert srv.release(ts[0]) == 0
        assert srv.release(ts[0]) == pa.PA_ERR_NOT_FOUND
        time.sleep(0.3)                                             # past the TTL
        for t in ts[1:]:
            assert srv.poll(t)[0] == pa.PA_ERR_NOT_FOUND
        st = srv.stats()
        assert st.expired == 4 and st.released == 1
        _drain(srv)
        assert srv.stats().bytes_in_use == 0


def test_larger_request_with_64_bit_ids(pa, cuda_ok):
    """A larger request with 64-bit ids (3 million nodes) matches pa_generate."""
    with pa.Server(budget_bytes=2 << 30) as srv:
        prm = pa.make_params(3_000_000, 2, 0.3, seed=3, id_bits=64)
        t = srv.submit(prm)
        rc, res = srv.wait(t, timeout_ns=60_000_000_000)
        assert rc == 0
        _check_alone(pa, prm, res)
        srv.release(t)


@pytest.mark.parametrize("outputs", ["csr", "both"])
def test_csr_outputs_equal_alone(pa, cuda_ok, outputs):
    """With CSR outputs every served graph's CSR equals pa_build_csr of the same
    request generated alone; without PA_OUT_PAIRS the pair buffer is not kept,
    and all memory returns to the budget after release."""
    out = pa.PA_OUT_CSR | (pa.PA_OUT_PAIRS if outputs == "both" else 0)
    rng = np.random.default_rng(3)
    prms = _requests(pa, 40, rng, max_exp=5.0)
    with pa.Server(budget_bytes=2 << 30, outputs=out) as srv:
        tickets = [srv.submit(q) for q in prms]
        for t, q in zip(tickets, prms):
            rc, res = srv.wait(t)
            assert rc == 0 and res.status == 0
            want_e, _ = pa.generate(q)
            want_rp, want_col = pa.build_csr(q, want_e)
            rp, col = pa.Server.csr_view(res, q.n, q.id_bits)
            assert torch.equal(rp, want_rp) and torch.equal(col, want_col)
            if outputs == "both":
                assert torch.equal(pa.Server.edges_view(res, q.id_bits), want_e)
            else:
                assert res.edges is None
            assert srv.release(t) == 0
        _drain(srv)
        assert srv.stats().bytes_in_use == 0


def test_small_request_overtakes_a_running_large_batch(pa, cuda_ok):
    """A small request submitted while a large batch runs goes to the express
    lane (its own high-priority stream) and finishes before that batch: with
    CSR outputs the large batch is a generation followed by a chain of CSR
    kernels, and the small request's kernels take the SMs at the first kernel
    boundary.  Both results equal the requests generated alone."""
    out = pa.PA_OUT_CSR | pa.PA_OUT_PAIRS
    big = pa.make_params(30_000_000, 16, 0.5, seed=11, id_bits=32)
    small = pa.make_params(20_000, 4, 0.5, seed=12)
    with pa.Server(budget_bytes=24 << 30, outputs=out) as srv:
        # warm both lanes up (first launches load kernels)
        for q in (pa.make_params(3_000_000, 16, 0.5, seed=1), small):
            t = srv.submit(q)
            assert srv.wait(t)[0] == 0
            srv.release(t)
        tb = srv.submit(big)
        deadline = time.time() + 10
        while srv.stats().running == 0 and time.time() < deadline:
            time.sleep(0.0002)
        time.sleep(0.002)                      # the large batch is on the GPU
        ts = srv.submit(small)
        rc_s, rs = srv.wait(ts)
        rc_b, rb = srv.wait(tb)
        assert rc_s == 0 and rc_b == 0 and rs.status == 0 and rb.status == 0
        assert rs.t_submit_ns > rb.t_start_ns          # submitted while the batch ran
        assert rs.t_done_ns < rb.t_done_ns, (rs.t_done_ns, rb.t_done_ns)
        for q, res in ((small, rs), (big, rb)):
            want_e, _ = pa.generate(q)
            assert torch.equal(pa.Server.edges_view(res, q.id_bits), want_e)
            want_rp, want_col = pa.build_csr(q, want_e)
            rp, col = pa.Server.csr_view(res, q.n, q.id_bits)
            assert torch.equal(rp, want_rp) and torch.equal(col, want_col)
            del want_e, want_rp, want_col
        srv.release(ts)
        srv.release(tb)
        _drain(srv)
        assert srv.stats().bytes_in_use == 0
