"""The router on one GPU: two servers on device 0 stand in for two GPUs (each
has its own control thread, pool and launches; nothing waits across them).
Every result must equal the same request generated alone, tickets must name
the server that holds them, and placement must use both servers."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests(pa, count, rng):
    out = []
    for i in range(count):
        d = int(rng.integers(1, 33))
        n = max(d + 1, int(round(10 ** rng.uniform(2, 5.5))))
        model = pa.PA_MODEL_BA if i % 5 == 0 else pa.PA_MODEL_COPY
        mode = pa.PA_SEED_STAR_REF if model else int(rng.integers(0, 2))
        out.append(pa.make_params(n, d, float(rng.uniform(0.1, 0.9)), seed=7000 + i,
                                  id_bits=32 if i % 3 else 64, seed_mode=mode, model=model))
    return out


def test_router_results_equal_alone_and_use_both_servers(pa, cuda_ok):
    rng = np.random.default_rng(4)
    reqs = _requests(pa, 40, rng)
    with pa.Router([0, 0], budget_bytes=4 << 30) as r:
        assert len(r) == 2
        tickets = [r.submit(q) for q in reqs]
        assert {r.server_of(t) for t in tickets} == {0, 1}
        for t, q in zip(tickets, reqs):
            rc, res = r.wait(t, 60_000_000_000)
            assert rc == 0 and res.status == 0
            assert r.device_of(t) == 0
            want, _ = pa.generate(q)
            assert torch.equal(pa.Server.edges_view(res, q.id_bits), want)
        st = r.stats()
        assert st.completed == 40 and st.failed == 0
        assert r.stats(0).completed + r.stats(1).completed == 40
        for t in tickets:
            assert r.release(t) == 0
        assert r.release(tickets[0]) == pa.PA_ERR_NOT_FOUND


def test_router_balances_by_budget_share(pa, cuda_ok):
    """Equal requests submitted at once alternate between equal servers."""
    with pa.Router([0, 0], budget_bytes=2 << 30) as r:
        q = pa.make_params(200_000, 8, 0.5, seed=1)
        tickets = [r.submit(q) for _ in range(10)]
        assert [r.server_of(t) for t in tickets] == [0, 1] * 5
        for t in tickets:
            rc, res = r.wait(t, 60_000_000_000)
            assert rc == 0 and res.status == 0
            r.release(t)


def test_router_csr_outputs(pa, cuda_ok):
    with pa.Router([0, 0], outputs=pa.PA_OUT_CSR) as r:
        q = pa.make_params(50_000, 4, 0.5, seed=3)
        t = r.submit(q)
        rc, res = r.wait(t, 60_000_000_000)
        assert rc == 0 and res.status == 0 and not res.edges
        rowptr, col = pa.Server.csr_view(res, q.n, q.id_bits)
        E, _ = pa.generate(q)
        want_rp, want_col = pa.build_csr(q, E)
        assert torch.equal(rowptr, want_rp) and torch.equal(col, want_col)
        r.release(t)


def test_router_forgets_expired_results(pa, cuda_ok):
    """A result dropped by its server's TTL stops counting against that server:
    after the expiry the next equal request goes back to server 0."""
    import time
    with pa.Router([0, 0], budget_bytes=1 << 30, ttl_ns=50_000_000) as r:
        q = pa.make_params(50_000, 4, 0.5, seed=11)
        t0 = r.submit(q)
        assert r.server_of(t0) == 0
        rc, _ = r.wait(t0, 60_000_000_000)
        assert rc == 0
        t1 = r.submit(q)                       # server 0 still holds t0's bytes
        assert r.server_of(t1) == 1
        assert r.wait(t1, 60_000_000_000)[0] == 0
        assert r.release(t1) == 0
        time.sleep(0.3)                        # past the TTL: t0 expires unreleased
        assert r.poll(t0)[0] == pa.PA_ERR_NOT_FOUND
        t2 = r.submit(q)
        assert r.server_of(t2) == 0
        assert r.wait(t2, 60_000_000_000)[0] == 0
        r.release(t2)
