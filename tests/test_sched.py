"""Admission queue of the request server (pa_sched_*): host logic, no GPU.

The policy: arrival order; a request that fits the free budget is admitted, one
that does not is passed over unless it has waited aging_ns, which stops the
scan.  A Python restatement of that rule is checked against the library on
random traces."""
import numpy as np
import pytest

OK, INVALID, CAPACITY, BUSY, NOT_FOUND = 0, 1, 5, 7, 8


def test_fifo_skip_ahead_and_release(pa):
    q = pa.Sched(100, aging_ns=1000)
    assert q.submit(1, 60, 0) == OK
    assert q.submit(2, 50, 0) == OK
    assert q.submit(3, 30, 0) == OK
    assert q.admit(10) == [1, 3]          # 2 does not fit behind 1; 3 does
    assert (q.in_use, q.queued) == (90, 1)
    assert q.release(1) == OK
    assert q.admit(20) == [2]
    assert q.in_use == 80


def test_aged_request_blocks_the_scan(pa):
    q = pa.Sched(100, aging_ns=50)
    q.submit(1, 80, 0)
    q.submit(2, 60, 0)                     # will not fit while 1 runs
    q.submit(3, 10, 0)
    assert q.admit(10) == [1, 3]           # 2 young: passed over
    q.submit(4, 10, 20)
    assert q.admit(100) == []              # 2 has aged: 4 waits behind it
    q.release(1)
    assert q.admit(101) == [2, 4]


def test_errors(pa):
    q = pa.Sched(100, aging_ns=0, max_queue=2)
    assert q.submit(1, 101, 0) == CAPACITY
    assert q.submit(1, 10, 0) == OK
    assert q.submit(1, 10, 0) == INVALID   # ticket already queued
    assert q.submit(2, 10, 0) == OK
    assert q.submit(3, 10, 0) == BUSY      # queue full
    assert q.release(9) == NOT_FOUND
    assert q.release(2, 5) == INVALID      # partial release of a queued request
    assert q.release(2) == OK              # withdrawn
    assert q.queued == 1
    assert q.admit(0) == [1]
    assert q.submit(1, 10, 0) == INVALID   # ticket held
    assert q.release(1, 4) == OK           # part of it (e.g. scratch) comes back
    assert q.in_use == 6
    assert q.release(1, 100) == OK         # more than held: all that is left
    assert q.in_use == 0
    assert q.release(1) == OK
    assert q.release(1) == NOT_FOUND


def _model(budget, aging, ops):
    queue, held, used, out = [], {}, 0, []
    for op in ops:
        if op[0] == "submit":
            _, t, b, now = op
            if b > budget:
                out.append(CAPACITY)
                continue
            queue.append((t, b, now))
            out.append(OK)
        elif op[0] == "admit":
            _, now, cap = op
            got, keep, stopped = [], [], False
            for t, b, ts in queue:
                if stopped or len(got) >= cap:
                    keep.append((t, b, ts))
                elif b <= budget - used:
                    used += b
                    held[t] = b
                    got.append(t)
                else:
                    stopped = now - ts >= aging
                    keep.append((t, b, ts))
            queue = keep
            out.append(got)
        else:
            _, t = op
            used -= held.pop(t)
            out.append(OK)
    return out, used


@pytest.mark.parametrize("seed", range(6))
def test_matches_policy_model(pa, seed):
    rng = np.random.default_rng(seed)
    budget, aging = 1000, 40
    q = pa.Sched(budget, aging_ns=aging)
    ops, now, next_t, admitted = [], 0, 1, []
    for _ in range(400):
        now += int(rng.integers(0, 10))
        r = rng.random()
        if r < 0.5:
            ops.append(("submit", next_t, int(rng.integers(1, 1200)), now))
            next_t += 1
        elif r < 0.8 or not admitted:
            ops.append(("admit", now, int(rng.integers(1, 6))))
            res, _ = _model(budget, aging, ops)
            admitted.extend(res[-1])
        else:
            ops.append(("release", admitted.pop(int(rng.integers(0, len(admitted))))))
    want, used = _model(budget, aging, ops)
    got = []
    for op in ops:
        if op[0] == "submit":
            got.append(q.submit(op[1], op[2], op[3]))
        elif op[0] == "admit":
            got.append(q.admit(op[1], op[2]))
        else:
            got.append(q.release(op[1]))
    assert got == want
    assert q.in_use == used


def test_lanes_admit_separately(pa):
    q = pa.Sched(100, aging_ns=50)
    assert q.submit(1, 70, 0, lane=0) == OK
    assert q.submit(2, 10, 0, lane=1) == OK
    assert q.submit(3, 60, 0, lane=0) == OK
    assert q.admit(1, lanes=1 << 1) == [2]          # lane 1 only
    assert q.admit(2, lanes=1 << 0) == [1]          # 3 does not fit
    assert q.submit(4, 10, 60, lane=1) == OK
    assert q.submit(5, 10, 60, lane=0) == OK
    # 3 has aged in lane 0: 5 waits behind it, but lane 1's 4 is not held back
    assert q.admit(100) == [4]
    q.release(1)
    assert q.admit(101) == [3, 5]


def _lane_model(budget, aging, ops):
    queue, held, used, out = [], {}, 0, []
    for op in ops:
        if op[0] == "submit":
            _, t, b, now, lane = op
            if b > budget:
                out.append(CAPACITY)
                continue
            queue.append((t, b, now, lane))
            out.append(OK)
        elif op[0] == "admit":
            _, now, cap, mask = op
            got, keep, open_ = [], [], mask
            for t, b, ts, lane in queue:
                if len(got) >= cap or not (open_ >> lane) & 1:
                    keep.append((t, b, ts, lane))
                elif b <= budget - used:
                    used += b
                    held[t] = b
                    got.append(t)
                else:
                    if now - ts >= aging:
                        open_ &= ~(1 << lane)
                    keep.append((t, b, ts, lane))
            queue = keep
            out.append(got)
        else:
            _, t = op
            used -= held.pop(t)
            out.append(OK)
    return out, used


@pytest.mark.parametrize("seed", range(6))
def test_lanes_match_policy_model(pa, seed):
    """The lane rule restated in Python, on random traces over three lanes."""
    rng = np.random.default_rng(100 + seed)
    budget, aging = 1000, 40
    q = pa.Sched(budget, aging_ns=aging)
    ops, now, next_t, admitted = [], 0, 1, []
    for _ in range(400):
        now += int(rng.integers(0, 10))
        r = rng.random()
        if r < 0.5:
            ops.append(("submit", next_t, int(rng.integers(1, 1200)), now, int(rng.integers(0, 3))))
            next_t += 1
        elif r < 0.8 or not admitted:
            ops.append(("admit", now, int(rng.integers(1, 6)), int(rng.integers(1, 8))))
            res, _ = _lane_model(budget, aging, ops)
            admitted.extend(res[-1])
        else:
            ops.append(("release", admitted.pop(int(rng.integers(0, len(admitted))))))
    want, used = _lane_model(budget, aging, ops)
    got = []
    for op in ops:
        if op[0] == "submit":
            got.append(q.submit(op[1], op[2], op[3], lane=op[4]))
        elif op[0] == "admit":
            got.append(q.admit(op[1], op[2], lanes=op[3]))
        else:
            got.append(q.release(op[1]))
    assert got == want
    assert q.in_use == used
