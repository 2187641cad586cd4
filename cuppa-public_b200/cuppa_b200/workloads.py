"""Synthetic workloads of the benchmark configurations (no datasets involved).

* batched_instances(): the 4,096-instance mix -- n = round(10^U(3,7)),
  d = U{1..32}, p = U(0.1, 0.9) (rounded to 1e-6), seed = 1000 + i, int32 ids,
  clique seed graph -- drawn from numpy.random.default_rng(0).  The list is
  committed as tests/golden/batched_instances.json and a test checks that this
  function reproduces it.
* serve_requests(duration_s, rate): the served stream -- Poisson arrivals
  (exponential gaps from default_rng(1)), n = round(10^U(4,8)), d = U{2..16},
  p = U(0.2, 0.8), seeds from a counter starting at 0.
"""
from __future__ import annotations

import numpy as np


def batched_instances(count: int = 4096):
    rng = np.random.default_rng(0)
    n = np.round(10 ** rng.uniform(3, 7, count)).astype(np.int64)
    d = rng.integers(1, 33, count)
    p = rng.uniform(0.1, 0.9, count)
    n = np.maximum(n, d + 1)
    return [{"n": int(a), "d": int(b), "p": round(float(c), 6), "seed": 1000 + i}
            for i, (a, b, c) in enumerate(zip(n, d, p))]


def serve_requests(duration_s: float, rate: float = 2000.0, n_max_exp: float = 8.0):
    rng = np.random.default_rng(1)
    t, out, i = 0.0, [], 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration_s:
            break
        n = int(round(10 ** rng.uniform(4, n_max_exp)))
        d = int(rng.integers(2, 17))
        p = round(float(rng.uniform(0.2, 0.8)), 6)
        out.append({"t": t, "n": max(n, d + 1), "d": d, "p": p, "seed": i})
        i += 1
    return out


def edges_of(n: int, d: int, clique: bool = True) -> int:
    seed_edges = d * (d + 1) // 2 if clique else d
    return seed_edges + (n - d - 1) * d
