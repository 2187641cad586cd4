"""Launch-shape autotuner per (n, d) bucket.

A bucket is (floor(log2 n), d, id_bits).  For a bucket the tuner times a few
launch shapes of the same graph -- the grid of the start kernel (one wave, half
a wave, two waves), the persistent kernel instead of the start kernel, and the
persistent kernel's tile passes -- with CUDA events, keeps the fastest, and
records it in a JSON table; tuned_params() applies the table's entry to a
request.  Every shape generates the same graph (the draws do not depend on the
launch), which the GPU test checks.
"""
from __future__ import annotations

import json
import math
import os

from . import PA_START_NONE, alloc_buffers, check, edge_count, generate_into, finish, make_params

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune.json")


def bucket(n: int, d: int, id_bits: int) -> str:
    return f"n2^{int(math.log2(max(n, 2)))}_d{d}_i{id_bits}"


def candidates(sms: int = 148, per_sm: int = 4):
    """Launch shapes tried for every bucket (pa_params fields; 0 = the default)."""
    wave = sms * per_sm
    return [
        {},
        {"blocks": wave // 2},
        {"blocks": wave * 2},
        {"start_nodes": PA_START_NONE},
        {"start_nodes": PA_START_NONE, "tile_passes": 1},
        {"start_nodes": PA_START_NONE, "tile_passes": 4},
    ]


def load(path: str = DEFAULT_TABLE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save(table: dict, path: str = DEFAULT_TABLE) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply(prm, shape: dict):
    for k, v in shape.items():
        setattr(prm, k, v)
    return prm


def tuned_params(n: int, d: int, p: float, seed: int = 42, id_bits: int = 32, seed_mode: int = 1,
                 table: dict | None = None):
    """make_params(...) with the bucket's tuned launch shape, if the table has one."""
    prm = make_params(n, d, p, seed=seed, id_bits=id_bits, seed_mode=seed_mode)
    t = load() if table is None else table
    entry = t.get(bucket(n, d, id_bits))
    return apply(prm, entry["shape"]) if entry else prm


def tune(n: int, d: int, p: float = 0.5, id_bits: int = 32, reps: int = 3, table: dict | None = None,
         path: str | None = DEFAULT_TABLE, stream=None):
    """Time every candidate shape on one graph of the bucket; record the best."""
    import torch
    s = stream or torch.cuda.Stream()
    props = torch.cuda.get_device_properties(0)
    times = []
    for shape in candidates(props.multi_processor_count):
        prm = apply(make_params(n, d, p, seed=1, id_bits=id_bits), shape)
        edges, scratch = alloc_buffers(prm)
        generate_into(prm, edges, scratch, s)          # warm-up
        check(finish(scratch, s).status, "autotune warm-up")
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(reps)]
        for a, b in ev:
            a.record(s)
            generate_into(prm, edges, scratch, s)
            b.record(s)
        check(finish(scratch, s).status, "autotune run")
        times.append((min(a.elapsed_time(b) for a, b in ev), shape))
        del edges, scratch
    best_ms, best = min(times, key=lambda x: x[0])
    t = (load(path) if path else {}) if table is None else table
    t[bucket(n, d, id_bits)] = {"shape": best, "ms": best_ms,
                               "edges_per_s": edge_count(make_params(n, d, p, id_bits=id_bits)) / best_ms * 1e3,
                               "tried": [{"shape": sh, "ms": ms} for ms, sh in times]}
    if path:
        save(t, path)
    return best, times


def main(argv=None):
    """python -m cuppa_b200.autotune [--out PATH] [--log2n 12 16 20 24] [--d 2 4 8 16 32]
    tunes every (2^e, d) int32 bucket and writes the table."""
    import argparse
    ap = argparse.ArgumentParser(description="launch-shape autotuner")
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--log2n", type=int, nargs="+", default=[12, 16, 20, 24])
    ap.add_argument("--d", type=int, nargs="+", default=[2, 4, 8, 16, 32])
    ap.add_argument("--id-bits", type=int, default=32)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    table = load(args.out)
    for e in args.log2n:
        for d in args.d:
            best, times = tune(2 ** e, d, 0.5, args.id_bits, reps=args.reps, table=table, path=None)
            print(bucket(2 ** e, d, args.id_bits), best, [round(t, 4) for t, _ in times], flush=True)
    save(table, args.out)


if __name__ == "__main__":
    main()
