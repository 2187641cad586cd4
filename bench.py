#!/usr/bin/env python3
"""Benchmark of the copy-model preferential-attachment generator.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3]
    python bench.py --impl reference ...

One step = one generation of the whole graph (pa_generate: the scratch clear,
the all-ones fill of the start kernel's region, the start kernel and, for
graphs beyond its 2^31-node limit, the persistent kernel) into buffers
already resident in HBM.
Metric: edges/s (whole job).  The default workload is the largest single-GPU
configuration: n = 2^30 nodes, d = 4, p = 0.5, int64 ids, (d+1)-clique seed,
Philox seed 1234 -- 4,294,967,286 edges, 68.7 GB of (src, dst) pairs.  The
output alone is ~545x the 126 MB L2, so no L2 flush is needed between steps.

Multi-GPU (torchrun, N > 1): one graph does not shard (every copy read may hit
any earlier node), so each rank generates its own full replica and `value`
counts the edges of all ranks over the slowest rank's time (weak scaling).

Besides the device-timed value the line carries:
  e2e          the same generation through the C ABI from host parameters,
               host-timed, including the device->host read of each step's
               result block (status and counters);
  roofline     algorithmic bytes of the generator kernel per launch over its
               CUDA-event duration, against the measured HBM copy bandwidth;
  cpu_baseline the sequential CPU oracle on a bounded sample (1 core);
  clocks       SM clocks and throttle reasons sampled during the timed region;
  parity       after the timed region, the device digest (pa_digest) of the
               last step's whole edge list against the oracle's digest of the
               same configuration (tests/golden/fullsize_digests.json);
  step_dram_frac  the whole step (kernel traffic from the committed ncu
               capture plus the all-ones fill) in DRAM bytes over the step
               time, against the same peak;
  batched, served  (default workload, one GPU) the batched and served figures
               of the metric: 4,096 mixed instances in one persistent launch per
               wave against one launch per graph, and Poisson request streams
               through the request server at 2,000 req/s (a 2 s window) and at
               a sustainable 100 req/s (5 s), with p50/p99 latency.

--impl reference times the reference's own sequential generator
(oracle/_ref/scm_ref, src/PA/SPA/SerialCopyModel3.cpp compiled from the
reference sources) on a bounded sample per step; where that binary is absent
it falls back to the CPU oracle restatement.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuppa-public_b200"))

CLIQUE, STAR_REF = 1, 0
COPY, BA = 0, 1
WORKLOADS = {
    "c3": dict(n=2 ** 30, d=4, p=0.5, seed=1234, id_bits=64, seed_mode=CLIQUE, fixture="c3_p0.5",
               name="copy-model PA, n=2^30, d=4, p=0.5, int64 ids, clique seed, Philox seed 1234"),
    "c3p0": dict(n=2 ** 30, d=4, p=0.0, seed=1234, id_bits=64, seed_mode=CLIQUE, fixture="c3_p0",
                 name="copy-model PA, n=2^30, d=4, p=0.0, int64 ids, clique seed, Philox seed 1234"),
    "c2": dict(n=10 ** 8, d=16, p=0.5, seed=7, id_bits=64, seed_mode=CLIQUE, fixture="c2",
               name="copy-model PA, n=10^8, d=16, p=0.5, int64 ids, clique seed, Philox seed 7"),
    "c3s": dict(n=2 ** 25, d=4, p=0.5, seed=1234, id_bits=64, seed_mode=CLIQUE, fixture="c3s",
                name="copy-model PA, n=2^25, d=4, p=0.5, int64 ids, clique seed, Philox seed 1234 "
                     "(profiling size)"),
    "c3m": dict(n=2 ** 26, d=4, p=0.5, seed=1234, id_bits=64, seed_mode=CLIQUE, fixture="c3m",
                name="copy-model PA, n=2^26, d=4, p=0.5, int64 ids, clique seed, Philox seed 1234 "
                     "(traffic capture size)"),
    "c1": dict(n=10 ** 5, d=4, p=0.5, seed=42, id_bits=32, seed_mode=CLIQUE, fixture="c1",
               name="copy-model PA, n=10^5, d=4, p=0.5, int32 ids, clique seed, Philox seed 42"),
    # the repeated-nodes Barabasi-Albert model of -A sba at the same size
    "sba": dict(n=2 ** 30, d=4, p=0.0, seed=1234, id_bits=64, seed_mode=STAR_REF, model=BA,
                fixture="sba_n2^30",
                name="repeated-nodes BA (-A sba), n=2^30, d=4, int64 ids, star seed, "
                     "Philox seed 1234",
                metric="edges/s on 1 B200 (BA PA generation)"),
}
METRIC = "edges/s on 1 B200 (copy-model PA generation)"
CPU_SAMPLE_NODES = 2 ** 24      # oracle sample: ~67M edges, a few seconds on one core
REF_SAMPLE_NODES = 2 ** 23      # reference scm sample per step: ~33.5M edges


def algorithmic_bytes_per_edge(w) -> float:
    """2s (pair write) + c*s (copy-target read), s = id bytes; c = 1-p for the
    copy model, 1/2 for BA (an even endpoint position is a target slot)."""
    s = w["id_bits"] // 8
    copy = 0.5 if w.get("model", COPY) == BA else 1.0 - w["p"]
    return 2 * s + copy * s


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(workload: str):
    """Per-launch DRAM bytes of the dominant kernel from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "kernel_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        return t.get(workload, {}).get("dram_bytes_per_launch")
    except Exception:
        return None


def load_fixture_digests(name):
    """The oracle's whole-graph digests of a configuration (committed fixture
    tests/golden/fullsize_digests.json, written by tests/golden/make_golden.py);
    None when the configuration has none."""
    path = os.path.join(ROOT, "tests", "golden", "fullsize_digests.json")
    try:
        with open(path) as f:
            cases = {c["name"]: c for c in json.load(f)["cases"]}
    except Exception:
        return None
    c = cases.get(name)
    if c is None:
        return None
    return {k: tuple(int(x, 16) for x in c[k]) for k in ("pairs", "rowptr", "col") if k in c}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while running."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest x over all ranks (every rank takes this collective step)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, steps: int, world: int, slowest_s: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / slowest_s


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def baseline_core() -> int:
    """The host core the sequential baselines are pinned to (the first one this
    process may use)."""
    try:
        return min(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return 0


def pinned(fn, *a, **kw):
    """Run fn on one core (Linux affinity of the calling thread), then restore."""
    try:
        old = os.sched_getaffinity(0)
        os.sched_setaffinity(0, {baseline_core()})
    except (AttributeError, OSError):
        return fn(*a, **kw)
    try:
        return fn(*a, **kw)
    finally:
        os.sched_setaffinity(0, old)


def pin_child():
    """preexec_fn for the reference binaries: one core."""
    try:
        os.sched_setaffinity(0, {baseline_core()})
    except (AttributeError, OSError):
        pass


def host_cores() -> int:
    return os.cpu_count() or 0


def cpu_baseline_oracle(w, nodes: int):
    """The sequential oracle, pinned to one core, on `nodes` nodes of the same
    (d, p, seed)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as orc
    n = min(nodes, w["n"])

    def run():
        t0 = time.perf_counter()
        if w.get("model", COPY) == BA:
            orc.generate_ba(n, w["d"], w["seed"])
        else:
            orc.generate(n, w["d"], w["p"], w["seed"], w["seed_mode"])
        return time.perf_counter() - t0
    what = ("Philox restatement of SerialBA.cpp" if w.get("model", COPY) == BA
            else "Philox restatement of SerialCopyModel3.cpp")
    dt = pinned(run)
    edges = orc.edge_count(n, w["d"], w["seed_mode"])
    return {"value": edges / dt, "unit": "edges/s", "cores": 1, "kind": "port",
            "host_cores": host_cores(), "pinned_core": baseline_core(),
            "sample": f"oracle ({what}), n={n}, d={w['d']}, "
                      f"p={w['p']}, {edges} edges in {dt:.2f} s, one thread on one core"}


def run_reference(args, w):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    ba = w.get("model", COPY) == BA
    ref = os.path.join(ROOT, "oracle", "_ref", "sba_ref" if ba else "scm_ref")
    n = REF_SAMPLE_NODES
    d = w["d"]
    edges = (n - d - 1) * d + d
    times = []
    if os.path.exists(ref):
        kind = "reference"
        if ba:
            sample = (f"reference -A sba (SerialBA.cpp, MT19937-64, int32 ids), n={n}, d={d}; "
                      "its own 'Computation Time' per step; single-threaded")
            cmd = [ref, str(n), str(d), "{td}", "-"]
        else:
            sample = (f"reference -A scm (SerialCopyModel3.cpp, MT19937-64, star seed, int32 ids), "
                      f"n={n}, d={d}, p={w['p']}; its own 'Computation Time' per step; "
                      "single-threaded")
            cmd = [ref, str(n), str(d), str(w["p"]), "{td}", "-"]
        with tempfile.TemporaryDirectory() as td:
            for i in range(args.warmup + args.steps):
                out = subprocess.run([td if a == "{td}" else a for a in cmd], cwd=td,
                                     preexec_fn=pin_child,
                                     capture_output=True, text=True, check=True).stdout
                t = [float(x.split(":")[1]) for x in out.splitlines()
                     if x.startswith("Computation Time")][0]
                if i >= args.warmup:
                    times.append(t)
    else:
        kind = "port"
        sample = f"oracle restatement (reference binary absent), n={n}, d={d}, p={w['p']}"
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle as orc
        edges = orc.edge_count(n, d, w["seed_mode"])
        def one():
            t0 = time.perf_counter()
            if ba:
                orc.generate_ba(n, d, w["seed"])
            else:
                orc.generate(n, d, w["p"], w["seed"], w["seed_mode"])
            return time.perf_counter() - t0
        for i in range(args.warmup + args.steps):
            dt = pinned(one)
            if i >= args.warmup:
                times.append(dt)
    total = sum(times)
    value = edges * len(times) / total
    line = {
        "impl": "reference", "metric": w.get("metric", METRIC), "value": value, "unit": "edges/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64" if w["id_bits"] == 64 else "int32",
        "data": "synthetic (generator parameters only)",
        "config": {"workload": w["name"], "sample_nodes": n},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": 1, "kind": kind,
                         "host_cores": host_cores(), "pinned_core": baseline_core(),
                         "sample": sample},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args, w):
    import torch
    import torch.distributed as dist
    import cuppa_b200 as pa

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    prm = pa.make_params(w["n"], w["d"], w["p"], seed=w["seed"], id_bits=w["id_bits"],
                         seed_mode=w["seed_mode"], tile_passes=args.tile_passes,
                         blocks=args.blocks, model=w.get("model", COPY))
    E = pa.edge_count(prm)
    edges, scratch = pa.alloc_buffers(prm)
    stream = torch.cuda.Stream()

    def step():
        pa.generate_into(prm, edges, scratch, stream)

    # warm-up (each checked)
    for _ in range(args.warmup):
        step()
        st = pa.finish(scratch, stream)
        pa.check(st.status, "warm-up generation")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-timed region: each step's phases marked by events recorded
    # on the launching stream inside pa_generate_timed
    ev = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(4))
          for _ in range(args.steps)]
    t_all0, t_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for e3 in ev:                      # create the CUDA events outside the timed region
        for x in e3:
            x.record(stream)
    barrier()
    with ClockSampler(local) as clk:
        t_all0.record(stream)
        for i in range(args.steps):
            pa.generate_timed(prm, edges, scratch, ev[i], stream)
        t_all1.record(stream)
        stream.synchronize()
    barrier()
    st = pa.finish(scratch, stream)
    pa.check(st.status, "timed generation")
    ms = max_over_ranks(t_all0.elapsed_time(t_all1), world, "cuda")
    fill_ms = [e[0].elapsed_time(e[1]) for e in ev]      # scratch clear + all-ones fill
    start_ms = [e[1].elapsed_time(e[2]) for e in ev]     # start kernel
    gen_ms = [e[2].elapsed_time(e[3]) for e in ev]       # persistent kernel
    value = job_rate(E, args.steps, world, ms / 1e3)

    # ---- end to end through the C ABI: host params -> generation -> result read
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pa.generate_into(prm, edges, scratch, stream)
        st = pa.finish(scratch, stream)          # stream sync + device->host result block
    t1 = time.perf_counter()
    pa.check(st.status, "e2e generation")
    e2e_s = max_over_ranks(t1 - t0, world, "cuda")
    e2e = {"value": job_rate(E, args.steps, world, e2e_s), "unit": "edges/s",
           "h2d_bytes_per_step": ctypes_sizeof_params(pa), "d2h_bytes_per_step": 64}
    # small graphs: the same end-to-end loop replaying a captured CUDA graph
    # (pa_plan_*), where issuing the clear, fill and launch one by one matters
    e2e_graph = None
    if E < (1 << 26):
        plan = pa.Plan(prm, edges, scratch)
        plan.launch(stream)
        pa.check(pa.finish(scratch, stream).status, "graph warm-up")
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            plan.launch(stream)
            st = pa.finish(scratch, stream)
        t1 = time.perf_counter()
        pa.check(st.status, "graph e2e generation")
        plan.close()
        g_s = max_over_ranks(t1 - t0, world, "cuda")
        e2e_graph = {"value": job_rate(E, args.steps, world, g_s), "unit": "edges/s",
                     "ms_per_step": 1e3 * g_s / args.steps,
                     "plain_ms_per_step": 1e3 * e2e_s / args.steps}

    # ---- parity of the last timed step's output (after all timing): the
    # device digest of the whole edge list against the oracle's
    want = load_fixture_digests(w.get("fixture"))
    parity = None
    if want is not None:
        got = pa.digest(edges[:E].reshape(-1), stream=stream)
        ok = got == want["pairs"]
        if world > 1:
            flag = torch.tensor([0.0 if ok else 1.0], device="cuda")
            dist.all_reduce(flag)
            ok = flag.item() == 0.0
        parity = ok
    elif world > 1:
        dist.all_reduce(torch.zeros(1, device="cuda"))     # same collective steps on every rank

    # ---- back to back into two buffers: each step's all-ones fill (pa_fill, a
    # small grid) runs on a second stream beside the previous step's generation,
    # which skips its own fill (PA_FLAG_PREFILLED).  K fills and K generations
    # lie inside the timed window; parity is checked on the last buffer.
    pipelined = None
    free_b, _ = torch.cuda.mem_get_info()
    ebytes = edges.numel() * edges.element_size()
    if world == 1 and args.pipeline and free_b > ebytes + (4 << 30):
        bufs = [edges, torch.empty_like(edges)]
        q = pa.make_params(w["n"], w["d"], w["p"], seed=w["seed"], id_bits=w["id_bits"],
                           seed_mode=w["seed_mode"], tile_passes=args.tile_passes,
                           blocks=args.blocks, model=w.get("model", COPY),
                           flags=pa.PA_FLAG_PREFILLED)
        fill_s = torch.cuda.Stream()
        ev_fill = [torch.cuda.Event(), torch.cuda.Event()]
        ev_gen = [torch.cuda.Event(), torch.cuda.Event()]

        def run_pipelined(k_steps):
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            fill_s.wait_event(a0)
            pa.fill(prm, bufs[0], fill_s)
            ev_fill[0].record(fill_s)
            for k in range(k_steps):
                b = k % 2
                stream.wait_event(ev_fill[b])
                pa.generate_into(q, bufs[b], scratch, stream)
                ev_gen[b].record(stream)
                if k + 1 < k_steps:
                    nb = (k + 1) % 2
                    if k >= 1:
                        fill_s.wait_event(ev_gen[nb])   # buffer nb's last generation is done
                    pa.fill(prm, bufs[nb], fill_s)
                    ev_fill[nb].record(fill_s)
            a1.record(stream)
            stream.synchronize()
            fill_s.synchronize()
            return a0.elapsed_time(a1)

        run_pipelined(args.warmup)
        pa.check(pa.finish(scratch, stream).status, "pipelined warm-up")
        barrier()
        with ClockSampler(local) as clk_p:
            ms_p = run_pipelined(args.steps)
        pa.check(pa.finish(scratch, stream).status, "pipelined generation")
        last = bufs[(args.steps - 1) % 2]
        p_ok = (pa.digest(last[:E].reshape(-1), stream=stream) == want["pairs"]
                if want is not None else None)
        pipelined = {"value": E * args.steps / (ms_p / 1e3), "unit": "edges/s",
                     "ms_per_step": ms_p / args.steps, "parity": p_ok, "buffers": 2,
                     "what": "graphs generated back to back into two buffers; each step's "
                             "all-ones fill (pa_fill) runs on a second stream beside the "
                             "previous step's generation (PA_FLAG_PREFILLED); K fills and K "
                             "generations inside the CUDA-event window",
                     "clocks": clk_p.summary()}
        if p_ok is False:
            parity = False
        del bufs, q
        torch.cuda.synchronize()

    if rank == 0:
        peak, peak_kind = load_peaks()
        bpe = algorithmic_bytes_per_edge(w)
        u_split = pa.start_split(prm)
        gen_edges = (w["n"] - u_split) * w["d"]            # the persistent kernel's share
        start_edges = E - gen_edges                         # the start kernel's (and the seed)
        # the dominant kernel: the one with the larger share of the step
        if statistics.mean(gen_ms) >= statistics.mean(start_ms):
            kernel, k_edges, kern_s = "gen_kernel", gen_edges, statistics.mean(gen_ms) / 1e3
        else:
            kernel, k_edges, kern_s = "start_kernel", start_edges, statistics.mean(start_ms) / 1e3
        achieved = k_edges * bpe / kern_s / 1e9
        traffic = load_traffic(args.workload)     # ncu DRAM bytes of one such launch
        launches = (1 if u_split > w["d"] + 1 else 0) + (1 if gen_edges > 0 else 0)
        line = {
            "metric": w.get("metric", METRIC), "value": value, "unit": "edges/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64" if w["id_bits"] == 64 else "int32",
            "data": "synthetic (generator parameters only; output is the graph)",
            "config": {"workload": w["name"], "edges": E,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": f"output {E * 2 * w['id_bits'] // 8 / 1e9:.1f} GB > 126 MB L2; "
                             "no flush needed"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "bytes_per_edge": bpe, "traffic": traffic,
                         # the DRAM the launch actually moves (whole 128-byte lines
                         # for random reads) over its measured time
                         "traffic_gbs": traffic / kern_s / 1e9 if traffic else None,
                         "traffic_frac": traffic / kern_s / 1e9 / peak if traffic else None,
                         "kernel": kernel, "launch_ms_mean": kern_s * 1e3,
                         "kernel_edges": k_edges},
            "phases_ms_mean": {"clear+fill (memsets)": statistics.mean(fill_ms),
                               "start_kernel": statistics.mean(start_ms),
                               "gen_kernel": statistics.mean(gen_ms),
                               "start_split_node": u_split},
            "e2e": e2e,
            "e2e_cuda_graph": e2e_graph,
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
            "device_stats": st.as_dict(),
            "parity": parity,
            "pipelined": pipelined,
            "parity_check": ("device pa_digest of the whole edge list of the last timed step "
                             "(2E ids, position-keyed) equal to the oracle's digest of the same "
                             f"configuration (tests/golden/fullsize_digests.json, '{w.get('fixture')}')"
                             if want is not None else "no whole-graph fixture for this workload"),
        }
        # the whole step in actual DRAM bytes: the kernel's ncu traffic plus the
        # all-ones fill of the start region (written once) over the step time
        fill_bytes = (u_split - (w["d"] + 1)) * w["d"] * 2 * (w["id_bits"] // 8)
        if traffic:
            step_bytes = traffic + fill_bytes
            line["step_dram_frac"] = step_bytes / (ms / args.steps / 1e3) / 1e9 / peak
            line["step_dram"] = {"bytes": step_bytes, "kernel_traffic": traffic,
                                 "fill_bytes": fill_bytes,
                                 "gbs": step_bytes / (ms / args.steps / 1e3) / 1e9,
                                 "peak": peak}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_oracle(w, CPU_SAMPLE_NODES)
    del edges, scratch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and args.workload == "c3" and not args.no_extras:
        # the batched and served figures of the metric, measured in the same run
        line["batched"] = measure_batched(args, 1, 0)[0]
        line["served"] = {
            "overload": measure_served(args, args.rate, args.serve_window, "csr", 1, 0)[0],
            "sustainable": measure_served(args, args.sustain_rate, args.sustain_seconds, "csr",
                                          1, 0)[0],
        }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if parity in (None, True) else 1


STREAM_W = dict(n=2 ** 30, d=4, p=0.5, seed=1234, id_bits=64, seed_mode=CLIQUE,
                name="copy-model PA, n=2^30, d=4, p=0.5, int64 ids, clique seed, Philox seed "
                     "1234, SLOTS layout, written as 'u v' text")
STREAM_REF_NODES = 2 ** 22      # reference sample per step: scm generation + its writer


def d2h_link_gbs(torch, nbytes=1 << 30, reps=5) -> float:
    """Plain pinned device->host copy bandwidth (the host link's roofline)."""
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    s = torch.cuda.Stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(s):
        dst.copy_(src, non_blocking=True)
        a.record(s)
        for _ in range(reps):
            dst.copy_(src, non_blocking=True)
        b.record(s)
    s.synchronize()
    return nbytes * reps / (a.elapsed_time(b) / 1e3) / 1e9


def stream_chunks(n, d, chunk_edges=1 << 24) -> int:
    """Chunks pa_stream_edges cuts rows d+1..n-1 into (whole tiles of 2048 // d rows)."""
    rows, tile_rows = n - d - 1, 2048 // d
    chunk_rows = -(-max(1, chunk_edges // d) // tile_rows) * tile_rows
    return -(-rows // min(chunk_rows, rows))


def run_stream(args):
    """Generation into the targets-only layout, then the edge list as text,
    formatted on the device and copied out in chunks to a discarding sink."""
    import ctypes
    import torch
    import cuppa_b200 as pa

    torch.cuda.set_device(0)
    w = STREAM_W
    prm = pa.make_params(w["n"], w["d"], w["p"], seed=w["seed"], id_bits=w["id_bits"],
                         seed_mode=w["seed_mode"], layout=pa.PA_LAYOUT_SLOTS)
    E = pa.edge_count(prm)
    slots, scratch = pa.alloc_buffers(prm)
    stream = torch.cuda.Stream()
    discard = pa._SINK(lambda ctx, data, nbytes: 0)
    total = ctypes.c_uint64()

    def step():
        pa.generate_into(prm, slots, scratch, stream)
        pa.check(pa.finish(scratch, stream).status, "generation")
        t0 = time.perf_counter()
        pa.check(pa.lib().pa_stream_edges(ctypes.byref(prm), ctypes.c_void_p(slots.data_ptr()),
                                          pa.PA_FORMAT_TEXT, 0,
                                          ctypes.cast(discard, ctypes.c_void_p), None,
                                          ctypes.c_void_p(stream.cuda_stream),
                                          ctypes.byref(total)), "pa_stream_edges")
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        stream_s = [step() for _ in range(args.steps)]
        t_all = time.perf_counter() - t0
    text_bytes = int(total.value)
    del slots, scratch
    torch.cuda.empty_cache()
    link = d2h_link_gbs(torch)
    # end to end: the one call a user makes (library memory, generate, write the file)
    t0 = time.perf_counter()
    st, nbytes = pa.generate_to_file(prm, "/dev/null")
    e2e_s = time.perf_counter() - t0
    pa.check(st.status, "pa_generate_to_file")
    achieved = text_bytes / statistics.mean(stream_s) / 1e9
    line = {
        "metric": "edges/s generated and written as text (copy-model PA)",
        "value": E * args.steps / t_all, "unit": "edges/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_all / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (generator parameters only; output is the graph's text)",
        "config": {"workload": w["name"], "edges": E, "text_bytes": text_bytes,
                   "sink": "discard (host memory, native callback)",
                   "timing": "host clock around generate + finish + pa_stream_edges"},
        "roofline": {"bound": "host link (D2H)", "achieved": achieved, "peak": link,
                     "unit": "GB/s", "frac": achieved / link, "peak_source": "measured in run",
                     "traffic": None, "kernel": "pa_stream_edges pipeline",
                     "stream_ms_mean": 1e3 * statistics.mean(stream_s)},
        "e2e": {"value": E / e2e_s, "unit": "edges/s", "h2d_bytes_per_step": 80,
                "d2h_bytes_per_step": nbytes,
                "call": "pa_generate_to_file(prm, '/dev/null', TEXT): alloc, generate, write, free"},
        # per step: the start kernel, then 3 formatting kernels per chunk
        "gpu_launches": (1 + 3 * stream_chunks(w["n"], w["d"])) * args.steps,
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_writer_sample(STREAM_REF_NODES, w["d"], w["p"])
    print(json.dumps(line), flush=True)
    return 0


def reference_writer_sample(n, d, p):
    """The reference's sequential path for the same job on one core: -A scm
    generation (scm_ref) plus PAHelper::writeGraphToDisk (write_ref), n nodes."""
    scm = os.path.join(ROOT, "oracle", "_ref", "scm_ref")
    wr = os.path.join(ROOT, "oracle", "_ref", "write_ref")
    if not (os.path.exists(scm) and os.path.exists(wr)):
        return None
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run([scm, str(n), str(d), str(p), td, "-"], cwd=td, preexec_fn=pin_child,
                             capture_output=True, text=True, check=True).stdout
        t_gen = [float(x.split(":")[1]) for x in out.splitlines()
                 if x.startswith("Computation Time")][0]
        out = subprocess.run([wr, str(n), str(d), str(p), "/dev/null"], preexec_fn=pin_child,
                             capture_output=True,
                             text=True, check=True).stdout
        t_wr = [float(x.split(":")[1]) for x in out.splitlines() if x.startswith("Write Time")][0]
    edges = (n - d) * d
    return {"value": edges / (t_gen + t_wr), "unit": "edges/s", "cores": 1, "kind": "reference",
            "host_cores": host_cores(), "pinned_core": baseline_core(),
            "sample": f"reference -A scm generation ({t_gen:.2f} s) + PAHelper::writeGraphToDisk "
                      f"to /dev/null ({t_wr:.2f} s), n={n}, d={d}, p={p}, int32, one thread"}


def rank_share(pa, prms, world: int, rank: int) -> list:
    """Instances this rank generates: its part of pa_batch_partition (largest
    first, each to the lightest part), the same split on every rank."""
    if world == 1:
        return list(range(len(prms)))
    part = pa.batch_partition(prms, world)
    return [i for i, p in enumerate(part) if p == rank]


def measure_batched(args, world: int, rank: int):
    """4,096 mixed instances: one persistent launch per wave vs one launch per
    graph, identical outputs checked by digest; graphs/s of both.  With N ranks
    the instances are split by pa_batch_partition and each rank runs its part
    (the total is fixed: strong scaling; no collective beyond the timing).
    Returns (figures, identical) on every rank."""
    import torch
    import torch.distributed as dist
    import cuppa_b200 as pa
    from cuppa_b200.workloads import batched_instances, edges_of

    inst = batched_instances(args.instances)

    def prm(i):
        x = inst[i]
        return pa.make_params(x["n"], x["d"], x["p"], seed=x["seed"], id_bits=32,
                              seed_mode=pa.PA_SEED_CLIQUE)

    mine = rank_share(pa, [prm(i) for i in range(len(inst))], world, rank)
    order = sorted(mine, key=lambda i: -edges_of(inst[i]["n"], inst[i]["d"]))
    budget = int(args.budget_gb * 1e9)
    waves, cur, used = [], [], 0
    for i in order:
        b = edges_of(inst[i]["n"], inst[i]["d"]) * 8 + inst[i]["n"] // 2 + 4096
        if cur and used + b > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += b
    if cur:
        waves.append(cur)

    stream = torch.cuda.Stream()
    t_batch = t_plain = dev_batch = 0.0
    digests_b, digests_p = {}, {}
    total_edges = 0
    with ClockSampler(torch.cuda.current_device()) as clk:
        for wave in waves:
            prms = [prm(i) for i in wave]
            total_edges += sum(pa.edge_count(q) for q in prms)
            # batched: one persistent launch for the wave
            batch = pa.Batch(prms)
            for _ in range(args.warmup if wave is waves[0] else 0):
                batch.generate(stream)
                pa.check(batch.finish(stream).status, "batched warm-up")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            batch.generate(stream)
            e1.record(stream)
            st = batch.finish(stream)   # waits
            t_batch += time.perf_counter() - t0
            dev_batch += e0.elapsed_time(e1) / 1e3
            pa.check(st.status, "batched generation")
            for k, i in enumerate(wave):
                digests_b[i] = pa.digest(batch.graph(k).reshape(-1), stream=stream)
            # plain: one pa_generate per graph, back to back on one stream
            scratch = torch.empty(max(pa.sizes(q)[1] for q in prms), dtype=torch.uint8,
                                  device="cuda")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k, q in enumerate(prms):
                pa.generate_into(q, batch.edges[k], scratch, stream)
            st = pa.finish(scratch, stream)
            t_plain += time.perf_counter() - t0
            pa.check(st.status, "plain generation")
            for k, i in enumerate(wave):
                digests_p[i] = pa.digest(batch.graph(k).reshape(-1), stream=stream)
            del batch, scratch
            torch.cuda.empty_cache()
    same = all(digests_b[i] == digests_p[i] for i in digests_b)
    n_graphs = len(inst)
    t_batch = max_over_ranks(t_batch, world, "cuda")
    t_plain = max_over_ranks(t_plain, world, "cuda")
    if world > 1:
        flags = torch.tensor([0.0 if same else 1.0, float(total_edges)], device="cuda")
        dist.all_reduce(flags)
        same, total_edges = flags[0].item() == 0.0, int(flags[1].item())
    fig = {
        "workload": f"{n_graphs} instances: n=round(10^U(3,7)), d=U{{1..32}}, p=U(0.1,0.9), "
                    "seed=1000+i, int32, clique seed",
        "graphs_per_s": n_graphs / t_batch, "ms": t_batch * 1e3,
        "plain_graphs_per_s": n_graphs / t_plain, "plain_ms": t_plain * 1e3,
        "speedup_vs_plain": t_plain / t_batch, "identical_outputs": same,
        "device_ms": dev_batch * 1e3,
        "edges": total_edges, "edges_per_s": total_edges / t_batch,
        "waves_rank0": len(waves), "wave_budget_gb": args.budget_gb,
        "timing": "host clock around each wave's launches and its completion wait",
        "clocks": clk.summary(),
    }
    return fig, same


def run_batched(args):
    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    fig, same = measure_batched(args, world, rank)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0 if same else 1
    line = {
        "metric": "graphs/s, batched mixed instances (one persistent launch per wave)",
        "value": fig["graphs_per_s"], "unit": "graphs/s", "n_gpus": world, "steps": 1,
        "warmup": args.warmup, "ms_per_step": fig["ms"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (generator parameters only)",
        "config": {"workload": fig["workload"], "edges": fig["edges"],
                   "waves_rank0": fig["waves_rank0"], "wave_budget_gb": args.budget_gb,
                   "parallelism": f"instances split over {world} ranks (pa_batch_partition)"
                   if world > 1 else "single"},
        "plain_graphs_per_s": fig["plain_graphs_per_s"], "plain_ms": fig["plain_ms"],
        "speedup_vs_plain": fig["speedup_vs_plain"], "identical_outputs": same,
        "edges_per_s_batched": fig["edges_per_s"],
        "clocks": fig["clocks"],
    }
    print(json.dumps(line), flush=True)
    return 0 if same else 1


def measure_served(args, rate: float, seconds: float, outputs_name: str, world: int,
                   rank: int):
    """Poisson request stream through the request server (pa_server_*): requests
    are submitted at their arrival times from one thread, results are waited
    for and released in submission order from another; latency is the server's
    own clock from submit to the control thread seeing the batch complete.
    With N ranks, rank r serves the requests whose index is r mod N (a round-robin
    router: one server per GPU, no collective on the data path); the job's value
    is all ranks' edges over the slowest rank's span, and p50/p99 are over all
    requests.  Returns (figures, all_ok) on every rank."""
    import queue
    import torch
    import torch.distributed as dist
    import cuppa_b200 as pa
    from cuppa_b200.workloads import edges_of, serve_requests

    all_reqs = serve_requests(seconds, rate)
    reqs = [r for i, r in enumerate(all_reqs) if i % world == rank]
    free_b, _ = torch.cuda.mem_get_info()
    budget = min(int(args.serve_budget_gb * 1e9), int(free_b * 0.9))
    prms = [pa.make_params(r["n"], r["d"], r["p"], seed=r["seed"], id_bits=32,
                           seed_mode=pa.PA_SEED_CLIQUE) for r in reqs]
    tickets = queue.Queue()
    lat, edges_done, statuses, small = [], 0, [], []
    express_edges = args.serve_express_edges or (1 << 22)   # the server's default
    outputs = {"pairs": pa.PA_OUT_PAIRS, "csr": pa.PA_OUT_CSR,
               "both": pa.PA_OUT_PAIRS | pa.PA_OUT_CSR}[outputs_name]
    with pa.Server(budget_bytes=budget, outputs=outputs, max_inflight=args.serve_max_inflight,
                   express_edges=args.serve_express_edges) as srv, \
            ClockSampler(torch.cuda.current_device()) as clk:
        # warm-up: a few requests, waited for and released
        for q in prms[: args.warmup]:
            t = srv.submit(q)
            srv.wait(t)
            srv.release(t)
        if world > 1:
            dist.barrier()          # every rank starts the arrival clock together
        t0 = time.perf_counter()

        def submitter():
            for r, q in zip(reqs, prms):
                delay = t0 + r["t"] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets.put((srv.submit(q), q))
            tickets.put(None)

        th = threading.Thread(target=submitter)
        th.start()
        first_submit, last_done = None, 0
        while True:
            item = tickets.get()
            if item is None:
                break
            t, q = item
            rc, res = srv.wait(t)
            statuses.append(res.status if rc == 0 else rc)
            lat.append((res.t_done_ns - res.t_submit_ns) / 1e6)
            small.append(res.n_edges <= express_edges)
            first_submit = res.t_submit_ns if first_submit is None else min(first_submit,
                                                                           res.t_submit_ns)
            last_done = max(last_done, res.t_done_ns)
            edges_done += res.n_edges
            srv.release(t)
        th.join()
        st = srv.stats().as_dict()
    span_s = (last_done - first_submit) / 1e9
    ok = all(x == 0 for x in statuses)
    n_req = len(reqs)
    if world > 1:
        span_s = max_over_ranks(span_s, world, "cuda")
        gathered = [None] * world
        dist.all_gather_object(gathered, (lat, edges_done, ok, n_req, small))
        lat = [x for g in gathered for x in g[0]]
        small = [x for g in gathered for x in g[4]]
        edges_done = sum(g[1] for g in gathered)
        ok = all(g[2] for g in gathered)
        n_req = sum(g[3] for g in gathered)
    lat_sorted = sorted(lat)

    def pct(x):
        return lat_sorted[min(len(lat_sorted) - 1, int(round(x / 100 * (len(lat_sorted) - 1))))]

    def pcts(sel):
        v = sorted(x for x, m in zip(lat, small) if m == sel)
        if not v:
            return None
        return {"requests": len(v), "p50_ms": v[len(v) // 2],
                "p99_ms": v[min(len(v) - 1, int(round(0.99 * (len(v) - 1))))]}

    offered_edges = sum(edges_of(r["n"], r["d"]) for r in all_reqs)
    fig = {
        "workload": f"Poisson {rate:g} req/s for {seconds:g} s: n=round(10^U(4,8)), d=U{{2..16}}, "
                    "p=U(0.2,0.8), int32, clique seed",
        "output": {"pairs": "edge list (PAIRS)", "csr": "undirected CSR",
                   "both": "edge list and undirected CSR"}[outputs_name]
                  + " kept on the device until released",
        "requests": n_req, "window_s": seconds, "budget_gb_per_gpu": budget / 1e9,
        "offered_requests_per_s": rate, "offered_edges_per_s": offered_edges / seconds,
        "served_requests_per_s": n_req / span_s, "edges_per_s": edges_done / span_s,
        "span_s": span_s, "p50_ms": pct(50), "p99_ms": pct(99), "max_ms": lat_sorted[-1],
        "express_sized": pcts(True), "bulk_sized": pcts(False),
        "all_ok": ok, "server_stats_rank0": st,
        "statuses_rank0": {str(c): statuses.count(c) for c in sorted(set(statuses))},
        "gpu_launches": st["batches"] * 2 + (st["completed"] * 11 if outputs & pa.PA_OUT_CSR else 0),
        "clocks": clk.summary(),
    }
    return fig, ok


def run_served(args):
    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    fig, ok = measure_served(args, args.rate, args.serve_seconds, args.serve_outputs, world, rank)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0 if ok else 1
    line = {
        "metric": "served edges/s with p50/p99 latency (continuous batching)",
        "value": fig["edges_per_s"], "unit": "edges/s", "n_gpus": world, "steps": 1,
        "warmup": args.warmup, "ms_per_step": fig["span_s"] * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (generator parameters only)",
        "config": {"workload": fig["workload"], "requests": fig["requests"],
                   "budget_gb_per_gpu": fig["budget_gb_per_gpu"],
                   "parallelism": f"requests round-robin over {world} servers (one per rank)"
                   if world > 1 else "single", "output": fig["output"]},
        "p50_ms": fig["p50_ms"], "p99_ms": fig["p99_ms"], "max_ms": fig["max_ms"],
        "express_sized": fig["express_sized"], "bulk_sized": fig["bulk_sized"],
        "requests_per_s": fig["served_requests_per_s"],
        "offered_requests_per_s": fig["offered_requests_per_s"],
        "offered_edges_per_s": fig["offered_edges_per_s"], "all_ok": ok,
        "server_stats_rank0": fig["server_stats_rank0"],
        "statuses_rank0": fig["statuses_rank0"], "gpu_launches": fig["gpu_launches"],
        "clocks": fig["clocks"],
    }
    print(json.dumps(line), flush=True)
    return 0 if ok else 1


def ctypes_sizeof_params(pa) -> int:
    import ctypes
    return ctypes.sizeof(pa.PaParams)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched", "served", "stream"],
                    default="c3")
    ap.add_argument("--tile-passes", type=int, default=0)
    ap.add_argument("--blocks", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--instances", type=int, default=4096, help="batched workload size")
    ap.add_argument("--budget-gb", type=float, default=100.0, help="batched wave budget")
    ap.add_argument("--serve-seconds", type=float, default=5.0, help="served: arrival window")
    ap.add_argument("--rate", type=float, default=2000.0, help="served: mean requests/s")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0, help="served: HBM budget")
    ap.add_argument("--serve-outputs", choices=["pairs", "csr", "both"], default="csr",
                    help="served: what each finished request keeps on the device")
    ap.add_argument("--serve-max-inflight", type=int, default=0,
                    help="served: batches per lane on the GPU at once (0 = the server's default)")
    ap.add_argument("--serve-express-edges", type=int, default=0,
                    help="served: largest request of the express lane (0 = the server's default)")
    ap.add_argument("--pipeline", action="store_true",
                    help="also measure generations back to back into two buffers, each step's "
                         "fill beside the previous step's generation")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the batched and served figures in its line")
    ap.add_argument("--serve-window", type=float, default=2.0,
                    help="default line: arrival window of the served run at --rate")
    ap.add_argument("--sustain-rate", type=float, default=100.0,
                    help="default line: a request rate the server sustains")
    ap.add_argument("--sustain-seconds", type=float, default=5.0,
                    help="default line: arrival window at --sustain-rate")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "served":
        return run_served(args)
    if args.workload == "stream":
        if args.impl == "reference":
            world, rank, _ = dist_setup()
            if rank != 0:
                return 0
            samples = [reference_writer_sample(STREAM_REF_NODES, STREAM_W["d"], STREAM_W["p"])
                       for _ in range(args.warmup + args.steps)][args.warmup:]
            if samples[0] is None:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "oracle/_ref/scm_ref or write_ref not built"}))
                return 0
            v = statistics.mean(x["value"] for x in samples)
            print(json.dumps({"impl": "reference", "metric": "edges/s generated and written as "
                              "text (copy-model PA)", "value": v, "unit": "edges/s",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "int32", "data": "synthetic",
                              "config": {"workload": STREAM_W["name"],
                                         "sample_nodes": STREAM_REF_NODES},
                              "cpu_baseline": samples[-1],
                              "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return run_stream(args)
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, w)
    return run_gpu(args, w)


if __name__ == "__main__":
    sys.exit(main())
