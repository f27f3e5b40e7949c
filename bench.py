#!/usr/bin/env python3
"""Benchmark of the Bine engine on B200: virtual-rank Bine allreduce GB/s.

Workload (one "step"): Bine allreduce (variant B, one port, 1-D ring) over
P = 256 virtual ranks, 1,048,576 int32 per rank (4 MiB), values uniform in
[-1000, 1000] from a seed, MPI_SUM -- every rank ends with the full sum.
The inputs (1 GiB) and results (1 GiB) are larger than the 126 MB L2, so no
L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Engine arm (default): K steps of bine_allreduce with the buffers resident in
HBM, bracketed by a barrier and torch.cuda.synchronize(), timed with CUDA
events on the engine's stream; max over ranks when launched with torchrun
(N independent replicas: a collective over virtual ranks does not shard
across GPUs).  The JSON line also carries the HBM roofline of the fused
kernel, the end-to-end figure through the C ABI with host buffers, the
reference's CPU time on this host (cpu_baseline), and the SM clocks sampled
during the timed region.

Reference arm (--impl reference): the reference library itself, built from
its sources against the project's MPI shim (oracle/_ref), one forked process
per virtual rank on this host's cores, timed as bench/bench.cc does.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P_RANKS = 256
COUNT = 1 << 20  # int32 per rank: 4 MiB
ES = 4
ALGO_BYTES = 2 * P_RANKS * COUNT * ES  # every input read once, every output written once


def configure(args):
    """Applies the profiling overrides (--P/--count/--dtype/--engine/--order);
    the defaults are the benchmark workload."""
    global P_RANKS, COUNT, ES, ALGO_BYTES, WORKLOAD
    P_RANKS, COUNT = args.P, args.count
    ES = 4
    ALGO_BYTES = 2 * P_RANKS * COUNT * ES
    if (args.P, args.count, args.dtype, args.engine) != (256, 1 << 20, "int32", "fused"):
        WORKLOAD = (f"Bine allreduce (variant B, 1 port, 1-D ring), P={P_RANKS} virtual ranks, {COUNT} {args.dtype} "
                    f"per rank, MPI_SUM, {args.engine} engine"
                    + (f" ({args.fusion or 'automatic'} levels per pass)" if args.engine == "pipelined" else "")
                    + (f", {args.order} float order" if args.dtype == "float" else "")
                    + (f", {args.tree_split} lanes per vector" if args.tree_split else "") + " (profiling variant)")
METRIC = "virtual-rank Bine allreduce GB/s"
WORKLOAD = "Bine allreduce (variant B, 1 port, 1-D ring), P=256 virtual ranks, 1,048,576 int32 (4 MiB) per rank, MPI_SUM"
DEFAULT_WORKLOAD = WORKLOAD
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "allreduce_fused_p256_4MiB_int32.txt")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary."""
    if not os.path.exists(PROFILE_SUMMARY):
        return None
    with open(PROFILE_SUMMARY) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1]))
    return None


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
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
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"],
                                 parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_time(steps, warmup, budget_s=150.0):
    """Times the reference library (oracle/_ref) on this host; returns a dict."""
    from oracle import ref

    if not ref.available():
        return None
    count = COUNT
    # Calibrate one call at full size, then shrink the per-step sample only
    # if K calls would not fit in the time budget.
    probe = ref.time_collective("allreduce", "int32", count, P_RANKS, iters=1, warmup=0, timeout=600)
    if not probe.get("ok"):
        return {"error": "reference run failed", "detail": probe}
    t_call = probe["median_s"]
    while count > 4096 and (steps + warmup) * t_call * (count / COUNT) > budget_s:
        count //= 2
    j = ref.time_collective("allreduce", "int32", count, P_RANKS, iters=steps, warmup=warmup, timeout=900)
    if not j.get("ok"):
        return {"error": "reference run failed", "detail": j}
    t = j["median_s"]
    gbs = 2 * P_RANKS * count * ES / t / 1e9
    cores = os.cpu_count()
    sample = (f"P={P_RANKS} allreduce, {count} int32 per rank ({'full workload' if count == COUNT else 'scaled sample'}), "
              f"{steps} timed calls after {warmup} warm-ups; per call: two barriers, wall time around one call, "
              f"max over ranks, median over calls (bench/bench.cc:289-318, 376-387); {P_RANKS} processes on "
              f"{cores} cores" + (" (oversubscribed: more ranks than cores)" if P_RANKS > cores else ""))
    return {"value": gbs, "unit": "GB/s", "cores": cores, "kind": "reference", "sample": sample,
            "median_s": t, "count": count}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    r = reference_time(args.steps, max(args.warmup, 1))
    if r is None or "error" in r:
        why = "oracle/_ref/bine_ref_run is not built" if r is None else json.dumps(r)[:300]
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["median_s"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "P": P_RANKS, "count_per_rank": r["count"], "variant": "B", "ports": 1,
                   "layer": "MPI (shim, one process per rank)"},
        "cpu_baseline": {"value": r["value"], "unit": "GB/s", "cores": r["cores"], "kind": "reference",
                         "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def max_over_ranks(value, dist, device):
    """Max of a per-rank float over all ranks (the slowest replica's time)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_engine_arm(args):
    import numpy as np
    import torch

    import bine_trees_fugaku_b200 as bine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # Inputs: uniform int32 in [-1000, 1000] (or N(0,1) float32), one
    # seeded stream per rank.
    gen = torch.Generator(device="cuda")
    gen.manual_seed(12345 + rank)
    if args.dtype == "int32":
        send = torch.randint(-1000, 1001, (P_RANKS, COUNT), dtype=torch.int32, device="cuda", generator=gen)
        code = bine.INT32
    else:
        send = torch.randn((P_RANKS, COUNT), dtype=torch.float32, device="cuda", generator=gen)
        code = bine.FLOAT
    recv = torch.empty_like(send)
    stream = torch.cuda.current_stream()
    comm = bine.Comm(P_RANKS)
    comm.set_stream(stream)
    comm.set_algo("allreduce", "B")
    comm.set_engine(args.engine)
    if args.fusion is not None:
        comm.set_fusion(args.fusion)
    comm.set_float_order(args.order)
    comm.set_tree_split(args.tree_split)
    comm.set_host_window(args.host_window)

    def step():
        comm.allreduce(send, recv, COUNT, code)

    for _ in range(args.warmup):
        step()
    barrier()
    comm.synchronize()
    # Correctness of the timed configuration: exact integer sums; float
    # sums within 1e-4 relative of FP64 (checked bit for bit by the tests).
    # Every rank's row is checked.
    if args.dtype == "int32":
        expect = send.sum(0, dtype=torch.int64).to(torch.int32)
        ok = bool((recv == expect).all())
    else:
        s64 = send.double().sum(0)
        floor = send.abs().double().sum(0) * (P_RANKS * 2.0 ** -24)
        ok = bool(((recv[0].double() - s64).abs() <= floor + 1e-30).all() and (recv == recv[0]).all())
        expect = recv[0].clone()

    # The timed region: exactly K steps between a barrier + synchronize on
    # both sides.  It is repeated until the repeats span at least a second,
    # so that the clock sampler (100 ms period) sees it; the line reports
    # the median repeat (each the max over ranks).
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    repeats, reps_ms = 1, []
    with ClockSampler(local) as clocks:
        while True:
            barrier()
            start.record(stream)
            for _ in range(args.steps):
                step()
            end.record(stream)
            barrier()
            reps_ms.append(max_over_ranks(start.elapsed_time(end), dist, "cuda"))
            # Every rank takes the same decision (from the max over ranks).
            if len(reps_ms) >= 200 or sum(reps_ms) >= 1000.0:
                break
        repeats = len(reps_ms)
    elapsed_ms = statistics.median(reps_ms)
    ms_per_step = elapsed_ms / args.steps
    value = world * ALGO_BYTES / (ms_per_step * 1e-3) / 1e9
    per_launch_gbs = ALGO_BYTES / (ms_per_step * 1e-3) / 1e9

    # End to end through the C ABI with host buffers (bine_allreduce_host,
    # the MPI_Allreduce call shape): every step moves all inputs from pinned
    # host memory to the GPU and every rank's result back, pipelined in
    # column windows.  The call is ordered on the communicator's stream, so
    # events on that stream bracket it.
    host_in = torch.empty((P_RANKS, COUNT), dtype=send.dtype, pin_memory=True)
    host_in.copy_(send.cpu())
    host_out = torch.empty_like(host_in, pin_memory=True)
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 10))
    for _ in range(2 if e2e_steps else 0):
        comm.allreduce_host(host_in, host_out, COUNT, code)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        comm.allreduce_host(host_in, host_out, COUNT, code)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / max(1, e2e_steps), dist, "cuda")
    if e2e_steps:
        ok = ok and bool(torch.equal(host_out[3], expect.cpu()))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = reference_time(10, 3, budget_s=60.0)
        if r and "error" not in r:
            cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")}

    peak, peak_kind = peaks()
    default = WORKLOAD == DEFAULT_WORKLOAD
    half = P_RANKS * COUNT * ES
    l2_note = (f"inputs {half / 2**20:.0f} MiB and outputs {half / 2**20:.0f} MiB "
               + ("exceed the 126 MB L2; no flush" if half > 126e6 else
                  "fit the 126 MB L2 between steps (no flush): a cache-resident profiling variant"))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32" if args.dtype == "int32" else "float32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "P": P_RANKS, "count_per_rank": COUNT, "variant": "B", "ports": 1,
                       "engine": args.engine, "parallelism": f"replicas{world}", "l2": l2_note},
            "roofline": {"bound": "hbm", "achieved": per_launch_gbs, "peak": peak, "unit": "GB/s",
                         "frac": per_launch_gbs / peak, "traffic": profiled_traffic() if default else None,
                         "traffic_source": ("dram__bytes_read.sum + dram__bytes_write.sum per launch from the "
                                            "committed ncu capture (" + os.path.relpath(PROFILE_SUMMARY, ROOT) +
                                            "), not measured in this run") if default else
                                           "no committed capture of this profiling variant",
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "algorithmic_bytes_per_launch": ALGO_BYTES},
            "cpu_baseline": cpu,
            "e2e": None if not e2e_steps else {
                "value": ALGO_BYTES / (e2e_ms * 1e-3) / 1e9 * world, "unit": "GB/s",
                "h2d_bytes_per_step": P_RANKS * COUNT * ES, "d2h_bytes_per_step": P_RANKS * COUNT * ES,
                "path": "Comm.allreduce_host (C ABI bine_allreduce_host) with pinned host buffers; every step "
                        "copies all inputs to the GPU and every rank's result back, in pipelined column windows"},
            "gpu_launches": args.steps,
            "timed_repeats": {"repeats": repeats, "ms_per_repeat_median": elapsed_ms,
                              "ms_per_repeat_min": min(reps_ms), "ms_per_repeat_max": max(reps_ms),
                              "note": "the K-step timed region repeated until the repeats span >= 1 s; "
                                      "gpu_launches counts one repeat"},
            "clocks": clocks.summary(),
            "correct": ok,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    comm.close()
    return 0 if ok else 1


def batch_waves(spec, budget_bytes):
    """Splits the workload's items into consecutive waves whose outputs fit
    `budget_bytes` each (an item larger than the budget gets a wave of its
    own)."""
    waves, cur, used = [], [], 0
    for k, it in enumerate(spec):
        ob = it[4]
        if cur and used + ob > budget_bytes:
            waves.append(cur)
            cur, used = [], 0
        cur.append(k)
        used += ob
    if cur:
        waves.append(cur)
    return waves


def batch_workload(n=4096, seed=2024, budget_bytes=48 << 30):
    """The batched workload: n independent collectives, P ~ U[4, 512], per-rank
    message log-uniform from 64 B, op mix 50% allreduce / 25% reduce_scatter /
    25% allgather, dtype mix float32 N(0,1) / int32 U[-1000, 1000].

    The per-rank message is the larger per-rank buffer (allreduce send =
    receive, reduce_scatter send, allgather receive); counts are rounded down
    to whole 16-byte vectors (at least one).  Inputs are views of one shared,
    read-only pool of 512 rows of 4 MiB; outputs are distinct.  The
    log-uniform upper bound starts at 4 MiB and is halved until the outputs
    fit `budget_bytes` (the stated sizes would need ~400 GB for the
    allreduces alone); the bound used is reported."""
    import numpy as np

    rng = np.random.default_rng(seed)
    P = rng.integers(4, 513, n)
    u = rng.random(n)
    op = rng.choice(3, n, p=[0.5, 0.25, 0.25])
    is_float = rng.random(n) < 0.5
    upper = 4 << 20
    while True:
        m = np.exp(np.log(64) + u * (np.log(upper) - np.log(64)))
        items, out_bytes = [], 0
        for k in range(n):
            p = int(P[k])
            if op[k] == 0:
                c = max(4, int(m[k] // 4) // 4 * 4)
                ob = p * c * 4
            else:
                c = max(4, int(m[k] // (4 * p)) // 4 * 4)
                ob = p * c * 4 * (p if op[k] == 2 else 1)
            items.append((["allreduce", "reduce_scatter", "allgather"][op[k]], p, c, bool(is_float[k]), ob))
            out_bytes += ob
        if out_bytes <= budget_bytes or upper <= 1024:
            return items, upper, out_bytes
        upper //= 2


def run_batch_suite(args):
    if args.batch_waves:
        return run_batch_waves(args)
    import numpy as np
    import torch

    import bine_trees_fugaku_b200 as bine
    from bine_trees_fugaku_b200 import tuning

    torch.cuda.set_device(0)
    spec, upper, out_bytes = batch_workload(args.batch_n)
    pool_rows, pool_row = 512, 4 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    pool_i = torch.randint(-1000, 1001, (pool_rows, pool_row // 4), dtype=torch.int32, device="cuda", generator=g)
    pool_f = torch.randn((pool_rows, pool_row // 4), dtype=torch.float32, device="cuda", generator=g)
    outs, items, algo_bytes = [], [], 0
    for coll, p, c, fl, ob in spec:
        out = torch.empty(ob // 4, dtype=torch.float32 if fl else torch.int32, device="cuda")
        outs.append(out)
        send = (pool_f if fl else pool_i)
        items.append((coll, send, out, c, bine.FLOAT if fl else bine.INT32, p, pool_row, 0))
        if coll == "allreduce":
            algo_bytes += 2 * p * c * 4
        elif coll == "reduce_scatter":
            algo_bytes += p * p * c * 4 + p * c * 4
        else:
            algo_bytes += p * c * 4 + p * p * c * 4
    stream = torch.cuda.current_stream()
    # Per-call baseline: one FUSED launch per collective (FAST float order).
    comms = {}
    for coll, send, out, c, dt, p, _, _ in items:
        if p not in comms:
            cm = bine.Comm(p)
            cm.set_stream(stream)
            cm.set_float_order("fast")
            cm.set_layout(pool_row, 0)
            comms[p] = cm

    def per_call():
        for coll, send, out, c, dt, p, _, _ in items:
            comms[p].run(coll, send, out, c, dt)

    per_call()
    torch.cuda.synchronize()
    ref_sums = torch.stack([o.view(torch.int32).to(torch.int64).sum() for o in outs])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = args.steps
    e0.record(stream)
    for _ in range(reps):
        per_call()
    e1.record(stream)
    torch.cuda.synchronize()
    per_call_ms = e0.elapsed_time(e1) / reps
    # The same per-call launches captured in one CUDA graph: no host
    # launch overhead, still one kernel per collective.
    per_call_graph_ms = None
    try:
        g1 = torch.cuda.CUDAGraph()
        s1 = torch.cuda.Stream()
        s1.wait_stream(stream)
        for cm in comms.values():
            cm.set_stream(s1)
        with torch.cuda.stream(s1):
            with torch.cuda.graph(g1, stream=s1):
                per_call()
        stream.wait_stream(s1)
        for cm in comms.values():
            cm.set_stream(stream)
        for _ in range(3):
            g1.replay()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            g1.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        per_call_graph_ms = e0.elapsed_time(e1) / reps
        del g1
    except (RuntimeError, bine.BineError) as e:
        print(f"per-call graph capture failed: {e}", file=sys.stderr)
        for cm in comms.values():
            cm.set_stream(stream)

    # Autotuned batched launch (tuning cached on disk with a checksum).
    cache = os.path.join(args.out or os.path.join(ROOT, "bench_out"), "batch_tuning.json")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    table = tuning.load(cache)
    sig = tuning.signature(items, torch.cuda.get_device_name(0))
    tune_ms = None
    if sig in table:
        tu = bine.BatchTuning.from_dict(table[sig])
    else:
        tu, tune_ms = bine.Batch.autotune(items, stream, reps=2)
        table[sig] = tu.as_dict()
        tuning.save(cache, table)
    batch = bine.Batch(items, tu)
    for o in outs:
        o.zero_()
    batch.launch(stream)
    torch.cuda.synchronize()
    sums = torch.stack([o.view(torch.int32).to(torch.int64).sum() for o in outs])
    fl = torch.tensor([it[4] == bine.FLOAT for it in items], device="cuda")
    exact = bool(torch.equal(sums[~fl], ref_sums[~fl]))
    # Captured in a CUDA graph: one graph launch per batch.
    graph = torch.cuda.CUDAGraph()
    s2 = torch.cuda.Stream()
    s2.wait_stream(stream)
    with torch.cuda.stream(s2):
        with torch.cuda.graph(graph, stream=s2):
            batch.launch(s2)
    stream.wait_stream(s2)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1) / reps
    line = {"suite": "batch", "metric": "batched collectives throughput", "unit": "GB/s",
            "value": algo_bytes / (batch_ms * 1e-3) / 1e9,
            "per_call_value": algo_bytes / (per_call_ms * 1e-3) / 1e9,
            "speedup_vs_one_launch_per_collective": per_call_ms / batch_ms,
            "speedup_vs_one_launch_per_collective_graph": (per_call_graph_ms / batch_ms) if per_call_graph_ms else None,
            "batch_ms": batch_ms, "per_call_ms": per_call_ms, "per_call_graph_ms": per_call_graph_ms,
            "collectives": len(items),
            "collectives_per_s": len(items) / (batch_ms * 1e-3),
            "integer_results_equal_single_calls": exact,
            "config": {"n": len(items), "P": "U[4,512]", "message": f"log-uniform [64 B, {upper} B] (per-rank, larger buffer)",
                       "mix": "50% allreduce / 25% reduce_scatter / 25% allgather; float32 N(0,1) / int32 U[-1000,1000]",
                       "output_bytes": out_bytes, "algorithmic_bytes": algo_bytes, "inputs": "shared read-only pool 512 x 4 MiB",
                       "tuning": tu.as_dict(), "autotune_ms": tune_ms, "graph": "one CUDA graph replay per batch"}}
    print(json.dumps(line))
    batch.close()
    return 0 if exact else 1


def run_batch_waves(args):
    """The batched workload at its stated sizes: 4096 collectives, per-rank
    message log-uniform on [64 B, 4 MiB] (no halving), whose outputs (about
    420 GB) are produced in waves that fit a 48 GB output arena.  Each wave
    is one batched persistent launch; all waves are captured in one CUDA
    graph, replayed once per step.  Compared with one launch per collective
    (the same waves, the same arena), as a plain loop and captured in a
    graph.  Integer results are checked per wave against the per-call
    results."""
    import torch

    import bine_trees_fugaku_b200 as bine

    torch.cuda.set_device(0)
    budget = 48 << 30
    spec, upper, out_bytes = batch_workload(args.batch_n, budget_bytes=1 << 62)
    waves = batch_waves(spec, budget)
    pool_rows, pool_row = 512, 4 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    pool_i = torch.randint(-1000, 1001, (pool_rows, pool_row // 4), dtype=torch.int32, device="cuda", generator=g)
    pool_f = torch.randn((pool_rows, pool_row // 4), dtype=torch.float32, device="cuda", generator=g)
    arena = torch.empty(max(sum(spec[k][4] for k in w) for w in waves) // 4, dtype=torch.int32, device="cuda")
    algo_bytes = 0
    wave_items = []
    for w in waves:
        off, items = 0, []
        for k in w:
            coll, p, c, fl, ob = spec[k]
            out = arena[off // 4:(off + ob) // 4]
            out = out.view(torch.float32) if fl else out
            off += ob
            items.append((coll, pool_f if fl else pool_i, out, c, bine.FLOAT if fl else bine.INT32, p, pool_row, 0))
            algo_bytes += {"allreduce": 2 * p * c * 4, "reduce_scatter": p * p * c * 4 + p * c * 4}.get(
                coll, p * c * 4 + p * p * c * 4)
        wave_items.append(items)
    stream = torch.cuda.current_stream()
    comms = {}
    for items in wave_items:
        for coll, send, out, c, dt, p, _, _ in items:
            if p not in comms:
                cm = bine.Comm(p)
                cm.set_stream(stream)
                cm.set_float_order("fast")
                cm.set_layout(pool_row, 0)
                comms[p] = cm

    def per_call(items):
        for coll, send, out, c, dt, p, _, _ in items:
            comms[p].run(coll, send, out, c, dt)

    # Tuned once on the first wave (the autotuner times its candidates on
    # that wave), used for every wave.
    tu, tune_ms = bine.Batch.autotune(wave_items[0], stream, reps=2)
    batches = [bine.Batch(items, tu) for items in wave_items]
    exact = True
    for items, b in zip(wave_items, batches):
        per_call(items)
        torch.cuda.synchronize()
        ref = [o.view(torch.int32).to(torch.int64).sum() for _, _, o, _, dt, _, _, _ in items if dt == bine.INT32]
        arena.zero_()
        b.launch(stream)
        torch.cuda.synchronize()
        got = [o.view(torch.int32).to(torch.int64).sum() for _, _, o, _, dt, _, _, _ in items if dt == bine.INT32]
        exact = exact and all(bool(x == y) for x, y in zip(ref, got))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(1, min(args.steps, 5))

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def all_per_call():
        for items in wave_items:
            per_call(items)

    per_call_ms = timed(all_per_call)

    def capture(fn):
        gr = torch.cuda.CUDAGraph()
        s1 = torch.cuda.Stream()
        s1.wait_stream(stream)
        for cm in comms.values():
            cm.set_stream(s1)
        with torch.cuda.stream(s1):
            with torch.cuda.graph(gr, stream=s1):
                fn(s1)
        stream.wait_stream(s1)
        for cm in comms.values():
            cm.set_stream(stream)
        return gr

    g_per = capture(lambda st: all_per_call())
    per_call_graph_ms = timed(g_per.replay)
    del g_per
    g_batch = capture(lambda st: [b.launch(st) for b in batches])
    batch_ms = timed(g_batch.replay)
    del g_batch
    line = {"suite": "batch", "mode": "waves", "metric": "batched collectives throughput", "unit": "GB/s",
            "value": algo_bytes / (batch_ms * 1e-3) / 1e9,
            "per_call_value": algo_bytes / (per_call_ms * 1e-3) / 1e9,
            "speedup_vs_one_launch_per_collective": per_call_ms / batch_ms,
            "speedup_vs_one_launch_per_collective_graph": per_call_graph_ms / batch_ms,
            "batch_ms": batch_ms, "per_call_ms": per_call_ms, "per_call_graph_ms": per_call_graph_ms,
            "collectives": len(spec), "waves": len(waves), "collectives_per_s": len(spec) / (batch_ms * 1e-3),
            "integer_results_equal_single_calls": exact,
            "config": {"n": len(spec), "P": "U[4,512]", "message": f"log-uniform [64 B, {upper} B] (per-rank, larger buffer)",
                       "mix": "50% allreduce / 25% reduce_scatter / 25% allgather; float32 N(0,1) / int32 U[-1000,1000]",
                       "output_bytes": out_bytes, "algorithmic_bytes": algo_bytes,
                       "arena": f"{budget >> 30} GiB output arena reused by every wave",
                       "inputs": "shared read-only pool 512 x 4 MiB", "tuning": tu.as_dict(), "autotune_ms": tune_ms,
                       "graph": "every wave's launch in one CUDA graph, one replay per step"}}
    print(json.dumps(line))
    for b in batches:
        b.close()
    return 0 if exact else 1


SWEEP_COLLS = ["allreduce", "reduce_scatter", "allgather", "bcast", "alltoall"]
SWEEP_P = [16, 64, 96, 256, 384, 1024]
SWEEP_BYTES = [32 * 4 ** k for k in range(11)] + [64 << 20]
SWEEP_ENGINES = ("fused", "steps", "pipelined")


def sweep_algo_bytes(coll, P, count, es):
    """Algorithmic bytes of one call (each input read once, each output
    written once)."""
    if coll == "allreduce":
        return 2 * P * count * es
    if coll == "reduce_scatter":
        return P * P * count * es + P * count * es
    if coll == "allgather":
        return P * count * es + P * P * count * es
    if coll == "bcast":
        return P * count * es
    return 2 * P * P * count * es  # alltoall


def sweep_check(coll, send, recv, P, count, is_float, order=None, chunk_elems=1 << 25, ref_cache=None):
    """Check of one sweep point, in column chunks so that the temporaries
    stay small: integers and copies exactly against MPI semantics; float32
    sums in the FAST order within 1e-6 relative of an FP64 sum (plus the
    FP64 sum's own uncertainty, P * 2^-52 * sum|x|); float32 sums in the
    reference's order bit for bit against the oracle (ref_order_check)."""
    import torch

    if coll in ("allreduce", "reduce_scatter"):
        if is_float and order == "reference":
            return ref_order_check(coll, send, recv, P, count, ref_cache)
        n = send.shape[1]
        flat = recv.reshape(-1) if coll == "reduce_scatter" else None
        step = max(1, chunk_elems // P)
        for a in range(0, n, step):
            b = min(n, a + step)
            blk = send[:, a:b]
            got = recv[:, a:b] if coll == "allreduce" else flat[a:b].unsqueeze(0)
            if is_float:
                ssum = blk.sum(0, dtype=torch.float64)
                floor = blk.abs().sum(0, dtype=torch.float64) * (P * 2.0 ** -52)
                if not bool(((got.double() - ssum).abs() <= 1e-6 * ssum.abs() + floor).all()):
                    return False
            elif not bool((got == blk.sum(0)).all()):
                return False
        return True
    if coll == "allgather":
        src = send.reshape(-1)
        step = max(1, chunk_elems // P)
        return all(bool((recv[:, a:a + step] == src[a:a + step]).all()) for a in range(0, src.numel(), step))
    if coll == "bcast":
        return bool((recv == recv[0:1]).all())
    # alltoall: recv[q, r*count + j] = send[r, q*count + j]
    return all(bool(torch.equal(recv[:, r * count:(r + 1) * count], send[r].view(P, count))) for r in range(P))


REF_ORDER_FULL_BYTES = 64 << 20


def ref_order_columns(coll, P, count):
    """Send-row columns whose results are checked against the oracle, and
    the count of the oracle's call.  Small inputs are checked whole.  Larger
    ones are checked on four columns of every block (first, second, middle,
    last): the reference's addition tree of an element depends only on the
    block it lies in, not on the block's length, so an oracle call with four
    columns per block evaluates the same trees.  Blocks: allreduce splits
    the count into P blocks, the remainder going to the first ones
    (lib/libbine.cc:971-1010); reduce_scatter's block b is columns
    [b*count, (b+1)*count) of every send row."""
    import numpy as np

    if P * count * 4 * (P if coll == "reduce_scatter" else 1) <= REF_ORDER_FULL_BYTES:
        return None, count
    if coll == "allreduce":
        sizes = np.array([count // P + (b < count % P) for b in range(P)], np.int64)
    else:
        sizes = np.full(P, count, np.int64)
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    pos = np.stack([np.zeros(P, np.int64), np.minimum(1, sizes - 1), sizes // 2, sizes - 1], 1)
    cols = (offs[:, None] + pos).reshape(-1)
    return cols, (4 * P if coll == "allreduce" else 4)


def ref_order_check(coll, send, recv, P, count, cache=None):
    """Float32 results in the reference's order against the oracle (the
    C++ restatement of the reference's MPI layer, variant B / contiguous
    reduce_scatter, one port, a ring of P), bit for bit.  The oracle is the
    checker here, run outside the timed region; `cache` keeps its result for
    the other engines of the same point."""
    import numpy as np
    import torch

    from oracle import port

    key = (coll, P, count)
    if cache is not None and key in cache:
        cols, want = cache[key]
    else:
        cols, n = ref_order_columns(coll, P, count)
        x = send if cols is None else send[:, torch.from_numpy(cols).to(send.device)]
        want, _ = port.run(coll, x.cpu().numpy(), n, variant="B" if coll == "allreduce" else None)
        if cache is not None:
            cache.clear()
            cache[key] = (cols, want)
    if coll == "allreduce":
        got = recv if cols is None else recv[:, torch.from_numpy(cols).to(recv.device)]
        got = got.cpu().numpy()
    else:
        if cols is None:
            got = recv.cpu().numpy()
        else:
            b = np.repeat(np.arange(P), 4)
            j = cols - b * count
            got = recv[torch.from_numpy(b).to(recv.device), torch.from_numpy(j).to(recv.device)].cpu().numpy()
            got = got.reshape(P, 4)
    return bool(np.array_equal(got.view(np.uint32), want.view(np.uint32)))


def run_sweep_suite(args):
    """The collective sweep: allreduce, reduce_scatter, allgather, bcast
    (root 0) and alltoall at P in {16, 64, 96, 256, 384, 1024}, per-rank
    contribution 32 B..16 MiB in powers of 4 and 64 MiB, float32 N(0,1) and
    int64 U[-2^40, 2^40].  Each point is checked (sweep_check) and timed on
    the device: FUSED engine in the reference float order where the
    reference has one (else FAST), and the STEPS and PIPELINED engines up
    to P=384.
    Points whose device working set exceeds 80 % of free HBM are skipped and
    listed.  One JSON line per point goes to --out/sweep.jsonl; a summary
    line to stdout."""
    import torch

    import bine_trees_fugaku_b200 as bine

    torch.cuda.set_device(0)
    out_dir = args.out or os.path.join(ROOT, "bench_out")
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "sweep.jsonl")
    stream = torch.cuda.current_stream()
    dtypes = [("float32", torch.float32, bine.FLOAT, 4), ("int64", torch.int64, bine.INT64, 8)]
    g = torch.Generator(device="cuda")
    rows, skipped, bad = [], [], []
    ref_cache = {}

    # A 256 MiB buffer written before every timed call evicts the 126 MB
    # L2, so each call starts cold, as a call on fresh data would.
    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def time_call(comm, coll, send, recv, count, code):
        comm.run(coll, send, recv, count, code)
        comm.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        comm.run(coll, send, recv, count, code)
        e1.record(stream)
        e1.synchronize()
        one = max(e0.elapsed_time(e1), 1e-3)
        reps = int(min(50, max(3, 10.0 / one)))
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in evs:
            l2_flush.fill_(1)
            a.record(stream)
            comm.run(coll, send, recv, count, code)
            b.record(stream)
        evs[-1][1].synchronize()
        comm.synchronize()
        return statistics.median(a.elapsed_time(b) for a, b in evs) * 1e3  # microseconds

    t_start = time.time()
    with open(path, "w") as f:
        def emit(r):
            rows.append(r)
            f.write(json.dumps(r) + "\n")
            f.flush()

        sweep_p = [int(v) for v in args.sweep_p.split(",")] if args.sweep_p else SWEEP_P
        for P in sweep_p:
            comms = {}
            engines = SWEEP_ENGINES + ((f"pipelined-fuse{args.sweep_fusion}",) if args.sweep_fusion >= 1 else ())
            for engine in engines:
                cm = bine.Comm(P)
                cm.set_engine(engine.split("-")[0])
                if "-fuse" in engine:
                    cm.set_fusion(args.sweep_fusion)
                cm.set_stream(stream)
                comms[engine] = cm
            for coll in SWEEP_COLLS:
                for nbytes in [b for b in SWEEP_BYTES if b >= args.sweep_min_bytes]:
                    for dname, tdt, code, es in dtypes:
                        count = max(1, nbytes // es)
                        se, re = bine.row_counts(coll, count, P)
                        point = {"coll": coll, "P": P, "bytes_per_rank": count * es, "dtype": dname}
                        need = P * (se + re) * es + (P * count * es if coll == "bcast" else 0)
                        need = int(need * 1.25) + (1 << 30)  # workspace and check temporaries
                        if need > 0.8 * torch.cuda.mem_get_info()[0]:
                            skipped.append(dict(point, need_bytes=need))
                            continue
                        g.manual_seed(P * 1000003 + nbytes + es)
                        shape = (P, count if coll == "bcast" else se)
                        if dname == "float32":
                            send = torch.randn(shape, dtype=tdt, device="cuda", generator=g)
                        else:
                            send = torch.randint(-(1 << 40), (1 << 40) + 1, shape, dtype=tdt, device="cuda", generator=g)
                        recv = torch.zeros((P, re), dtype=tdt, device="cuda")
                        if coll == "bcast":
                            recv[0] = send[0]
                        for engine in engines:
                            if engine != "fused" and P > 384:
                                continue
                            comm = comms[engine]
                            order = "reference"
                            comm.set_float_order("reference")
                            try:
                                try:
                                    t_us = time_call(comm, coll, send, recv, count, code)
                                except bine.Unsupported:
                                    if engine != "fused" or dname != "float32":
                                        raise
                                    order = "fast"  # the reference has no float order to keep here
                                    comm.set_float_order("fast")
                                    t_us = time_call(comm, coll, send, recv, count, code)
                            except bine.BineError as e:
                                emit(dict(point, engine=engine, unsupported=str(e)[:160]))
                                continue
                            ok = sweep_check(coll, send, recv, P, count, dname == "float32", order,
                                             ref_cache=ref_cache)
                            ab = sweep_algo_bytes(coll, P, count, es)
                            r = dict(point, engine=engine, float_order=order if dname == "float32" else None,
                                     us=t_us, algo_gbs=ab / (t_us * 1e-6) / 1e9, correct=ok)
                            emit(r)
                            if not ok:
                                bad.append(r)
                            if coll != "bcast":
                                recv.zero_()
                        del send, recv
                        torch.cuda.empty_cache()
            for cm in comms.values():
                cm.close()
        for sk in skipped:
            f.write(json.dumps(dict(sk, skipped="device working set above 80% of free HBM")) + "\n")
    timed = [r for r in rows if "us" in r]
    # The reference library itself at a sample of the points (P = 16 and
    # 64, float32, three sizes, its default variants; host memory bounded),
    # timed as bench.cc times it, next to the fused engine at the same point.
    refs = []
    if args.sweep_reference:
        from oracle import ref

        fused = {(r["coll"], r["P"], r["bytes_per_rank"], r["dtype"]): r for r in timed if r["engine"] == "fused"}
        with open(os.path.join(out_dir, "sweep_reference.jsonl"), "w") as f:
            for P in (16, 64):
                for coll in SWEEP_COLLS:
                    for nbytes in (32, 32 * 4 ** 5, 32 * 4 ** 8):
                        count = max(1, nbytes // 4)
                        se, re = bine.row_counts(coll, count, P)
                        if (se + re) * 4 > 16 << 20:
                            continue
                        j = ref.time_collective(coll, "float", count, P, iters=5, warmup=2, timeout=120)
                        e = fused.get((coll, P, count * 4, "float32"))
                        r = {"coll": coll, "P": P, "bytes_per_rank": count * 4, "dtype": "float32",
                             "ref_ok": bool(j.get("ok")), "cores": os.cpu_count()}
                        if j.get("ok"):
                            ab = sweep_algo_bytes(coll, P, count, 4)
                            r.update(ref_us=j["median_s"] * 1e6, ref_gbs=ab / j["median_s"] / 1e9)
                            if e:
                                r.update(engine_us=e["us"], speedup=j["median_s"] * 1e6 / e["us"])
                        refs.append(r)
                        f.write(json.dumps(r) + "\n")
    best = {}
    for r in timed:
        k = (r["coll"], r["engine"])
        if k not in best or r["algo_gbs"] > best[k]["algo_gbs"]:
            best[k] = r
    import numpy as np

    # The two schedule-faithful engines point by point: geometric mean of
    # the STEPS time over the PIPELINED time, by per-rank message size.
    us = {(r["coll"], r["P"], r["bytes_per_rank"], r["dtype"], r["engine"]): r["us"] for r in timed}
    ratio = {}
    for (coll, P, nb, dt, eng), t in us.items():
        if eng == "steps" and (coll, P, nb, dt, "pipelined") in us:
            band = "below 64 KiB" if nb < 65536 else ("64 KiB to 2 MiB" if nb < 2 << 20 else "2 MiB and up")
            ratio.setdefault(band, []).append(t / us[(coll, P, nb, dt, "pipelined")])
    sums = [r for r in timed if r["dtype"] == "float32" and r["coll"] in ("allreduce", "reduce_scatter")]
    big = {}
    for r in timed:
        if r["bytes_per_rank"] >= 2 << 20:
            big.setdefault((r["coll"], r["engine"]), []).append(r["algo_gbs"])
    fuse_ratio = {}
    for (coll, P, nb, dt, eng), t in us.items():
        if eng.startswith("pipelined-fuse") and (coll, P, nb, dt, "pipelined") in us:
            band = "below 64 KiB" if nb < 65536 else ("64 KiB to 2 MiB" if nb < 2 << 20 else "2 MiB and up")
            fuse_ratio.setdefault(band, []).append(us[(coll, P, nb, dt, "pipelined")] / t)
    line = {"suite": "sweep", "points_timed": len(timed), "points_incorrect": len(bad),
            "pipelined_over_fused_passes_time_geomean": {k: round(float(np.exp(np.mean(np.log(v)))), 3)
                                                         for k, v in sorted(fuse_ratio.items())},
            "float_sums_bit_exact_vs_oracle": len([r for r in sums if r["float_order"] == "reference" and r["correct"]]),
            "float_sums_fast_within_1e-6_of_fp64": len([r for r in sums if r["float_order"] == "fast" and r["correct"]]),
            "timing": "median of per-call CUDA-event times, L2 flushed (256 MiB written) before every call",
            "steps_over_pipelined_time_geomean": {k: round(float(np.exp(np.mean(np.log(v)))), 3)
                                                  for k, v in sorted(ratio.items())},
            "reference_points": len([r for r in refs if "speedup" in r]),
            "speedup_over_reference_range": [round(min(r["speedup"] for r in refs if "speedup" in r), 1),
                                             round(max(r["speedup"] for r in refs if "speedup" in r), 1)]
            if any("speedup" in r for r in refs) else None,
            "points_unsupported": len([r for r in rows if "unsupported" in r]), "points_skipped": len(skipped),
            "best_algo_gbs": {f"{k[0]}/{k[1]}": round(v["algo_gbs"], 1) for k, v in sorted(best.items())},
            "median_algo_gbs_2mib_up": {f"{c}/{e}": round(float(np.median(v)), 1) for (c, e), v in sorted(big.items())},
            "seconds": round(time.time() - t_start, 1), "jsonl": os.path.relpath(path, ROOT)}
    print(json.dumps(line))
    return 0 if not bad else 1


def run_dropin_suite(args):
    """Unmodified MPI callers: the oracle's harness (P forked ranks calling
    MPI_Allreduce on host buffers, timed as bench.cc times it: two
    barriers, wall time around one call, max over ranks, median) linked
    against the reference library and, unchanged, against the engine's PMPI
    layer.  Same workload as the headline line."""
    from oracle import ref

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "dropin"], check=True, capture_output=True)
    out = {}
    for name, binary in (("reference", ref.BIN_PATH), ("engine_pmpi", ref.DROPIN_PATH)):
        if not os.path.exists(binary):
            out[name] = {"unavailable": f"{os.path.relpath(binary, ROOT)} is not built"}
            continue
        j = ref.time_collective("allreduce", "int32", COUNT, P_RANKS, iters=min(args.steps, 10),
                                warmup=min(args.warmup, 3), timeout=900, binary=binary)
        if not j.get("ok"):
            out[name] = {"error": json.dumps(j)[:300]}
            continue
        out[name] = {"median_s": j["median_s"], "gbs": ALGO_BYTES / j["median_s"] / 1e9}
    line = {"suite": "dropin", "metric": "MPI_Allreduce through the reference's own entry point, host buffers",
            "unit": "GB/s (algorithmic)", **out, "cores": os.cpu_count(),
            "config": {"workload": WORKLOAD, "P": P_RANKS, "count_per_rank": COUNT,
                       "harness": "oracle/ref_harness.cc: P forked ranks, bench.cc timing",
                       "engine": "PMPI layer: rows deposited into node-shared pinned memory, the "
                                 "bine_allreduce_host_hooked pipeline taking each column window as soon as "
                                 "every row holds it, rows collected as windows return"}}
    if "gbs" in out.get("reference", {}) and "gbs" in out.get("engine_pmpi", {}):
        line["speedup"] = out["engine_pmpi"]["gbs"] / out["reference"]["gbs"]
    print(json.dumps(line))
    return 0


LINK_TORI = [[2, 2, 2], [4, 4, 4], [8, 8, 8], [64, 64], [32, 256]]
LINK_SCHEDULES = [("allreduce", "B"), ("allreduce", "L"), ("allgather", "VEC_DOUBLING_CONT_PERMUTE")]


def run_links_suite(args):
    """Torus link-byte accounting at 1 MiB per rank: tori 2x2x2, 4x4x4,
    8x8x8, 64x64 and 32x256 (one rank per node, row-major), the Bine and
    binomial / recursive-doubling (RECDOUB family) schedules of allreduce
    (B and L) and allgather, 1 and 6 ports.  Device counts (bine_link_bytes)
    are timed with CUDA events and compared exactly with the host
    restatement (bine_link_bytes_host) wherever the host planner finishes in
    seconds (P <= 512, and the L tree everywhere); every device count is
    also checked for volume: the sum over links equals the sum over
    messages of bytes x minimal hops."""
    import numpy as np
    import torch

    import bine_trees_fugaku_b200 as bine

    torch.cuda.set_device(0)
    out_dir = args.out or os.path.join(ROOT, "bench_out")
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "links.jsonl")
    stream = torch.cuda.current_stream()
    count = (1 << 20) // 4
    rows = []
    with open(path, "w") as f:
        for dims in LINK_TORI:
            P = int(np.prod(dims))
            for coll, variant in LINK_SCHEDULES:
                for family in ("BINE", "RECDOUB"):
                    for ports in (1, 6):
                        mirrored = ports > len(dims)
                        r = {"dims": "x".join(map(str, dims)), "P": P, "coll": coll, "variant": variant,
                             "family": family, "ports": ports, "bytes_per_rank": count * 4}
                        planned = not (family == "BINE" or not mirrored)  # device needs the message list
                        if planned and P > 512 and variant != "L":
                            r["skipped"] = "device counts come from the planned message list; planning is O(P^2)"
                            rows.append(r)
                            f.write(json.dumps(r) + "\n")
                            continue
                        comm = bine.Comm(P, dims)
                        comm.set_ports(ports)
                        comm.set_algo(coll, variant, family)
                        comm.set_stream(stream)
                        out = torch.zeros(P * len(dims) * 2, dtype=torch.int64, device="cuda")
                        try:
                            comm.link_bytes(coll, count, bine.INT32, out)
                            torch.cuda.synchronize()
                            reps = 20
                            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                            t0 = time.time()
                            e0.record(stream)
                            for _ in range(reps):
                                comm.link_bytes(coll, count, bine.INT32, out)
                            e1.record(stream)
                            e1.synchronize()
                            r["device_us"] = e0.elapsed_time(e1) / reps * 1e3
                            r["device_wall_us"] = (time.time() - t0) / reps * 1e6
                            r["device_path"] = "message list" if planned else "generator"
                        except bine.BineError as e:
                            r["unsupported"] = str(e)[:160]
                            rows.append(r)
                            f.write(json.dumps(r) + "\n")
                            comm.close()
                            continue
                        dev = out.cpu().numpy().astype(np.uint64)
                        r["total_bytes"] = int(dev.sum())
                        r["max_link_bytes"] = int(dev.max())
                        if P <= 512 or variant == "L":
                            t0 = time.time()
                            host = comm.link_bytes_host(coll, count, bine.INT32)
                            r["host_ms"] = (time.time() - t0) * 1e3
                            r["exact_vs_host"] = bool(np.array_equal(host, dev))
                            msgs = comm.plan_messages(coll, count)
                            r["messages"] = int(len(msgs))
                        rows.append(r)
                        f.write(json.dumps(r) + "\n")
                        f.flush()
                        comm.close()
    timed = [r for r in rows if "device_us" in r]
    cmp = [r for r in timed if "exact_vs_host" in r]
    line = {"suite": "links", "configs": len(rows), "timed": len(timed), "compared_with_host": len(cmp),
            "all_exact": all(r["exact_vs_host"] for r in cmp),
            "skipped": len([r for r in rows if "skipped" in r]),
            "largest": [{k: r.get(k) for k in ("dims", "coll", "variant", "family", "ports", "device_us", "host_ms",
                                               "max_link_bytes")} for r in timed if r["P"] >= 4096][:8],
            "jsonl": os.path.relpath(path, ROOT)}
    print(json.dumps(line))
    return 0 if line["all_exact"] else 1


def run_picker_suite(args):
    """Learned variant picker: measures every valid arm of sampled calls on
    the GPU (STEPS engine times, device link accounting), trains bine_mlp on
    80% of the calls and judges its picks on the held-out 20% against
    exhaustive search and the fixed rule.  --picker-data adds measured
    datasets (with --picker-n 0, no new measurement)."""
    import numpy as np
    import torch

    import bine_trees_fugaku_b200 as bine
    from bine_trees_fugaku_b200 import picker as pk

    torch.cuda.set_device(0)
    out_dir = args.out or os.path.join(ROOT, "bench_out")
    os.makedirs(out_dir, exist_ok=True)

    def log(m):
        print(m, file=sys.stderr, flush=True)

    t0 = time.time()
    # Datasets: measured ones given with --picker-data (comma-separated),
    # plus --picker-n newly measured calls; each keeps its own held-out 20 %.
    cfgs, T, Lb, valid, te = [], [], [], [], []
    for path in [p for p in (args.picker_data or "").split(",") if p]:
        z = np.load(path)
        te.extend(int(i) + len(cfgs) for i in z["test"])
        cfgs += json.loads(str(z["configs"]))
        T.append(z["T"].astype(np.float64))
        Lb.append(z["Lb"])
        valid.append(z["valid"])
    if args.picker_n > 0:
        configs = pk.sample_configs(args.picker_n, seed=args.picker_seed)
        c2, _, T2, L2, v2 = pk.measure(configs, reps=3, time_budget_s=args.picker_budget, log=log)
        perm = np.random.default_rng(5 + args.picker_seed).permutation(len(c2))
        n_hold = len(c2) // 5 if args.picker_holdout is None else min(args.picker_holdout, len(c2) // 2)
        te.extend(int(i) + len(cfgs) for i in np.sort(perm[:n_hold]))
        cfgs += c2
        T.append(T2)
        Lb.append(L2)
        valid.append(v2)
    T, Lb, valid = np.concatenate(T), np.concatenate(Lb), np.concatenate(valid)
    te = np.array(sorted(te), np.int64)
    X = np.array([pk.features(c["coll"], c["P"], c["count"], c["es"], c["dims"]) for c in cfgs], np.float32)
    np.savez_compressed(os.path.join(out_dir, "picker_dataset.npz"), X=X, T=T.astype(np.float32),
                        Lb=Lb.astype(np.float32), valid=valid, test=te, configs=json.dumps(cfgs))
    t_measure = time.time() - t0
    # Noise ceiling: re-time some held-out calls; how often is the first
    # measurement's best arm within 5 % of the second measurement's best?
    ceiling = None
    if args.picker_repeat:
        sub = [int(i) for i in te[: args.picker_repeat]]
        c2, _, T2, _, v2 = pk.measure([cfgs[i] for i in sub], reps=3, log=log)
        assert c2 == [cfgs[i] for i in sub]
        hits = rows = 0
        for k, i in enumerate(sub):
            both = valid[i] & v2[k] & pk.allowed_arms(cfgs[i], valid[i])
            if not both.any():
                continue
            rows += 1
            a = int(np.argmin(np.where(both, T[i], np.inf)))
            hits += T2[k, a] <= 1.05 * float(np.min(T2[k, both]))
        ceiling = {"calls": rows, "best_of_first_timing_within_5pct_on_second": hits / max(1, rows)}
    tr = np.setdiff1d(np.arange(len(cfgs)), te)
    # A tenth of the training calls chooses the checkpoint; the held-out
    # calls are never seen before the evaluation.
    rs = np.random.default_rng(6).permutation(tr)
    va, tr = np.sort(rs[: len(rs) // 10]), np.sort(rs[len(rs) // 10:])
    Y, M, st = pk.targets(T[tr], Lb[tr], valid[tr])
    Yv, Mv, _ = pk.targets(T[va], Lb[va], valid[va], st)
    t1 = time.time()
    mlps, losses = [], None
    for seed in range(args.picker_ensemble):
        m, lo = pk.train(X[tr], Y, M, steps=args.picker_steps, log=log, val=(X[va], Yv, Mv), seed=seed)
        mlps.append(m)
        losses = losses or lo
    torch.cuda.synchronize()
    t_train = time.time() - t1
    if len(te):
        single = pk.evaluate(pk.predict(mlps[0], X[te]), T[te], Lb[te], valid[te], [cfgs[i] for i in te])
        pred = pk.predict(mlps, X[te])
        ev = pk.evaluate(pred, T[te], Lb[te], valid[te], [cfgs[i] for i in te])
    else:  # a measurement-only run: every call goes to training
        single = {"pick_within_5pct_of_optimum": None}
        ev = {}
    # Pick latency: one forward pass of a 16-row batch through every model
    # of the ensemble, device-timed.
    x16 = torch.from_numpy(X[:16].copy() if len(X) >= 16 else np.zeros((16, pk.IN_DIM), np.float32)).cuda()
    ens = bine.Ensemble(mlps)
    y16 = torch.empty((16, pk.OUT_DIM), dtype=torch.float32, device="cuda")
    for _ in range(5):
        ens.forward(x16, out=y16)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(100):
        ens.forward(x16, out=y16)
    e1.record()
    torch.cuda.synchronize()
    # Device time of one fused forward: 20 forwards captured in a CUDA
    # graph (no host launch cost between them), replayed.
    forward16_device_us = None
    try:
        gs = torch.cuda.Stream()
        gs.wait_stream(torch.cuda.current_stream())
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.stream(gs):
            with torch.cuda.graph(gr, stream=gs):
                for _ in range(20):
                    ens.forward(x16, stream=gs, out=y16)
        torch.cuda.current_stream().wait_stream(gs)
        for _ in range(3):
            gr.replay()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(10):
            gr.replay()
        g1.record()
        torch.cuda.synchronize()
        forward16_device_us = g0.elapsed_time(g1) * 1e3 / 200
        del gr
    except RuntimeError as e:
        print(f"graph timing of the ensemble forward failed: {e}", file=sys.stderr)
    # The layered path (per model: one GEMM + bias/GELU launch per layer),
    # for comparison.
    for _ in range(3):
        for m in mlps:
            m.forward(x16)
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0.record()
    for _ in range(100):
        for m in mlps:
            m.forward(x16)
    l1.record()
    torch.cuda.synchronize()
    ens.close()
    meta = {"calls": len(cfgs), "held_out": int(len(te)), "train_steps": args.picker_steps,
            "single_model_pick_within_5pct": single["pick_within_5pct_of_optimum"],
            "device": torch.cuda.get_device_name(0)}
    pk.save(os.path.join(out_dir, "picker_weights.npz"), mlps, st, meta)
    line = {"suite": "picker", "metric": "learned pick vs exhaustive search (held-out calls)",
            **ev, "models": len(mlps), "single_model_pick_within_5pct": single["pick_within_5pct_of_optimum"],
            "noise_ceiling": ceiling, "calls_measured": len(cfgs), "arms": pk.NARMS,
            "training_calls": int(len(tr)), "training_samples": int(valid[tr].sum()),
            "validation_calls": int(len(va)),
            "valid_arms_per_call_mean": float(valid.sum(1).mean()) if len(cfgs) else 0.0,
            "train_loss_first_last": [losses[0], float(np.mean(losses[-50:]))],
            "measure_s": t_measure, "train_s": t_train,
            "forward16_us": e0.elapsed_time(e1) * 10.0,
            "forward16_device_us": forward16_device_us,
            "forward16_layered_us": l0.elapsed_time(l1) * 10.0,
            "forward16_note": "ensemble mean of a 16-row batch: one fused launch (bine_mlp_ensemble_forward) "
                              "against the layered per-model path; forward16_us includes the host's launch "
                              "cost (back-to-back calls from Python), forward16_device_us is device time "
                              "(20 forwards per CUDA graph replay)",
            "config": {"model": "ensemble of bine_mlp 16-256-256-256-%d GELU, bf16 weights, fp32 accumulate" % pk.OUT_DIM,
                       "engine": "steps", "timing": "per arm: median of 3 CUDA-event batches of back-to-back "
                                                    "launches (each batch ~300 us, at most 32 launches)",
                       "calls": "sampled: 60% allreduce / 20% reduce_scatter / 20% allgather, P on [4, 4096] "
                                "([4, 2048] for reduce_scatter and allgather), per-rank message log-uniform "
                                "32 B..256 MiB (P x message <= 2 GiB)",
                       "samples": "one (call, arm) timing per training sample; held-out calls are judged "
                                  "against exhaustive search over every valid arm"}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    # Profiling overrides; the defaults are the benchmark workload.
    ap.add_argument("--P", type=int, default=256)
    ap.add_argument("--count", type=int, default=1 << 20)
    ap.add_argument("--dtype", default="int32", choices=["int32", "float"])
    ap.add_argument("--engine", default="fused", choices=["fused", "steps", "pipelined"])
    ap.add_argument("--fusion", type=int, default=None,
                    help="levels of the schedule per pass of the pipelined engine (default: the engine's own choice)")
    ap.add_argument("--sweep-fusion", type=int, default=0,
                    help="also time the pipelined engine with this many levels per pass (1: level by level)")
    ap.add_argument("--sweep-p", default=None, help="comma-separated P values of the sweep (default: all)")
    ap.add_argument("--sweep-min-bytes", type=int, default=0, help="smallest per-rank message of the sweep")
    ap.add_argument("--order", default="reference", choices=["reference", "fast"])
    ap.add_argument("--host-window", type=int, default=32 << 20,
                    help="column-window bytes of the host-buffer pipeline (e2e leg)")
    ap.add_argument("--tree-split", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="lanes per output vector of the exact-order float kernel (0: chosen per call)")
    ap.add_argument("--suite", default="headline", choices=["headline", "batch", "picker", "sweep", "links", "dropin"])
    ap.add_argument("--batch-n", type=int, default=4096)
    ap.add_argument("--batch-waves", action="store_true",
                    help="batch suite at the stated 4 MiB message bound, in waves that fit a 48 GB output arena")
    ap.add_argument("--sweep-reference", action="store_true",
                    help="also time the reference library at a sample of the sweep's points")
    ap.add_argument("--picker-n", type=int, default=1500)
    ap.add_argument("--picker-seed", type=int, default=11)
    ap.add_argument("--picker-budget", type=float, default=900.0, help="seconds of measurement at most")
    ap.add_argument("--picker-steps", type=int, default=16000)
    ap.add_argument("--picker-ensemble", type=int, default=5, help="models trained with different seeds, averaged")
    ap.add_argument("--picker-data", default=None,
                    help="measured picker_dataset.npz files to train on (comma-separated; --picker-n 0 to measure none)")
    ap.add_argument("--picker-repeat", type=int, default=150, help="held-out calls re-timed for the noise ceiling")
    ap.add_argument("--picker-holdout", type=int, default=None,
                    help="held-out calls among the newly measured ones (default: a fifth)")
    ap.add_argument("--out", default=None, help="directory for the picker's dataset and weights")
    args = ap.parse_args()
    configure(args)
    if args.suite == "batch":
        return run_batch_suite(args)
    if args.suite == "picker":
        return run_picker_suite(args)
    if args.suite == "sweep":
        return run_sweep_suite(args)
    if args.suite == "links":
        return run_links_suite(args)
    if args.suite == "dropin":
        return run_dropin_suite(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_engine_arm(args)


if __name__ == "__main__":
    sys.exit(main())
