"""Learned variant picker for the step engine.

For each call it picks the schedule the STEPS engine runs: the Bine variant
(for allreduce the latency-optimal tree "L" against the bandwidth-optimal
reduce-scatter + allgather "B", "B_COALESCE", "B_CONT"), the port count
and the segment size (the engine's unit of work per block).  These are the
choices the reference leaves to LIBBINE_* variables and its sweep scripts.
The picker never changes a result:

* integer sums and copies are exact whatever the arm;
* a float32 sum in the reference's order is a different addition tree for
  every variant and port count (the port count splits the vector into
  different blocks, lib/libbine.cc:986-1010), so for those calls the picker
  keeps the caller's variant and port count and chooses the segment only,
  which moves the same data in different units.  Only FAST-order float
  calls on the FUSED engine, whose sums do not follow the schedule, are
  free in every knob.

* Features (one row per call): op one-hot, log2 P, log2 message bytes,
  torus shape (number of dimensions and log2 of each), dtype one-hot, and
  derived terms (bytes per block, distance from a power of two, message
  against the default segment).
* Targets per arm: log2 measured GPU time and log2 of the busiest torus
  link's bytes, both generated by this engine (bench.py --suite picker).
* Model: bine_mlp (3 x 256, GELU, bf16 weights, fp32 accumulation),
  trained on the GPU with the engine's own kernels.
* Evaluated against exhaustive search (every valid arm measured).  Fallback: the
  reference's fixed rule (fixed_rule below), used when no model is loaded
  or the model's pick is not valid for the call.
* Picker.choose applies the model's best provable arm; Picker.tune times
  the model's best few arms once per call shape and keeps the fastest.
"""
import json
import math
import os

import numpy as np

# --------------------------------------------------------------- arm space
SEGMENTS = [0, 4096, 65536]  # LIBBINE_SEGMENT_SIZE values the reference sweeps (0: engine default)
PORTS = [1, 2, 6]
ARMS = []
for v in ["L", "B", "B_COALESCE", "B_CONT"]:
    for p in PORTS:
        for s in SEGMENTS:
            ARMS.append(("allreduce", v, p, s))
for s in SEGMENTS:
    ARMS.append(("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 1, s))
for v in ["VEC_DOUBLING_CONT_PERMUTE", "VEC_DOUBLING_CONT_SEND", "VEC_DOUBLING_BLOCKS"]:
    for p in PORTS:
        for s in SEGMENTS:
            ARMS.append(("allgather", v, p, s))
# The reference's RING family (the bucket allreduce, its comparator): one
# schedule whatever the port setting.
for s in SEGMENTS:
    ARMS.append(("allreduce", "RING", 1, s))
NARMS = len(ARMS)
IN_DIM = 16
OUT_DIM = ((2 * NARMS + 15) // 16) * 16
OPS = ["allreduce", "reduce_scatter", "allgather"]
# Planning the per-block B schedules costs O(P^2 * ports) on the host, and
# the bucket ring sends P messages per step for every step of every ring
# (67 M moves at P = 4096 on one ring); arms beyond these sizes are not
# offered.
MAX_P = {"B": 128, "B_COALESCE": 256, "RING": 256}


def is_p2(x):
    return x > 0 and (x & (x - 1)) == 0


def message_bytes(coll, P, count, es):
    """Per-rank message: the larger per-rank buffer."""
    if coll == "allreduce":
        return count * es
    return count * es * P  # reduce_scatter send row / allgather receive row


FEATURE_VERSION = 2


def features(coll, P, count, es, dims=None):
    dims = list(dims or [P])
    msg = max(1, message_bytes(coll, P, count, es))
    f = np.zeros(IN_DIM, np.float32)
    f[OPS.index(coll)] = 1.0
    f[3] = math.log2(P) / 12.0
    f[4] = math.log2(msg) / 28.0
    f[5] = len(dims) / 3.0
    for i, d in enumerate(dims[:3]):
        f[6 + i] = math.log2(d) / 12.0
    f[9] = 1.0 if es == 4 else 0.0
    f[10] = 1.0 if es != 4 else 0.0
    f[11] = 1.0 if is_p2(P) else 0.0
    f[12] = math.log2(max(1, count)) / 28.0
    f[13] = math.log2(max(1.0, msg / P)) / 28.0  # bytes per block
    lp = math.log2(P)
    f[14] = lp - math.floor(lp)  # distance above the power of two below P
    f[15] = min(1.0, msg / (32.0 * 1024))  # below/above the default 32 KiB segment
    return f


def statically_valid(arm, coll, P, count, dims=None):
    """Arms the engine can plan for this call (the planner has the final
    word: cases it rejects are invalid too)."""
    c, v, ports, seg = arm
    if c != coll:
        return False
    if coll == "allreduce":
        if v in MAX_P and P > MAX_P[v]:
            return False
        if v == "B_CONT" and not is_p2(P):
            return False
        if v == "RING":
            return count >= 1
        if v != "L" and count < ports * P:
            return False
        if v == "L" and count < ports:
            return False
        return True
    if coll == "reduce_scatter":
        return is_p2(P)
    if coll == "allgather":
        if v in ("VEC_DOUBLING_CONT_PERMUTE", "VEC_DOUBLING_CONT_SEND") and not is_p2(P):
            return False
        if v == "VEC_DOUBLING_CONT_SEND" and ports != 1:
            return False
        if v == "VEC_DOUBLING_BLOCKS" and ports != 1:
            return False  # the block-by-block allgather ignores LIBBINE_NUM_PORTS
        return count >= ports
    return False


def fixed_rule(coll, P, count, es):
    """The reference's own selection, composed from its defaults and sweep
    scripts: variant B (lib/libbine.cc:56) when count >= ports*P
    (lib/libbine.cc:1036), else L; ports 1 up to 128 KiB per rank, else 6
    (bench/run_allreduce.sh:21-31); segment 0 up to 16 KiB, 4 KiB up to
    128 KiB, else 64 KiB (bench/run_allreduce.sh:3-17).  Per-block B beyond
    the planning cap becomes B_COALESCE (the same data movement, coalesced);
    reduce_scatter keeps its single variant; allgather keeps its default
    CONT_PERMUTE where it runs and the block-by-block variant elsewhere."""
    msg = message_bytes(coll, P, count, es)
    ports = 1 if msg <= 128 * 1024 else 6
    seg = 0 if msg <= 16 * 1024 else (4096 if msg <= 128 * 1024 else 65536)
    if coll == "allreduce":
        while ports > 1 and count < ports:
            ports = 2 if ports == 6 else 1
        if count >= ports * P:
            v = "B" if P <= MAX_P["B"] else "B_COALESCE"
            if v == "B_COALESCE" and P > MAX_P["B_COALESCE"]:
                v = "B_CONT" if is_p2(P) else "L"
        else:
            v = "L"
        if v == "L":
            while ports > 1 and count < ports:
                ports = 2 if ports == 6 else 1
        arm = ("allreduce", v, ports, seg)
    elif coll == "reduce_scatter":
        arm = ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 1, seg)
    else:
        v = "VEC_DOUBLING_CONT_PERMUTE" if is_p2(P) else "VEC_DOUBLING_BLOCKS"
        if v == "VEC_DOUBLING_BLOCKS":
            ports = 1
        while ports > 1 and count < ports:
            ports = 2 if ports == 6 else 1
        arm = ("allgather", v, ports, seg)
    return ARMS.index(arm)


FLOAT_CODES = (2, 3)  # BINE_FLOAT, BINE_DOUBLE
REDUCTIONS = ("allreduce", "reduce_scatter")
DEFAULT_VARIANT = {"allreduce": "B", "reduce_scatter": "VEC_HALVING_CONT_PERMUTE",
                   "allgather": "VEC_DOUBLING_CONT_PERMUTE"}


def order_bound(coll, datatype, engine="steps", float_order="reference"):
    """Whether the call's result bits depend on the variant and port count:
    float sums in the reference's order (the STEPS and PIPELINED engines
    always keep it; the FUSED engine unless set to FAST)."""
    return coll in REDUCTIONS and datatype in FLOAT_CODES and not (engine == "fused" and float_order == "fast")


def keep_of(comm, coll):
    """The caller's (variant, ports) for `coll` on `comm` ("RING" for the
    RING family, whose schedule ignores both)."""
    if comm.family.get(coll) == "RING":
        return "RING", 1
    return comm.algo.get(coll, DEFAULT_VARIANT[coll]), comm.ports


def arm_keeps(arm, keep):
    return keep is None or (arm[1], arm[2]) == tuple(keep)


def fallback_arm(config, valid=None):
    """The arm the fixed rule ends up running: its own pick, or, where the
    engine refuses that (valid[a] False), the first valid latency-optimal
    tree (allreduce) or block-by-block allgather, as Picker does without a
    model; None when nothing runs."""
    c = config
    first = fixed_rule(c["coll"], c["P"], c["count"], c["es"])
    if valid is None or valid[first]:
        return first
    for a, arm in enumerate(ARMS):
        if valid[a] and arm[0] == c["coll"] and arm[1] in ("L", "VEC_DOUBLING_BLOCKS"):
            return a
    return None


def allowed_arms(config, valid=None):
    """Arm mask of a measured call for the evaluation: every arm for integer
    calls; for float reductions (reference order) the arms with the variant
    and port count the fixed rule runs (fallback_arm), i.e. the segment
    choice alone."""
    m = np.ones(NARMS, bool)
    if config["coll"] in REDUCTIONS and config.get("dtype") == "float":
        fa = fallback_arm(config, valid)
        if fa is None:
            return np.zeros(NARMS, bool)
        m = np.array([arm_keeps(a, ARMS[fa][1:3]) for a in ARMS])
    return m


def apply_arm(comm, arm):
    coll, v, ports, seg = arm
    if v == "RING":
        comm.set_algo(coll, DEFAULT_VARIANT[coll], "RING")
    else:
        comm.set_algo(coll, v)
    comm.set_ports(ports)
    comm.set_segment(seg)


# ------------------------------------------------------------ data sampling
P_GRID = sorted({int(round(2 ** (k / 4.0))) for k in range(8, 49)} | {6, 12, 24, 48, 96, 384})
# reduce_scatter / allgather schedules move every block separately
# (P^2 log P moves: 4.2 M at P = 2048, 16.8 M at P = 4096, where one
# variant takes 15-23 s to plan and prove); they are sampled up to 2048.
MAX_P_VECTOR = 2048


def sample_configs(n, seed, max_total_bytes=2 << 30):
    """Calls: op 60/20/20 allreduce/reduce_scatter/allgather, P log-uniform
    on a grid over [4, 4096] ([4, 2048] for the vector collectives),
    per-rank message log-uniform 32 B..256 MiB (capped so P x message <=
    max_total_bytes), int32 or float32, one in three on a 2-D or 3-D torus
    when P is a power of two >= 16."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        coll = str(rng.choice(OPS, p=[0.6, 0.2, 0.2]))
        grid = P_GRID if coll == "allreduce" else [p for p in P_GRID if p <= MAX_P_VECTOR]
        P = int(rng.choice(grid))
        es = 4
        dt = "int32" if rng.random() < 0.5 else "float"
        m = 32 * 2 ** (rng.random() * 23)
        m = min(m, max_total_bytes / P)
        count = max(1, int(m // es)) if coll == "allreduce" else max(1, int(m // (es * P)))
        dims = [P]
        if is_p2(P) and P >= 16 and rng.random() < 1 / 3:
            k = int(math.log2(P))
            if rng.random() < 0.5:
                a = k // 2
                dims = [2 ** a, 2 ** (k - a)]
            else:
                a = k // 3
                b = (k - a) // 2
                dims = [2 ** a, 2 ** b, 2 ** (k - a - b)]
        out.append({"coll": coll, "P": P, "count": count, "es": es, "dtype": dt, "dims": dims})
    return out


def time_arm(comm, coll, send, recv, count, code, stream, reps=3, target_us=300.0, max_batch=32):
    """Microseconds per call: `reps` batches of back-to-back launches
    between two CUDA events (the batch grows until it spans ~target_us),
    median of the per-launch averages."""
    import torch

    def batch(n):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            comm.run(coll, send, recv, count, code)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e3 / n

    first = batch(1)
    n = int(min(max_batch, max(1, target_us // max(first, 1e-3))))
    ts = [batch(n) for _ in range(reps)]
    comm.synchronize()
    return float(np.median(ts))


def measure(configs, reps=3, time_budget_s=None, log=None, planners=None):
    """Measures every valid arm of every call on the GPU with the STEPS
    engine (time_arm), and the busiest link's bytes from the engine's device
    link accounting.  Returns (configs measured, X [n, IN_DIM], T_us
    [n, NARMS], L_bytes [n, NARMS], valid [n, NARMS]) in the order of
    `configs`; arms the engine refuses are invalid.  Stops early, keeping
    whole calls, once time_budget_s passes (the measured calls are then a
    subset).

    Planning and proving a call's schedules is host work that takes longer
    than timing them, so `planners` worker threads (default: the host's
    cores less two, at most 16) each take the next call, build its
    communicator and prove every statically valid arm (the planner releases
    the interpreter lock), while this thread times the prepared calls one
    at a time on the GPU: timings never overlap each other."""
    import queue
    import threading
    import time

    import torch

    import bine_trees_fugaku_b200 as bine

    stream = torch.cuda.current_stream()
    planners = planners or max(1, min(16, (os.cpu_count() or 4) - 2))
    t_start = time.time()
    ready = queue.Queue(maxsize=2 * planners)
    lock = threading.Lock()
    state = {"next": 0, "stop": False}

    def over_budget():
        return time_budget_s is not None and time.time() - t_start > time_budget_s

    def planner():
        while True:
            with lock:
                if state["stop"] or over_budget() or state["next"] >= len(configs):
                    break
                i = state["next"]
                state["next"] += 1
            cfg = configs[i]
            coll, P, count, dims = cfg["coll"], cfg["P"], cfg["count"], cfg["dims"]
            comm = bine.Comm(P, dims if len(dims) > 1 else None)
            comm.set_engine("steps")
            ok = []
            for a, arm in enumerate(ARMS):
                if not statically_valid(arm, coll, P, count, dims):
                    continue
                try:
                    apply_arm(comm, arm)
                    comm.plan_verify(coll, count)  # plans and proves once; run() reuses both
                    ok.append(a)
                except bine.BineError:
                    continue
            ready.put((i, comm, ok))
        ready.put(None)

    threads = [threading.Thread(target=planner, daemon=True) for _ in range(planners)]
    for t in threads:
        t.start()
    rows = {}
    finished = 0
    try:
        while finished < planners:
            item = ready.get()
            if item is None:
                finished += 1
                continue
            i, comm, ok = item
            cfg = configs[i]
            coll, P, count, es, dims = cfg["coll"], cfg["P"], cfg["count"], cfg["es"], cfg["dims"]
            comm.set_stream(stream)
            se, re = bine.row_counts(coll, count, P)
            dtype = torch.int32 if cfg["dtype"] == "int32" else torch.float32
            code = bine.INT32 if cfg["dtype"] == "int32" else bine.FLOAT
            send = torch.ones((P, se), dtype=dtype, device="cuda")
            recv = torch.zeros((P, re), dtype=dtype, device="cuda")
            links = torch.zeros(P * len(dims) * 2, dtype=torch.int64, device="cuda")
            t_row = np.full(NARMS, np.nan)
            l_row = np.full(NARMS, np.nan)
            for a in ok:
                arm = ARMS[a]
                try:
                    apply_arm(comm, arm)
                    comm.run(coll, send, recv, count, code)  # uploads the device tables once
                    comm.synchronize()
                except bine.BineError:
                    continue
                t_row[a] = time_arm(comm, coll, send, recv, count, code, stream, reps)
                comm.link_bytes(coll, count, code, links)
                l_row[a] = float(links.max().item())
            del send, recv, links
            comm.close()
            rows[i] = (t_row, l_row)
            if log and len(rows) % 500 == 0:
                log(f"measured {len(rows)}/{len(configs)} calls in {time.time() - t_start:.0f} s")
    finally:
        with lock:
            state["stop"] = True
        # Drain so that planners blocked on a full queue can finish.
        alive = [t for t in threads if t.is_alive()]
        while alive:
            try:
                item = ready.get(timeout=0.1)
                if item is not None:
                    item[1].close()
            except queue.Empty:
                pass
            alive = [t for t in threads if t.is_alive()]
    done = sorted(rows)
    cfgs = [configs[i] for i in done]
    T = np.array([rows[i][0] for i in done]).reshape(-1, NARMS)
    Lb = np.array([rows[i][1] for i in done]).reshape(-1, NARMS)
    X = np.array([features(c["coll"], c["P"], c["count"], c["es"], c["dims"]) for c in cfgs],
                 np.float32).reshape(-1, IN_DIM)
    return cfgs, X, T, Lb, ~np.isnan(T)


# ------------------------------------------------------------- the model
def targets(T, Lb, valid, stats=None, relative=True):
    """Standardised log2 targets; returns (Y [n, OUT_DIM], mask, stats).
    `stats` reuses another split's standardisation.  relative: each call's
    targets are taken relative to its best arm (log2 time over the fastest,
    log2 busiest-link bytes over the least), so the model spends no capacity
    on a call's overall scale, which no pick depends on."""
    n = T.shape[0]
    lt = np.where(valid, np.log2(np.maximum(T, 1e-3)), 0.0)
    ll = np.where(valid, np.log2(np.maximum(Lb, 0.0) + 1.0), 0.0)
    if relative:
        any_valid = valid.any(1, keepdims=True)
        lt = np.where(valid, lt - np.where(any_valid, np.min(np.where(valid, lt, np.inf), 1, keepdims=True), 0), 0.0)
        ll = np.where(valid, ll - np.where(any_valid, np.min(np.where(valid, ll, np.inf), 1, keepdims=True), 0), 0.0)
    st = stats or {"t_mean": float(lt[valid].mean()), "t_std": float(lt[valid].std() + 1e-9),
                   "l_mean": float(ll[valid].mean()), "l_std": float(ll[valid].std() + 1e-9)}
    Y = np.zeros((n, OUT_DIM), np.float32)
    M = np.zeros((n, OUT_DIM), np.float32)
    st.setdefault("relative", bool(relative))
    Y[:, :NARMS] = (lt - st["t_mean"]) / st["t_std"]
    Y[:, NARMS:2 * NARMS] = (ll - st["l_mean"]) / st["l_std"]
    M[:, :NARMS] = valid
    M[:, NARMS:2 * NARMS] = valid
    return Y, M, st


def train(X, Y, M, steps=3000, batch=256, lr=1e-3, seed=0, log=None, val=None, check_every=250):
    """Trains bine_mlp on the GPU (Adam, cosine learning rate); returns
    (mlp, losses).  With val = (Xv, Yv, Mv) the parameters with the lowest
    masked validation MSE seen at the checkpoints are kept."""
    import torch

    import bine_trees_fugaku_b200 as bine

    mlp = bine.MLP(IN_DIM, 256, OUT_DIM, batch, seed=seed)
    rng = np.random.default_rng(seed)
    n = X.shape[0]
    Xd, Yd, Md = (torch.from_numpy(a).cuda() for a in (X, Y, M))
    losses = []
    best = (np.inf, None)
    for s in range(steps):
        idx = torch.from_numpy(rng.integers(0, n, batch)).cuda()
        cur = lr * 0.5 * (1 + math.cos(math.pi * s / steps))
        loss = mlp.train_step(Xd[idx].contiguous(), Yd[idx].contiguous(), Md[idx].contiguous(), cur)
        losses.append(loss)
        if val is not None and ((s + 1) % check_every == 0 or s + 1 == steps):
            Xv, Yv, Mv = val
            d = (predict(mlp, Xv) - Yv) * Mv
            v = float((d * d).sum() / max(1.0, Mv.sum()))
            if v < best[0]:
                best = (v, mlp.get_params())
            if log:
                log(f"step {s + 1} train {loss:.4f} val {v:.4f}")
        elif log and s % 500 == 0:
            log(f"step {s} loss {loss:.4f}")
    if best[1] is not None:
        mlp.set_params(best[1])
    return mlp, losses


def predict(mlp, X):
    """Model outputs [n, OUT_DIM] (standardised log2 time, log2 link bytes);
    for a list of models (an ensemble), the mean of their outputs.  One
    fused launch (bine_mlp_ensemble_forward) per call."""
    import torch

    import bine_trees_fugaku_b200 as bine

    ens = mlp if isinstance(mlp, bine.Ensemble) else bine.Ensemble(mlp if isinstance(mlp, (list, tuple)) else [mlp])
    n = X.shape[0]
    pad = (-n) % 16
    Xp = np.concatenate([X, np.zeros((pad, IN_DIM), np.float32)]) if pad else X
    out = ens.forward(torch.from_numpy(np.ascontiguousarray(Xp, np.float32)).cuda()).cpu().numpy()
    if ens is not mlp:
        ens.close()
    return out[:n]


def evaluate(pred, T, Lb, valid, configs, shortlist=3):
    """Learned picks against exhaustive search (the measured optimum over
    every valid arm) and against the fixed rule, on held-out calls.

    Time objective: the arm with the lowest predicted time; its measured
    time over the optimum's.  Shortlist: the fastest measured of the
    `shortlist` arms the model ranks best (what Picker.tune settles on).
    Link objective: the arm with the lowest predicted busiest-link bytes;
    its bytes over the minimum."""
    rows, within, ratio, speed, fixed_within, fixed_invalid = 0, 0, [], [], 0, 0
    link_exact, link_ratio, short_within = 0, [], 0
    for i in range(T.shape[0]):
        # Float reductions: only arms that keep the reference order's
        # variant and ports (the result bits) compete.
        v = valid[i] & allowed_arms(configs[i], valid[i])
        if not v.any():
            continue
        rows += 1
        a = int(np.argmin(np.where(v, pred[i, :NARMS], np.inf)))
        t_opt = float(np.min(T[i, v]))
        within += T[i, a] <= 1.05 * t_opt
        ratio.append(T[i, a] / t_opt)
        # Shortlist: the best measured of the model's `shortlist` best arms.
        top = np.argsort(np.where(v, pred[i, :NARMS], np.inf))[:min(shortlist, int(v.sum()))]
        short_within += float(np.min(T[i, top])) <= 1.05 * t_opt
        c = configs[i]
        fa = fixed_rule(c["coll"], c["P"], c["count"], c["es"])
        if v[fa]:
            speed.append(T[i, fa] / T[i, a])
            fixed_within += T[i, fa] <= 1.05 * t_opt
        else:
            fixed_invalid += 1
        al = int(np.argmin(np.where(v, pred[i, NARMS:2 * NARMS], np.inf)))
        l_opt = float(np.min(Lb[i, v]))
        link_exact += Lb[i, al] <= l_opt
        link_ratio.append((Lb[i, al] + 1) / (l_opt + 1))
    gm = lambda x: float(np.exp(np.mean(np.log(x)))) if x else None
    return {"held_out_calls": rows,
            "pick_within_5pct_of_optimum": within / max(1, rows),
            "pick_time_over_optimum_geomean": gm(ratio),
            "pick_time_over_optimum_max": float(max(ratio)) if ratio else None,
            f"shortlist{shortlist}_within_5pct_of_optimum": short_within / max(1, rows),
            "fixed_rule_within_5pct_of_optimum": fixed_within / max(1, rows - fixed_invalid),
            "speedup_vs_fixed_rule_geomean": gm(speed),
            "calls_where_fixed_rule_is_refused": fixed_invalid,
            "link_pick_is_minimum": link_exact / max(1, rows),
            "link_bytes_over_minimum_geomean": gm(link_ratio)}


DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "picker_weights.npz")


def save(path, mlps, stats, meta):
    """Saves the weights of one model or of an ensemble (a list) as the
    bf16 values the forward pass uses (the master copies are fp32; forward
    rounds them to bf16), one row per model."""
    mlps = mlps if isinstance(mlps, (list, tuple)) else [mlps]
    meta = dict(meta, feature_version=FEATURE_VERSION, models=len(mlps))
    p = np.stack([m.get_params() for m in mlps])
    bits = (p.view(np.uint32) + 0x7FFF + ((p.view(np.uint32) >> 16) & 1)) >> 16  # round to nearest even
    np.savez_compressed(path, params_bf16=bits.astype(np.uint16), stats=json.dumps(stats),
                        meta=json.dumps(meta), arms=json.dumps(ARMS), dims=np.array([IN_DIM, 256, OUT_DIM]))


def load_params(path):
    """(params as float32 [models, n], dims, stats, meta, arms) of a saved
    picker."""
    z = np.load(path)
    p = (z["params_bf16"].astype(np.uint32) << 16).view(np.float32)
    return np.atleast_2d(p), tuple(int(v) for v in z["dims"]), json.loads(str(z["stats"])), \
        json.loads(str(z["meta"])), json.loads(str(z["arms"]))


class Picker:
    """Runtime picker.  With trained weights it ranks the arms by predicted
    time (bine_mlp forward on the GPU, averaged over the ensemble) and takes the first one the planner
    proves correct for the call; without weights it takes the fixed rule,
    then the latency-optimal tree (allreduce) or the block-by-block
    allgather when the planner refuses the rule's arm.  Picks are cached
    per call shape."""

    def __init__(self, path=DEFAULT_WEIGHTS):
        import bine_trees_fugaku_b200 as bine

        self.mlp = None
        self.cache = {}
        if path and os.path.exists(path):
            p, dims, _, meta, arms = load_params(path)
            if [tuple(a) for a in arms] != ARMS or dims != (IN_DIM, 256, OUT_DIM) or \
                    meta.get("feature_version") != FEATURE_VERSION:
                raise ValueError(f"{path}: arm space, features or model shape differ from this build")
            self.models = []
            for row in p:  # an ensemble: predictions are averaged
                m = bine.MLP(dims[0], dims[1], dims[2], 16, seed=0)
                m.set_params(row)
                self.models.append(m)
            self.mlp = bine.Ensemble(self.models)

    def ranking(self, coll, P, count, es, dims=None, keep=None):
        """Candidate arm indices, best first.  keep = (variant, ports)
        restricts them to arms with that variant and port count."""
        ok = [a for a, arm in enumerate(ARMS) if statically_valid(arm, coll, P, count, dims) and arm_keeps(arm, keep)]
        if self.mlp is None or not ok:
            first = fixed_rule(coll, P, count, es)
            if keep is not None:
                seg = ARMS[first][3]
                same = [a for a in ok if ARMS[a][3] == seg]
                return same + [a for a in ok if a not in same]
            rest = [a for a in ok if ARMS[a][1] in ("L", "VEC_DOUBLING_BLOCKS") and a != first]
            return [first] + rest
        x = np.zeros((16, IN_DIM), np.float32)
        x[0] = features(coll, P, count, es, dims)
        t = predict(self.mlp, x)[0, :NARMS]
        return sorted(ok, key=lambda a: t[a])

    def _candidates(self, comm, coll, count, datatype, limit):
        """Provable arms for the call, best first (at most `limit`), and the
        caller's (variant, ports) when the result bits depend on them."""
        import bine_trees_fugaku_b200 as bine

        es = bine.DTYPE_SIZE[datatype]
        keep = keep_of(comm, coll) if order_bound(coll, datatype, comm.engine, comm.float_order) else None
        cands = []
        for a in self.ranking(coll, comm.nranks, count, es, comm.dims, keep):
            apply_arm(comm, ARMS[a])
            try:
                comm.plan_verify(coll, count)
            except bine.Unsupported:
                continue
            cands.append(a)
            if len(cands) == limit:
                break
        if keep is not None:
            # The caller's own schedule, restored whatever the outcome; with
            # no arm of the arm space it must at least run as it is.
            if keep[0] == "RING":
                comm.set_algo(coll, DEFAULT_VARIANT[coll], "RING")
            else:
                comm.set_algo(coll, keep[0])
            comm.set_ports(keep[1])
            if not cands:
                comm.plan_verify(coll, count)
        return cands, keep

    def _apply(self, comm, coll, count, es, a, keep):
        """Applies arm `a`, or with keep and no arm of the arm space, the
        fixed rule's segment alone on the caller's schedule."""
        if a is not None:
            apply_arm(comm, ARMS[a])
            return ARMS[a]
        seg = ARMS[fixed_rule(coll, comm.nranks, count, es)][3]
        comm.set_segment(seg)
        return (coll, keep[0], keep[1], seg)

    def tune(self, comm, coll, count, datatype, trials=3, reps=3):
        """Times the `trials` best-ranked provable arms once for this call
        shape on scratch buffers (the caller's data is not touched) and
        caches the fastest; later choose() calls apply it.  Returns the arm.
        Float sums in the reference's order keep the caller's variant and
        port count (only the segment is tuned)."""
        import torch

        import bine_trees_fugaku_b200 as bine

        es = bine.DTYPE_SIZE[datatype]
        cands, keep = self._candidates(comm, coll, count, datatype, trials)
        key = (coll, comm.nranks, tuple(comm.dims), count, datatype, keep)
        if not cands:
            if keep is not None:
                self.cache[key] = None
                return self._apply(comm, coll, count, es, None, keep)
            raise bine.Unsupported(bine.ERR_UNSUPPORTED, f"no Bine schedule runs {coll} at P={comm.nranks}")
        se, re = bine.row_counts(coll, count, comm.nranks)
        tdt = {bine.INT32: torch.int32, bine.INT64: torch.int64, bine.FLOAT: torch.float32,
               bine.DOUBLE: torch.float64, bine.CHAR: torch.int8}[datatype]
        send = torch.zeros((comm.nranks, max(1, se)), dtype=tdt, device="cuda")
        recv = torch.zeros((comm.nranks, re), dtype=tdt, device="cuda")
        stream = torch.cuda.current_stream()
        comm.set_stream(stream)
        best = None
        for a in cands:
            apply_arm(comm, ARMS[a])
            t = time_arm(comm, coll, send, recv, count, datatype, stream, reps)
            if best is None or t < best[0]:
                best = (t, a)
        self.cache[key] = best[1]
        return self._apply(comm, coll, count, es, best[1], keep)

    def choose(self, comm, coll, count, datatype):
        """Applies the best provable arm to `comm` and returns it.
        `datatype` is the call's element type (bine.INT32, bine.FLOAT, ...):
        float sums in the reference's order keep the caller's variant and
        port count, so the result bits never change."""
        import bine_trees_fugaku_b200 as bine

        es = bine.DTYPE_SIZE[datatype]
        keep = keep_of(comm, coll) if order_bound(coll, datatype, comm.engine, comm.float_order) else None
        key = (coll, comm.nranks, tuple(comm.dims), count, datatype, keep)
        if key not in self.cache:
            cands, _ = self._candidates(comm, coll, count, datatype, 1)
            self.cache[key] = cands[0] if cands else None
        a = self.cache[key]
        if a is None and keep is None:
            raise bine.Unsupported(bine.ERR_UNSUPPORTED, f"no Bine schedule runs {coll} at P={comm.nranks}")
        return self._apply(comm, coll, count, es, a, keep)
