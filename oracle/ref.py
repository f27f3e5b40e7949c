"""Runner for the reference library itself (oracle/_ref/bine_ref_run).

The binary is the unmodified reference compiled from its sources against the
project's MPI shim (``make -C oracle ref``); each call forks one process per
rank on this host.  Every collective is forced onto the reference's MPI
layer (its default is the Fugaku-only uTofu layer, lib/libbine.cc:47-54).
"""
import json
import os
import subprocess
import tempfile

import numpy as np

from .common import DTYPES, DEFAULT_VARIANT, buffer_counts

_HERE = os.path.dirname(os.path.abspath(__file__))
BIN_PATH = os.path.join(_HERE, "_ref", "bine_ref_run")
ENV_COLL = {"allreduce": "ALLREDUCE", "reduce_scatter": "REDUCE_SCATTER", "allgather": "ALLGATHER",
            "bcast": "BCAST", "reduce": "REDUCE", "alltoall": "ALLTOALL", "scatter": "SCATTER",
            "gather": "GATHER"}
DT_ARG = {"int32": "int32", "int64": "int64", "float": "float", "double": "double", "char": "char"}


def available():
    return os.path.exists(BIN_PATH)


def base_env(coll=None, variant=None, dims=None, ports=1, family="BINE", distance=None):
    env = dict(os.environ)
    for v in ENV_COLL.values():
        env[f"LIBBINE_{v}_ALGO_LAYER"] = "MPI"
    env["LIBBINE_PREALLOC_SIZE"] = "0"
    if coll:
        C = ENV_COLL[coll]
        env[f"LIBBINE_{C}_ALGO"] = variant or DEFAULT_VARIANT[coll]
        env[f"LIBBINE_{C}_ALGO_FAMILY"] = family
        if distance:
            env[f"LIBBINE_{C}_DISTANCE"] = distance
    env["LIBBINE_NUM_PORTS"] = str(ports)
    if dims:
        env["LIBBINE_DIMENSIONS"] = "x".join(str(d) for d in dims)
    else:
        env.pop("LIBBINE_DIMENSIONS", None)
    return env


class RefResult:
    def __init__(self, ok, out, info, stderr, trace):
        self.ok, self.out, self.info, self.stderr, self.trace = ok, out, info, stderr, trace


TRACE_DTYPE = np.dtype([("src", np.int32), ("dst", np.int32), ("tag", np.int32), ("call", np.int32),
                        ("bytes", np.uint64)])


# The same harness linked against the engine's PMPI layer instead of the
# reference library (``make -C oracle dropin``).
DROPIN_PATH = os.path.join(_HERE, "_build", "bine_dropin_run")


def run(coll, x, count, *, variant=None, dims=None, ports=1, root=0, family="BINE", distance=None,
        trace=False, timeout=120.0, shim_timeout=20.0, binary=None, extra_env=None):
    """Runs the reference (or, with binary=DROPIN_PATH, the engine behind
    the same MPI entry points) on rank-major input x[P, send_count];
    returns RefResult."""
    x = np.ascontiguousarray(x)
    P = x.shape[0]
    dt = {np.dtype(v[1]): k for k, v in DTYPES.items()}[x.dtype]
    sc, rc = buffer_counts(coll, count, P)
    assert x.shape[1] == sc
    with tempfile.TemporaryDirectory() as td:
        fin, fout, ftr = (os.path.join(td, n) for n in ("in.bin", "out.bin", "trace.bin"))
        x.tofile(fin)
        cmd = [binary or BIN_PATH, "--coll", coll, "--dtype", DT_ARG[dt], "--count", str(count), "--P", str(P),
               "--root", str(root), "--in", fin, "--out", fout, "--timeout", str(shim_timeout)]
        if trace:
            cmd += ["--trace", ftr]
        env = base_env(coll, variant, dims, ports, family, distance)
        env.update(extra_env or {})
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
        except subprocess.TimeoutExpired as e:
            return RefResult(False, None, {"ok": False, "status": ["timeout"]}, str(e), None)
        lines = p.stdout.strip().splitlines()
        info = json.loads(lines[-1]) if lines else {"ok": False}
        out = None
        if info.get("ok") and os.path.exists(fout):
            out = np.fromfile(fout, dtype=x.dtype).reshape(P, rc)
        tr = np.fromfile(ftr, dtype=TRACE_DTYPE) if trace and os.path.exists(ftr) else None
        return RefResult(bool(info.get("ok")), out, info, p.stderr, tr)


def time_collective(coll, dtype, count, P, *, iters=10, warmup=10, variant=None, dims=None, ports=1, root=0,
                    timeout=600.0, binary=None):
    """Times the reference (or, with binary=DROPIN_PATH, the engine behind
    the same MPI entry points) as bench/bench.cc does; returns the harness
    JSON."""
    cmd = [binary or BIN_PATH, "--coll", coll, "--dtype", DT_ARG[dtype], "--count", str(count), "--P", str(P),
           "--root", str(root), "--gen", "uniform", "--iters", str(iters), "--warmup", str(warmup),
           "--timeout", str(timeout)]
    p = subprocess.run(cmd, capture_output=True, text=True, env=base_env(coll, variant, dims, ports),
                       timeout=timeout + 60)
    lines = p.stdout.strip().splitlines()
    return json.loads(lines[-1]) if lines else {"ok": False, "stderr": p.stderr[-500:]}
