"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout that has the reference at REF (default: $BINE_REFERENCE,
else a directory "reference" beside this repository) and the reference
library built by `make -C oracle ref`:

    python tests/golden/make_golden.py [REF] [--large-only]

Fixtures (all outputs of reference code, never hand-written):
  remap_rank.json      simulation/remap_rank.c (compiled from its source)
                       for every rank of a set of sizes;
  binomial_remap.json  simulation/binomial.py get_remapped_rank(q, P);
  simulator.json       "bw new vs ideal" printed by simulation/simulator.py
                       for ALLREDUCE on 2x2x2, 4x4x4 and 8x8x8 tori;
  ref_collectives.npz  results and message traces of the reference library
                       (lib/*.cc via oracle/_ref/bine_ref_run) for small
                       seeded inputs of every MPI-layer variant;
  ref_large.json       per case of tests/golden/large_cases.py (P = 128,
                       256, 384, 1024 and the full-size P = 8 allreduce):
                       whether the reference completed, whether its result
                       is the MPI result, and SHA-256 digests of its result
                       rows and message trace.
"""
import importlib.util
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from oracle.common import buffer_counts  # noqa: E402
from tests.golden.cases import CASES, case_input  # noqa: E402
from tests.golden import large_cases  # noqa: E402


def remap_rank_c(refdir):
    src = os.path.join(refdir, "simulation", "remap_rank.c")
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "remap_rank")
        subprocess.run(["gcc", "-O2", "-o", exe, src, "-lm"], check=True)
        out = {}
        for P in [2, 4, 8, 16, 32, 64, 128, 256, 6, 10, 12, 18, 96]:
            vals = []
            for r in range(P):
                line = subprocess.run([exe, str(P), str(r)], capture_output=True, text=True, check=True).stdout
                vals.append(int(line.split("remap_rank:")[1]))
            out[str(P)] = vals
    return out


def binomial_remap(refdir):
    path = os.path.join(refdir, "simulation", "binomial.py")
    spec = importlib.util.spec_from_file_location("ref_binomial", path)
    mod = importlib.util.module_from_spec(spec)
    # binomial.py runs validate_all() at import; it only prints and asserts.
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        spec.loader.exec_module(mod)
    return {str(P): [0] + [mod.get_remapped_rank(q, P) for q in range(1, P)] for P in [4, 8, 16, 32, 64, 128, 256]}


def simulator_ratios(refdir):
    out = {}
    for d in ["2x2x2", "4x4x4", "8x8x8"]:
        p = subprocess.run([sys.executable, os.path.join(refdir, "simulation", "simulator.py"), "-c", "ALLREDUCE",
                            "-d", d], capture_output=True, text=True, check=True)
        line = [l for l in p.stdout.splitlines() if "bw new vs ideal" in l][0]
        parts = line.replace(":", " ").split()
        out[d] = {"new_vs_ideal": float(parts[parts.index("ideal") + 1]), "line": line}
    return out


def ref_collectives():
    arrays = {}
    index = []
    for i, case in enumerate(CASES):
        x = case_input(case)
        r = ref.run(case["coll"], x, case["count"], variant=case["variant"], dims=case.get("dims"),
                    ports=case.get("ports", 1), root=case.get("root", 0), family=case.get("family", "BINE"),
                    distance=case.get("distance"), trace=True)
        entry = dict(case)
        entry["ok"] = r.ok
        if r.ok:
            arrays[f"out{i}"] = r.out
            t = r.trace
            arrays[f"msg{i}"] = np.stack([t["src"], t["dst"], t["bytes"].astype(np.int64)], 1)
        index.append(entry)
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    return arrays


def ref_large():
    """Digests of the reference's results on tests/golden/large_cases.py:
    per case whether the reference completed, whether its result is the MPI
    result, and the SHA-256 of the result rows and of the message trace."""
    out = []
    for case in large_cases.CASES:
        x = large_cases.case_input(case)
        r = ref.run(case["coll"], x, case["count"], variant=case["variant"], dims=case.get("dims"),
                    ports=case.get("ports", 1), root=case.get("root", 0), family=case.get("family", "BINE"),
                    distance=case.get("distance"), trace=True, timeout=900, shim_timeout=60)
        entry = dict(case)
        entry["ok"] = r.ok
        if r.ok:
            t = r.trace
            entry["digest"] = large_cases.result_digest(case, r.out)
            entry["trace_digest"] = large_cases.trace_digest(t["src"], t["dst"], t["bytes"].astype(np.int64))
            entry["messages"] = int(len(t))
            entry["mpi"] = large_cases.matches_mpi(case, x, r.out)
        else:
            entry["status"] = r.info.get("status", [])[:4]
        print(json.dumps({k: entry[k] for k in ("coll", "variant", "P", "dtype", "count", "ok")}
                         | {"mpi": entry.get("mpi")}), flush=True)
        out.append(entry)
    return out


def main():
    repo = os.path.dirname(os.path.dirname(HERE))
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    refdir = args[0] if args else os.environ.get("BINE_REFERENCE", os.path.join(os.path.dirname(repo), "reference"))
    if not ref.available():
        sys.exit("build the reference first: make -C oracle ref")
    if "--large-only" not in sys.argv:
        small(refdir)
    with open(os.path.join(HERE, "ref_large.json"), "w") as f:
        json.dump(ref_large(), f, indent=0)


def small(refdir):
    with open(os.path.join(HERE, "remap_rank.json"), "w") as f:
        json.dump(remap_rank_c(refdir), f)
    with open(os.path.join(HERE, "binomial_remap.json"), "w") as f:
        json.dump(binomial_remap(refdir), f)
    with open(os.path.join(HERE, "simulator.json"), "w") as f:
        json.dump(simulator_ratios(refdir), f, indent=1)
    np.savez_compressed(os.path.join(HERE, "ref_collectives.npz"), **ref_collectives())


if __name__ == "__main__":
    main()
