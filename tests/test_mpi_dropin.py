"""The engine behind the reference's own MPI entry points.

oracle/ref_harness.cc is the harness that runs the reference library: P
forked ranks calling MPI_Allreduce, MPI_Reduce_scatter, MPI_Allgather,
MPI_Bcast_f, MPI_Alltoall, MPI_Scatter, MPI_Gather or MPI_Reduce, with the
algorithm picked by the reference's LIBBINE_* variables.  `make -C oracle
dropin` links the same harness, unchanged, against the engine's PMPI layer
(bine_trees_fugaku_b200/csrc/bine_mpi.cc) instead of the reference library.

* CPU: the layer exports the reference's entry points, and on a host without
  a GPU every rank returns the engine's error instead of hanging.
* GPU: golden cases (outputs of the reference library itself) through the
  drop-in build return the reference's bytes, float32 included; where the
  reference returned wrong data, the MPI result.
"""
import os
import subprocess

import numpy as np
import pytest

from golden_data import load_ref_collectives
from oracle import ref
from oracle.common import expected, receiving_ranks
from tests.golden.cases import case_input

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENTRY_POINTS = ["MPI_Init", "MPI_Finalize", "MPI_Allreduce", "MPI_Reduce_scatter", "MPI_Allgather", "MPI_Bcast_f",
                "MPI_Alltoall", "MPI_Scatter", "MPI_Gather", "MPI_Reduce"]
# The reference names its broadcast MPI_Bcast_f and leaves MPI_Bcast to the
# MPI library (lib/libbine.cc:1252; bench/bench.cc:20, 136): a program's own
# MPI_Bcast calls must not be routed through the GPU.
NOT_INTERPOSED = ["MPI_Bcast"]


def build():
    lib = os.path.join(ROOT, "bine_trees_fugaku_b200", "lib", "libbine_b200.so")
    if not os.path.exists(lib):
        pytest.skip("engine library not built")
    p = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "dropin"], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    return ref.DROPIN_PATH


def test_layer_exports_the_reference_entry_points():
    build()
    so = os.path.join(ROOT, "oracle", "_build", "libbine_mpi.so")
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in ENTRY_POINTS:
        assert n in names, n
    for n in NOT_INTERPOSED:
        assert n not in names, n


def test_without_a_gpu_every_rank_reports_the_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    binary = build()
    x = np.arange(4 * 64, dtype=np.int32).reshape(4, 64)
    r = ref.run("allreduce", x, 64, binary=binary, timeout=180, shim_timeout=60)
    assert not r.ok
    assert r.info["status"] == ["exit:1"] * 4
    assert "bine_mpi:" in r.stderr


CASES = [c for c in load_ref_collectives() if c["ok"]]


def case_id(c):
    return (f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-d{c.get('dims')}-p{c.get('ports', 1)}"
            f"-r{c.get('root', 0)}-{c.get('family', 'BINE')}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES[::3], ids=case_id)
def test_dropin_returns_the_reference_bytes(case):
    binary = build()
    x = case_input(case)
    root = case.get("root", 0)
    r = ref.run(case["coll"], x, case["count"], variant=case["variant"], dims=case.get("dims"),
                ports=case.get("ports", 1), root=root, family=case.get("family", "BINE"),
                distance=case.get("distance"), binary=binary, timeout=120, shim_timeout=60)
    assert r.ok, (r.info, r.stderr[-500:])
    rr = receiving_ranks(case["coll"], case["P"], root)
    if np.array_equal(case["out"][rr].view(np.uint8), r.out[rr].view(np.uint8)):
        return
    # Different bytes only where the reference itself returned wrong data;
    # the engine then returns the MPI result (float sums whose reference
    # order does not exist run in the FP64-accumulated order).
    exp = expected(case["coll"], x, case["P"], case["count"], root)
    if case["dtype"] == "float" and case["coll"] in ("allreduce", "reduce_scatter", "reduce"):
        assert not np.allclose(case["out"][rr], exp[rr], rtol=1e-4, atol=1e-4)
        assert np.allclose(r.out[rr], exp[rr], rtol=1e-5, atol=1e-5)
    else:
        assert not np.array_equal(case["out"][rr], exp[rr])
        assert np.array_equal(r.out[rr], exp[rr])
