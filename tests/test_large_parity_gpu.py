"""Bit-exact parity with the reference library at large P, on the GPU.

tests/golden/ref_large.json holds, for every case of
tests/golden/large_cases.py, digests of the reference's own results (lib/*.cc
run by its MPI layer under the oracle's shim): allreduce B, B_COALESCE,
B_CONT and L, reduce_scatter, reduce, allgather, bcast, alltoall (Bine and
Bruck), scatter and gather at P = 128, 256, 384 and 1024, roots other than
0, the recursive-doubling family, tori of 128 and 384 ranks, and the
full-size P = 8 allreduce (1,048,576 int32 and float32 per rank).

Every case runs on the FUSED, STEPS and PIPELINED engines in the reference's
float order and must reproduce the reference's result bytes exactly, float32
included.  Where the reference fails or returns data that is not the MPI
result, the engines that follow its schedule must refuse the call
(BINE_ERR_UNSUPPORTED), and the FUSED engine must return the MPI result:
exact for integers and copies, and within 1e-6 relative of an FP64 sum for
float32 reductions in the FAST order.
"""
import json
import os

import numpy as np
import pytest
import torch

import bine_trees_fugaku_b200 as bine
from oracle.common import buffer_counts, expected, receiving_ranks
from tests.golden import large_cases as lc

pytestmark = pytest.mark.gpu

with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_large.json")) as _f:
    CASES = json.load(_f)
CODE = {"int32": bine.INT32, "float": bine.FLOAT}
REDUCTIONS = ("allreduce", "reduce_scatter", "reduce")


def case_id(c):
    extra = "".join(f"-{k}{c[k]}" for k in ("ports", "root", "family", "dims") if k in c)
    return f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-n{c['count']}{extra}"


def make_comm(case, engine, order="reference"):
    comm = bine.Comm(case["P"], case.get("dims"))
    comm.set_ports(case.get("ports", 1))
    comm.set_algo(case["coll"], case["variant"], case.get("family", "BINE"), case.get("distance"))
    comm.set_engine(engine)
    comm.set_float_order(order)
    comm.set_stream(torch.cuda.current_stream())
    return comm


def run(comm, case, x):
    P, count, root = case["P"], case["count"], case.get("root", 0)
    _, rc = buffer_counts(case["coll"], count, P)
    send = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    recv = torch.zeros((P, rc), dtype=send.dtype, device="cuda")
    if case["coll"] == "bcast":
        recv[root] = send[root]
    comm.run(case["coll"], send, recv, count, CODE[case["dtype"]], root)
    comm.synchronize()
    return recv.cpu().numpy()


def within_1e6_of_fp64(case, x, out):
    P, count, root = case["P"], case["count"], case.get("root", 0)
    rr = receiving_ranks(case["coll"], P, root)
    s = x.astype(np.float64).sum(0)
    exact = {"allreduce": lambda: np.tile(s, (P, 1)), "reduce": lambda: np.tile(s, (P, 1)),
             "reduce_scatter": lambda: s.reshape(P, count)}[case["coll"]]()[rr]
    # The FP64 sum itself is only good to about P * 2^-53 * sum|x|.
    ax = np.abs(x.astype(np.float64)).sum(0)
    floor = {"allreduce": lambda: np.tile(ax, (P, 1)), "reduce": lambda: np.tile(ax, (P, 1)),
             "reduce_scatter": lambda: ax.reshape(P, count)}[case["coll"]]()[rr] * P * 2.0 ** -52
    return bool((np.abs(out[rr].astype(np.float64) - exact) <= 1e-6 * np.abs(exact) + floor).all())


@pytest.mark.parametrize("engine", ["fused", "steps", "pipelined"])
@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_engine_matches_reference_at_large_p(case, engine):
    x = lc.case_input(case)
    float_reduction = case["dtype"] == "float" and case["coll"] in REDUCTIONS
    comm = make_comm(case, engine)
    try:
        if case["ok"] and case["mpi"]:
            out = run(comm, case, x)
            assert lc.result_digest(case, out) == case["digest"], "result bytes differ from the reference's"
            return
        # The reference fails here or returns data that is not the MPI result.
        if engine != "fused" or float_reduction:
            with pytest.raises(bine.Unsupported):
                run(comm, case, x)
        if engine == "fused":
            comm.set_float_order("fast")
            out = run(comm, case, x)
            if float_reduction:
                assert within_1e6_of_fp64(case, x, out)
            else:
                rr = receiving_ranks(case["coll"], case["P"], case.get("root", 0))
                assert np.array_equal(out[rr], expected(case["coll"], x, case["P"], case["count"],
                                                        case.get("root", 0))[rr])
    finally:
        comm.close()
