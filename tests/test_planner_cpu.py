"""The engine's host planner (schedule IR, exact trees, messages, link
accounting) checked on the CPU against the reference's outputs.

The IR is executed with numpy (tests/irexec.py) only to check the plan;
the product runs it on the GPU.
"""
import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine
from golden_data import load_json, load_ref_collectives
from irexec import eval_trees, run_moves
from oracle import port
from oracle.common import buffer_counts, receiving_ranks
from tests.golden.cases import case_input

CASES = load_ref_collectives()


def make_comm(case):
    comm = bine.Comm(case["P"], case.get("dims"))
    comm.set_ports(case.get("ports", 1))
    comm.set_algo(case["coll"], case["variant"], case.get("family", "BINE"), case.get("distance"))
    return comm


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}"
                         f"-d{c.get('dims')}-p{c.get('ports', 1)}-r{c.get('root', 0)}-{c.get('family', 'BINE')}")
def test_plan_matches_reference(case):
    x = case_input(case)
    comm = make_comm(case)
    root = case.get("root", 0)
    try:
        out = run_moves(comm, case["coll"], case["count"], x, root)
    except bine.Unsupported:
        # Must be a case the oracle rejects as well.
        with pytest.raises(port.ReferenceUnsupported):
            port.run(case["coll"], x, case["count"], variant=case["variant"], dims=case.get("dims"),
                     ports=case.get("ports", 1), root=root, family=case.get("family", "BINE"),
                     distance=case.get("distance"))
        return
    assert case["ok"]
    rr = receiving_ranks(case["coll"], case["P"], root)
    assert np.array_equal(out[rr].view(np.uint8), case["out"][rr].view(np.uint8))
    m = comm.plan_messages(case["coll"], case["count"], root)
    es = x.dtype.itemsize
    mine = sorted(zip(m[:, 1].tolist(), m[:, 2].tolist(), (m[:, 3] * es).tolist()))
    ref = sorted(zip(case["msgs"][:, 0].tolist(), case["msgs"][:, 1].tolist(), case["msgs"][:, 2].tolist()))
    assert mine == ref
    if case["coll"] in ("allreduce", "reduce_scatter", "reduce"):
        t = eval_trees(comm, case["coll"], case["count"], x, root)
        assert np.array_equal(t[rr].view(np.uint8), case["out"][rr].view(np.uint8))


@pytest.mark.parametrize("variant,P,ports", [("B", 64, 1), ("B", 128, 1), ("B_COALESCE", 96, 2), ("L", 64, 3),
                                             ("L", 96, 1), ("B_CONT", 128, 1)])
def test_plan_trees_match_oracle_larger(variant, P, ports):
    count = 3 * P * ports + 7
    x = np.random.default_rng(P).standard_normal((P, count)).astype(np.float32)
    expect, _ = port.run("allreduce", x, count, variant=variant, ports=ports)
    comm = bine.Comm(P)
    comm.set_ports(ports)
    comm.set_algo("allreduce", variant)
    got = eval_trees(comm, "allreduce", count, x)
    assert np.array_equal(got.view(np.uint32), expect.view(np.uint32))


@pytest.mark.parametrize("dims", ["2x2x2", "4x4x4", "8x8x8"])
def test_link_accounting_reproduces_simulator(dims):
    """Distance-weighted traffic of rank 0's reduce-scatter messages equals
    simulation/simulator.py's "bw new vs ideal" for the Bine allreduce."""
    gold = load_json("simulator.json")[dims]["new_vs_ideal"]
    d = [int(v) for v in dims.split("x")]
    P = int(np.prod(d))
    comm = bine.Comm(P, d)
    count = P * 64
    msgs = comm.plan_messages("allreduce", count)
    steps = sum(int(np.log2(v)) for v in d)
    rs = msgs[(msgs[:, 1] == 0) & (msgs[:, 0] >= 1) & (msgs[:, 0] <= steps)]  # level 0 copies send -> recv
    coords = lambda r: np.unravel_index(r, d)
    total = weighted = 0
    for lvl, src, dst, n in rs:
        a, b = np.array(coords(src)), np.array(coords(dst))
        (k,) = np.nonzero(a != b)[0]
        delta = (b[k] - a[k]) % d[k]
        hops = min(delta, d[k] - delta)
        total += n
        weighted += n * hops
    assert abs(total / weighted - gold) < 1e-12


@pytest.mark.parametrize("coll,ports,count", [("allreduce", 1, 64 * 64), ("allreduce", 6, 64 * 6 * 5 + 7),
                                              ("alltoall", 1, 3)])
def test_link_bytes_conserve_message_volume(coll, ports, count):
    d = [4, 4, 4]
    comm = bine.Comm(64, d)
    comm.set_ports(ports)
    lb = comm.link_bytes_host(coll, count, bine.INT32)
    msgs = comm.plan_messages(coll, count)
    expect = 0
    for _, s, t, n in msgs:
        a, b = np.array(np.unravel_index(s, d)), np.array(np.unravel_index(t, d))
        for k in np.nonzero(a != b)[0]:
            delta = (b[k] - a[k]) % d[k]
            expect += n * 4 * min(delta, d[k] - delta)
    assert int(lb.sum()) == expect
    assert lb.shape == (64 * 3 * 2,)


@pytest.mark.parametrize("ports", [1, 6])
def test_reduce_scatter_volume_per_step_is_uniform_over_blocks(ports):
    """Every block is sent at reduce-scatter step i by P/2^(i+1) ranks (the
    identity the large-torus link test relies on), checked on the planner."""
    d = [4, 4, 4]
    P = 64
    comm = bine.Comm(P, d)
    comm.set_ports(ports)
    count = P * ports * 3 + 5
    msgs = comm.plan_messages("allreduce", count)
    S = 6
    # Port p reduces its own slice of count_p elements (lib/libbine.cc:986-1010).
    per_port = [count // ports + (p < count % ports) for p in range(ports)]
    for i in range(S):
        lvl = msgs[msgs[:, 0] == i + 1]
        # Each of a port's blocks leaves P / 2^(i+1) ranks at step i.
        assert int(lvl[:, 3].sum()) == sum(c * (P >> (i + 1)) for c in per_port), i
    total_rs = sum(int(msgs[msgs[:, 0] == i + 1][:, 3].sum()) for i in range(S))
    assert total_rs == sum(P * c * (2 ** S - 1) // 2 ** S for c in per_port)


@pytest.mark.parametrize("case", [c for c in CASES if c["ok"]], ids=lambda c: f"{c['coll']}-{c['variant']}-P{c['P']}"
                         f"-{c['dtype']}-d{c.get('dims')}-p{c.get('ports', 1)}-r{c.get('root', 0)}-{c.get('family', 'BINE')}")
def test_verify_flags_exactly_the_wrong_reference_results(case):
    """The planner's symbolic proof fails exactly where the reference
    completes with data that is not the MPI result."""
    from oracle.common import expected
    x = case_input(case)
    comm = make_comm(case)
    root = case.get("root", 0)
    try:
        comm.plan_stats(case["coll"], case["count"], root)
    except bine.Unsupported:
        return  # not even plannable (undefined behaviour in the reference)
    rr = receiving_ranks(case["coll"], case["P"], root)
    exp = expected(case["coll"], x, case["P"], case["count"], root)
    if case["dtype"] == "float" and case["coll"] in ("allreduce", "reduce_scatter", "reduce"):
        right = np.allclose(case["out"][rr], exp[rr], rtol=1e-4, atol=1e-4)
    else:
        right = np.array_equal(case["out"][rr], exp[rr])
    if right:
        comm.plan_verify(case["coll"], case["count"], root)
    else:
        with pytest.raises(bine.Unsupported):
            comm.plan_verify(case["coll"], case["count"], root)
