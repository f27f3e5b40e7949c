"""The oracle (C++ restatement) pinned against the reference's own outputs.

Fixtures in tests/golden/ come from reference code run by
tests/golden/make_golden.py: simulation/remap_rank.c, simulation/binomial.py
and the reference library (lib/*.cc) built against the MPI shim.
"""
import numpy as np
import pytest

from golden_data import load_json, load_ref_collectives
from oracle import port, ref
from oracle.common import buffer_counts, expected, receiving_ranks
from tests.golden.cases import case_input

CASES = load_ref_collectives()


def test_remap_rank_known_answers():
    gold = load_json("remap_rank.json")
    assert gold["8"] == [0, 4, 6, 1, 3, 7, 5, 2]
    for P, vals in gold.items():
        P = int(P)
        assert [port.remap_rank(P, r) for r in range(P)] == vals, P


def test_binomial_py_remap_known_answers():
    for P, vals in load_json("binomial_remap.json").items():
        P = int(P)
        assert [port.remap_rank(P, q) for q in range(P)] == vals, P


def _msgs(m):
    return sorted(zip(m[:, 0].tolist(), m[:, 1].tolist(), m[:, 2].tolist()))


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}"
                         f"-d{c.get('dims')}-p{c.get('ports', 1)}-r{c.get('root', 0)}-{c.get('family', 'BINE')}")
def test_oracle_matches_reference(case):
    x = case_input(case)
    kw = dict(variant=case["variant"], dims=case.get("dims"), ports=case.get("ports", 1), root=case.get("root", 0),
              family=case.get("family", "BINE"), distance=case.get("distance"))
    try:
        out, msgs = port.run(case["coll"], x, case["count"], trace=True, **kw)
    except port.ReferenceUnsupported as e:
        # The oracle rejects the case: the reference must fail on it too, or
        # return something other than the MPI result, or only get through by
        # reading/writing past its buffers (undefined behaviour).
        if case["ok"]:
            rr = receiving_ranks(case["coll"], case["P"], case.get("root", 0))
            exp = expected(case["coll"], x, case["P"], case["count"], case.get("root", 0))
            wrong = not np.array_equal(case["out"][rr], exp[rr]) if case["dtype"] == "int32" else \
                not np.allclose(case["out"][rr], exp[rr], rtol=1e-4, atol=1e-4)
            assert wrong or "past" in str(e) or "out-of-bounds" in str(e), str(e)
        return
    assert case["ok"], "the oracle runs a case the reference fails on"
    rr = receiving_ranks(case["coll"], case["P"], case.get("root", 0))
    assert np.array_equal(out[rr].view(np.uint8), case["out"][rr].view(np.uint8))
    mine = sorted(zip(msgs["src"].tolist(), msgs["dst"].tolist(), msgs["bytes"].astype(np.int64).tolist()))
    assert mine == _msgs(case["msgs"])


@pytest.mark.skipif(not ref.available(), reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("coll,variant,P", [("allreduce", "B", 32), ("allreduce", "L", 64), ("allreduce", "B", 24),
                                            ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 32),
                                            ("allgather", "VEC_DOUBLING_BLOCKS", 20), ("alltoall", "LOG", 32),
                                            ("bcast", "BINOMIAL_TREE", 18)])
def test_oracle_matches_live_reference(coll, variant, P):
    count = 2 * P + 1 if coll == "allreduce" else 3
    sc, _ = buffer_counts(coll, count, P)
    x = np.random.default_rng(P).standard_normal((P, sc)).astype(np.float32)
    out, msgs = port.run(coll, x, count, variant=variant, trace=True)
    r = ref.run(coll, x, count, variant=variant, trace=True)
    assert r.ok, r.stderr[-500:]
    assert np.array_equal(out.view(np.uint32), r.out.view(np.uint32))
    a = sorted(zip(msgs["src"].tolist(), msgs["dst"].tolist(), msgs["bytes"].tolist()))
    b = sorted(zip(r.trace["src"].tolist(), r.trace["dst"].tolist(), r.trace["bytes"].tolist()))
    assert a == b


def _large_cases():
    import json
    import os

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_large.json")
    with open(path) as f:
        return json.load(f)


LARGE = _large_cases()
# The restatement runs one thread per rank with per-block messages: cases
# whose P^2 message counts would take it beyond a few seconds on a CPU are
# pinned on the GPU only (tests/test_large_parity_gpu.py).
SLOW = {("allgather", "VEC_DOUBLING_BLOCKS"), ("allreduce", "B"), ("allreduce", "B_COALESCE"),
        ("reduce", "REDUCE_SCATTER_GATHER"), ("bcast", "SCATTER_ALLGATHER")}


def _large_quick(c):
    return c["P"] <= 256 or ((c["coll"], c["variant"]) not in SLOW and c["P"] <= 1024)


@pytest.mark.parametrize("case", [c for c in LARGE if _large_quick(c)],
                         ids=lambda c: f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-n{c['count']}"
                         + "".join(f"-{k}{c[k]}" for k in ("ports", "root", "family", "dims") if k in c))
def test_oracle_matches_reference_digests_at_large_p(case):
    """The restatement against digests of the reference's own results at
    P = 128..1024 (tests/golden/ref_large.json): identical result bytes and
    message multiset where the reference gives the MPI result; where it
    fails or returns other data, the restatement reports the reference as
    unsupported."""
    from tests.golden import large_cases as lc

    x = lc.case_input(case)
    kw = dict(variant=case["variant"], dims=case.get("dims"), ports=case.get("ports", 1), root=case.get("root", 0),
              family=case.get("family", "BINE"), distance=case.get("distance"))
    try:
        out, msgs = port.run(case["coll"], x, case["count"], trace=True, **kw)
    except port.ReferenceUnsupported:
        assert not (case["ok"] and case["mpi"]), "the restatement refuses a case the reference runs correctly"
        return
    assert case["ok"], "the restatement runs a case the reference fails on"
    assert lc.result_digest(case, out) == case["digest"]
    assert lc.trace_digest(msgs["src"], msgs["dst"], msgs["bytes"].astype(np.int64)) == case["trace_digest"]


@pytest.mark.skipif(not ref.available(), reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("case", [c for c in LARGE if c["P"] <= 256 and c["ok"] and c["count"] < 1 << 20][::7],
                         ids=lambda c: f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-n{c['count']}")
def test_large_digests_reproduce_on_the_live_reference(case):
    """A sample of the large-P fixtures recomputed by the reference library
    itself (oracle/_ref): the digests are current."""
    from tests.golden import large_cases as lc

    x = lc.case_input(case)
    r = ref.run(case["coll"], x, case["count"], variant=case["variant"], dims=case.get("dims"),
                ports=case.get("ports", 1), root=case.get("root", 0), family=case.get("family", "BINE"),
                distance=case.get("distance"), timeout=300, shim_timeout=60)
    assert r.ok, r.stderr[-500:]
    assert lc.result_digest(case, r.out) == case["digest"]
