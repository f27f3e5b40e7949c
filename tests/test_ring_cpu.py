"""The bucket (multi-dimensional ring) allreduce, the reference's RING family
comparator (BineCommon::bucket_allreduce, lib/libbine_common.cc:2486-2663,
over ringRedScatAG, lib/libbine_common.cc:2372-2484).

The reference runs it on uTofu only, so its library cannot produce golden
outputs for it; two independent restatements pin it instead:
  * the oracle (oracle/bine_oracle.cc, bucket_allreduce), which follows the
    reference's own loops over a message layer, checked against MPI
    semantics (exact integer sums, FP64-bounded float sums);
  * the engine's planner (gen_allreduce_ring), whose schedule IR, executed
    with numpy, and whose extracted addition trees must give the oracle's
    bytes, float32 included, with the same message multiset.
"""
import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine
from irexec import eval_trees, run_moves
from oracle import port
from oracle.common import expected

CASES = [([8], 100), ([8], 1000), ([16], 3), ([6], 5), ([7], 64), ([4, 4], 77), ([5, 3], 999), ([2, 3, 4], 1001),
         ([4, 4, 4], 64 * 6 * 3 + 5), ([2, 2, 2], 48), ([32], 4096 + 7), ([2, 8], 40), ([3, 2, 2], 17)]


def comm_for(dims):
    P = int(np.prod(dims))
    comm = bine.Comm(P, dims if len(dims) > 1 else None)
    comm.set_algo("allreduce", "B", "RING")
    return comm, P


def oracle_run(x, count, dims, trace=False):
    return port.run("allreduce", x, count, family="RING", dims=dims if len(dims) > 1 else None, trace=trace)


@pytest.mark.parametrize("dims,count", CASES, ids=lambda v: str(v))
def test_ring_oracle_computes_the_mpi_sum(dims, count):
    P = int(np.prod(dims))
    rng = np.random.default_rng(P * 1000 + count)
    x = rng.integers(-1000, 1001, (P, count)).astype(np.int32)
    out, _ = oracle_run(x, count, dims)
    assert np.array_equal(out, expected("allreduce", x, P, count))
    xf = rng.standard_normal((P, count)).astype(np.float32)
    outf, _ = oracle_run(xf, count, dims)
    err = np.abs(outf.astype(np.float64) - xf.astype(np.float64).sum(0))
    assert (err <= P * 2.0 ** -24 * np.abs(xf.astype(np.float64)).sum(0) + 1e-30).all()


@pytest.mark.parametrize("dims,count", CASES, ids=lambda v: str(v))
def test_ring_schedule_matches_the_oracle_bit_for_bit(dims, count):
    comm, P = comm_for(dims)
    comm.plan_verify("allreduce", count)
    for dt in (np.int32, np.float32):
        rng = np.random.default_rng(P + count)
        x = (rng.integers(-1000, 1001, (P, count)) if dt == np.int32 else rng.standard_normal((P, count))).astype(dt)
        want, msgs = oracle_run(x, count, dims, trace=True)
        assert np.array_equal(run_moves(comm, "allreduce", count, x).view(np.uint32), want.view(np.uint32))
        if dt == np.float32:
            assert np.array_equal(eval_trees(comm, "allreduce", count, x).view(np.uint32), want.view(np.uint32))
        pm = comm.plan_messages("allreduce", count)
        mine = sorted(zip(pm[:, 1].tolist(), pm[:, 2].tolist(), (pm[:, 3] * 4).tolist()))
        theirs = sorted(zip(msgs["src"].tolist(), msgs["dst"].tolist(), msgs["bytes"].astype(np.int64).tolist()))
        assert mine == theirs
    comm.close()


def test_ring_step_structure():
    """A 1-D ring of P: two buckets (one per direction), P - 1 reduce-scatter
    and P - 1 allgather steps, each step one message per rank and bucket;
    the work-row copy and the receive-row copy are levels of their own."""
    comm, P = comm_for([8])
    count = 8 * 2 * 10
    st = comm.plan_stats("allreduce", count)
    assert st["levels"] == 1 + (P - 1) + 1 + (P - 1)
    pm = comm.plan_messages("allreduce", count)
    assert len(pm) == 2 * (P - 1) * 2 * P
    assert set((pm[:, 2] - pm[:, 1]) % P) == {1, P - 1}  # neighbours only
    assert set(pm[:, 3]) == {count // 2 // P}
    comm.close()


@pytest.mark.parametrize("coll,line", [("reduce_scatter", "lib/libbine_coll_reduce_scatter.cc:826"),
                                       ("allgather", "lib/libbine_coll_allgather.cc:1514"),
                                       ("bcast", "lib/libbine.cc:1284")])
def test_ring_family_elsewhere_is_refused_with_the_reason(coll, line):
    comm = bine.Comm(8)
    comm.set_algo(coll, list(bine.VARIANTS[coll])[0], "RING")
    with pytest.raises(bine.Unsupported) as e:
        comm.plan_stats(coll, 16)
    assert line in str(e.value)
    comm.close()


def test_ring_link_bytes_use_neighbour_links_only():
    """Every ring message crosses one link of its dimension: on a 4x4 torus
    each directed link carries the same bytes."""
    comm, P = comm_for([4, 4])
    count = 4 * 16 * 12
    lb = comm.link_bytes_host("allreduce", count, bine.INT32)
    msgs = comm.plan_messages("allreduce", count)
    assert int(lb.sum()) == int(msgs[:, 3].sum()) * 4
    assert len(set(lb.tolist())) == 1
    comm.close()
