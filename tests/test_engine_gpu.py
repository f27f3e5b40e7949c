"""GPU parity of the engine, through the C ABI, against the reference.

* Every golden case (outputs of the reference library itself) is run on the
  FUSED, STEPS and PIPELINED engines and compared bit for bit, float32
  included.
* Larger cases are compared with the oracle (the C++ restatement).
* Full-size properties (P = 256, 4 MiB per rank) use exact integer sums and
  the FP64 tolerance of the reordered float path.
Bit-exactness excludes NaN payloads (no input here produces NaNs).
"""
import numpy as np
import pytest
import torch

import bine_trees_fugaku_b200 as bine
from golden_data import load_ref_collectives
from oracle import port
from oracle.common import buffer_counts, expected, receiving_ranks
from tests.golden.cases import case_input

pytestmark = pytest.mark.gpu

CASES = load_ref_collectives()
NP2CODE = {np.dtype(np.int32): bine.INT32, np.dtype(np.int64): bine.INT64, np.dtype(np.float32): bine.FLOAT,
           np.dtype(np.float64): bine.DOUBLE, np.dtype(np.int8): bine.CHAR}


def make_comm(P, coll, variant, dims=None, ports=1, family="BINE", distance=None, engine="fused", order="reference"):
    comm = bine.Comm(P, dims)
    comm.set_ports(ports)
    comm.set_algo(coll, variant, family, distance)
    comm.set_engine(engine)
    comm.set_float_order(order)
    comm.set_stream(torch.cuda.current_stream())
    return comm


def run(comm, coll, x, count, root=0):
    P = x.shape[0]
    _, rc = buffer_counts(coll, count, P)
    send = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    recv = torch.zeros((P, rc), dtype=send.dtype, device="cuda")
    if coll == "bcast":
        recv[root] = send[root]
    comm.run(coll, send, recv, count, NP2CODE[x.dtype], root)
    comm.synchronize()
    return recv.cpu().numpy()


def case_id(c):
    return (f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-d{c.get('dims')}-p{c.get('ports', 1)}"
            f"-r{c.get('root', 0)}-{c.get('family', 'BINE')}")


@pytest.mark.parametrize("engine", ["fused", "steps", "pipelined", "pipelined-seg256", "pipelined-fuse3",
                                    "pipelined-fuse6-seg256", "pipelined-fuse64"])
@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_engine_matches_reference(case, engine):
    x = case_input(case)
    root = case.get("root", 0)
    segment = 256 if engine.endswith("seg256") else 0  # many small segments, level dependencies
    fusion = int(engine.split("-fuse")[1].split("-")[0]) if "-fuse" in engine else 1  # levels per pass
    engine = engine.split("-")[0]
    comm = make_comm(case["P"], case["coll"], case["variant"], case.get("dims"), case.get("ports", 1),
                     case.get("family", "BINE"), case.get("distance"), engine)
    comm.set_segment(segment)
    comm.set_fusion(fusion)
    rr = receiving_ranks(case["coll"], case["P"], root)
    reduction = case["coll"] in ("allreduce", "reduce_scatter", "reduce")
    right = reference_is_right(case, x)
    try:
        out = run(comm, case["coll"], x, case["count"], root)
    except bine.Unsupported:
        # Only cases where the reference fails or returns wrong data may be
        # refused, and only by the engine that follows the reference's
        # schedule or by the exact float order.
        assert engine in ("steps", "pipelined") or (reduction and case["dtype"] == "float")
        assert not right
        return
    if right:
        assert np.array_equal(out[rr].view(np.uint8), case["out"][rr].view(np.uint8))
    else:
        # Reference-unsupported: MPI semantics (exact for integers and copies).
        exp = expected(case["coll"], x, case["P"], case["count"], root)
        assert np.array_equal(out[rr], exp[rr])


def reference_is_right(case, x):
    """The reference ran this case, without undefined behaviour, and returned
    the MPI result (exactly for integers and copies, to 1e-4 for float sums
    whose order differs from an FP64 sum)."""
    if not case["ok"]:
        return False
    try:
        port.run(case["coll"], x, case["count"], variant=case["variant"], dims=case.get("dims"),
                 ports=case.get("ports", 1), root=case.get("root", 0), family=case.get("family", "BINE"),
                 distance=case.get("distance"))
    except port.ReferenceUnsupported:
        return False
    root = case.get("root", 0)
    rr = receiving_ranks(case["coll"], case["P"], root)
    exp = expected(case["coll"], x, case["P"], case["count"], root)
    if case["dtype"] == "float" and case["coll"] in ("allreduce", "reduce_scatter", "reduce"):
        return bool(np.allclose(case["out"][rr], exp[rr], rtol=1e-4, atol=1e-4))
    return bool(np.array_equal(case["out"][rr], exp[rr]))


@pytest.mark.parametrize("engine", ["fused", "steps", "pipelined"])
@pytest.mark.parametrize("coll,variant,P,count,dims,ports", [
    ("allreduce", "B", 64, 64 * 1000 + 13, None, 1),
    ("allreduce", "B", 96, 96 * 512, None, 1),
    ("allreduce", "B_COALESCE", 48, 48 * 777, None, 2),
    ("allreduce", "B_CONT", 128, 128 * 256, None, 1),
    ("allreduce", "L", 64, 50_000, None, 1),
    ("allreduce", "L", 72, 30_000, [6, 12], 2),
    ("allreduce", "B", 64, 64 * 600, [4, 4, 4], 6),
    ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 64, 1024, None, 1),
    ("reduce", "BINOMIAL_TREE", 64, 20_000, None, 1),
    ("reduce", "REDUCE_SCATTER_GATHER", 32, 20_001, None, 1),
    # Block boundaries off the 16-byte grid: vector bodies plus element
    # heads and tails.
    ("allreduce", "B", 96, 50_000, None, 1),
    ("allreduce", "B_COALESCE", 48, 48 * 777 + 5, None, 2),
    ("allreduce", "L", 72, 30_001, [6, 12], 2),
    ("allreduce", "B", 384, 131_072, None, 1),
    ("allreduce", "B", 1000, 64_007, None, 1),  # programs of 1,000 leaves: over 48 KB of shared memory
    # Row-aligned tiles holding the ends of several segments (one tree
    # shape, ranks per lane): 2 to 8 segments per tile.
    ("allreduce", "B", 96, 96 * 40 + 3, None, 1),
    ("allreduce", "B", 384, 384 * 100 + 1, None, 1),
    ("allreduce", "B", 200, 200 * 1000 + 17, None, 1),
    ("allreduce", "B", 1000, 1000 * 130 + 3, None, 1),
    ("allreduce", "B_COALESCE", 96, 96 * 333 + 5, None, 1),
    # Several tree shapes: row tiles per shape side by side, edges between
    # segments of different shapes.
    ("allreduce", "B", 46, 46 * 2000 + 1, None, 1),
    ("allreduce", "B", 76, 76 * 3000 + 5, None, 1),
    ("allreduce", "B", 118, 118 * 500 + 3, None, 1),
    ("allreduce", "B", 70, 70 * 1000 + 9, None, 1),
])
def test_float_exact_order_large(engine, coll, variant, P, count, dims, ports):
    sc, _ = buffer_counts(coll, count, P)
    x = np.random.default_rng(P + count).standard_normal((P, sc)).astype(np.float32)
    expect, _ = port.run(coll, x, count, variant=variant, dims=dims, ports=ports)
    comm = make_comm(P, coll, variant, dims, ports, engine=engine)
    out = run(comm, coll, x, count)
    rr = receiving_ranks(coll, P)
    assert np.array_equal(out[rr].view(np.uint32), expect[rr].view(np.uint32))


@pytest.mark.parametrize("P,count,form", [
    (96, 96 * 40 + 3, 3), (384, 384 * 100 + 1, 3), (1000, 1000 * 130 + 3, 3),
    (200, 200 * 1000 + 17, 3),  # three tree shapes (10, 82 and 108 segments)
    (76, 76 * 3000 + 5, 3),     # seven shapes
    (70, 70 * 1000 + 9, 2),     # nine shapes: more than a call may have
    (96, 524_288, 3), (384, 524_288, 3), (1000, 1_048_576, 3),
    (256, 1 << 20, 3),   # power of two: segments on the grid already, one shape
    (96, 96 * 8, 2),     # 2-vector segments: a 32-vector tile would touch 16
])
def test_row_aligned_tiles_are_used(P, count, form):
    """The exact-order allreduce plans row-aligned tiles (form 3) where the
    trees have at most 8 shapes and a tile touches at most 8 segments of
    one shape, and keeps per-segment tiles otherwise (more shapes, or short
    segments); the cases above that compare bits with the oracle therefore
    run both."""
    comm = make_comm(P, "allreduce", "B")
    got, lanes = comm.tree_form("allreduce", count, bine.FLOAT)
    assert (got, lanes > 1) == (form, True)


@pytest.mark.parametrize("lanes", [1, 2, 4, 8])
@pytest.mark.parametrize("coll,variant,P,count,dims,ports", [
    ("allreduce", "B", 256, 256 * 64, None, 1),
    ("allreduce", "B", 96, 50_000, None, 1),
    ("allreduce", "B", 96, 96 * 512, None, 1),
    ("allreduce", "B_COALESCE", 48, 48 * 776, None, 2),
    ("allreduce", "L", 64, 50_000, None, 1),
    ("allreduce", "L", 72, 30_000, [6, 12], 2),
    ("allreduce", "B", 64, 64 * 600, [4, 4, 4], 6),
    ("allreduce", "B", 384, 384 * 100 + 1, None, 1),
    ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 64, 1024, None, 1),
    ("reduce", "BINOMIAL_TREE", 64, 20_000, None, 1),
])
def test_float_exact_order_split_lanes(lanes, coll, variant, P, count, dims, ports):
    """The exact-order float kernel with every lane count per output vector
    (the tree cut into 1, 2, 4 or 8 subtrees and recombined by shuffles)
    returns the oracle's bits."""
    sc, _ = buffer_counts(coll, count, P)
    x = np.random.default_rng(P * 7 + count).standard_normal((P, sc)).astype(np.float32)
    expect, _ = port.run(coll, x, count, variant=variant, dims=dims, ports=ports)
    comm = make_comm(P, coll, variant, dims, ports)
    comm.set_tree_split(lanes)
    out = run(comm, coll, x, count)
    rr = receiving_ranks(coll, P)
    assert np.array_equal(out[rr].view(np.uint32), expect[rr].view(np.uint32))


@pytest.mark.parametrize("coll", ["allgather", "bcast", "alltoall", "scatter", "gather"])
@pytest.mark.parametrize("P,count,dt", [(64, 4096, np.float32), (32, 1001, np.int64), (16, 37, np.int8),
                                        (256, 1024, np.int32)])
def test_copies_large(coll, P, count, dt):
    sc, _ = buffer_counts(coll, count, P)
    x = (np.random.default_rng(P).standard_normal((P, sc)) * 100).astype(dt)
    root = 3 % P
    comm = make_comm(P, coll, list(bine.VARIANTS[coll])[0])
    out = run(comm, coll, x, count, root)
    rr = receiving_ranks(coll, P, root)
    assert np.array_equal(out[rr], expected(coll, x, P, count, root)[rr])


def test_full_size_int32_allreduce_is_exact():
    """P = 256 virtual ranks, 4 MiB of int32 each (the benchmark workload)."""
    P, count = 256, 1 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    send = torch.randint(-1000, 1001, (P, count), dtype=torch.int32, device="cuda", generator=g)
    recv = torch.empty_like(send)
    comm = make_comm(P, "allreduce", "B")
    comm.allreduce(send, recv, count, bine.INT32)
    comm.synchronize()
    expect = send.sum(0, dtype=torch.int64).to(torch.int32)
    assert torch.equal(recv, expect.expand(P, count))


@pytest.mark.parametrize("engine", ["steps", "pipelined"])
@pytest.mark.parametrize("P,count", [(256, 1 << 18), (1024, 1 << 14)])
def test_full_size_int32_allreduce_steps_engine(P, count, engine):
    g = torch.Generator(device="cuda")
    g.manual_seed(2)
    send = torch.randint(-1000, 1001, (P, count), dtype=torch.int32, device="cuda", generator=g)
    recv = torch.empty_like(send)
    comm = make_comm(P, "allreduce", "B", engine=engine)
    comm.allreduce(send, recv, count, bine.INT32)
    comm.synchronize()
    assert torch.equal(recv, send.sum(0, dtype=torch.int64).to(torch.int32).expand(P, count))


def test_fast_float_order_within_1e6_of_fp64():
    """Reordered float32 path: |y - y64| <= 1e-6 |y64| elementwise, y64 the FP64 sum."""
    P, count = 256, 1 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    send = torch.randn((P, count), dtype=torch.float32, device="cuda", generator=g)
    recv = torch.empty_like(send)
    comm = make_comm(P, "allreduce", "B", order="fast")
    comm.allreduce(send, recv, count, bine.FLOAT)
    comm.synchronize()
    y64 = send.double().sum(0)
    err = (recv[0].double() - y64).abs()
    assert bool((err <= 1e-6 * y64.abs() + 1e-30).all())
    assert torch.equal(recv[0], recv[-1])


def test_full_size_float_reference_order_matches_oracle_columns():
    """P = 256, 4 MiB float32 per rank in the reference order; sampled
    columns are checked against the oracle run on the same columns' blocks."""
    P, count = 256, 1 << 20
    x = np.random.default_rng(4).standard_normal((P, count)).astype(np.float32)
    comm = make_comm(P, "allreduce", "B")
    send = torch.from_numpy(x).cuda()
    recv = torch.empty_like(send)
    comm.allreduce(send, recv, count, bine.FLOAT)
    comm.synchronize()
    got = recv[0].cpu().numpy()
    # The reference's block b of rank r covers the same columns for every
    # count that is a multiple of P: run the oracle on 4 columns per block.
    blk = count // P
    cols = np.concatenate([b * blk + np.array([0, 1, blk // 2, blk - 1]) for b in range(P)])
    small = x[:, cols]
    expect, _ = port.run("allreduce", small, small.shape[1], variant="B")
    assert np.array_equal(got[cols].view(np.uint32), expect[0].view(np.uint32))
    assert torch.equal(recv[0], recv[P - 1])


def test_in_place_and_strided_layouts():
    P, count = 32, 4099  # odd count: element-wise tail path
    x = np.random.default_rng(5).integers(-1000, 1001, (P, count)).astype(np.int32)
    comm = make_comm(P, "allreduce", "B")
    buf = torch.from_numpy(x).cuda()
    comm.allreduce(buf, buf, count, bine.INT32)  # MPI_IN_PLACE
    comm.synchronize()
    assert np.array_equal(buf.cpu().numpy(), expected("allreduce", x, P, count))
    stride = 8192 * 4
    big = torch.zeros((P, 8192), dtype=torch.int32, device="cuda")
    big[:, :count] = torch.from_numpy(x).cuda()
    out = torch.zeros_like(big)
    comm.set_layout(stride, stride)
    comm.allreduce(big, out, count, bine.INT32)
    comm.synchronize()
    assert np.array_equal(out[:, :count].cpu().numpy(), expected("allreduce", x, P, count))
    assert int(out[:, count:].abs().sum()) == 0


@pytest.mark.parametrize("engine", ["steps", "pipelined"])
def test_step_engine_barrier_timeout_is_reported_and_recoverable(engine):
    """A wait that can never end (fault injected on the host: a grid barrier
    waiting for one arrival too many, or a segment waiting for a completion
    value no segment writes) expires after the configured bound; the engine
    reports BINE_ERR_TIMEOUT and the next call works."""
    P, count = 16, 16 * 64
    x = np.random.default_rng(6).integers(-1000, 1001, (P, count)).astype(np.int32)
    comm = make_comm(P, "allreduce", "B", engine=engine)
    comm.set_step_timeout(200)
    comm.debug_set_barrier_extra(1)
    send = torch.from_numpy(x).cuda()
    recv = torch.zeros_like(send)
    comm.allreduce(send, recv, count, bine.INT32)
    with pytest.raises(bine.Timeout):
        comm.synchronize()
    comm.debug_set_barrier_extra(0)
    comm.allreduce(send, recv, count, bine.INT32)
    comm.synchronize()
    assert np.array_equal(recv.cpu().numpy(), expected("allreduce", x, P, count))


@pytest.mark.parametrize("dims,coll,variant,ports,family", [
    ([8], "allreduce", "B", 1, "BINE"), ([4, 4], "allreduce", "B", 2, "BINE"), ([2, 2, 2], "allreduce", "B", 6, "BINE"),
    ([4, 4, 4], "allreduce", "B", 6, "BINE"), ([4, 4, 4], "allreduce", "L", 1, "BINE"),
    ([4, 4, 4], "allreduce", "L", 1, "RECDOUB"), ([8, 8], "allreduce", "B", 1, "RECDOUB"),
    ([4, 8], "allgather", "VEC_DOUBLING_CONT_PERMUTE", 1, "BINE"), ([6, 4], "allreduce", "B", 1, "BINE"),
    ([4, 4, 4], "alltoall", "LOG", 1, "BINE"), ([16], "bcast", "BINOMIAL_TREE", 1, "BINE"),
    ([4, 4], "allreduce", "B", 1, "RING"), ([2, 4, 8], "allreduce", "B", 1, "RING"),
])
def test_device_link_bytes_match_host(dims, coll, variant, ports, family):
    P = int(np.prod(dims))
    comm = bine.Comm(P, dims)
    comm.set_ports(ports)
    comm.set_algo(coll, variant, family)
    comm.set_stream(torch.cuda.current_stream())
    count = P * ports * 37 + 5 if coll == "allreduce" else 13
    host = comm.link_bytes_host(coll, count, bine.FLOAT)
    out = torch.zeros(len(host), dtype=torch.int64, device="cuda")
    comm.link_bytes(coll, count, bine.FLOAT, out)
    comm.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), host)


@pytest.mark.parametrize("dims", [[64, 64], [32, 256], [8, 8, 8]])
@pytest.mark.parametrize("variant,ports", [("B", 1), ("B", 6), ("L", 1)])
def test_device_link_bytes_large_tori_conserve_volume(dims, variant, ports):
    """1 MiB per rank on the largest tori: the total over links equals the
    sum over messages of bytes x minimal hops, computed here from the step
    distances (rho_k on the ring of each step's dimension)."""
    P = int(np.prod(dims))
    count = (1 << 20) // 4
    comm = bine.Comm(P, dims)
    comm.set_ports(ports)
    comm.set_algo("allreduce", variant)
    comm.set_stream(torch.cuda.current_stream())
    out = torch.zeros(P * len(dims) * 2, dtype=torch.int64, device="cuda")
    comm.link_bytes("allreduce", count, bine.INT32, out)
    comm.synchronize()
    total = int(out.sum())
    rho = lambda k: (1 - (-2) ** (k + 1)) // 3
    expect = 0
    for port in range(ports):
        cp = count // ports + (port < count % ports)
        # steps round-robin over dims starting at port % ndims
        seq, nxt, cur = [], [0] * len(dims), port % len(dims)
        S = sum(int(np.log2(d)) for d in dims)
        for i in range(S):
            seq.append((cur, nxt[cur]))
            nxt[cur] += 1
            if i != S - 1:
                cur = (cur + 1) % len(dims)
                while nxt[cur] >= int(np.log2(dims[cur])):
                    cur = (cur + 1) % len(dims)
        for i, (d, k) in enumerate(seq):
            L = dims[d]
            dist = rho(k) % L
            hops = min(dist, L - dist)
            if variant == "L":
                expect += P * cp * 4 * hops
            else:
                # Every block of the port is sent by P/2^(i+1) ranks at
                # reduce-scatter step i, and comes back in the allgather.
                expect += 2 * ((P * cp * 4) >> (i + 1)) * hops
    assert total == expect


def test_batched_launch_matches_semantics_and_single_calls():
    """A mixed batch in one persistent launch: integer results equal the
    single-call results bit for bit, float32 sums are within 1e-6 of FP64."""
    rng = np.random.default_rng(9)
    items, xs, outs = [], [], []
    for k in range(300):
        coll = ["allreduce", "reduce_scatter", "allgather"][k % 3]
        P = int(rng.integers(4, 65))
        c = int(rng.integers(1, 64)) * 4
        fl = bool(k % 2)
        sc, rc = buffer_counts(coll, c, P)
        x = rng.standard_normal((P, sc)).astype(np.float32) if fl else \
            rng.integers(-1000, 1001, (P, sc)).astype(np.int32)
        send = torch.from_numpy(x).cuda()
        out = torch.zeros((P, rc), dtype=send.dtype, device="cuda")
        items.append((coll, send, out, c, bine.FLOAT if fl else bine.INT32, P))
        xs.append(x)
        outs.append(out)
    best, ms = bine.Batch.autotune(items, torch.cuda.current_stream(), reps=1)
    assert ms > 0
    b = bine.Batch(items, best)
    b.launch(torch.cuda.current_stream())
    torch.cuda.synchronize()
    for (coll, send, out, c, dt, P), x in zip(items, xs):
        got = out.cpu().numpy()
        if dt == bine.INT32:
            assert np.array_equal(got, expected(coll, x, P, c))
            single = torch.zeros_like(out)
            cm = make_comm(P, coll, list(bine.VARIANTS[coll])[0])
            cm.run(coll, send, single, c, dt)
            cm.synchronize()
            assert torch.equal(single, out)
        else:
            exp64 = x.astype(np.float64)
            if coll == "allgather":
                assert np.array_equal(got, expected(coll, x, P, c))
            else:
                full = exp64.sum(0)
                ref = np.tile(full, (P, 1)) if coll == "allreduce" else full.reshape(P, c)
                assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-30)
    b.close()


@pytest.mark.parametrize("P,count,dt", [(256, (1 << 16) + 13, np.int32), (64, 300_000, np.int64), (7, 5, np.int8),
                                        (512, 40_000, np.int32)])
def test_allreduce_host_buffers_integers(P, count, dt):
    """bine_allreduce_host on pinned host tensors: several column windows,
    a ragged last window, exact integer sums (wrapping like C)."""
    rng = np.random.default_rng(P + count)
    x = rng.integers(-100, 101, (P, count)).astype(dt)
    send = torch.from_numpy(x).pin_memory()
    recv = torch.zeros_like(send).pin_memory()
    comm = make_comm(P, "allreduce", "B")
    comm.allreduce_host(send, recv, count, NP2CODE[x.dtype])
    assert np.array_equal(recv.numpy(), expected("allreduce", x, P, count))


@pytest.mark.parametrize("split", [0, 1, 8])
def test_allreduce_host_buffers_float_reference_order(split):
    """Exact-order float through column windows (P=256: 32,768 columns per
    window) returns the device call's bits."""
    P, count = 256, 256 * 200
    x = np.random.default_rng(11).standard_normal((P, count)).astype(np.float32)
    comm = make_comm(P, "allreduce", "B")
    comm.set_tree_split(split)
    dev = run(comm, "allreduce", x, count)
    send = torch.from_numpy(x).pin_memory()
    recv = torch.zeros_like(send).pin_memory()
    comm.allreduce_host(send, recv, count, bine.FLOAT)
    assert np.array_equal(recv.numpy().view(np.uint32), dev.view(np.uint32))


@pytest.mark.parametrize("P,count", [(96, 96 * 333 + 7), (1000, 1000 * 262 + 11), (200, 200 * 700 + 3)])
def test_allreduce_host_buffers_float_row_aligned_tiles(P, count):
    """Non-power-of-two P, exact float order through column windows: the
    row-aligned tiles clipped at window edges return the device call's
    bits."""
    x = np.random.default_rng(P + 5).standard_normal((P, count)).astype(np.float32)
    comm = make_comm(P, "allreduce", "B")
    dev = run(comm, "allreduce", x, count)
    send = torch.from_numpy(x).pin_memory()
    recv = torch.zeros_like(send).pin_memory()
    comm.set_host_window(1 << 20)
    comm.allreduce_host(send, recv, count, bine.FLOAT)
    assert np.array_equal(recv.numpy().view(np.uint32), dev.view(np.uint32))


def test_allreduce_host_pageable_in_place_and_strided():
    P, count = 16, 5000
    x = np.random.default_rng(3).integers(-1000, 1001, (P, count)).astype(np.int32)
    comm = make_comm(P, "allreduce", "B")
    buf = x.copy()  # pageable numpy memory, in place
    comm.allreduce_host(buf, buf, count, bine.INT32)
    assert np.array_equal(buf, expected("allreduce", x, P, count))
    big = np.zeros((P, 6000), np.int32)
    big[:, :count] = x
    out = np.full((P, 6000), 7, np.int32)
    comm.set_layout(6000 * 4, 6000 * 4)
    comm.allreduce_host(big, out, count, bine.INT32)
    assert np.array_equal(out[:, :count], expected("allreduce", x, P, count))
    assert np.all(out[:, count:] == 7)


@pytest.mark.parametrize("engine", ["fused", "steps", "pipelined"])
@pytest.mark.parametrize("coll", bine.COLLS)
def test_zero_and_ragged_counts(engine, coll):
    """count 0 leaves every output byte as it was; counts below P (1 and
    3 elements per rank) give the MPI result, or, on the engine that follows
    the reference's schedule, a clean refusal where the reference cannot
    run them."""
    P, root = 16, 0
    comm = make_comm(P, coll, list(bine.VARIANTS[coll])[0], engine=engine)
    sentinel = torch.full((P, 64), 7, dtype=torch.int32, device="cuda")
    comm.run(coll, sentinel.clone(), sentinel, 0, bine.INT32, root)
    comm.synchronize()
    assert int((sentinel != 7).sum()) == 0
    for count in (1, 3):
        sc, _ = buffer_counts(coll, count, P)
        x = np.random.default_rng(count).integers(-1000, 1001, (P, sc)).astype(np.int32)
        try:
            out = run(comm, coll, x, count, root)
        except bine.Unsupported:
            assert engine in ("steps", "pipelined")
            continue
        rr = receiving_ranks(coll, P, root)
        assert np.array_equal(out[rr], expected(coll, x, P, count, root)[rr])


def test_pipelined_engine_repeated_launches_and_graph_replay():
    """The pipelined kernel leaves its completion state ready for the next
    launch: back-to-back calls, and replays of a CUDA graph holding one
    call, give the exact sums each time, with inputs changed in between."""
    P, count = 64, 64 * 1000
    comm = make_comm(P, "allreduce", "B", engine="pipelined")
    g = torch.Generator(device="cuda")
    g.manual_seed(8)
    send = torch.randint(-1000, 1001, (P, count), dtype=torch.int32, device="cuda", generator=g)
    recv = torch.empty_like(send)
    for k in range(3):
        send.add_(k)
        comm.allreduce(send, recv, count, bine.INT32)
        comm.synchronize()
        assert torch.equal(recv, send.sum(0, dtype=torch.int64).to(torch.int32).expand(P, count))
    stream = torch.cuda.Stream()
    comm.set_stream(stream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        comm.allreduce(send, recv, count, bine.INT32)
    for k in range(3):
        send.mul_(-1).add_(k)
        recv.zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(recv, send.sum(0, dtype=torch.int64).to(torch.int32).expand(P, count))
    comm.synchronize()


def test_hooked_host_allreduce_runs_windows_in_order_and_can_be_abandoned():
    """bine_allreduce_host_hooked: the hooks see consecutive column windows
    covering the call, before-window ahead of after-window; results equal
    bine_allreduce_host's; a hook that returns nonzero abandons the call
    with BINE_ERR_ABORTED and the next call works."""
    P, count = 8, 50_000
    x = torch.randint(-1000, 1001, (P, count), dtype=torch.int32).pin_memory()
    plain, hooked = torch.empty_like(x).pin_memory(), torch.zeros_like(x).pin_memory()
    comm = make_comm(P, "allreduce", "B")
    comm.set_host_window(64 << 10)  # several windows
    comm.allreduce_host(x, plain, count, bine.INT32)
    seen = []
    comm.allreduce_host_hooked(x, hooked, count, bine.INT32, before=lambda f, n: seen.append(("in", f, n)),
                               after=lambda f, n: seen.append(("out", f, n)))
    assert torch.equal(hooked, plain)
    assert torch.equal(plain, x.sum(0, dtype=torch.int64).to(torch.int32).expand(P, count))
    for kind in ("in", "out"):
        w = [(f, n) for k, f, n in seen if k == kind]
        assert len(w) > 2 and w[0][0] == 0 and all(a[0] + a[1] == b[0] for a, b in zip(w, w[1:]))
        assert w[-1][0] + w[-1][1] == count
    order = [(k, f) for k, f, _ in seen]
    assert all(order.index(("in", f)) < order.index(("out", f)) for _, f, _ in seen)
    with pytest.raises(bine.BineError) as e:
        comm.allreduce_host_hooked(x, hooked, count, bine.INT32, before=lambda f, n: f > 0)
    assert e.value.code == bine.ERR_ABORTED
    hooked.zero_()
    comm.allreduce_host_hooked(x, hooked, count, bine.INT32)
    assert torch.equal(hooked, plain)


@pytest.mark.parametrize("engine", ["steps", "pipelined"])
@pytest.mark.parametrize("variant,P", [("B", 16), ("B", 24), ("L", 4), ("L", 16), ("L", 24), ("B_COALESCE", 12)])
def test_in_place_allreduce_on_the_step_engines(engine, variant, P):
    """MPI_IN_PLACE (sendbuf == recvbuf) on the engines that run the
    reference's schedule: the L butterfly reads a peer's input in the step
    that writes the peer's result, so the input rows are staged first; two
    calls in a row give the out-of-place bytes, float32 included."""
    count = P * 37 + 5
    for dt, code in ((np.int32, bine.INT32), (np.float32, bine.FLOAT)):
        rng = np.random.default_rng(P)
        x = (rng.integers(-1000, 1001, (P, count)) if dt == np.int32 else rng.standard_normal((P, count))).astype(dt)
        comm = make_comm(P, "allreduce", variant, engine=engine)
        send = torch.from_numpy(x).cuda()
        expect = torch.empty_like(send)
        comm.allreduce(send, expect, count, code)
        for _ in range(2):
            buf = send.clone()
            comm.allreduce(buf, buf, count, code)
            comm.synchronize()
            assert torch.equal(buf.view(torch.uint8), expect.view(torch.uint8))


@pytest.mark.parametrize("coll,P,count", [
    ("reduce_scatter", 1024, 8), ("reduce_scatter", 256, 4), ("allreduce", 512, 64), ("allreduce", 64, 32),
    ("reduce", 1024, 16), ("allgather", 1024, 8), ("allgather", 300, 4), ("bcast", 512, 8), ("bcast", 1000, 12),
])
def test_small_calls_at_large_p(coll, P, count):
    """Few output columns at large P: column tiles of 16 or 8 columns (16 or
    32 row groups) for the sums, destination groups for allgather and
    bcast; results exact."""
    comm = make_comm(P, coll, list(bine.VARIANTS[coll])[0])
    for dt in (np.int32, np.int64):
        sc, _ = buffer_counts(coll, count, P)
        x = np.random.default_rng(P + count).integers(-1000, 1001, (P, sc)).astype(dt)
        out = run(comm, coll, x, count, 0)
        rr = receiving_ranks(coll, P, 0)
        assert np.array_equal(out[rr], expected(coll, x, P, count, 0)[rr])


@pytest.mark.parametrize("engine", ["fused", "steps", "pipelined"])
@pytest.mark.parametrize("coll", ["allreduce", "reduce_scatter", "reduce", "allgather", "alltoall", "scatter", "gather"])
@pytest.mark.parametrize("layout", ["same_base", "offset_rows"])
def test_overlapping_arrays_match_separate_arrays(engine, coll, layout):
    """Input and output arrays that share bytes: the same base address with
    each array's own packed rows (MPI_IN_PLACE-like), or output rows that
    start one input row further on.  Such calls stage their input rows first
    (except an allreduce or reduce on the FUSED engine whose arrays are one),
    so every engine gives the bytes of separate arrays, float32 included."""
    P = 16
    count = P * 37 + 5 if coll == "allreduce" else 37
    sc, rc = buffer_counts(coll, count, P)
    variant = list(bine.VARIANTS[coll])[0]
    comm = make_comm(P, coll, variant, engine=engine)
    rr = receiving_ranks(coll, P, 0)
    for dt, code in ((np.int32, bine.INT32), (np.float32, bine.FLOAT)):
        rng = np.random.default_rng(P + sc)
        x = (rng.integers(-1000, 1001, (P, sc)) if dt == np.int32 else rng.standard_normal((P, sc))).astype(dt)
        want = run(comm, coll, x, count)
        shift = 0 if layout == "same_base" else sc
        tdt = torch.int32 if dt == np.int32 else torch.float32
        flat = torch.zeros(shift + P * max(sc, rc), dtype=tdt, device="cuda")
        for _ in range(2):
            flat.zero_()
            flat[:P * sc] = torch.from_numpy(x.ravel()).cuda()
            send, recv = flat[:P * sc], flat[shift:shift + P * rc]
            comm.run(coll, send, recv, count, code, 0)
            comm.synchronize()
            got = recv.view(P, rc).cpu().numpy()
            assert np.array_equal(got[rr].view(np.uint32), want[rr].view(np.uint32)), (dt, layout)


@pytest.mark.parametrize("engine", ["fused", "steps", "pipelined"])
@pytest.mark.parametrize("dims,count", [([8], 1000), ([4, 4], 77), ([2, 3, 4], 1001), ([256], 256 * 2 * 64 + 3),
                                        ([8, 8, 4], 256 * 6 * 8 + 1), ([6], 5)])
def test_ring_allreduce_matches_the_oracle(engine, dims, count):
    """The bucket (ring) allreduce, the reference's RING family, on every
    engine: the oracle's bytes, float32 in its addition order included."""
    P = int(np.prod(dims))
    comm = make_comm(P, "allreduce", "B", dims=dims if len(dims) > 1 else None, family="RING", engine=engine)
    for dt in (np.int32, np.float32):
        rng = np.random.default_rng(P + count)
        x = (rng.integers(-1000, 1001, (P, count)) if dt == np.int32 else rng.standard_normal((P, count))).astype(dt)
        want, _ = port.run("allreduce", x, count, family="RING", dims=dims if len(dims) > 1 else None)
        got = run(comm, "allreduce", x, count)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), dt
    comm.close()


@pytest.mark.parametrize("levels", [3, 6, 10])
@pytest.mark.parametrize("coll,variant,P,count", [
    ("allreduce", "B", 256, 256 * 64 + 7), ("allreduce", "B", 96, 96 * 40), ("allreduce", "L", 64, 4096),
    ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 128, 300), ("allgather", "VEC_DOUBLING_CONT_PERMUTE", 128, 301),
    ("alltoall", "LOG", 128, 33), ("bcast", "BINOMIAL_TREE", 128, 5000), ("reduce", "BINOMIAL_TREE", 64, 999)])
def test_fused_pipelined_engine_matches_the_level_by_level_engine(coll, variant, P, count, levels):
    """Level fusion on larger schedules: the PIPELINED engine with fused
    passes gives the STEPS engine's bytes (float32 in the reference order
    included), on two calls in a row and in place."""
    rr = receiving_ranks(coll, P, 0)
    for dt in (np.int32, np.float32):
        sc, _ = buffer_counts(coll, count, P)
        rng = np.random.default_rng(P + count + levels)
        x = (rng.integers(-1000, 1001, (P, sc)) if dt == np.int32 else rng.standard_normal((P, sc))).astype(dt)
        want = run(make_comm(P, coll, variant, engine="steps"), coll, x, count)
        comm = make_comm(P, coll, variant, engine="pipelined")
        comm.set_fusion(levels)
        for _ in range(2):
            got = run(comm, coll, x, count)
            assert np.array_equal(got[rr].view(np.uint8), want[rr].view(np.uint8)), (dt, levels)
        if coll == "allreduce":
            buf = torch.from_numpy(x).cuda()
            comm.allreduce(buf, buf, count, NP2CODE[x.dtype])
            comm.synchronize()
            assert np.array_equal(buf.cpu().numpy().view(np.uint8), want.view(np.uint8))


def test_fused_pipelined_engine_timeout_is_reported_and_recoverable():
    """The fused kernel's segment waits are bounded like the unfused ones."""
    P, count = 16, 16 * 64
    x = np.random.default_rng(6).integers(-1000, 1001, (P, count)).astype(np.int32)
    comm = make_comm(P, "allreduce", "B", engine="pipelined")
    comm.set_fusion(3)
    comm.set_step_timeout(200)
    comm.debug_set_barrier_extra(1)
    send = torch.from_numpy(x).cuda()
    recv = torch.zeros_like(send)
    comm.allreduce(send, recv, count, bine.INT32)
    with pytest.raises(bine.Timeout):
        comm.synchronize()
    comm.debug_set_barrier_extra(0)
    comm.allreduce(send, recv, count, bine.INT32)
    comm.synchronize()
    assert np.array_equal(recv.cpu().numpy(), expected("allreduce", x, P, count))
