"""Level fusion for the PIPELINED engine (bine_comm_set_fusion), on the CPU.

The fused form of a schedule (bine_plan_fused) groups consecutive levels
into passes whose moves evaluate, from the state at the start of the pass,
only what later passes read or what is a result; conflicting writes go to
fresh workspace slots.  Checked here, independently of the planner:

* executed with numpy, pass by pass, every fused schedule gives the
  reference library's own result bytes (tests/golden/ref_collectives.npz),
  float32 included, at several pass depths;
* fusion cuts the elements the engine reads and writes toward the
  algorithmic minimum;
* its dataflow plan (bine_plan_flow with fusion set) orders every
  cross-pass element conflict by a dependency path, no two moves of one
  pass conflict, and running the items in a random order the dependencies
  allow gives the reference's bytes.
"""
import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine
from golden_data import load_ref_collectives
from irexec import run_fused
from oracle.common import receiving_ranks
from tests.golden.cases import case_input

CASES = [c for c in load_ref_collectives() if c["ok"]]


def make_comm(case, levels=1, segment=0):
    comm = bine.Comm(case["P"], case.get("dims"))
    comm.set_ports(case.get("ports", 1))
    comm.set_algo(case["coll"], case["variant"], case.get("family", "BINE"), case.get("distance"))
    comm.set_segment(segment)
    comm.set_fusion(levels)
    return comm


def case_id(c):
    return (f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-d{c.get('dims')}-p{c.get('ports', 1)}"
            f"-r{c.get('root', 0)}-{c.get('family', 'BINE')}")


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_fused_schedules_give_the_reference_bytes(case):
    x = case_input(case)
    root = case.get("root", 0)
    comm = make_comm(case)
    try:
        comm.plan_verify(case["coll"], case["count"], root)
    except bine.Unsupported:
        return
    rr = receiving_ranks(case["coll"], case["P"], root)
    for levels in (1, 2, 3, 6, 64):
        got, _, _ = run_fused(comm, case["coll"], case["count"], x, root, levels)
        assert np.array_equal(got[rr].view(np.uint8), case["out"][rr].view(np.uint8)), levels


def algo_elems(coll, P, count):
    return {"allreduce": 2 * P * count, "alltoall": 2 * P * P * count, "reduce_scatter": P * P * count + P * count,
            "allgather": P * count + P * P * count, "bcast": P * count}[coll]


@pytest.mark.parametrize("coll,variant,P,count,levels,unfused,bound", [
    ("allreduce", "B", 256, 1 << 15, 3, 3.4, 1.45),
    ("allreduce", "B", 96, 96 * 100, 4, 3.4, 1.3),
    ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 256, 256, 4, 4.9, 1.35),
    ("allgather", "VEC_DOUBLING_CONT_PERMUTE", 256, 256, 6, 3.9, 1.3),
    ("bcast", "BINOMIAL_TREE", 256, 1 << 12, 4, 1.9, 1.15),
    ("alltoall", "LOG", 256, 64, 10, 17.9, 3.05),
    ("alltoall", "LOG", 64, 64, 8, 10.0, 3.05),
])
def test_fusion_cuts_the_elements_moved(coll, variant, P, count, levels, unfused, bound):
    """Elements read and written by the fused passes over the algorithmic
    minimum (each input read once, each output written once), against the
    level-by-level schedule."""
    comm = bine.Comm(P)
    comm.set_algo(coll, variant)
    st = comm.plan_stats(coll, count)
    assert st["traffic_elems"] >= unfused * algo_elems(coll, P, count)
    mv, lv, dv, _ = comm.plan_fused(coll, count, 0, levels)
    moved = int((mv[:, 1] * (mv[:, 3] + mv[:, 5])).sum())
    assert moved <= bound * algo_elems(coll, P, count)


def accesses(mv, lv, dv, move, start, cnt):
    """(row, first, end, is_write) of one piece of a fused move; rows are
    (buffer, rank)."""
    _, n, lb, nl, db, nd = (int(v) for v in mv[move])
    out = [((int(b), int(r)), int(o) + start, int(o) + start + cnt, False) for r, b, _, o in lv[lb:lb + nl]]
    out += [((int(b), int(r)), int(o) + start, int(o) + start + cnt, True) for r, b, o in dv[db:db + nd]]
    return out


def check_plan(mv, lv, dv, pieces, items, deps):
    """Structure, pass independence and dependency paths for every
    cross-pass element conflict."""
    cover = [[] for _ in range(len(mv))]
    for i, (pb, pe, db, de, lev) in enumerate(items.tolist()):
        assert 0 < pe - pb <= 256
        for p in range(pb, pe):
            m, s, c = pieces[p].tolist()
            assert mv[m][0] == lev and c > 0
            cover[m].append((s, c))
        for d in deps[db:de].tolist():
            assert (0 <= d < i and items[d][4] < lev) or (d < 0 and -d - 1 < lev)
    for m, segs in enumerate(cover):
        pos = 0
        for s, c in sorted(segs):
            assert s == pos
            pos += c
        assert pos == mv[m][1]
    # Moves of one pass: a written element is touched by no other move,
    # except that a move may read what it writes (in place, same elements).
    for lev in np.unique(mv[:, 0]).tolist():
        owner = {}
        for m in np.nonzero(mv[:, 0] == lev)[0].tolist():
            for row, s, e, w in accesses(mv, lv, dv, m, 0, int(mv[m][1])):
                for x in range(s, e):
                    prev = owner.get((row, x))
                    if prev is not None and prev[0] != m:
                        assert not (w or prev[1]), f"moves {prev[0]} and {m} of pass {lev} conflict"
                    if prev is None or w:
                        owner[(row, x)] = (m, w)
    level_of = items[:, 4]
    anc = [0] * len(items)
    level_all = [0] * (int(level_of.max()) + 1)
    writer, readers = {}, {}
    for i, (pb, pe, db, de, lev) in enumerate(items.tolist()):
        a = 0
        for d in deps[db:de].tolist():
            a |= (anc[d] | (1 << d)) if d >= 0 else level_all[-d - 1]
        anc[i] = a
        need = set()
        acc = [t for p in range(pb, pe) for t in accesses(mv, lv, dv, *pieces[p].tolist())]
        for row, s, e, w in acc:
            if not w:
                lw, rd = writer.setdefault(row, {}), readers.setdefault(row, {})
                for x in range(s, e):
                    if x in lw:
                        need.add(lw[x])
                    rd.setdefault(x, set()).add(i)
        for row, s, e, w in acc:
            if w:
                lw, rd = writer.setdefault(row, {}), readers.setdefault(row, {})
                for x in range(s, e):
                    if x in lw:
                        need.add(lw[x])
                    need |= rd.get(x, set())
                    lw[x] = i
                    rd[x] = set()
        for r in need:
            if level_of[r] < lev:
                assert (a >> r) & 1, f"item {i} (pass {lev}) is not ordered after item {r} (pass {level_of[r]})"
        level_all[lev] |= a | (1 << i)


def run_items(case, x, mv, lv, dv, tmp, pieces, items, deps, seed):
    """Executes the items in a random order the dependencies allow."""
    P, coll, root = case["P"], case["coll"], case.get("root", 0)
    se, re = bine.row_counts(coll, case["count"], P)
    bufs = [x.copy() if se else np.zeros((P, 0), x.dtype), np.zeros((P, re), x.dtype),
            np.zeros((P, max(1, tmp)), x.dtype)]
    if coll == "bcast":
        bufs[1][root] = x[root]
    level_of = items[:, 4].tolist()
    nlev = max(level_of) + 1
    left = np.bincount(level_of, minlength=nlev).tolist()
    by_item, by_level = [[] for _ in range(len(items))], [[] for _ in range(nlev)]
    waits = [0] * len(items)
    for i, (pb, pe, db, de, lev) in enumerate(items.tolist()):
        for d in deps[db:de].tolist():
            if d >= 0:
                by_item[d].append(i)
                waits[i] += 1
            elif left[-d - 1] > 0:
                by_level[-d - 1].append(i)
                waits[i] += 1
    ready = [i for i in range(len(items)) if waits[i] == 0]
    rng = np.random.default_rng(seed)
    ran = 0
    while ready:
        k = int(rng.integers(len(ready)))
        ready[k], ready[-1] = ready[-1], ready[k]
        i = ready.pop()
        results = []
        for p in range(items[i][0], items[i][1]):
            m, s, c = pieces[p].tolist()
            _, n, lb, nl, db, nd = mv[m]
            stack = []
            for r, b, adds, off in lv[lb:lb + nl]:
                stack.append(bufs[b][r, off + s:off + s + c].copy())
                for _ in range(adds):
                    top = stack.pop()
                    stack[-1] = (stack[-1] + top).astype(x.dtype)
            results += [(b, r, off + s, stack[0]) for r, b, off in dv[db:db + nd]]
        for b, r, off, v in results:
            bufs[b][r, off:off + len(v)] = v
        ran += 1
        freed = list(by_item[i])
        left[level_of[i]] -= 1
        if left[level_of[i]] == 0:
            freed += by_level[level_of[i]]
        for j in freed:
            waits[j] -= 1
            if waits[j] == 0:
                ready.append(j)
    assert ran == len(items), "dependency cycle"
    return bufs[1]


@pytest.mark.parametrize("case", CASES[::3], ids=case_id)
def test_fused_dataflow_plan_orders_every_conflict_and_matches_reference(case):
    x = case_input(case)
    es = x.dtype.itemsize
    root = case.get("root", 0)
    for levels, segment, target in ((3, 0, 592), (6, 64, 3), (64, 256, 1)):
        comm = make_comm(case, levels, segment)
        try:
            pieces, items, deps = comm.plan_flow(case["coll"], case["count"], root, es, target)
        except bine.Unsupported:
            return
        mv, lv, dv, tmp = comm.plan_fused(case["coll"], case["count"], root, levels)
        if len(items) > 4000:
            continue
        check_plan(mv, lv, dv, pieces, items, deps)
        out = run_items(case, x, mv, lv, dv, tmp, pieces, items, deps, seed=levels + segment)
        rr = receiving_ranks(case["coll"], case["P"], root)
        assert np.array_equal(out[rr].view(np.uint8), case["out"][rr].view(np.uint8))


def test_automatic_fusion_uses_the_per_collective_levels():
    """bine_comm_set_fusion(0): each collective takes its own levels per pass
    (allreduce, reduce_scatter and reduce 6; allgather, bcast, scatter and
    gather 12; alltoall 13); the dataflow plan is that fused plan."""
    table = {"allreduce": ("B", 6), "reduce_scatter": ("VEC_HALVING_CONT_PERMUTE", 6),
             "allgather": ("VEC_DOUBLING_CONT_PERMUTE", 12), "bcast": ("BINOMIAL_TREE", 12),
             "reduce": ("BINOMIAL_TREE", 6), "alltoall": ("LOG", 13)}
    for coll, (variant, levels) in table.items():
        count = 16 * 9 + 1 if coll in ("allreduce", "bcast", "reduce") else 5
        auto = bine.Comm(16)
        auto.set_algo(coll, variant)
        auto.set_fusion(0)
        fixed = bine.Comm(16)
        fixed.set_algo(coll, variant)
        fixed.set_fusion(levels)
        a = auto.plan_flow(coll, count, 0, 4, 592)
        b = fixed.plan_flow(coll, count, 0, 4, 592)
        assert all(np.array_equal(x, y) for x, y in zip(a, b)), coll
