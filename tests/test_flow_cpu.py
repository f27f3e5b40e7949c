"""The pipelined engine's dataflow plan (bine_plan_flow), checked on the CPU.

The plan cuts every move of the schedule into pieces, packs pieces into
items and gives each item the earlier items it must wait for.  Checked here,
independently of how the planner derives it:

* the pieces tile every move exactly and items stay within one level;
* every element-level conflict (read after write, write after write, write
  after read) between items of different levels is ordered by a dependency
  path;
* no two moves of one level conflict (the premise of both step engines);
* running the items in a random order the dependencies allow gives the
  reference's results, bit for bit.
"""
import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine
from golden_data import load_ref_collectives
from oracle.common import receiving_ranks
from tests.golden.cases import case_input

CASES = [c for c in load_ref_collectives() if c["ok"]]


def make_comm(case, segment=0):
    comm = bine.Comm(case["P"], case.get("dims"))
    comm.set_ports(case.get("ports", 1))
    comm.set_algo(case["coll"], case["variant"], case.get("family", "BINE"), case.get("distance"))
    comm.set_segment(segment)
    comm.set_fusion(1)  # the level-by-level plan (fused plans: tests/test_fusion_cpu.py)
    return comm


def plan(comm, case, es, target):
    root = case.get("root", 0)
    try:
        mv, n, add = comm.plan_moves(case["coll"], case["count"], root)
        pieces, items, deps = comm.plan_flow(case["coll"], case["count"], root, es, target)
    except bine.Unsupported:
        return None
    return mv, n, add, pieces, items, deps


def touched(mv, add, move, start, cnt, alias):
    """(row, first, end, is_write) of one piece; rows are (space, rank), the
    send and receive rows sharing a space when `alias`."""
    _, dr, db, do, ar, ab, ao, br, bb, bo = (int(v) for v in mv[move])

    def space(b):
        return 2 if b == 2 else (0 if alias else b)

    out = [((space(ab), ar), ao + start, ao + start + cnt, False)]
    if add[move]:
        out.append(((space(bb), br), bo + start, bo + start + cnt, False))
    out.append(((space(db), dr), do + start, do + start + cnt, True))
    return out


def check_structure(mv, n, pieces, items, deps):
    levels = mv[:, 0]
    cover = [[] for _ in range(len(mv))]
    for i, (pb, pe, db, de, lv) in enumerate(items.tolist()):
        assert 0 < pe - pb <= 256
        if i:
            assert lv >= items[i - 1][4] and pb == items[i - 1][1] and db == items[i - 1][3]
        for p in range(pb, pe):
            m, s, c = pieces[p].tolist()
            assert levels[m] == lv and c > 0
            cover[m].append((s, c))
        for d in deps[db:de].tolist():
            assert (0 <= d < i and items[d][4] < lv) or (d < 0 and -d - 1 < lv)
    for m, segs in enumerate(cover):
        pos = 0
        for s, c in sorted(segs):
            assert s == pos
            pos += c
        assert pos == n[m]
    assert items[-1][1] == len(pieces) and items[-1][3] == len(deps)


def check_conflicts(mv, add, pieces, items, deps):
    """Every cross-level element conflict is ordered by a dependency path;
    no two moves of one level conflict."""
    level_of = items[:, 4]
    anc = [0] * len(items)  # ancestors as bit sets
    level_all = [0] * (int(level_of.max()) + 1)  # per level: OR of (ancestors | item)
    writer, readers = {}, {}
    for i, (pb, pe, db, de, lv) in enumerate(items.tolist()):
        a = 0
        for d in deps[db:de].tolist():
            a |= (anc[d] | (1 << d)) if d >= 0 else level_all[-d - 1]
        anc[i] = a
        need = set()
        acc = [t for p in range(pb, pe) for t in touched(mv, add, *pieces[p].tolist(), alias=False)]
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
            if level_of[r] < lv:
                assert (a >> r) & 1, f"item {i} (level {lv}) is not ordered after item {r} (level {level_of[r]})"
        level_all[lv] |= a | (1 << i)


def check_level_independence(mv, n, add):
    """Moves of one level touch disjoint elements wherever one of them
    writes (send and receive rows distinct)."""
    for lv in np.unique(mv[:, 0]).tolist():
        owner = {}
        for m in np.nonzero(mv[:, 0] == lv)[0].tolist():
            for row, s, e, w in touched(mv, add, m, 0, int(n[m]), alias=False):
                for x in range(s, e):
                    prev = owner.get((row, x))
                    if prev is not None and prev[0] != m:
                        assert not (w or prev[1]), f"moves {prev[0]} and {m} of level {lv} conflict"
                    if prev is None or w:
                        owner[(row, x)] = (m, w)


def run_flow(case, x, mv, add, pieces, items, deps, seed):
    """Executes the items in a random order the dependencies allow."""
    P, coll, root = case["P"], case["coll"], case.get("root", 0)
    comm = make_comm(case)
    st = comm.plan_stats(coll, case["count"], root)
    se, re = bine.row_counts(coll, case["count"], P)
    bufs = [x.copy() if se else np.zeros((P, 0), x.dtype), np.zeros((P, re), x.dtype),
            np.zeros((P, max(1, st["tmp_elems"])), x.dtype)]
    if coll == "bcast":
        bufs[1][root] = x[root]
    # Kahn's algorithm with a random choice among the ready items.
    level_of = items[:, 4].tolist()
    nlev = max(level_of) + 1
    left = np.bincount(level_of, minlength=nlev).tolist()  # unfinished items per level
    by_item = [[] for _ in range(len(items))]  # dependents through item entries
    by_level = [[] for _ in range(nlev)]  # dependents through level entries
    waits = [0] * len(items)
    for i, (pb, pe, db, de, lv) in enumerate(items.tolist()):
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
            _, dr, db, do, ar, ab, ao, br, bb, bo = mv[m]
            v = bufs[ab][ar, ao + s:ao + s + c].copy()
            if add[m]:
                v = (v + bufs[bb][br, bo + s:bo + s + c]).astype(x.dtype)
            results.append((db, dr, do + s, v))
        for db, dr, do, v in results:
            bufs[db][dr, do:do + len(v)] = v
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


def case_id(c):
    return (f"{c['coll']}-{c['variant']}-P{c['P']}-{c['dtype']}-d{c.get('dims')}-p{c.get('ports', 1)}"
            f"-r{c.get('root', 0)}-{c.get('family', 'BINE')}")


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_flow_plan_orders_every_conflict_and_matches_reference(case):
    x = case_input(case)
    es = x.dtype.itemsize
    # The engine's sizing, then small segments with few items per level:
    # many pieces, items packing several moves, level dependencies.
    for segment, target in ((0, 592), (64, 3), (256, 1)):
        comm = make_comm(case, segment)
        got = plan(comm, case, es, target)
        if got is None:
            return
        mv, n, add, pieces, items, deps = got
        if len(items) > 4000:  # keeps the element-level check to seconds
            continue
        if segment == 0:
            check_level_independence(mv, n, add)
        check_structure(mv, n, pieces, items, deps)
        check_conflicts(mv, add, pieces, items, deps)
        out = run_flow(case, x, mv, add, pieces, items, deps, seed=segment + target)
        rr = receiving_ranks(case["coll"], case["P"], case.get("root", 0))
        assert np.array_equal(out[rr].view(np.uint8), case["out"][rr].view(np.uint8))


@pytest.mark.parametrize("coll,variant,P,count,ports", [
    ("allreduce", "B", 64, 64 * 5 + 3, 1), ("allreduce", "L", 48, 200, 2),
    ("allgather", "VEC_DOUBLING_BLOCKS", 32, 7, 1), ("alltoall", "LOG", 32, 3, 1),
    ("bcast", "SCATTER_ALLGATHER", 32, 100, 1)])
def test_flow_plan_larger_schedules_order_every_conflict(coll, variant, P, count, ports):
    case = {"coll": coll, "variant": variant, "P": P, "count": count, "ports": ports}
    if variant == "SCATTER_ALLGATHER":
        case["distance"] = "INCREASING"
    comm = make_comm(case, 16)
    mv, n, add, pieces, items, deps = plan(comm, case, 4, 40)
    check_structure(mv, n, pieces, items, deps)
    check_conflicts(mv, add, pieces, items, deps)

