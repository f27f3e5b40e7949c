"""Test helpers: run the engine's planned schedule on the CPU with numpy.

This is test infrastructure, not a product path: it checks that the host
planner's schedule IR (bine_plan_moves) and its reduction trees
(bine_plan_trees) compute what the oracle computes, bit for bit, before any
GPU runs them.  numpy's float32 addition is IEEE round-to-nearest, as is the
device's __fadd_rn.
"""
import numpy as np

import bine_trees_fugaku_b200 as bine


def run_moves(comm, coll, count, x, root=0):
    """Executes the schedule level by level with value semantics."""
    P = comm.nranks
    mv, n, add = comm.plan_moves(coll, count, root)
    st = comm.plan_stats(coll, count, root)
    se, re = bine.row_counts(coll, count, P)
    bufs = [x.copy() if se else np.zeros((P, 0), x.dtype), np.zeros((P, re), x.dtype),
            np.zeros((P, max(1, st["tmp_elems"])), x.dtype)]
    if coll == "bcast":
        bufs[1][root] = x[root]
    levels = mv[:, 0]
    for lvl in np.unique(levels):
        idx = np.nonzero(levels == lvl)[0]
        results = []
        for i in idx:
            _, dr, db, do, ar, ab, ao, br, bb, bo = mv[i]
            k = n[i]
            v = bufs[ab][ar, ao:ao + k].copy()
            if add[i]:
                v = (v + bufs[bb][br, bo:bo + k]).astype(x.dtype)
            results.append((db, dr, do, v))
        for db, dr, do, v in results:
            bufs[db][dr, do:do + len(v)] = v
    return bufs[1]


def eval_trees(comm, coll, count, x, root=0):
    """Evaluates the planner's postfix reduction programs with numpy."""
    P = comm.nranks
    prog, segs = comm.plan_trees(coll, count, root)
    _, re = bine.row_counts(coll, count, P)
    out = np.zeros((P, re), x.dtype)
    for off, n, rank, pb, pl, depth in segs:
        pos = np.arange(off, off + n)
        stack = []
        for r, adds, shift in prog[pb:pb + pl]:
            stack.append(x[r, pos + shift])
            for _ in range(adds):
                top = stack.pop()
                stack[-1] = (stack[-1] + top).astype(x.dtype)
        assert len(stack) == 1
        if rank < 0:
            out[:, off:off + n] = stack[0]
        else:
            out[rank, off:off + n] = stack[0]
    return out


def run_fused(comm, coll, count, x, root=0, levels=3):
    """Executes the fused form of the schedule (bine_plan_fused) pass by
    pass with value semantics; returns (receive rows, elements read and
    written, passes)."""
    P = comm.nranks
    mv, lv, dv, tmp = comm.plan_fused(coll, count, root, levels)
    se, re = bine.row_counts(coll, count, P)
    bufs = [x.copy() if se else np.zeros((P, 0), x.dtype), np.zeros((P, re), x.dtype),
            np.zeros((P, max(1, tmp)), x.dtype)]
    if coll == "bcast":
        bufs[1][root] = x[root]
    traffic = 0
    for p in np.unique(mv[:, 0]):
        results = []
        for _, n, lb, nl, db, nd in mv[mv[:, 0] == p]:
            stack = []
            for r, b, adds, off in lv[lb:lb + nl]:
                stack.append(bufs[b][r, off:off + n].copy())
                for _ in range(adds):
                    top = stack.pop()
                    stack[-1] = (stack[-1] + top).astype(x.dtype)
            assert len(stack) == 1
            traffic += n * (nl + nd)
            for r, b, off in dv[db:db + nd]:
                results.append((b, r, off, stack[0]))
        for b, r, off, v in results:
            bufs[b][r, off:off + len(v)] = v
    return bufs[1], traffic, len(np.unique(mv[:, 0]))
