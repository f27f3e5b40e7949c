"""Large-P cases for which tests/golden/ref_large.json holds digests of the
reference library's own results.

P = 128, 256, 384 and 1024 virtual ranks are too many rows to store, so the
fixture keeps, per case, the SHA-256 of the receiving ranks' result bytes
(row-major, little-endian) and of the sorted message trace; the inputs are
regenerated here from each case's seed.  A digest comparison is bit-exact.
Also here: the full-size P = 8 allreduce (1,048,576 elements per rank,
int32 uniform in [-1000, 1000] and float32 N(0, 1)).
"""
import hashlib

import numpy as np

from oracle.common import buffer_counts, expected, receiving_ranks

LARGE_P = (128, 256, 384, 1024)
_DT = {"int32": np.int32, "float": np.float32}


def _cases():
    out = []

    def add(coll, variant, P, dtype, count, **kw):
        c = {"coll": coll, "variant": variant, "P": P, "dtype": dtype, "count": count,
             "seed": 50000 + 17 * P + len(out)}
        c.update(kw)
        out.append(c)

    for P in LARGE_P:
        for dt in ("float", "int32"):
            # Ragged blocks (count not a multiple of P) and 16-byte blocks.
            add("allreduce", "B", P, dt, 2 * P + 3)
            add("allreduce", "B", P, dt, 8 * P)
            add("allreduce", "L", P, dt, 2 * P + 3)
        add("allreduce", "B_COALESCE", P, "float", 3 * P + 1)
        add("allreduce", "B_CONT", P, "float", 8 * P)
        add("allreduce", "L", P, "float", 8 * P + 5, ports=2)
        add("allreduce", "B", P, "float", 4 * P + 7, ports=3)
        add("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", P, "float", 3)
        add("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", P, "float", 8)
        add("reduce", "BINOMIAL_TREE", P, "float", 37)
        add("reduce", "REDUCE_SCATTER_GATHER", P, "float", 4 * P + 1)
        for var in ("VEC_DOUBLING_CONT_PERMUTE", "VEC_DOUBLING_CONT_SEND", "VEC_DOUBLING_BLOCKS"):
            add("allgather", var, P, "float", 3)
        add("bcast", "BINOMIAL_TREE", P, "float", 37)
        add("bcast", "SCATTER_ALLGATHER", P, "float", 4 * P + 1, distance="INCREASING")
        add("alltoall", "LOG", P, "float", 2)
        add("alltoall", "LOG", P, "float", 2, family="BRUCK")
        add("scatter", "BINOMIAL_TREE_CONT_PERMUTE", P, "float", 3)
        add("gather", "BINOMIAL_TREE_CONT_PERMUTE", P, "float", 3)
    # Roots other than 0 and the recursive-doubling family at P = 256.
    for coll, var in (("bcast", "BINOMIAL_TREE"), ("reduce", "BINOMIAL_TREE"),
                      ("scatter", "BINOMIAL_TREE_CONT_PERMUTE"), ("gather", "BINOMIAL_TREE_CONT_PERMUTE")):
        for root in (6, 77):
            add(coll, var, 256, "float", 5, root=root)
    for var in ("B", "L"):
        add("allreduce", var, 256, "float", 2 * 256 + 3, family="RECDOUB")
    # Tori of 128 and 384 ranks.
    for dims in ([8, 4, 4], [8, 8, 6]):
        P = int(np.prod(dims))
        for var in ("B", "L"):
            add("allreduce", var, P, "float", 2 * P + 3, dims=dims)
    # The full-size P = 8 allreduce, int32 and float32.
    for dt in ("int32", "float"):
        add("allreduce", "B", 8, dt, 1 << 20, seed=8)
    return out


CASES = _cases()


def case_input(case):
    P, count = case["P"], case["count"]
    sc, _ = buffer_counts(case["coll"], count, P)
    rng = np.random.default_rng(case["seed"])
    if case["dtype"] == "float":
        return rng.standard_normal((P, sc)).astype(np.float32)
    return rng.integers(-1000, 1001, (P, sc)).astype(np.int32)


def result_digest(case, out):
    """SHA-256 of the receiving ranks' rows of `out` (the collective's
    defined result)."""
    rr = receiving_ranks(case["coll"], case["P"], case.get("root", 0))
    return hashlib.sha256(np.ascontiguousarray(out[rr]).tobytes()).hexdigest()


def trace_digest(src, dst, nbytes):
    """SHA-256 of the message multiset: sorted (src, dst, bytes) int64 rows."""
    m = np.stack([np.asarray(src, np.int64), np.asarray(dst, np.int64), np.asarray(nbytes, np.int64)], 1)
    m = m[np.lexsort((m[:, 2], m[:, 1], m[:, 0]))]
    return hashlib.sha256(m.tobytes()).hexdigest()


def matches_mpi(case, x, out):
    """Whether `out` is the MPI result: exact for integers and copies, and
    within the error bound of an n-term float32 sum for float reductions."""
    P, count, root = case["P"], case["count"], case.get("root", 0)
    rr = receiving_ranks(case["coll"], P, root)
    exp = expected(case["coll"], x, P, count, root)
    if case["dtype"] == "float" and case["coll"] in ("allreduce", "reduce_scatter", "reduce"):
        # |fl(sum) - sum| <= (P-1) u sum|x| for any summation order.
        ax = np.abs(x.astype(np.float64))
        scale = {"allreduce": lambda: np.tile(ax.sum(0), (P, 1)),
                 "reduce": lambda: np.tile(ax.sum(0), (P, 1)),
                 "reduce_scatter": lambda: ax.sum(0).reshape(P, count)}[case["coll"]]()
        err = np.abs(out[rr].astype(np.float64) - exp[rr].astype(np.float64))
        return bool((err <= P * 2.0 ** -24 * scale[rr] + 1e-30).all())
    return bool(np.array_equal(out[rr], exp[rr]))
