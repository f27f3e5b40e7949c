"""Shared vocabulary of the oracle: collectives, variants, dtypes, buffer sizes.

Per-rank buffer sizes follow bench/bench.cc:178-207; default variants and
distance types follow lib/libbine.cc:28-73.
"""
import numpy as np

COLLS = ["allreduce", "reduce_scatter", "allgather", "bcast", "reduce", "alltoall", "scatter", "gather"]
COLL_ID = {c: i for i, c in enumerate(COLLS)}

DTYPES = {"int32": (0, np.int32), "int64": (1, np.int64), "float": (2, np.float32),
          "double": (3, np.float64), "char": (4, np.int8)}

# Variant names are the reference's LIBBINE_<COLL>_ALGO values.
VARIANTS = {
    "allreduce": {"L": 0, "B": 1, "B_CONT": 3, "B_COALESCE": 4},
    "allgather": {"VEC_DOUBLING_CONT_PERMUTE": 0, "VEC_DOUBLING_CONT_SEND": 1, "VEC_DOUBLING_BLOCKS": 2},
    "reduce_scatter": {"VEC_HALVING_CONT_PERMUTE": 0},
    "bcast": {"BINOMIAL_TREE": 0, "SCATTER_ALLGATHER": 2},
    "reduce": {"BINOMIAL_TREE": 0, "REDUCE_SCATTER_GATHER": 1},
    "alltoall": {"LOG": 0},
    "scatter": {"BINOMIAL_TREE_CONT_PERMUTE": 0},
    "gather": {"BINOMIAL_TREE_CONT_PERMUTE": 0},
}
DEFAULT_VARIANT = {"allreduce": "B", "allgather": "VEC_DOUBLING_CONT_PERMUTE",
                   "reduce_scatter": "VEC_HALVING_CONT_PERMUTE", "bcast": "BINOMIAL_TREE",
                   "reduce": "BINOMIAL_TREE", "alltoall": "LOG", "scatter": "BINOMIAL_TREE_CONT_PERMUTE",
                   "gather": "BINOMIAL_TREE_CONT_PERMUTE"}
FAMILIES = {"BINE": 1, "RECDOUB": 2, "BRUCK": 3, "RING": 4}


def buffer_counts(coll, count, P):
    """Per-rank (send, recv) element counts for the reference's `count` argument."""
    if coll in ("allreduce", "bcast", "reduce"):
        return count, count
    if coll in ("reduce_scatter", "scatter"):
        return count * P, count
    if coll in ("allgather", "gather"):
        return count, count * P
    if coll == "alltoall":
        return count * P, count * P
    raise ValueError(coll)


def expected(coll, x, P, count, root=0):
    """MPI semantics of the collective on rank-major input x[P, send_count].

    Integer sums wrap like the C types.  Rows of ranks that receive nothing
    (non-roots of reduce and gather) are returned as None entries by callers;
    here they are zero.  Float reductions are summed in float64 and rounded,
    which is the FP64 reference for the reordered fast variant.
    """
    if coll in ("allreduce", "reduce", "reduce_scatter"):
        if np.issubdtype(x.dtype, np.floating):
            s = x.astype(np.float64).sum(0).astype(x.dtype)
        else:
            s = x.sum(0, dtype=x.dtype)
        if coll == "allreduce":
            return np.tile(s, (P, 1))
        if coll == "reduce":
            out = np.zeros((P, count), x.dtype)
            out[root] = s
            return out
        return s.reshape(P, count)
    if coll == "allgather":
        return np.tile(x.reshape(-1), (P, 1))
    if coll == "bcast":
        return np.tile(x[root], (P, 1))
    if coll == "alltoall":
        return x.reshape(P, P, count).transpose(1, 0, 2).reshape(P, P * count)
    if coll == "scatter":
        return x[root].reshape(P, count)
    if coll == "gather":
        out = np.zeros((P, P * count), x.dtype)
        out[root] = x.reshape(-1)
        return out
    raise ValueError(coll)


def receiving_ranks(coll, P, root=0):
    """Ranks whose result buffer the collective defines."""
    if coll in ("reduce", "gather"):
        return [root]
    return list(range(P))
