"""Small seeded cases for which tests/golden/ref_collectives.npz holds the
reference library's own results and message traces."""
import numpy as np

from oracle.common import buffer_counts

_DT = {"int32": np.int32, "float": np.float32}


def _cases():
    out = []
    variants = [("allreduce", "B"), ("allreduce", "B_COALESCE"), ("allreduce", "B_CONT"), ("allreduce", "L"),
                ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE"), ("allgather", "VEC_DOUBLING_CONT_PERMUTE"),
                ("allgather", "VEC_DOUBLING_CONT_SEND"), ("allgather", "VEC_DOUBLING_BLOCKS"),
                ("bcast", "BINOMIAL_TREE"), ("bcast", "SCATTER_ALLGATHER"), ("reduce", "BINOMIAL_TREE"),
                ("reduce", "REDUCE_SCATTER_GATHER"), ("alltoall", "LOG"), ("scatter", "BINOMIAL_TREE_CONT_PERMUTE"),
                ("gather", "BINOMIAL_TREE_CONT_PERMUTE")]
    for coll, var in variants:
        for P in (4, 8, 16, 6, 12):
            for dt in ("int32", "float"):
                count = 3 * P + 5 if coll == "allreduce" else 5
                c = {"coll": coll, "variant": var, "P": P, "dtype": dt, "count": count, "seed": 1000 + P}
                if var == "SCATTER_ALLGATHER":
                    c["distance"] = "INCREASING"
                out.append(c)
    # Tori, ports, roots and the recursive-doubling family.
    for dims in ([2, 2, 2], [4, 4], [2, 8, 2], [6, 6], [4, 6, 4]):
        P = int(np.prod(dims))
        for var in ("B", "L"):
            for ports in (1, 2, 6):
                out.append({"coll": "allreduce", "variant": var, "P": P, "dims": dims, "ports": ports,
                            "dtype": "float", "count": 6 * P + 3, "seed": 7 + P})
    for var in ("B", "L", "B_CONT"):
        out.append({"coll": "allreduce", "variant": var, "P": 16, "family": "RECDOUB", "dtype": "float",
                    "count": 77, "seed": 3})
    for coll, var in (("bcast", "BINOMIAL_TREE"), ("reduce", "BINOMIAL_TREE"), ("scatter", "BINOMIAL_TREE_CONT_PERMUTE"),
                      ("gather", "BINOMIAL_TREE_CONT_PERMUTE")):
        out.append({"coll": coll, "variant": var, "P": 16, "root": 5, "dtype": "float", "count": 9, "seed": 11})
    for coll, var in (("reduce_scatter", "VEC_HALVING_CONT_PERMUTE"), ("allgather", "VEC_DOUBLING_CONT_PERMUTE")):
        out.append({"coll": coll, "variant": var, "P": 16, "ports": 3, "dtype": "int32", "count": 7, "seed": 5})
    # Bruck's alltoall, the reference's comparator (any P).
    for P in (4, 8, 16, 6, 12):
        for dt in ("int32", "float"):
            out.append({"coll": "alltoall", "variant": "LOG", "P": P, "family": "BRUCK", "dtype": dt, "count": 5,
                        "seed": 2000 + P})
    return out


CASES = _cases()


def case_input(case):
    P, count = case["P"], case["count"]
    sc, _ = buffer_counts(case["coll"], count, P)
    rng = np.random.default_rng(case["seed"])
    if case["dtype"] == "float":
        return rng.standard_normal((P, sc)).astype(np.float32)
    return rng.integers(-1000, 1001, (P, sc)).astype(np.int32)
