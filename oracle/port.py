"""ctypes binding of the C++ restatement (oracle/bine_oracle.cc).

Build it with ``make -C oracle port`` (``__graft_entry__.build()`` does).
"""
import ctypes
import os

import numpy as np

from .common import COLL_ID, DTYPES, FAMILIES, VARIANTS, DEFAULT_VARIANT, buffer_counts

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libbine_oracle.so")

OK, ERR_ARG, ERR_REFERENCE_UNSUPPORTED, ERR_INTERNAL = 0, 1, 2, 3


class _Call(ctypes.Structure):
    _fields_ = [("coll", ctypes.c_int), ("algo", ctypes.c_int), ("family", ctypes.c_int),
                ("distance", ctypes.c_int), ("dtype", ctypes.c_int), ("nranks", ctypes.c_int),
                ("ndims", ctypes.c_int), ("dims", ctypes.c_int * 3), ("ports", ctypes.c_int),
                ("root", ctypes.c_int), ("count", ctypes.c_long)]


class Msg(ctypes.Structure):
    _fields_ = [("src", ctypes.c_int32), ("dst", ctypes.c_int32), ("bytes", ctypes.c_uint64)]


MSG_DTYPE = np.dtype([("src", np.int32), ("dst", np.int32), ("bytes", np.uint64)])

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle restatement not built: {LIB_PATH} (run `make -C oracle port`)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_run.restype = ctypes.c_int
        _lib.oracle_run.argtypes = [ctypes.POINTER(_Call), ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        _lib.oracle_last_error.restype = ctypes.c_char_p
        _lib.oracle_remap_rank.restype = ctypes.c_uint32
        _lib.oracle_remap_rank.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib.oracle_get_nu.restype = ctypes.c_uint32
        _lib.oracle_get_nu.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib.oracle_remap_distance_doubling.restype = ctypes.c_int
        _lib.oracle_remap_distance_doubling.argtypes = [ctypes.c_uint32]
    return _lib


class ReferenceUnsupported(Exception):
    """The reference asserts, exits, deadlocks or corrupts data on this case."""


def run(coll, x, count, *, variant=None, dims=None, ports=1, root=0, family="BINE", distance=None,
        trace=False):
    """Runs one collective of the restatement.

    x: rank-major input, shape (P, send_count) with the element dtype.
    Returns (out[P, recv_count], msgs or None).
    """
    x = np.ascontiguousarray(x)
    P = x.shape[0]
    dt_name = {np.dtype(v[1]): k for k, v in DTYPES.items()}[x.dtype]
    sc, rc = buffer_counts(coll, count, P)
    assert x.shape[1] == sc, (x.shape, sc)
    variant = variant or DEFAULT_VARIANT[coll]
    c = _Call()
    c.coll = COLL_ID[coll]
    c.algo = VARIANTS[coll][variant]
    c.family = FAMILIES[family]
    c.distance = -1 if distance is None else {"INCREASING": 0, "DECREASING": 1}[distance]
    c.dtype = DTYPES[dt_name][0]
    c.nranks = P
    if dims:
        c.ndims = len(dims)
        for i, d in enumerate(dims):
            c.dims[i] = d
    else:
        c.ndims = 0
    c.ports = ports
    c.root = root
    c.count = count
    out = np.zeros((P, rc), x.dtype)
    nmsg = ctypes.c_size_t(0)
    cap = 1 << 20 if trace else 0
    msgs = np.zeros(cap, MSG_DTYPE) if trace else None
    rcode = lib().oracle_run(ctypes.byref(c), x.ctypes.data, out.ctypes.data,
                             msgs.ctypes.data if trace else None, cap, ctypes.byref(nmsg))
    if rcode == ERR_REFERENCE_UNSUPPORTED:
        raise ReferenceUnsupported(lib().oracle_last_error().decode())
    if rcode != OK:
        raise RuntimeError(f"oracle_run failed ({rcode}): {lib().oracle_last_error().decode()}")
    if trace:
        msgs = msgs[: min(nmsg.value, cap)].copy()
    return out, msgs


def remap_rank(nranks, rank):
    return lib().oracle_remap_rank(nranks, rank)


def get_nu(rank, nranks):
    return lib().oracle_get_nu(rank, nranks)


def remap_distance_doubling(num):
    return lib().oracle_remap_distance_doubling(num)


def compute_peers(rank, port, dims, family="BINE"):
    dims = list(dims)
    arr = (ctypes.c_int * 3)(*(dims + [0] * (3 - len(dims))))
    peers = (ctypes.c_int * 64)()
    n = lib().oracle_compute_peers(rank, port, FAMILIES[family], len(dims), arr, peers)
    return list(peers[:n])


def get_tree(root, port, dims, family="BINE", distance="INCREASING"):
    dims = list(dims)
    P = int(np.prod(dims))
    arr = (ctypes.c_int * 3)(*(dims + [0] * (3 - len(dims))))
    outs = [np.zeros(P, np.uint32) for _ in range(5)]
    rc = lib().oracle_get_tree(root, port, FAMILIES[family], {"INCREASING": 0, "DECREASING": 1}[distance],
                               len(dims), arr, *[o.ctypes.data_as(ctypes.c_void_p) for o in outs])
    if rc != OK:
        raise ReferenceUnsupported(lib().oracle_last_error().decode())
    return dict(zip(["parent", "reached_at_step", "remapped_ranks", "remapped_ranks_max", "subtree_roots"], outs))


def block_step(rank, port, dims, family="BINE"):
    dims = list(dims)
    P = int(np.prod(dims))
    arr = (ctypes.c_int * 3)(*(dims + [0] * (3 - len(dims))))
    out = np.zeros(P, np.uint32)
    lib().oracle_block_step(rank, port, FAMILIES[family], len(dims), arr, out.ctypes.data_as(ctypes.c_void_p))
    return out
