"""B200-native engine for the Bine-tree collectives over virtual ranks.

Python mirror of the engine's C ABI (include/bine_b200.h), loaded with ctypes
from the in-tree library lib/libbine_b200.so.  A ``Comm`` holds P virtual
ranks on one GPU; its methods keep the argument lists of the reference's MPI
entry points (lib/libbine.cc): ``allreduce(sendbuf, recvbuf, count, datatype,
op)``, ``bcast(buffer, count, datatype, root)`` and so on, where every
buffer is a rank-major device array -- a CUDA torch tensor of shape
(P, row) or a raw device pointer.

There is no fallback: if the library is missing, importing the engine
raises, and every call runs the CUDA kernels.
"""
import ctypes
import os

import numpy as np

from .build import LIB_PATH

INT32, INT64, FLOAT, DOUBLE, CHAR = 0, 1, 2, 3, 4
SUM = 0
SUCCESS, ERR_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_TIMEOUT, ERR_NOMEM, ERR_INTERNAL, ERR_ABORTED = range(8)
# bine_window_hook_t: (user, first column, columns) -> 0 to go on
WINDOW_HOOK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong)
ENGINE_FUSED, ENGINE_STEPS, ENGINE_PIPELINED = 0, 1, 2
ORDER_REFERENCE, ORDER_FAST = 0, 1
FAMILY = {"BINE": 1, "RECDOUB": 2, "BRUCK": 3, "RING": 4}
DISTANCE = {None: -1, "INCREASING": 0, "DECREASING": 1}

COLLS = ["allreduce", "reduce_scatter", "allgather", "bcast", "reduce", "alltoall", "scatter", "gather"]
COLL_ID = {c: i for i, c in enumerate(COLLS)}
# Variant names are the reference's LIBBINE_<COLL>_ALGO values.
VARIANTS = {
    "allreduce": {"L": 0, "B": 1, "B_CONT": 3, "B_COALESCE": 4},
    "reduce_scatter": {"VEC_HALVING_CONT_PERMUTE": 0},
    "allgather": {"VEC_DOUBLING_CONT_PERMUTE": 0, "VEC_DOUBLING_CONT_SEND": 1, "VEC_DOUBLING_BLOCKS": 2},
    "bcast": {"BINOMIAL_TREE": 0, "SCATTER_ALLGATHER": 2},
    "reduce": {"BINOMIAL_TREE": 0, "REDUCE_SCATTER_GATHER": 1},
    "alltoall": {"LOG": 0},
    "scatter": {"BINOMIAL_TREE_CONT_PERMUTE": 0},
    "gather": {"BINOMIAL_TREE_CONT_PERMUTE": 0},
}
DTYPE_SIZE = {INT32: 4, INT64: 8, FLOAT: 4, DOUBLE: 8, CHAR: 1}
NP_DTYPE = {INT32: np.int32, INT64: np.int64, FLOAT: np.float32, DOUBLE: np.float64, CHAR: np.int8}


class BatchItem(ctypes.Structure):
    """bine_batch_item_t"""
    _fields_ = [("coll", ctypes.c_int), ("datatype", ctypes.c_int), ("nranks", ctypes.c_int),
                ("reserved", ctypes.c_int), ("count", ctypes.c_long), ("sendbuf", ctypes.c_void_p),
                ("recvbuf", ctypes.c_void_p), ("send_stride", ctypes.c_size_t), ("recv_stride", ctypes.c_size_t)]


class BatchTuning(ctypes.Structure):
    """bine_batch_tuning_t"""
    _fields_ = [("rank_bound", ctypes.c_int * 4), ("tile_cols", ctypes.c_int * 4), ("grid_mult", ctypes.c_int),
                ("order", ctypes.c_int)]

    def as_dict(self):
        return {"rank_bound": list(self.rank_bound), "tile_cols": list(self.tile_cols),
                "grid_mult": self.grid_mult, "order": self.order}

    @classmethod
    def from_dict(cls, d):
        t = cls()
        for k in range(4):
            t.rank_bound[k] = d["rank_bound"][k]
            t.tile_cols[k] = d["tile_cols"][k]
        t.grid_mult, t.order = d["grid_mult"], d["order"]
        return t


class BineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"bine error {code}: {msg}")
        self.code = code


class Unsupported(BineError):
    """The selected reference algorithm cannot run this case."""


class Timeout(BineError):
    """A bounded device-side wait expired."""


_lib = None


def lib():
    """Loads lib/libbine_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"the engine library is not built: {LIB_PATH} "
                          "(run `python -m bine_trees_fugaku_b200.build`)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, ci, sz, i64p = ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64)
    L.bine_last_error_string.restype = ctypes.c_char_p
    L.bine_mlp_last_error.restype = ctypes.c_char_p
    sig = {
        "bine_comm_create": [i, i, ctypes.POINTER(ci), ctypes.POINTER(vp)],
        "bine_comm_destroy": [vp],
        "bine_comm_set_stream": [vp, vp],
        "bine_comm_set_layout": [vp, sz, sz],
        "bine_comm_set_ports": [vp, i],
        "bine_comm_set_algo": [vp, i, i, i, i],
        "bine_comm_set_engine": [vp, i],
        "bine_comm_set_segment": [vp, ctypes.c_longlong],
        "bine_comm_set_fusion": [vp, i],
        "bine_plan_fused": [vp, i, ctypes.c_long, i, i, i64p, sz, ctypes.POINTER(sz), i64p, sz, ctypes.POINTER(sz),
                            i64p, sz, ctypes.POINTER(sz), i64p],
        "bine_comm_set_float_order": [vp, i],
        "bine_comm_set_step_timeout": [vp, ctypes.c_uint],
        "bine_debug_set_barrier_extra": [vp, ctypes.c_uint],
        "bine_comm_set_tree_split": [vp, ctypes.c_int],
        "bine_allreduce_host": [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp],
        "bine_allreduce_host_hooked": [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, WINDOW_HOOK, WINDOW_HOOK,
                                       vp],
        "bine_comm_set_host_window": [vp, ctypes.c_longlong],
        "bine_comm_synchronize": [vp],
        "bine_allreduce": [vp, vp, i, i, i, vp],
        "bine_reduce_scatter": [vp, vp, ctypes.POINTER(ci), i, i, vp],
        "bine_allgather": [vp, i, i, vp, i, i, vp],
        "bine_bcast": [vp, i, i, i, vp],
        "bine_alltoall": [vp, i, i, vp, i, i, vp],
        "bine_scatter": [vp, i, i, vp, i, i, i, vp],
        "bine_gather": [vp, i, i, vp, i, i, i, vp],
        "bine_reduce": [vp, vp, i, i, i, i, vp],
        "bine_plan_stats": [vp, i, ctypes.c_long, i, i64p],
        "bine_plan_verify": [vp, i, ctypes.c_long, i],
        "bine_link_bytes": [vp, i, ctypes.c_long, i, i, vp],
        "bine_plan_moves": [vp, i, ctypes.c_long, i, i64p, i64p, sz, ctypes.POINTER(sz)],
        "bine_plan_messages": [vp, i, ctypes.c_long, i, i64p, sz, ctypes.POINTER(sz)],
        "bine_plan_flow": [vp, i, ctypes.c_long, i, i, i, i64p, sz, ctypes.POINTER(sz), ctypes.POINTER(ctypes.c_int32),
                           sz, ctypes.POINTER(sz), ctypes.POINTER(ctypes.c_int32), sz, ctypes.POINTER(sz)],
        "bine_plan_trees": [vp, i, ctypes.c_long, i, i64p, sz, ctypes.POINTER(sz), i64p, sz, ctypes.POINTER(sz)],
        "bine_debug_tree_form": [vp, i, ctypes.c_long, i, i, ctypes.POINTER(i), ctypes.POINTER(i)],
        "bine_plan_tree_form": [vp, i, ctypes.c_long, i, i, i64p],
        "bine_plan_tree_cover": [vp, i, ctypes.c_long, i, i, i64p, sz, ctypes.POINTER(sz)],
        "bine_link_bytes_host": [vp, i, ctypes.c_long, i, i, ctypes.POINTER(ctypes.c_uint64), sz],
        "bine_mlp_create": [i, i, i, i, ctypes.c_ulonglong, ctypes.POINTER(vp)],
        "bine_mlp_destroy": [vp],
        "bine_mlp_num_params": [vp, ctypes.POINTER(sz)],
        "bine_mlp_get_params": [vp, vp],
        "bine_mlp_set_params": [vp, vp],
        "bine_mlp_forward": [vp, vp, i, vp, vp],
        "bine_mlp_gradients": [vp, vp, vp, vp, i, vp, ctypes.POINTER(ctypes.c_float)],
        "bine_mlp_train_step": [vp, vp, vp, vp, i, ctypes.c_float, vp, ctypes.POINTER(ctypes.c_float)],
        "bine_mlp_ensemble_create": [ctypes.POINTER(vp), i, ctypes.POINTER(vp)],
        "bine_mlp_ensemble_forward": [vp, vp, i, vp, vp],
        "bine_mlp_ensemble_destroy": [vp],
        "bine_batch_create": [ctypes.POINTER(BatchItem), i, ctypes.POINTER(BatchTuning), ctypes.POINTER(vp)],
        "bine_batch_launch": [vp, vp],
        "bine_batch_destroy": [vp],
        "bine_batch_autotune": [ctypes.POINTER(BatchItem), i, vp, i, ctypes.POINTER(BatchTuning),
                                ctypes.POINTER(ctypes.c_float)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    _lib = L
    return L


def last_error():
    return lib().bine_last_error_string().decode()


def check(rc):
    if rc == SUCCESS:
        return
    msg = last_error()
    if rc == ERR_UNSUPPORTED:
        raise Unsupported(rc, msg)
    if rc == ERR_TIMEOUT:
        raise Timeout(rc, msg)
    raise BineError(rc, msg)


def _ptr(buf):
    """Device pointer of a CUDA tensor or an integer address."""
    if buf is None:
        return None
    if isinstance(buf, int):
        return buf
    if hasattr(buf, "data_ptr"):
        if not buf.is_cuda:
            raise ValueError("buffers must be CUDA tensors (device memory)")
        return buf.data_ptr()
    raise TypeError(f"unsupported buffer type {type(buf)}")


def _host_ptr(buf):
    """Address of a host buffer: a CPU torch tensor or a numpy array."""
    if isinstance(buf, np.ndarray):
        return buf.ctypes.data
    if getattr(buf, "is_cuda", False):
        raise ValueError("bine_allreduce_host takes host buffers")
    return buf.data_ptr()


def dtype_of_tensor(t):
    import torch
    return {torch.int32: INT32, torch.int64: INT64, torch.float32: FLOAT, torch.float64: DOUBLE,
            torch.int8: CHAR}[t.dtype]


class Comm:
    """P virtual ranks on the current CUDA device (a torus of `dims`)."""

    def __init__(self, nranks, dims=None):
        dims = list(dims or [])
        arr = (ctypes.c_int * max(1, len(dims)))(*dims) if dims else None
        h = ctypes.c_void_p()
        check(lib().bine_comm_create(nranks, len(dims), arr, ctypes.byref(h)))
        self._h = h
        self.nranks = nranks
        self.dims = dims or [nranks]
        # Settings as last set (the picker reads them): per-collective
        # variant (None: the reference's default), ports, engine, float order.
        self.algo = {}
        self.family = {}
        self.ports = 1
        self.engine = "fused"
        self.float_order = "reference"
        self.fusion = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().bine_comm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------- settings
    def set_stream(self, stream):
        """Orders calls on a torch.cuda.Stream (or a raw cudaStream_t)."""
        h = stream if isinstance(stream, int) else (stream.cuda_stream if stream is not None else 0)
        check(lib().bine_comm_set_stream(self._h, h))

    def set_layout(self, send_stride=0, recv_stride=0):
        check(lib().bine_comm_set_layout(self._h, send_stride, recv_stride))

    def set_ports(self, ports):
        check(lib().bine_comm_set_ports(self._h, ports))
        self.ports = ports

    def set_algo(self, coll, variant, family="BINE", distance=None):
        check(lib().bine_comm_set_algo(self._h, COLL_ID[coll], VARIANTS[coll][variant], FAMILY[family],
                                       DISTANCE[distance]))
        self.algo[coll] = variant
        self.family[coll] = family

    def set_engine(self, engine):
        check(lib().bine_comm_set_engine(self._h, {"fused": ENGINE_FUSED, "steps": ENGINE_STEPS,
                                                             "pipelined": ENGINE_PIPELINED}.get(engine, engine)))
        self.engine = {ENGINE_FUSED: "fused", ENGINE_STEPS: "steps", ENGINE_PIPELINED: "pipelined"}.get(engine, engine)

    def set_segment(self, segment_bytes):
        check(lib().bine_comm_set_segment(self._h, segment_bytes))

    def set_fusion(self, levels):
        """Levels of the reference's schedule per pass of the PIPELINED
        engine (1: every level on its own; 0, the default: per collective)."""
        check(lib().bine_comm_set_fusion(self._h, levels))
        self.fusion = levels

    def set_float_order(self, order):
        check(lib().bine_comm_set_float_order(self._h, {"reference": ORDER_REFERENCE, "fast": ORDER_FAST}.get(order, order)))
        self.float_order = {ORDER_REFERENCE: "reference", ORDER_FAST: "fast"}.get(order, order)

    def set_step_timeout(self, ms):
        check(lib().bine_comm_set_step_timeout(self._h, ms))

    def set_host_window(self, window_bytes):
        """Column-window bytes of allreduce_host's pipeline."""
        check(lib().bine_comm_set_host_window(self._h, window_bytes))

    def set_tree_split(self, lanes):
        """Lanes per output vector of the exact-order float reduction
        (0: chosen per call)."""
        check(lib().bine_comm_set_tree_split(self._h, lanes))

    def debug_set_barrier_extra(self, extra):
        check(lib().bine_debug_set_barrier_extra(self._h, extra))

    def synchronize(self):
        check(lib().bine_comm_synchronize(self._h))

    # ------------------------------------------------------ collectives
    def allreduce(self, sendbuf, recvbuf, count, datatype, op=SUM):
        check(lib().bine_allreduce(_ptr(sendbuf), _ptr(recvbuf), count, datatype, op, self._h))

    def allreduce_host(self, sendbuf, recvbuf, count, datatype, op=SUM):
        """bine_allreduce_host: host (CPU) tensors or numpy arrays, pinned
        for full bandwidth; returns when recvbuf holds the result."""
        check(lib().bine_allreduce_host(_host_ptr(sendbuf), _host_ptr(recvbuf), count, datatype, op, self._h))

    def allreduce_host_hooked(self, sendbuf, recvbuf, count, datatype, before=None, after=None, op=SUM):
        """bine_allreduce_host_hooked: `before(first, n)` runs before the
        input columns [first, first + n) go to the GPU, `after(first, n)`
        once those output columns are in host memory; a truthy return
        abandons the call (BineError with code ERR_ABORTED)."""
        def wrap(fn):
            return WINDOW_HOOK(lambda _u, first, n: 1 if fn(first, n) else 0) if fn else WINDOW_HOOK()
        hb, ha = wrap(before), wrap(after)  # kept alive for the call
        check(lib().bine_allreduce_host_hooked(_host_ptr(sendbuf), _host_ptr(recvbuf), count, datatype, op, self._h,
                                               hb, ha, None))

    def _equal_counts(self, count):
        """ctypes array of nranks copies of `count`, cached: building it per
        call costs more host time than a small call takes on the GPU."""
        cache = self.__dict__.setdefault("_counts_cache", {})
        if count not in cache:
            if len(cache) > 64:
                cache.clear()
            cache[count] = (ctypes.c_int * self.nranks)(*([count] * self.nranks))
        return cache[count]

    def reduce_scatter(self, sendbuf, recvbuf, recvcounts, datatype, op=SUM):
        if isinstance(recvcounts, ctypes.Array):
            rc = recvcounts
        else:
            rc = (ctypes.c_int * self.nranks)(*recvcounts)
        check(lib().bine_reduce_scatter(_ptr(sendbuf), _ptr(recvbuf), rc, datatype, op, self._h))

    def allgather(self, sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype):
        check(lib().bine_allgather(_ptr(sendbuf), sendcount, sendtype, _ptr(recvbuf), recvcount, recvtype, self._h))

    def bcast(self, buffer, count, datatype, root):
        check(lib().bine_bcast(_ptr(buffer), count, datatype, root, self._h))

    def alltoall(self, sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype):
        check(lib().bine_alltoall(_ptr(sendbuf), sendcount, sendtype, _ptr(recvbuf), recvcount, recvtype, self._h))

    def scatter(self, sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, root):
        check(lib().bine_scatter(_ptr(sendbuf), sendcount, sendtype, _ptr(recvbuf), recvcount, recvtype, root,
                                 self._h))

    def gather(self, sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, root):
        check(lib().bine_gather(_ptr(sendbuf), sendcount, sendtype, _ptr(recvbuf), recvcount, recvtype, root,
                                self._h))

    def reduce(self, sendbuf, recvbuf, count, datatype, op=SUM, root=0):
        check(lib().bine_reduce(_ptr(sendbuf), _ptr(recvbuf), count, datatype, op, root, self._h))

    def run(self, coll, sendbuf, recvbuf, count, datatype, root=0):
        """Dispatches by name with the reference's `count` meaning."""
        if coll == "allreduce":
            return self.allreduce(sendbuf, recvbuf, count, datatype)
        if coll == "reduce_scatter":
            return self.reduce_scatter(sendbuf, recvbuf, self._equal_counts(count), datatype)
        if coll == "allgather":
            return self.allgather(sendbuf, count, datatype, recvbuf, count, datatype)
        if coll == "bcast":
            return self.bcast(recvbuf, count, datatype, root)
        if coll == "reduce":
            return self.reduce(sendbuf, recvbuf, count, datatype, SUM, root)
        if coll == "alltoall":
            return self.alltoall(sendbuf, count, datatype, recvbuf, count, datatype)
        if coll == "scatter":
            return self.scatter(sendbuf, count, datatype, recvbuf, count, datatype, root)
        if coll == "gather":
            return self.gather(sendbuf, count, datatype, recvbuf, count, datatype, root)
        raise ValueError(coll)

    # -------------------------------------------- host schedule queries
    def plan_stats(self, coll, count, root=0):
        out = (ctypes.c_int64 * 5)()
        check(lib().bine_plan_stats(self._h, COLL_ID[coll], count, root, out))
        return dict(zip(["levels", "moves", "messages", "tmp_elems", "traffic_elems"], list(out)))

    def plan_verify(self, coll, count, root=0):
        """Raises Unsupported when the reference's schedule is wrong here."""
        check(lib().bine_plan_verify(self._h, COLL_ID[coll], count, root))

    def link_bytes(self, coll, count, datatype, out, root=0):
        """Per-link byte counts computed on the GPU into `out` (a CUDA
        uint64/int64 tensor of 2*ndims*P entries)."""
        check(lib().bine_link_bytes(self._h, COLL_ID[coll], count, datatype, root, _ptr(out)))

    def plan_moves(self, coll, count, root=0):
        n = ctypes.c_size_t(0)
        check(lib().bine_plan_moves(self._h, COLL_ID[coll], count, root, None, None, 0, ctypes.byref(n)))
        mv = np.zeros((max(1, n.value), 10), np.int64)
        sz = np.zeros(max(1, n.value), np.int64)
        check(lib().bine_plan_moves(self._h, COLL_ID[coll], count, root,
                                    mv.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                    sz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n.value, ctypes.byref(n)))
        return mv[: n.value], sz[: n.value] // 2, sz[: n.value] % 2

    def plan_flow(self, coll, count, root=0, elem_size=4, target_items=592):
        """Dataflow form of the schedule as the PIPELINED engine runs it:
        (pieces [n, 3] = move, start, n; items [n, 5] = piece begin/end,
        dependency begin/end, level; deps: item index or -(level + 1))."""
        npc, nit, ndp = ctypes.c_size_t(0), ctypes.c_size_t(0), ctypes.c_size_t(0)
        check(lib().bine_plan_flow(self._h, COLL_ID[coll], count, root, elem_size, target_items, None, 0,
                                   ctypes.byref(npc), None, 0, ctypes.byref(nit), None, 0, ctypes.byref(ndp)))
        pieces = np.zeros((max(1, npc.value), 3), np.int64)
        items = np.zeros((max(1, nit.value), 5), np.int32)
        deps = np.zeros(max(1, ndp.value), np.int32)
        i32p = ctypes.POINTER(ctypes.c_int32)
        check(lib().bine_plan_flow(self._h, COLL_ID[coll], count, root, elem_size, target_items,
                                   pieces.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), npc.value, ctypes.byref(npc),
                                   items.ctypes.data_as(i32p), nit.value, ctypes.byref(nit),
                                   deps.ctypes.data_as(i32p), ndp.value, ctypes.byref(ndp)))
        return pieces[: npc.value], items[: nit.value], deps[: ndp.value]

    def plan_fused(self, coll, count, root=0, levels=3):
        """Fused form of the call's schedule: (moves [n, 6] = (pass, elements,
        first leaf, leaves, first destination, destinations), leaves [n, 4] =
        (rank, buffer, additions, offset), destinations [n, 3] = (rank,
        buffer, offset), workspace elements per rank)."""
        nm, nl, nd, tmp = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int64()
        check(lib().bine_plan_fused(self._h, COLL_ID[coll], count, root, levels, None, 0, ctypes.byref(nm), None, 0,
                                    ctypes.byref(nl), None, 0, ctypes.byref(nd), ctypes.byref(tmp)))
        mv = np.zeros((max(1, nm.value), 6), np.int64)
        lv = np.zeros((max(1, nl.value), 4), np.int64)
        dv = np.zeros((max(1, nd.value), 3), np.int64)
        p64 = ctypes.POINTER(ctypes.c_int64)
        check(lib().bine_plan_fused(self._h, COLL_ID[coll], count, root, levels, mv.ctypes.data_as(p64), nm.value,
                                    ctypes.byref(nm), lv.ctypes.data_as(p64), nl.value, ctypes.byref(nl),
                                    dv.ctypes.data_as(p64), nd.value, ctypes.byref(nd), None))
        return mv[:nm.value], lv[:nl.value], dv[:nd.value], tmp.value

    def plan_messages(self, coll, count, root=0):
        n = ctypes.c_size_t(0)
        check(lib().bine_plan_messages(self._h, COLL_ID[coll], count, root, None, 0, ctypes.byref(n)))
        m = np.zeros((max(1, n.value), 4), np.int64)
        check(lib().bine_plan_messages(self._h, COLL_ID[coll], count, root,
                                       m.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n.value, ctypes.byref(n)))
        return m[: n.value]

    def plan_trees(self, coll, count, root=0):
        npg, nsg = ctypes.c_size_t(0), ctypes.c_size_t(0)
        check(lib().bine_plan_trees(self._h, COLL_ID[coll], count, root, None, 0, ctypes.byref(npg), None, 0,
                                    ctypes.byref(nsg)))
        prog = np.zeros((max(1, npg.value), 3), np.int64)
        segs = np.zeros((max(1, nsg.value), 6), np.int64)
        p64 = ctypes.POINTER(ctypes.c_int64)
        check(lib().bine_plan_trees(self._h, COLL_ID[coll], count, root, prog.ctypes.data_as(p64), npg.value,
                                    ctypes.byref(npg), segs.ctypes.data_as(p64), nsg.value, ctypes.byref(nsg)))
        return prog[: npg.value], segs[: nsg.value]

    def plan_tree_form(self, coll, count, datatype, root=0):
        """Host-only plan of the exact-order float kernels for this call:
        dict of form (0 element kernel only, 1 one lane per vector, 2 lanes
        per vector with per-segment tiles, 3 lanes per vector with
        row-aligned tiles), lanes, shapes, tiles, edges and element pieces."""
        o = np.zeros(6, np.int64)
        check(lib().bine_plan_tree_form(self._h, COLL_ID[coll], count, datatype, root,
                                        o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return dict(zip(("form", "lanes", "shapes", "tiles", "edges", "pieces"), (int(v) for v in o)))

    def plan_tree_cover(self, coll, count, datatype, root=0):
        """Host-only: the output runs each exact-order kernel of the plan
        writes, as an array of (first element, elements, kind) rows (kind 1
        vector tile, 2 edge vector, 3 element piece)."""
        n = ctypes.c_size_t(0)
        check(lib().bine_plan_tree_cover(self._h, COLL_ID[coll], count, datatype, root, None, 0, ctypes.byref(n)))
        runs = np.zeros((max(1, n.value), 3), np.int64)
        check(lib().bine_plan_tree_cover(self._h, COLL_ID[coll], count, datatype, root,
                                         runs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n.value,
                                         ctypes.byref(n)))
        return runs[: n.value]

    def tree_form(self, coll, count, datatype, root=0):
        """(form, lanes) of the exact-order float kernel for this call: form
        0 element kernel only, 1 one lane per vector, 2 lanes per vector
        with per-segment tiles, 3 lanes per vector with row-aligned tiles."""
        form, lanes = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().bine_debug_tree_form(self._h, COLL_ID[coll], count, datatype, root, ctypes.byref(form),
                                         ctypes.byref(lanes)))
        return form.value, lanes.value

    def link_bytes_host(self, coll, count, datatype, root=0):
        n = self.nranks * len(self.dims) * 2
        out = np.zeros(n, np.uint64)
        check(lib().bine_link_bytes_host(self._h, COLL_ID[coll], count, datatype, root,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n))
        return out


def row_counts(coll, count, P):
    """Per-rank (send, receive) element counts for the reference's `count`."""
    if coll in ("allreduce", "reduce"):
        return count, count
    if coll == "bcast":
        return 0, count
    if coll in ("reduce_scatter", "scatter"):
        return count * P, count
    if coll in ("allgather", "gather"):
        return count, count * P
    if coll == "alltoall":
        return count * P, count * P
    raise ValueError(coll)


class Batch:
    """Many allreduce / reduce_scatter / allgather calls in one persistent
    launch (bine_batch_*).  `items` are (coll, sendbuf, recvbuf, count,
    datatype, nranks[, send_stride, recv_stride]) tuples of CUDA tensors
    laid out (nranks, row); strides in bytes, 0 = packed rows."""

    def __init__(self, items, tuning=None):
        self._items = self.make_items(items)
        self._h = ctypes.c_void_p()
        tu = ctypes.byref(tuning) if tuning is not None else None
        check(lib().bine_batch_create(self._items, len(items), tu, ctypes.byref(self._h)))

    @staticmethod
    def make_items(items):
        arr = (BatchItem * max(1, len(items)))()
        for k, it in enumerate(items):
            coll, send, recv, count, dt, P = it[:6]
            arr[k].send_stride = it[6] if len(it) > 6 else 0
            arr[k].recv_stride = it[7] if len(it) > 7 else 0
            arr[k].coll = COLL_ID[coll]
            arr[k].datatype = dt
            arr[k].nranks = P
            arr[k].count = count
            arr[k].sendbuf = _ptr(send)
            arr[k].recvbuf = _ptr(recv)
        return arr

    def launch(self, stream=None):
        h = stream if isinstance(stream, int) else (stream.cuda_stream if stream is not None else 0)
        check(lib().bine_batch_launch(self._h, h))

    def close(self):
        if getattr(self, "_h", None):
            lib().bine_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def autotune(items, stream=None, reps=3):
        arr = Batch.make_items(items)
        best = BatchTuning()
        ms = ctypes.c_float()
        h = stream if isinstance(stream, int) else (stream.cuda_stream if stream is not None else 0)
        check(lib().bine_batch_autotune(arr, len(items), h, reps, ctypes.byref(best), ctypes.byref(ms)))
        return best, ms.value


def mlp_layout(in_dim, hidden, out_dim):
    """Parameter arena of bine_mlp: per layer (weight offset, bias offset,
    out, in); weights row-major [out, in], every block padded to 16 floats."""
    dims = [in_dim, hidden, hidden, hidden, out_dim]
    off, out = 0, []
    for l in range(4):
        w = off
        off = (off + dims[l] * dims[l + 1] + 15) // 16 * 16
        b = off
        off = (off + dims[l + 1] + 15) // 16 * 16
        out.append((w, b, dims[l + 1], dims[l]))
    return out


class MLP:
    """bine_mlp_*: in -> H -> H -> H -> out MLP (GELU, bf16 weights and
    activations, fp32 accumulation) trained with the engine's own kernels."""

    def __init__(self, in_dim, hidden, out_dim, max_batch, seed=0):
        self.dims = (in_dim, hidden, out_dim)
        self.max_batch = max_batch
        self._h = ctypes.c_void_p()
        self._check(lib().bine_mlp_create(in_dim, hidden, out_dim, max_batch, seed, ctypes.byref(self._h)))
        n = ctypes.c_size_t()
        self._check(lib().bine_mlp_num_params(self._h, ctypes.byref(n)))
        self.nparams = n.value

    def _check(self, rc):
        if rc != SUCCESS:
            raise BineError(rc, lib().bine_mlp_last_error().decode())

    def layout(self):
        """(weight offset, bias offset, out, in) per layer in the parameter arena."""
        return mlp_layout(*self.dims)

    def get_params(self):
        out = np.zeros(self.nparams, np.float32)
        self._check(lib().bine_mlp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        self._check(lib().bine_mlp_set_params(self._h, p.ctypes.data))

    def forward(self, x, stream=None):
        """x: CUDA float32 tensor [n, in] (n multiple of 16) -> [n, out]."""
        import torch
        y = torch.empty((x.shape[0], self.dims[2]), dtype=torch.float32, device=x.device)
        h = stream.cuda_stream if stream is not None else 0
        self._check(lib().bine_mlp_forward(self._h, x.data_ptr(), x.shape[0], y.data_ptr(), h))
        return y

    def gradients(self, x, t, mask):
        g = np.zeros(self.nparams, np.float32)
        loss = ctypes.c_float()
        self._check(lib().bine_mlp_gradients(self._h, x.data_ptr(), t.data_ptr(), mask.data_ptr(), x.shape[0],
                                             g.ctypes.data, ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, x, t, mask, lr, stream=None):
        loss = ctypes.c_float()
        h = stream.cuda_stream if stream is not None else 0
        self._check(lib().bine_mlp_train_step(self._h, x.data_ptr(), t.data_ptr(), mask.data_ptr(), x.shape[0], lr,
                                              h, ctypes.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "_h", None):
            lib().bine_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """bine_mlp_ensemble_*: the mean output of 1..8 MLPs of one shape
    (hidden width 256), computed by one fused launch."""

    def __init__(self, mlps):
        self.mlps = list(mlps)
        self.dims = self.mlps[0].dims
        arr = (ctypes.c_void_p * len(self.mlps))(*[m._h.value for m in self.mlps])
        self._h = ctypes.c_void_p()
        self._check(lib().bine_mlp_ensemble_create(arr, len(self.mlps), ctypes.byref(self._h)))

    def _check(self, rc):
        if rc != SUCCESS:
            raise BineError(rc, lib().bine_mlp_last_error().decode())

    def forward(self, x, stream=None, out=None):
        """x: CUDA float32 tensor [n, in] (n multiple of 16) -> mean [n, out]."""
        import torch
        y = out if out is not None else torch.empty((x.shape[0], self.dims[2]), dtype=torch.float32, device=x.device)
        h = stream.cuda_stream if stream is not None else 0
        self._check(lib().bine_mlp_ensemble_forward(self._h, x.data_ptr(), x.shape[0], y.data_ptr(), h))
        return y

    def close(self):
        if getattr(self, "_h", None):
            lib().bine_mlp_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
