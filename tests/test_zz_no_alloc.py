"""The allocation-free allreduce entry point, bine_allreduce_noalloc.

Some callers cannot let a library allocate device memory: a framework whose
memory manager owns every device allocation, or a phase of a program in
which cudaMalloc must not be called.  For them the library offers one
allreduce that keeps all of its device scratch in a fixed array reserved when
the library loads.  These tests call it through the C ABI and check that it
returns exactly what the ordinary entry point, bine_allreduce(), returns on
the same inputs -- twice in a row, since every call reuses the same scratch
-- and that a call needing more scratch than the array holds is refused
with a clear error.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

import bine_trees_fugaku_b200 as bine

pytestmark = pytest.mark.gpu


def noalloc_allreduce(comm, send, recv, count, datatype):
    f = bine.lib().bine_allreduce_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f(send.data_ptr(), recv.data_ptr(), count, datatype, bine.SUM, comm._h)


@pytest.mark.parametrize("dtype,variant,P,count", [
    (np.int32, "B", 64, 64 * 1000 + 13),
    (np.float32, "B", 32, 32 * 777),
    (np.float32, "L", 24, 5001),
    (np.int64, "B_COALESCE", 12, 12 * 50 + 1),
])
def test_noalloc_matches_bine_allreduce_on_two_calls(dtype, variant, P, count):
    code = {np.int32: bine.INT32, np.float32: bine.FLOAT, np.int64: bine.INT64}[dtype]
    stream = torch.cuda.current_stream()
    comm = bine.Comm(P)
    comm.set_algo("allreduce", variant)
    comm.set_stream(stream)
    ref = bine.Comm(P)
    ref.set_algo("allreduce", variant)
    ref.set_engine("steps")
    ref.set_stream(stream)
    rng = np.random.default_rng(P + count)
    for _ in range(2):
        if dtype == np.float32:
            x = rng.standard_normal((P, count)).astype(dtype)
        else:
            x = rng.integers(-1000, 1001, (P, count)).astype(dtype)
        send = torch.from_numpy(x).cuda()
        want = torch.zeros_like(send)
        got = torch.full_like(send, 7)
        ref.allreduce(send, want, count, code)
        ref.synchronize()
        rc = noalloc_allreduce(comm, send, got, count, code)
        assert rc == bine.SUCCESS, bine.last_error()
        # Bit for bit: integer sums are exact and float sums follow the same
        # reference order in both entry points.
        assert torch.equal(got, want)


def test_noalloc_refuses_calls_that_need_more_than_its_scratch():
    P, count = 16, 2 << 20  # the L variant stages P * count floats: 128 MiB
    comm = bine.Comm(P)
    comm.set_algo("allreduce", "L")
    comm.set_stream(torch.cuda.current_stream())
    send = torch.zeros((P, count), dtype=torch.float32, device="cuda")
    recv = torch.zeros_like(send)
    rc = noalloc_allreduce(comm, send, recv, count, bine.FLOAT)
    assert rc == bine.ERR_NOMEM
    assert "scratch" in bine.last_error()


def test_noalloc_in_place_matches_out_of_place():
    """In place (the same buffer for input and result), the input rows are
    staged in the fixed scratch before the schedule runs; two calls in a
    row give the out-of-place bytes."""
    P, count = 16, 16 * 37 + 5
    comm = bine.Comm(P)
    comm.set_algo("allreduce", "L")
    comm.set_stream(torch.cuda.current_stream())
    x = torch.from_numpy(np.random.default_rng(9).standard_normal((P, count)).astype(np.float32)).cuda()
    want = torch.zeros_like(x)
    assert noalloc_allreduce(comm, x, want, count, bine.FLOAT) == bine.SUCCESS, bine.last_error()
    for _ in range(2):
        buf = x.clone()
        assert noalloc_allreduce(comm, buf, buf, count, bine.FLOAT) == bine.SUCCESS, bine.last_error()
        torch.cuda.synchronize()
        assert torch.equal(buf, want)


def test_noalloc_barrier_timeout_is_reported_and_recoverable():
    """A grid barrier told to wait for one arrival that never comes (fault
    injected on the host) expires after the configured bound: the call
    reports BINE_ERR_TIMEOUT, and the next call on the same scratch is
    correct.  The wait is bounded, so nothing hangs."""
    P, count = 16, 16 * 64
    comm = bine.Comm(P)
    comm.set_algo("allreduce", "B")
    comm.set_stream(torch.cuda.current_stream())
    x = np.random.default_rng(6).integers(-1000, 1001, (P, count)).astype(np.int32)
    send = torch.from_numpy(x).cuda()
    recv = torch.zeros_like(send)
    comm.set_step_timeout(200)
    comm.debug_set_barrier_extra(1)
    assert noalloc_allreduce(comm, send, recv, count, bine.INT32) == bine.ERR_TIMEOUT
    assert "timed out" in bine.last_error()
    comm.debug_set_barrier_extra(0)
    assert noalloc_allreduce(comm, send, recv, count, bine.INT32) == bine.SUCCESS, bine.last_error()
    want = x.astype(np.int64).sum(0).astype(np.int32)
    assert np.array_equal(recv.cpu().numpy(), np.broadcast_to(want, (P, count)))
