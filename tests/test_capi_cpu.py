"""The C ABI library loads and exports every entry point include/*.h
declares; argument checks work without a GPU."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(bine_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(bine.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_comm_argument_checks():
    with pytest.raises(bine.BineError):
        bine.Comm(0)
    with pytest.raises(bine.BineError):
        bine.Comm(12, [3, 5])  # does not multiply to 12
    with pytest.raises(bine.BineError):
        bine.Comm(8, [8, 1])  # size-1 dimension
    c = bine.Comm(8)
    with pytest.raises(bine.BineError):
        c.set_ports(7)
    with pytest.raises(KeyError):
        c.set_algo("allreduce", "NOPE")


def test_unsupported_cases_report_the_reference_line():
    c = bine.Comm(6)
    c.set_algo("allreduce", "B_CONT")
    with pytest.raises(bine.Unsupported) as e:
        c.plan_stats("allreduce", 60)
    assert "lib/libbine_common.cc" in str(e.value)
    c.set_algo("allreduce", "B")
    with pytest.raises(bine.Unsupported):
        c.plan_stats("allreduce", 5)  # count < ports * P (lib/libbine.cc:1036)


def test_collective_argument_errors_are_reported_before_any_device_work():
    """The checks the reference leaves to asserts (lib/libbine.cc:1035-1036,
    1170-1171) come back as BINE_ERR_ARG, on a host without a GPU too; a
    zero count is a no-op that succeeds without touching the device."""
    c = bine.Comm(8)
    fake = 1 << 20  # an address never dereferenced: every case fails or returns first
    err = lambda f: pytest.raises(bine.BineError, match="bine error 1:")  # noqa: E731
    with err(None):
        c.allreduce(fake, fake, -1, bine.INT32)
    with err(None):
        c.allreduce(fake, fake, 16, 99)
    with err(None):
        c.allreduce(fake, fake, 16, bine.INT32, op=1)
    with err(None):
        c.reduce(fake, fake, 16, bine.INT32, root=8)
    with err(None):
        c.bcast(fake, 16, bine.INT32, -1)
    with err(None):
        c.allreduce(None, fake, 16, bine.INT32)
    c.set_layout(16, 16)  # stride of 16 bytes < 16 int32 per rank
    with err(None):
        c.allreduce(fake, fake, 16, bine.INT32)
    c.set_layout(0, 0)
    for coll in bine.COLLS:
        c.run(coll, fake, fake, 0, bine.INT32)  # count 0: nothing to do
    c.allreduce_host(np.zeros((8, 1), np.int32), np.zeros((8, 1), np.int32), 0, bine.INT32)
    with err(None):
        c.set_tree_split(3)
    with err(None):
        c.set_host_window(100)
    with err(None):
        c.set_segment(-5)


def test_hooked_host_allreduce_argument_errors_and_zero_count():
    """bine_allreduce_host_hooked rejects a null communicator and any op but
    SUM before touching the device; with count 0 it succeeds without calling
    either hook."""
    L = bine.lib()
    z = np.zeros((8, 1), np.int32)
    null_hook = bine.WINDOW_HOOK()
    assert L.bine_allreduce_host_hooked(z.ctypes.data, z.ctypes.data, 1, bine.INT32, bine.SUM, None,
                                        null_hook, null_hook, None) == bine.ERR_ARG
    c = bine.Comm(8)
    with pytest.raises(bine.BineError, match="bine error 1:"):
        c.allreduce_host_hooked(z, z, 1, bine.INT32, op=1)
    calls = []
    c.allreduce_host_hooked(z, z, 0, bine.INT32, before=lambda f, n: calls.append(f), after=lambda f, n: calls.append(f))
    assert calls == []
