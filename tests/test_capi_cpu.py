"""The C ABI library loads and exports every entry point include/*.h
declares; argument checks work without a GPU."""
import ctypes
import glob
import os
import re

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
