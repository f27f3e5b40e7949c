"""The benchmark sweep's correctness checks (bench.py sweep_check), on the CPU.

The sweep checks float32 sums in the reference's order bit for bit against
the oracle: whole inputs when they are small, and otherwise four columns of
every block, because an element's addition tree depends only on the block it
lies in.  Here the sampled path is forced on small inputs and must accept the
oracle's own full result and reject a result with one sampled element off by
one ulp; the FAST-order check accepts FP64-rounded sums and rejects an error
of 1e-5 relative.
"""
import numpy as np
import pytest
import torch

import bench
from oracle import port


@pytest.mark.parametrize("coll,P,count", [("allreduce", 16, 16 * 37 + 5), ("allreduce", 12, 12 * 50),
                                          ("reduce_scatter", 16, 29)])
@pytest.mark.parametrize("sampled", [False, True])
def test_reference_order_check_is_bit_exact(coll, P, count, sampled, monkeypatch):
    if sampled:
        monkeypatch.setattr(bench, "REF_ORDER_FULL_BYTES", 0)
    se = count if coll == "allreduce" else count * P
    x = np.random.default_rng(P + count).standard_normal((P, se)).astype(np.float32)
    full, _ = port.run(coll, x, count, variant="B" if coll == "allreduce" else None)
    send, recv = torch.from_numpy(x), torch.from_numpy(full.copy())
    assert bench.sweep_check(coll, send, recv, P, count, True, "reference", ref_cache={})
    cols, _ = bench.ref_order_columns(coll, P, count)
    bad = full.copy()
    if coll == "allreduce":
        j = int(cols[-1]) if cols is not None else count - 1
        bad[P - 1, j] = np.nextafter(bad[P - 1, j], np.float32(np.inf))
    else:
        bad[P - 1, count - 1] = np.nextafter(bad[P - 1, count - 1], np.float32(np.inf))
    assert not bench.sweep_check(coll, send, torch.from_numpy(bad), P, count, True, "reference", ref_cache={})


def test_sampled_columns_cover_four_positions_of_every_block(monkeypatch):
    monkeypatch.setattr(bench, "REF_ORDER_FULL_BYTES", 0)
    P, count = 8, 8 * 10 + 3
    cols, n = bench.ref_order_columns("allreduce", P, count)
    sizes = [count // P + (b < count % P) for b in range(P)]
    offs = np.cumsum([0] + sizes[:-1])
    assert n == 4 * P and len(cols) == 4 * P
    for b in range(P):
        assert list(cols[4 * b:4 * b + 4]) == [offs[b], offs[b] + 1, offs[b] + sizes[b] // 2, offs[b] + sizes[b] - 1]


def test_fast_order_check_bound():
    P, count = 64, 1000
    x = np.random.default_rng(3).standard_normal((P, count)).astype(np.float32)
    s = x.astype(np.float64).sum(0)
    send = torch.from_numpy(x)
    good = torch.from_numpy(np.tile(s.astype(np.float32), (P, 1)))
    assert bench.sweep_check("allreduce", send, good, P, count, True, "fast")
    off = s.astype(np.float32).copy()
    off[7] = np.float32(s[7] * (1 + 1e-5) + 1e-3)
    assert not bench.sweep_check("allreduce", send, torch.from_numpy(np.tile(off, (P, 1))), P, count, True, "fast")
