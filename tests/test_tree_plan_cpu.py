"""Host plan of the exact-order float reduction kernels (no GPU).

bine_plan_tree_form runs the planner's tree and tile logic without
uploading anything: which kernel form a call gets, how many tree shapes
its segments have, how many row tiles and straddling edge vectors the
row-aligned form plans, and how many element pieces are left for the
element kernels.  The GPU tests compare the results of these plans bit for
bit with the oracle; these tests pin the plans themselves."""
import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine

L = 4  # float32 elements per 16-byte vector


def plan(P, count, variant="B"):
    c = bine.Comm(P)
    c.set_algo("allreduce", variant)
    try:
        return c.plan_tree_form("allreduce", count, bine.FLOAT), c.plan_trees("allreduce", count)
    finally:
        c.close()


def straddling_boundaries(segs):
    """Segment starts (other than the first) inside a 16-byte vector."""
    offs = np.sort(segs[:, 0])
    return int(np.sum(offs[1:] % L != 0))


@pytest.mark.parametrize("P,count", [(96, 524_288), (384, 524_288), (1000, 1_048_576), (96, 96 * 40 + 4)])
def test_one_shape_calls_plan_row_tiles_and_cover_every_edge(P, count):
    f, (prog, segs) = plan(P, count)
    assert f["form"] == 3 and f["shapes"] == 1 and f["lanes"] > 1
    # Every vector that straddles two segments is an edge evaluated whole,
    # so no element piece is left (the count is a whole number of vectors).
    assert f["edges"] == straddling_boundaries(segs)
    assert f["pieces"] == 0
    # Row tiles cover every body vector: at least one tile per tile width.
    width = (256 // f["lanes"]) * L
    assert f["tiles"] >= count // width


def test_counts_on_the_vector_grid_have_no_edges():
    f, (_, segs) = plan(96, 96 * 5504)
    assert straddling_boundaries(segs) == 0
    assert f["form"] == 3 and f["edges"] == 0 and f["pieces"] == 0


def test_a_partial_last_vector_stays_an_element_piece():
    f, (_, segs) = plan(1000, 1_048_577)
    assert f["form"] == 3 and f["pieces"] == 1
    assert f["edges"] == straddling_boundaries(segs)


@pytest.mark.parametrize("P,count,shapes", [(200, 200 * 1000 + 17, 3), (76, 76 * 3000 + 5, 7), (46, 46 * 2000 + 1, 3)])
def test_several_tree_shapes_keep_the_row_aligned_form(P, count, shapes):
    f, (prog, segs) = plan(P, count)
    distinct = {tuple(prog[s[3]:s[3] + s[4], 1]) for s in segs}
    assert len(distinct) == shapes
    assert f["form"] == 3 and f["shapes"] == shapes


def test_more_than_eight_shapes_fall_back_to_per_segment_tiles():
    f, (prog, segs) = plan(70, 70 * 1000 + 9)
    assert len({tuple(prog[s[3]:s[3] + s[4], 1]) for s in segs}) == 9
    assert f["form"] == 2 and f["shapes"] == 0 and f["edges"] == 0


def test_segments_too_short_for_row_tiles_fall_back():
    # 8-element segments: a 32-vector tile would hold 16 of them.
    f, _ = plan(96, 96 * 8)
    assert f["form"] == 2


def test_debug_form_matches_the_plan():
    c = bine.Comm(384)
    c.set_algo("allreduce", "B")
    try:
        f = c.plan_tree_form("allreduce", 524_288, bine.FLOAT)
        assert c.tree_form("allreduce", 524_288, bine.FLOAT) == (f["form"], f["lanes"])
    finally:
        c.close()


def test_plan_rejects_integer_types_and_non_reductions():
    c = bine.Comm(16)
    try:
        with pytest.raises(bine.BineError):
            c.plan_tree_form("allreduce", 1024, bine.INT32)
        with pytest.raises(bine.BineError):
            c.plan_tree_form("allgather", 1024, bine.FLOAT)
    finally:
        c.close()


def coverage(P, count, variant="B"):
    c = bine.Comm(P)
    c.set_algo("allreduce", variant)
    try:
        runs = c.plan_tree_cover("allreduce", count, bine.FLOAT)
    finally:
        c.close()
    hits = np.zeros(count + 1, np.int64)
    np.add.at(hits, runs[:, 0], 1)
    np.add.at(hits, runs[:, 0] + runs[:, 1], -1)
    return np.cumsum(hits)[:count], runs


@pytest.mark.parametrize("P,count", [
    (96, 524_288), (96, 96 * 40 + 3), (384, 384 * 100 + 1), (1000, 1000 * 130 + 3), (1000, 1_048_577),
    (200, 200 * 1000 + 17), (76, 76 * 3000 + 5), (46, 46 * 2000 + 1), (70, 70 * 1000 + 9), (96, 96 * 8),
    (256, 1 << 16), (24, 24 * 1000 + 3),
])
def test_every_output_element_is_written_exactly_once(P, count):
    """The runs the kernels of the plan write (row-tile lane vectors as the
    kernel finds their segment, edge vectors, element pieces; or the tiles
    of the per-segment forms) cover the output row once each, with no
    element written twice: the condition for every kernel to run beside the
    others without a race, and for no element to be left unwritten."""
    cover, runs = coverage(P, count)
    assert cover.min() == 1 and cover.max() == 1
    assert np.all(runs[:, 1] > 0)
