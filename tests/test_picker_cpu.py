"""Host logic of the learned variant picker: arm space, features, the fixed
rule, validity against the planner's proofs, targets and the evaluation
arithmetic.  No GPU."""
import json

import numpy as np
import pytest

import bine_trees_fugaku_b200 as bine
from bine_trees_fugaku_b200 import picker as pk


def test_arm_space_shape():
    assert len(pk.ARMS) == pk.NARMS == len(set(pk.ARMS))
    assert pk.OUT_DIM % 16 == 0 and pk.OUT_DIM >= 2 * pk.NARMS
    assert pk.IN_DIM % 16 == 0
    for coll in pk.OPS:
        assert any(a[0] == coll for a in pk.ARMS)


def test_features_are_bounded_and_distinguish_calls():
    a = pk.features("allreduce", 256, 1 << 20, 4)
    b = pk.features("allreduce", 256, 1 << 10, 4)
    c = pk.features("allgather", 256, 1 << 10, 4, [16, 16])
    for f in (a, b, c):
        assert f.shape == (pk.IN_DIM,) and f.dtype == np.float32
        assert np.all(f >= 0) and np.all(f <= 1.5)
    assert not np.array_equal(a, b) and not np.array_equal(b, c)


@pytest.mark.parametrize("coll,P,count,want", [
    ("allreduce", 64, 1 << 20, ("allreduce", "B", 6, 65536)),       # 4 MiB: 6 ports, 64 KiB segments
    ("allreduce", 64, 1024, ("allreduce", "B", 1, 0)),              # 4 KiB: 1 port, no segmenting
    ("allreduce", 64, 16, ("allreduce", "L", 1, 0)),                # count < P: latency tree
    ("allreduce", 256, 1 << 16, ("allreduce", "B_COALESCE", 6, 65536)),  # per-block B beyond the planning cap
    ("allreduce", 1024, 1 << 16, ("allreduce", "B_CONT", 6, 65536)),
    ("allreduce", 1000, 1 << 16, ("allreduce", "L", 6, 65536)),
    ("reduce_scatter", 64, 256, ("reduce_scatter", "VEC_HALVING_CONT_PERMUTE", 1, 4096)),
    ("allgather", 64, 256, ("allgather", "VEC_DOUBLING_CONT_PERMUTE", 1, 4096)),
    ("allgather", 48, 256, ("allgather", "VEC_DOUBLING_BLOCKS", 1, 4096)),
])
def test_fixed_rule(coll, P, count, want):
    assert pk.ARMS[pk.fixed_rule(coll, P, count, 4)] == want


def test_statically_valid_arms_are_planned_or_refused_cleanly():
    """Every arm the picker offers either plans and proves, or the planner
    refuses it with BINE_ERR_UNSUPPORTED (never another error)."""
    for cfg in pk.sample_configs(40, seed=5):
        if cfg["P"] > 128:
            continue
        comm = bine.Comm(cfg["P"], cfg["dims"] if len(cfg["dims"]) > 1 else None)
        for arm in pk.ARMS:
            if arm[3] or not pk.statically_valid(arm, cfg["coll"], cfg["P"], cfg["count"], cfg["dims"]):
                continue
            pk.apply_arm(comm, arm)
            try:
                comm.plan_verify(cfg["coll"], cfg["count"])
            except bine.Unsupported:
                pass
        comm.close()


def test_sampled_calls_respect_limits():
    cfgs = pk.sample_configs(500, seed=1)
    for c in cfgs:
        assert 4 <= c["P"] <= 4096 and c["count"] >= 1
        assert int(np.prod(c["dims"])) == c["P"]
        assert c["P"] * pk.message_bytes(c["coll"], c["P"], c["count"], c["es"]) <= (2 << 30) + c["P"] * 4
        if c["coll"] != "allreduce":
            assert c["P"] <= pk.MAX_P_VECTOR
    assert {c["coll"] for c in cfgs} == set(pk.OPS)


def test_picker_without_weights_falls_back_past_refused_arms():
    """At P=23 the reference's B deadlocks; the fixed rule names B, the
    planner refuses it, and the picker falls back to the L tree."""
    p = pk.Picker(path=None)
    comm = bine.Comm(23)
    arm = p.choose(comm, "allreduce", 95239, bine.INT32)
    assert arm[1] == "L"
    comm.plan_verify("allreduce", 95239)
    comm.close()
    comm = bine.Comm(64)
    assert p.choose(comm, "allreduce", 1 << 20, bine.INT32) == ("allreduce", "B", 6, 65536)
    comm.close()


def test_picker_reports_when_nothing_runs():
    """reduce_scatter at non-power-of-two P: the reference's only variant
    returns wrong data, so no arm is offered."""
    p = pk.Picker(path=None)
    comm = bine.Comm(91)
    with pytest.raises(bine.Unsupported):
        p.choose(comm, "reduce_scatter", 852, bine.INT32)
    comm.close()


def test_targets_mask_invalid_arms():
    T = np.array([[10.0, np.nan] + [np.nan] * (pk.NARMS - 2), [20.0, 40.0] + [np.nan] * (pk.NARMS - 2)])
    Lb = np.where(np.isnan(T), np.nan, 1024.0)
    valid = ~np.isnan(T)
    Y, M, st = pk.targets(T, Lb, valid, relative=False)
    assert Y.shape == (2, pk.OUT_DIM) and M.shape == (2, pk.OUT_DIM)
    assert M[0, 0] == 1 and M[0, 1] == 0 and M[1, 1] == 1 and M[:, 2 * pk.NARMS:].sum() == 0
    assert np.all(np.isfinite(Y))
    lt = np.log2([10.0, 20.0, 40.0])
    assert st["t_mean"] == pytest.approx(lt.mean())
    # Relative targets: each call's best arm is 0 before standardisation
    # (log2 times 0; 0 and 1), and the ordering within a call is kept.
    Yr, Mr, sr = pk.targets(T, Lb, valid)
    assert sr["t_mean"] == pytest.approx(1.0 / 3.0) and sr["relative"]
    assert Yr[1, 0] < Yr[1, 1] and np.array_equal(Mr, M)


def test_evaluate_perfect_and_fixed_rule_arithmetic():
    cfgs = [{"coll": "allreduce", "P": 64, "count": 1 << 20, "es": 4, "dims": [64]}]
    T = np.full((1, pk.NARMS), np.nan)
    Lb = np.full((1, pk.NARMS), np.nan)
    fa = pk.fixed_rule("allreduce", 64, 1 << 20, 4)
    best = pk.ARMS.index(("allreduce", "B_CONT", 6, 65536))
    T[0, fa], T[0, best] = 200.0, 100.0
    Lb[0, fa], Lb[0, best] = 1000.0, 3000.0
    valid = ~np.isnan(T)
    pred = np.zeros((1, pk.OUT_DIM))
    pred[0, :pk.NARMS] = np.log2(np.nan_to_num(T[0], nan=1e9))
    pred[0, pk.NARMS:2 * pk.NARMS] = np.log2(np.nan_to_num(Lb[0], nan=1e12))
    ev = pk.evaluate(pred, T, Lb, valid, cfgs)
    assert ev["pick_within_5pct_of_optimum"] == 1.0
    assert ev["speedup_vs_fixed_rule_geomean"] == pytest.approx(2.0)
    assert ev["fixed_rule_within_5pct_of_optimum"] == 0.0
    assert ev["link_pick_is_minimum"] == 1.0


def test_saved_weights_are_the_bf16_forward_values(tmp_path):
    class Fake:
        def get_params(self):
            return np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.14159], np.float32)

    path = tmp_path / "w.npz"
    pk.save(str(path), Fake(), {"t_mean": 0.0}, {"calls": 0})
    p, dims, st, meta, arms = pk.load_params(str(path))
    assert p.shape == (1, 5) and list(p[0]) == [1.0, 1.0, 1.0078125, -2.5, 3.140625]
    pk.save(str(path), [Fake(), Fake()], {"t_mean": 0.0}, {"calls": 0})
    p, _, _, meta, _ = pk.load_params(str(path))
    assert p.shape == (2, 5) and meta["models"] == 2
    assert dims == (pk.IN_DIM, 256, pk.OUT_DIM) and [tuple(a) for a in arms] == pk.ARMS
    assert json.dumps(st) and meta["calls"] == 0


def test_picker_keeps_variant_and_ports_of_reference_order_float_sums():
    """A float32 sum in the reference's order is a different addition tree
    per variant and port count, so the picker chooses only the segment for
    it; integer calls and FAST-order calls on the FUSED engine are free."""
    p = pk.Picker(path=None)
    comm = bine.Comm(64)
    comm.set_engine("steps")
    comm.set_algo("allreduce", "L")
    comm.set_ports(2)
    arm = p.choose(comm, "allreduce", 1 << 20, bine.FLOAT)
    assert arm[:3] == ("allreduce", "L", 2)
    assert (comm.algo["allreduce"], comm.ports) == ("L", 2)
    free = bine.Comm(64)
    free.set_engine("steps")
    assert p.choose(free, "allreduce", 1 << 20, bine.INT32) == ("allreduce", "B", 6, 65536)
    fast = bine.Comm(64)
    fast.set_float_order("fast")
    assert p.choose(fast, "allreduce", 1 << 20, bine.FLOAT) == ("allreduce", "B", 6, 65536)
    assert pk.order_bound("allreduce", bine.FLOAT, "fused", "reference")
    assert pk.order_bound("reduce_scatter", bine.DOUBLE, "pipelined", "fast")
    assert not pk.order_bound("allreduce", bine.FLOAT, "fused", "fast")
    assert not pk.order_bound("allgather", bine.FLOAT, "steps", "reference")
    assert not pk.order_bound("allreduce", bine.INT64, "steps", "reference")
    for c in (comm, free, fast):
        c.close()


def test_evaluation_restricts_float_reductions_to_the_segment_choice():
    cfg = {"coll": "allreduce", "P": 64, "count": 1 << 20, "es": 4, "dtype": "float"}
    m = pk.allowed_arms(cfg)
    fa = pk.ARMS[pk.fixed_rule("allreduce", 64, 1 << 20, 4)]
    assert m.sum() == len(pk.SEGMENTS)
    assert all(pk.ARMS[a][1:3] == fa[1:3] for a in np.nonzero(m)[0])
    assert pk.allowed_arms(dict(cfg, dtype="int32")).all()
