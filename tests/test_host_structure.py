"""C++ structure compiler vs the oracle (CPU only, through the C ABI).

Block keys, shapes, strides and offsets must be bit-exact
(tenet-core/src/fusion_space.rs:2211-2262, 3953-4104); recoupling and compose
tables are replayed in numpy and compared with the oracle's Host-path
restatement to 1e-12 relative.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule, su2_f
from oracle.tensor import TensorMap as OT
from tests.helpers import product_rule, product_space, replay_compose, replay_transform

U1R = Rule([U1])
SU2R = Rule([SU2])
FZ2R = Rule([FZ2])
I3 = Rule([FZ2, U1, SU2])

V_U1 = Leg.new(U1R, [((-2,), 4), ((-1,), 8), ((0,), 12), ((1,), 8), ((2,), 4)])
V_U1_SMALL = Leg.new(U1R, [((-1,), 2), ((0,), 3), ((1,), 2)])
V_SU2 = Leg.new(SU2R, [((0,), 2), ((1,), 2), ((2,), 1)])
W_SU2 = Leg.new(SU2R, [((0,), 3), ((1,), 2), ((2,), 2), ((3,), 1)])
P_SU2 = Leg.new(SU2R, [((1,), 1)])
V_FZ2 = Leg.new(FZ2R, [((0,), 2), ((1,), 3)])
V_I3 = Leg.new(I3, [((0, 0, 0), 2), ((1, 1, 1), 2), ((0, 2, 0), 1), ((1, -1, 1), 1)])
P_I3 = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])

SPACES = {
    "u1_config": (U1R, [V_U1, V_U1], [V_U1, V_U1]),
    "u1_small_dual": (U1R, [V_U1_SMALL, V_U1_SMALL.dual()], [V_U1_SMALL]),
    "su2_rank4": (SU2R, [V_SU2, V_SU2], [V_SU2, V_SU2]),
    "su2_mps": (SU2R, [W_SU2, P_SU2], [W_SU2]),
    "su2_rank3_1": (SU2R, [W_SU2, P_SU2, P_SU2], [W_SU2]),
    "fz2": (FZ2R, [V_FZ2, V_FZ2], [V_FZ2, V_FZ2.dual()]),
    "i3": (I3, [V_I3, P_I3], [P_I3, V_I3]),
}


def oracle_keys(space: OHom):
    return [blk["key"] for blk in space.blocks]


@pytest.mark.parametrize("name", sorted(SPACES))
def test_layout_and_keys_bit_exact(name):
    rule, cod, dom = SPACES[name]
    ref = OHom(rule, cod, dom)
    sp = product_space(rule, cod, dom)
    assert sp.size == ref.size
    assert [(lab, r, c, o) for lab, r, c, o in sp.sectors()] == [(c, r, cc, o) for c, r, cc, o in ref.sectors]
    got = sp.blocks()
    assert len(got) == len(ref.blocks)
    for (off, shape, strides, sidx), blk in zip(got, ref.blocks):
        assert off == blk["offset"] and shape == blk["shape"] and strides == blk["strides"] and sidx == blk["sector"]
    assert sp.block_keys() == oracle_keys(ref)


PERMS = [
    ("u1_config", [0, 3], [2, 1]),
    ("u1_config", [1, 0], [3, 2]),
    ("u1_config", [2, 3], [0, 1]),
    ("u1_small_dual", [2, 0], [1]),
    ("su2_rank4", [1, 0], [3, 2]),
    ("su2_rank4", [0, 3], [2, 1]),
    ("su2_rank4", [3], [0, 1, 2]),
    ("su2_mps", [0], [2, 1]),
    ("su2_rank3_1", [0, 1], [2, 3]),
    ("su2_rank3_1", [2, 1, 0], [3]),
    ("su2_rank3_1", [3, 1], [0, 2]),
    ("fz2", [1, 0], [3, 2]),
    ("fz2", [3, 0], [1, 2]),
    ("i3", [0, 3], [2, 1]),
    ("i3", [1, 0], [3, 2]),
]


@pytest.mark.parametrize("name,p1,p2", PERMS)
def test_permute_tables_replay_matches_oracle(name, p1, p2):
    rule, cod, dom = SPACES[name]
    rng = np.random.default_rng(7)
    src = OT(OHom(rule, cod, dom), rng.standard_normal(OHom(rule, cod, dom).size))
    ref = src.permute(p1, p2)
    from tenet_b200.typed import TransformPlan

    sp = product_space(rule, cod, dom)
    plan = TransformPlan(sp, "permute", p1, p2, (), 0)
    assert plan.dst.size == ref.space.size
    assert plan.dst.block_keys() == oracle_keys(ref.space)
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=1e-12, atol=1e-12 * np.abs(ref.data).max())


@pytest.mark.parametrize("name,n", [("su2_rank4", 3), ("su2_rank4", 1), ("su2_rank4", 0), ("fz2", 4), ("i3", 1)])
def test_repartition_tables_replay_matches_oracle(name, n):
    rule, cod, dom = SPACES[name]
    rng = np.random.default_rng(3)
    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, rng.standard_normal(sp0.size))
    ref = src.repartition(n)
    from tenet_b200.typed import TransformPlan

    plan = TransformPlan(product_space(rule, cod, dom), "repartition", (), (), (), n)
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=1e-12, atol=1e-12 * np.abs(ref.data).max())


def test_braid_with_levels_matches_oracle():
    rule, cod, dom = SPACES["su2_rank3_1"]
    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(5).standard_normal(sp0.size))
    levels = [2, 0, 3, 1]
    ref = src.braid([1, 2], [3, 0], levels)
    from tenet_b200.typed import TransformPlan

    plan = TransformPlan(product_space(rule, cod, dom), "braid", [1, 2], [3, 0], levels, 0)
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", ["u1_config", "su2_rank4", "i3"])
def test_compose_jobs_replay_matches_oracle(name):
    rule, cod, dom = SPACES[name]
    rng = np.random.default_rng(11)
    a_sp = OHom(rule, cod, dom)
    b_sp = OHom(rule, dom, cod)
    a = OT(a_sp, rng.standard_normal(a_sp.size))
    b = OT(b_sp, rng.standard_normal(b_sp.size))
    ref = a.compose(b)
    from tenet_b200.typed import ComposePlan

    plan = ComposePlan(product_space(rule, cod, dom), product_space(rule, dom, cod))
    assert plan.dst.size == ref.space.size
    got = replay_compose(plan.export(), a.data, b.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=1e-12, atol=1e-12 * np.abs(ref.data).max())


def test_host_f_symbols_match_exact_racah():
    rule = product_rule(SU2R)
    worst = 0.0
    for a in range(0, 7):
        for b in range(0, 7):
            for c in range(0, 7):
                for e in range(abs(a - b), a + b + 1, 2):
                    for f in range(abs(b - c), b + c + 1, 2):
                        for d in range(abs(e - c), e + c + 1, 2):
                            ref = su2_f(a, b, c, d, e, f)
                            got = rule.fsymbol(a, b, c, d, e, f)
                            worst = max(worst, abs(got - ref))
    assert worst < 4e-16


def test_rejects_invalid_input():
    from tenet_b200 import _lib, typed

    rule = typed.U1FusionRule()
    v = typed.GradedSpace(rule, [(0, 2), (1, 1)])
    sp = typed.HomSpace(rule, [v], [v])
    with pytest.raises(_lib.TenetError):
        typed.TransformPlan(sp, "permute", [0, 0], [], (), 0)
    with pytest.raises(_lib.TenetError):
        typed.TransformPlan(sp, "repartition", (), (), (), 5)
    w = typed.GradedSpace(rule, [(0, 3)])
    with pytest.raises(_lib.TenetError):
        typed.ComposePlan(typed.HomSpace(rule, [v], [v]), typed.HomSpace(rule, [w], [v]))
    with pytest.raises(ValueError):
        typed.GradedSpace(rule, [(0, 1), (0, 2)])


def test_u1_config_plan_sizes():
    from tenet_b200.typed import ComposePlan, TransformPlan

    rule, cod, dom = SPACES["u1_config"]
    sp = product_space(rule, cod, dom)
    cp = ComposePlan(sp, sp)
    assert cp.njobs == 9
    assert cp.flops == sum(2 * r ** 3 for r in [16, 64, 160, 256, 304, 256, 160, 64, 16])
    xp = TransformPlan(sp, "permute", [0, 3], [2, 1], (), 0)
    assert xp.bytes_moved == 16 * 283392


def test_block_extent_limit_is_an_error_not_a_fault():
    """Transform tiles stage multi-indices as 16-bit values: a block extent above
    65535 is rejected on the host with TNT_INVALID_ARGUMENT (no device work)."""
    import tenet_b200 as tb
    from tenet_b200 import _lib

    rule = tb.U1FusionRule()
    V = tb.GradedSpace(rule, [(0, 70000)])
    W = tb.GradedSpace(rule, [(0, 2)])
    sp = tb.typed.HomSpace(rule, [V, W], [W])
    with pytest.raises(_lib.TenetError, match="65535"):
        tb.typed.TransformPlan(sp, "permute", [1, 0], [2], None, 0)
