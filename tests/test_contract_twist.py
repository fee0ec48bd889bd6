"""Fermionic contraction: the supertrace twist and TensorMap::twist (CPU only).

The oracle is checked against the laws the reference's own facade tests state
(tenet/tests/typed_facade.rs:6475-6550): an explicit output order equals the
default contraction followed by the same permutation, and composition equals
contraction with the right operand twisted on its dual codomain legs, while
the plain contraction differs from composition when a contracted leg is dual
and fermionic.  The C++ plan tables (twist plan, contract right-operand plan)
are then replayed in numpy against the oracle.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from tests.helpers import product_space, replay_transform

I3 = Rule([FZ2, U1, SU2])
U1R = Rule([U1])
FZ2R = Rule([FZ2])

# The leg pair of the reference's fZ2 x U(1) x SU(2) law fixture
# (typed_facade.rs:6424-6462): q is built dual.
P_I3 = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 2)])
Q_I3 = Leg.new(I3, [((1, -1, 1), 1), ((0, 0, 2), 1), ((0, 2, 0), 2)]).dual()
# The U(1) pair (typed_facade.rs:6349-6375): q dual.
P_U1 = Leg.new(U1R, [((-1,), 1), ((0,), 2), ((1,), 1)])
Q_U1 = Leg.new(U1R, [((0,), 1), ((1,), 2)]).dual()
V_FZ2 = Leg.new(FZ2R, [((0,), 2), ((1,), 3)])

LAW_CASES = {"i3": (I3, P_I3, Q_I3, True), "u1": (U1R, P_U1, Q_U1, False)}


def _pair(rule, p, q, seed):
    sp = OHom(rule, [p, q], [p, q])
    rng = np.random.default_rng(seed)
    return OT(sp, rng.standard_normal(sp.size)), OT(sp, rng.standard_normal(sp.size))


@pytest.mark.parametrize("name", sorted(LAW_CASES))
def test_oracle_contract_laws(name):
    rule, p, q, nontrivial = LAW_CASES[name]
    a, b = _pair(rule, p, q, 5)
    default = a.contract(b, [2, 3], [0, 1], [0, 1, 2, 3])
    ordered = a.contract(b, [2, 3], [0, 1], [1, 3, 0, 2])
    np.testing.assert_array_equal(ordered.data, default.permute([1, 3], [0, 2]).data)
    dual_cod = [i for i, leg in enumerate(b.space.codomain) if leg.is_dual]
    assert dual_cod == [1]
    composed = a.compose(b)
    twisted = a.contract(b.twist(dual_cod), [2, 3], [0, 1], [0, 1, 2, 3])
    np.testing.assert_allclose(twisted.data, composed.data, rtol=0, atol=1e-13 * np.abs(composed.data).max())
    differs = not np.allclose(default.data, composed.data, rtol=0, atol=1e-12)
    assert differs == nontrivial
    assert np.abs(composed.data).max() > 0


def test_oracle_twist_is_a_sign_per_block():
    sp = OHom(I3, [P_I3, Q_I3], [P_I3, Q_I3])
    t = OT(sp, np.random.default_rng(2).standard_normal(sp.size))
    np.testing.assert_array_equal(t.twist([0, 0]).data, t.data)
    np.testing.assert_array_equal(t.twist([1]).twist([1]).data, t.data)
    once = t.twist([0, 3])
    flipped = 0
    for b, blk in enumerate(sp.blocks):
        cod, dom = blk["key"]
        sign = I3.twist(cod[0][0]) * I3.twist(dom[0][1])
        np.testing.assert_array_equal(sp.block_view(once.data, b), sign * sp.block_view(t.data, b))
        flipped += sign < 0
    assert flipped > 0


TWISTS = [
    ("i3", I3, [P_I3, Q_I3], [P_I3, Q_I3], [1]),
    ("i3", I3, [P_I3, Q_I3], [P_I3, Q_I3], [0, 2, 3]),
    ("fz2", FZ2R, [V_FZ2, V_FZ2], [V_FZ2, V_FZ2.dual()], [3]),
    ("fz2", FZ2R, [V_FZ2, V_FZ2], [V_FZ2, V_FZ2.dual()], [0, 1]),
]


@pytest.mark.parametrize("name,rule,cod,dom,legs", TWISTS)
def test_twist_plan_replay_matches_oracle(name, rule, cod, dom, legs):
    from tenet_b200.typed import TransformPlan

    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(9).standard_normal(sp0.size))
    ref = src.twist(legs)
    plan = TransformPlan(product_space(rule, cod, dom), "twist", legs, (), (), 0)
    assert plan.dst.size == sp0.size
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_array_equal(got, ref.data)


RHS = [
    ("i3", I3, [P_I3, Q_I3], [P_I3, Q_I3], [0, 1], [2, 3]),
    ("i3", I3, [P_I3, Q_I3], [P_I3, Q_I3], [1, 3], [0, 2]),
    ("i3", I3, [P_I3, Q_I3], [P_I3, Q_I3], [3], [0, 1, 2]),
    ("fz2", FZ2R, [V_FZ2, V_FZ2], [V_FZ2, V_FZ2.dual()], [2, 3], [1, 0]),
]


@pytest.mark.parametrize("name,rule,cod,dom,ctr,opn", RHS)
def test_contract_rhs_plan_replay_matches_oracle(name, rule, cod, dom, ctr, opn):
    """The right operand's permute with the supertrace twist fused into one plan."""
    from tenet_b200.typed import TransformPlan

    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(13).standard_normal(sp0.size))
    perm = src.permute(ctr, opn)
    dual = [p for p in range(len(ctr)) if perm.space.codomain[p].is_dual]
    ref = perm.twist(dual) if dual else perm
    plan = TransformPlan(product_space(rule, cod, dom), "contract_rhs", ctr, opn, (), 0)
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=1e-12, atol=1e-12 * np.abs(ref.data).max())


def test_contract_rhs_plan_is_the_permute_plan_for_bosonic_rules():
    from tenet_b200.typed import TransformPlan

    sp = product_space(U1R, [P_U1, Q_U1], [P_U1, Q_U1])
    a = TransformPlan(sp, "contract_rhs", [1, 3], [0, 2], (), 0).export()
    b = TransformPlan(sp, "permute", [1, 3], [0, 2], (), 0).export()
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_twist_plan_rejects_out_of_range_leg():
    from tenet_b200._lib import TenetError
    from tenet_b200.typed import TransformPlan

    sp = product_space(I3, [P_I3, Q_I3], [P_I3, Q_I3])
    with pytest.raises(TenetError):
        TransformPlan(sp, "twist", [4], (), (), 0)
