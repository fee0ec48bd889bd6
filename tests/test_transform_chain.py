"""Fused recoupling chains (``tnt_transform_chain_plan``), CPU side.

A chain of permutes, braids, repartitions, adjoints and twists compiles into
one transform whose tables, replayed in numpy, equal the oracle applying the
steps one by one (1e-12), on SU(2) and fermionic fZ2 x U(1) x SU(2) spaces;
the destination space is bit-exact.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from tests.helpers import product_space, replay_transform

SU2R = Rule([SU2])
I3 = Rule([FZ2, U1, SU2])
V = Leg.new(SU2R, [((0,), 2), ((1,), 2), ((2,), 1)])
W = Leg.new(SU2R, [((0,), 3), ((1,), 2), ((2,), 2), ((3,), 1)])
V3 = Leg.new(I3, [((0, 0, 0), 2), ((1, 1, 1), 2), ((0, 2, 0), 1)])

CASES = {
    "su2_permute_permute": (SU2R, [V, W], [V, W], [("permute", [1, 0], [3, 2]), ("permute", [0, 3], [2, 1])]),
    "su2_adjoint_permute": (SU2R, [V, W], [W], [("adjoint",), ("permute", [2, 0], [1])]),
    "su2_repartition_braid": (SU2R, [V, W], [V, W], [("repartition", 1), ("braid", [1, 0], [2, 3], [3, 1, 0, 2])]),
    "i3_permute_twist": (I3, [V3, V3], [V3, V3.dual()], [("permute", [3, 0], [1, 2]), ("twist", [0, 2])]),
    "i3_twist_adjoint_repartition": (I3, [V3, V3], [V3, V3.dual()],
                                     [("twist", [1]), ("adjoint",), ("repartition", 3)]),
}


def _program(steps):
    prog = []
    for st in steps:
        if st[0] in ("permute", "braid"):
            prog += [0 if st[0] == "permute" else 1, len(st[1]), *st[1], len(st[2]), *st[2]]
            if st[0] == "braid":
                prog += list(st[3])
        elif st[0] == "repartition":
            prog += [2, st[1]]
        elif st[0] == "adjoint":
            prog += [3]
        else:
            prog += [4, len(st[1]), *st[1]]
    return prog


def _oracle(t, steps):
    for st in steps:
        if st[0] == "permute":
            t = t.permute(st[1], st[2])
        elif st[0] == "braid":
            t = t.braid(st[1], st[2], st[3])
        elif st[0] == "repartition":
            t = t.repartition(st[1])
        elif st[0] == "adjoint":
            t = t.adjoint()
        else:
            t = t.twist(st[1])
    return t


@pytest.mark.parametrize("name", sorted(CASES))
def test_chain_replay_matches_stepwise_oracle(name):
    from tenet_b200.typed import TransformPlan

    rule, cod, dom, steps = CASES[name]
    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(21).standard_normal(sp0.size))
    ref = _oracle(src, steps)
    plan = TransformPlan(product_space(rule, cod, dom), "chain", _program(steps), (), (), len(steps))
    assert plan.dst.block_keys() == [b["key"] for b in ref.space.blocks]
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max())


def test_chain_moves_the_payload_once():
    from tenet_b200.typed import TransformPlan

    rule, cod, dom, steps = CASES["su2_permute_permute"]
    sp = product_space(rule, cod, dom)
    chain = TransformPlan(sp, "chain", _program(steps), (), (), len(steps))
    one = TransformPlan(sp, "permute", steps[0][1], steps[0][2], (), 0)
    assert chain.bytes_moved == one.bytes_moved


def test_malformed_chain_programs_are_rejected():
    from tenet_b200._lib import TenetError
    from tenet_b200.typed import TransformPlan

    rule, cod, dom, _ = CASES["su2_permute_permute"]
    sp = product_space(rule, cod, dom)
    for prog, n in (([9], 1), ([0, 2, 0, 1, 2, 2, 3], 2), ([0, 2, 0, 1, 2, 2, 3, 7], 1), ([0, 2, 0, 0, 2, 2, 3], 1)):
        with pytest.raises(TenetError):
            TransformPlan(sp, "chain", prog, (), (), n)
