"""Seeded random recouplings: the C++ plan tables against the oracle (CPU).

Random legs (U(1), SU(2), fZ2 x U(1) x SU(2), dual flags mixed), random
codomain/domain splits of rank 2-4 and random axis permutations, replayed in
numpy from the exported tables and compared with the oracle's permute
(1e-12); keys of the destination space bit-exact.  Also random two- and
three-step chains against the stepwise oracle.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from tests.helpers import product_space, replay_transform

RULES = {
    "U1": (Rule([U1]), [(-1,), (0,), (1,), (2,)]),
    "SU2": (Rule([SU2]), [(0,), (1,), (2,), (3,)]),
    "I3": (Rule([FZ2, U1, SU2]), [(0, 0, 0), (1, 1, 1), (0, 2, 0), (1, -1, 1), (0, 0, 2)]),
}


def _random_space(rng, name):
    rule, labels = RULES[name]
    rank = int(rng.integers(2, 5))
    legs = []
    for _ in range(rank):
        k = int(rng.integers(1, len(labels) + 1))
        pick = rng.choice(len(labels), size=k, replace=False)
        leg = Leg.new(rule, [(labels[i], int(rng.integers(1, 3))) for i in sorted(pick)])
        legs.append(leg.dual() if rng.random() < 0.3 else leg)
    n1 = int(rng.integers(0, rank + 1))
    return rule, legs[:n1], legs[n1:]


def _cases(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        name = list(RULES)[len(out) % len(RULES)]
        rule, cod, dom = _random_space(rng, name)
        sp = OHom(rule, cod, dom)
        if sp.size == 0 or sp.size > 20000:
            continue
        n = len(cod) + len(dom)
        perm = [int(x) for x in rng.permutation(n)]
        k = int(rng.integers(0, n + 1))
        out.append((name, rule, cod, dom, perm[:k], perm[k:], int(rng.integers(0, n + 1))))
    return out


@pytest.mark.parametrize("case", _cases(36, 2024), ids=lambda c: f"{c[0]}-{len(c[2])}{len(c[3])}-{c[4]}{c[5]}")
def test_random_permute_tables_match_oracle(case):
    from tenet_b200.typed import TransformPlan

    name, rule, cod, dom, p1, p2, _ = case
    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(len(p1) + 7).standard_normal(sp0.size))
    ref = src.permute(p1, p2)
    plan = TransformPlan(product_space(rule, cod, dom), "permute", p1, p2, (), 0)
    assert plan.dst.block_keys() == [b["key"] for b in ref.space.blocks]
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max(initial=1.0))


@pytest.mark.parametrize("case", _cases(18, 77), ids=lambda c: f"{c[0]}-{len(c[2])}{len(c[3])}")
def test_random_chains_match_stepwise_oracle(case):
    from tenet_b200.typed import TransformPlan

    name, rule, cod, dom, p1, p2, nrep = case
    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(nrep + 3).standard_normal(sp0.size))
    n = len(cod) + len(dom)
    ref = src.permute(p1, p2).repartition(nrep).adjoint()
    prog = [0, len(p1), *p1, len(p2), *p2, 2, nrep, 3]
    twist = FZ2 in rule.factors
    if twist:
        legs = [0, n - 1] if n > 1 else [0]
        ref = ref.twist(legs)
        prog += [4, len(legs), *legs]
    plan = TransformPlan(product_space(rule, cod, dom), "chain", prog, (), (), 4 if twist else 3)
    assert plan.dst.block_keys() == [b["key"] for b in ref.space.blocks]
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max(initial=1.0))


def _compose_cases(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        name = list(RULES)[len(out) % len(RULES)]
        rule, cod, mid = _random_space(rng, name)
        _, dom, _ = _random_space(rng, name)
        if not mid:
            continue
        a_sp, b_sp = OHom(rule, cod, mid), OHom(rule, mid, dom)
        if a_sp.size == 0 or b_sp.size == 0 or a_sp.size > 20000 or b_sp.size > 20000:
            continue
        out.append((name, rule, cod, mid, dom))
    return out


@pytest.mark.parametrize("case", _compose_cases(18, 99), ids=lambda c: f"{c[0]}-{len(c[2])}{len(c[3])}{len(c[4])}")
def test_random_compose_jobs_match_oracle(case):
    from tenet_b200.typed import ComposePlan
    from tests.helpers import replay_compose

    name, rule, cod, mid, dom = case
    a_sp, b_sp = OHom(rule, cod, mid), OHom(rule, mid, dom)
    rng = np.random.default_rng(len(cod) * 7 + len(dom))
    a, b = OT(a_sp, rng.standard_normal(a_sp.size)), OT(b_sp, rng.standard_normal(b_sp.size))
    ref = a.compose(b)
    plan = ComposePlan(product_space(rule, cod, mid), product_space(rule, mid, dom))
    assert plan.dst.size == ref.space.size
    assert plan.dst.block_keys() == [b["key"] for b in ref.space.blocks]
    got = replay_compose(plan.export(), a.data, b.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max(initial=1.0))


@pytest.mark.parametrize("case", _cases(12, 4242), ids=lambda c: f"{c[0]}-{len(c[2])}{len(c[3])}-braid")
def test_random_braids_with_levels_match_oracle(case):
    """Braids with random levels: for the symmetric (bosonic or fermionic)
    rules here a braid equals the permute, and both match the oracle."""
    from tenet_b200.typed import TransformPlan

    name, rule, cod, dom, p1, p2, _ = case
    sp0 = OHom(rule, cod, dom)
    src = OT(sp0, np.random.default_rng(len(p2) + 11).standard_normal(sp0.size))
    n = len(cod) + len(dom)
    levels = [int(x) for x in np.random.default_rng(n).permutation(n)]
    ref = src.braid(p1, p2, levels)
    plan = TransformPlan(product_space(rule, cod, dom), "braid", p1, p2, levels, 0)
    assert plan.dst.block_keys() == [b["key"] for b in ref.space.blocks]
    got = replay_transform(plan.export(), src.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max(initial=1.0))
    np.testing.assert_allclose(ref.data, src.permute(p1, p2).data, rtol=0,
                               atol=1e-12 * np.abs(ref.data).max(initial=1.0))
