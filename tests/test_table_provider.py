"""Checked table providers (generic fusion beyond the built-in factors), on the CPU.

Rep(S3) -- trivial, sign and the two-dimensional standard representation,
2 x 2 -> 1 + sign + 2 -- is the smallest non-abelian multiplicity-free rule
that is not SU(2).  Its tables come from Clebsch-Gordan isometries
(``tenet_b200.providers``); the same tables drive the device rule
(``TableFusionRule``, checked by ``tnt_rule_create_table``) and the oracle
(``oracle.sectors.TableRule``).  Checked here:

* the law checks accept Rep(S3) and the built-in SU(2) symbols satisfy the
  same pentagon / hexagon forms, and broken tables are rejected with the law
  they break;
* sector ids, layouts and block keys of random Rep(S3) spaces are bit-exact
  against the oracle, and random permutes, braids with levels, repartitions
  and composes replayed from the exported tables match the oracle to 1e-12.
"""

import itertools

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, Rule
from oracle.tensor import TensorMap as OT
from tests.helpers import product_space, replay_compose, replay_transform, table_rules


@pytest.fixture(scope="module")
def s3():
    from tenet_b200 import providers

    return providers.rep_s3()


@pytest.fixture(scope="module")
def rules(s3):
    return table_rules(s3)


def test_rep_s3_tables(s3):
    from tenet_b200 import providers

    assert list(s3.dims) == [1.0, 1.0, 2.0]
    assert [c for c in range(3) if s3.nsym[2, 2, c]] == [0, 1, 2]
    assert s3.rsym[2, 2, 1] == pytest.approx(-1.0)  # the sign channel of 2 x 2 is antisymmetric
    assert providers.check_tables(s3) == []


def test_law_forms_hold_for_builtin_su2():
    """The pentagon and hexagon in the form the checks use hold for the
    built-in SU(2) symbols (doubled spins up to 6, outer labels up to 1)."""
    r = Rule([SU2])
    S = 7
    F = np.zeros((S,) * 6)
    R = np.zeros((S,) * 3)
    for a, b, c in itertools.product(range(S), repeat=3):
        R[a, b, c] = r.R((a,), (b,), (c,))
    tri = lambda x, y, z: abs(x - y) <= z <= x + y and (x + y + z) % 2 == 0
    for a, b, c, d, e, f in itertools.product(range(S), repeat=6):
        if tri(a, b, e) and tri(e, c, d) and tri(b, c, f) and tri(a, f, d):
            F[a, b, c, d, e, f] = r.F((a,), (b,), (c,), (d,), (e,), (f,))
    small = slice(0, 2)
    # pentagon: F(f,c,d;e;g,l) F(a,b,l;e;f,k) = sum_h F(a,b,c;g;f,h) F(a,h,d;e;g,k) F(b,c,d;k;h,l)
    lhs = np.einsum("fcdegl,ablefk->abcdefgkl", F[:, small, small], F[small, small])
    rhs = np.einsum("abcgfh,ahdegk,bcdkhl->abcdefgkl", F[small, small, small], F[small, :, small], F[small, small, small])
    assert np.abs(lhs - rhs).max() <= 1e-12
    # hexagon: R(c,a,e) F(a,c,b;d;e,g) R(c,b,g) = sum_f F(c,a,b;d;e,f) R(c,f,d) F(a,b,c;d;f,g)
    lhs = np.einsum("cae,acbdeg,cbg->abcdeg", R[small, small], F[small, small, small], R[small, small])
    rhs = np.einsum("cabdef,cfd,abcdfg->abcdeg", F[small, small, small], R[small], F[small, small, small])
    assert np.abs(lhs - rhs).max() <= 1e-12


@pytest.mark.parametrize("breakage,message", [
    ("flip_f", "orthogonal"), ("gauge_f", "pentagon"), ("outer", "multiplicity"), ("dims", "dimensions"),
    ("r_sym", "symmetric"), ("fs", "Frobenius"), ("dual", "dual"),
])
def test_broken_tables_are_rejected(s3, breakage, message):
    import copy

    from tenet_b200 import _lib, typed

    p = copy.deepcopy(s3)
    if breakage == "flip_f":
        idx = tuple(int(x) for x in np.argwhere(np.abs(p.fsym[2, 2, 2, 2]) > 0.1)[0])
        p.fsym[(2, 2, 2, 2) + idx] *= 1.5
    elif breakage == "gauge_f":
        p.fsym[2, 2, 2, 2, 0, 1] *= -1.0  # still orthogonal, no longer a consistent gauge
        p.fsym[2, 2, 2, 2, 1, 1] *= -1.0
        p.fsym[2, 2, 2, 2, 2, 1] *= -1.0
    elif breakage == "outer":
        p.nsym = p.nsym.copy()
        p.nsym[2, 2, 2] = 2
    elif breakage == "dims":
        p.dims = np.array([1.0, 1.0, 2.5])
    elif breakage == "r_sym":
        p.rsym[2, 2, 2] = 0.5
    elif breakage == "fs":
        p.fs = np.array([1.0, 1.0, -1.0])
    elif breakage == "dual":
        p.dual = np.array([0, 2, 1], dtype=np.int32)
    with pytest.raises(_lib.TenetError) as err:
        typed.TableFusionRule(p)
    assert message in str(err.value)


def test_symbols_through_the_abi(rules, s3):
    orule, rule = rules
    for a, b, c, d, e, f in itertools.product(range(3), repeat=6):
        assert rule.fsymbol(a, b, c, d, e, f) == s3.fsym[a, b, c, d, e, f]
    assert [rule.dim(a) for a in range(3)] == [1.0, 1.0, 2.0]
    assert [rule.sector_id(a) for a in range(3)] == [0, 1, 2]


def _random_space(rng, orule):
    rank = int(rng.integers(2, 5))
    legs = []
    for _ in range(rank):
        k = int(rng.integers(1, 4))
        pick = sorted(rng.choice(3, size=k, replace=False))
        legs.append(Leg.new(orule, [((int(i),), int(rng.integers(1, 3))) for i in pick]))
    n1 = int(rng.integers(0, rank + 1))
    return legs[:n1], legs[n1:]


def _cases(orule, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        cod, dom = _random_space(rng, orule)
        sp = OHom(orule, cod, dom)
        if sp.size == 0 or sp.size > 20000:
            continue
        n = len(cod) + len(dom)
        perm = [int(x) for x in rng.permutation(n)]
        k = int(rng.integers(0, n + 1))
        out.append((cod, dom, perm[:k], perm[k:], [int(x) for x in rng.permutation(n)], int(rng.integers(0, n + 1))))
    return out


@pytest.mark.parametrize("i", range(16))
def test_random_rep_s3_recouplings_match_oracle(rules, i):
    from tenet_b200.typed import TransformPlan

    orule, rule = rules
    cod, dom, p1, p2, levels, nrep = _cases(orule, 16, 606)[i]
    sp0 = OHom(orule, cod, dom)
    dsp = product_space(orule, cod, dom)
    assert dsp.block_keys() == [b["key"] for b in sp0.blocks]
    assert dsp.size == sp0.size
    src = OT(sp0, np.random.default_rng(i).standard_normal(sp0.size))
    tol = 1e-12 * max(1.0, np.abs(src.data).max())
    for kind, ref, args in (("permute", src.permute(p1, p2), (p1, p2, (), 0)),
                            ("braid", src.braid(p1, p2, levels), (p1, p2, levels, 0)),
                            ("repartition", src.repartition(nrep), ((), (), (), nrep))):
        plan = TransformPlan(dsp, kind, *args)
        assert plan.dst.block_keys() == [b["key"] for b in ref.space.blocks], kind
        got = replay_transform(plan.export(), src.data, plan.dst.size)
        np.testing.assert_allclose(got, ref.data, rtol=0, atol=tol, err_msg=kind)


@pytest.mark.parametrize("i", range(6))
def test_random_rep_s3_composes_match_oracle(rules, i):
    from tenet_b200.typed import ComposePlan

    orule, rule = rules
    rng = np.random.default_rng(900 + i)
    while True:
        cod, mid = _random_space(rng, orule)
        _, dom = _random_space(rng, orule)
        if not mid:
            continue
        a_sp, b_sp = OHom(orule, cod, mid), OHom(orule, mid, dom)
        if 0 < a_sp.size <= 20000 and 0 < b_sp.size <= 20000:
            break
    a, b = OT(a_sp, rng.standard_normal(a_sp.size)), OT(b_sp, rng.standard_normal(b_sp.size))
    ref = a.compose(b)
    plan = ComposePlan(product_space(orule, cod, mid), product_space(orule, mid, dom))
    assert plan.dst.block_keys() == [blk["key"] for blk in ref.space.blocks]
    got = replay_compose(plan.export(), a.data, b.data, plan.dst.size)
    np.testing.assert_allclose(got, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max(initial=1.0))
