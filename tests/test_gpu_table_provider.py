"""A checked table provider (Rep(S3)) on the device against the oracle.

The recoupling transform kernel runs the provider's F/R-derived coefficients
(groups beyond SU(2)'s sizes take the general path), the grouped GEMM the
coupled sectors of its fusion, and the batched SVD / truncation the blocks
weighted by its quantum dimensions; each result matches the oracle driven by
the same tables (payloads 1e-12, singular values 1e-12, kept counts exact).
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill
from tests.helpers import product_leg, table_rules

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    from tenet_b200 import Runtime, providers

    orule, rule = table_rules(providers.rep_s3())
    V = Leg.new(orule, [((0,), 3), ((1,), 2), ((2,), 4)])
    W = Leg.new(orule, [((1,), 2), ((2,), 3)])
    return Runtime(0), orule, rule, V, W


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def dev(rt, rule, cod, dom, data):
    from tenet_b200 import typed

    return typed.TensorMap.from_host(rt, [product_leg(rule, l) for l in cod], [product_leg(rule, l) for l in dom],
                                     data)


@pytest.mark.parametrize("p1,p2", [([0, 3], [2, 1]), ([1, 0], [3, 2]), ([2], [0, 3, 1]), ([3, 2, 1], [0])])
def test_table_rule_permute_and_braid_match_oracle(env, p1, p2):
    rt, orule, rule, V, W = env
    cod, dom = [V, W], [W.dual(), V]
    sp = OHom(orule, cod, dom)
    src = OT(sp, normal_fill(7, sp.size))
    d = dev(rt, rule, cod, dom, src.data)
    ref = src.permute(p1, p2)
    got = d.permute(p1, p2)
    assert got.space.block_keys() == [b["key"] for b in ref.space.blocks]
    assert rel(got.to_host(), ref.data) <= 1e-12
    levels = [2, 0, 3, 1]
    refb = src.braid(p1, p2, levels)
    gotb = d.braid(p1, p2, levels)
    assert rel(gotb.to_host(), refb.data) <= 1e-12


def test_table_rule_compose_and_svd_match_oracle(env):
    from tenet_b200 import Truncation

    rt, orule, rule, V, W = env
    a_sp, b_sp = OHom(orule, [V, W], [W, V]), OHom(orule, [W, V], [V, V])
    a = OT(a_sp, normal_fill(11, a_sp.size))
    b = OT(b_sp, normal_fill(12, b_sp.size))
    ref = a.compose(b)
    da, db = dev(rt, rule, [V, W], [W, V], a.data), dev(rt, rule, [W, V], [V, V], b.data)
    c = da.compose(db)
    assert c.space.block_keys() == [blk["key"] for blk in ref.space.blocks]
    assert rel(c.to_host(), ref.data) <= 1e-12
    # truncated SVD: weighted rank budget uses the quantum dimensions (2 for the standard irrep)
    _, kept, err = ref.svd_trunc(("rank", 20))
    res = c.svd_trunc(Truncation.rank(20))
    assert res.kept == kept
    assert abs(res.error - err) <= 1e-10 * max(1.0, err)
