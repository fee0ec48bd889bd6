"""Fermionic contract and twist on the device vs the oracle.

The right operand's permute carries the supertrace twist inside its transform
plan, so a fermionic contraction runs the same three kernels as a bosonic one
(transform, grouped GEMM, transform).  Parity: 1e-12 relative to the largest
entry; the compose/contract law of the reference's facade tests
(tenet/tests/typed_facade.rs:6529-6547) holds bit for bit.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

I3 = Rule([FZ2, U1, SU2])
P_I3 = Leg.new(I3, [((0, 0, 0), 3), ((1, 1, 1), 4), ((1, -1, 1), 2), ((0, 2, 0), 2)])
Q_I3 = Leg.new(I3, [((1, -1, 1), 2), ((0, 0, 2), 3), ((0, 2, 0), 4), ((0, 0, 0), 2)]).dual()


def _close(got, ref):
    scale = max(np.abs(ref).max(), 1e-300)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * scale)


def _device(rt, t_o):
    import tenet_b200.typed as tb

    rule = product_rule(t_o.rule)
    cod = [product_leg(rule, l) for l in t_o.space.codomain]
    dom = [product_leg(rule, l) for l in t_o.space.domain]
    return tb.TensorMap.from_host(rt, cod, dom, t_o.data)


@pytest.fixture(scope="module")
def rt():
    import tenet_b200.typed as tb

    return tb.Runtime(0)


def _operands(seed):
    sp = OHom(I3, [P_I3, Q_I3], [P_I3, Q_I3])
    rng = np.random.default_rng(seed)
    return OT(sp, rng.standard_normal(sp.size)), OT(sp, rng.standard_normal(sp.size))


@pytest.mark.parametrize(
    "lhs_axes,rhs_axes,out",
    [([2, 3], [0, 1], [0, 1, 2, 3]), ([2, 3], [0, 1], [1, 3, 0, 2]), ([3], [1], [0, 1, 2, 3, 4, 5]),
     ([1, 2], [3, 0], [0, 1, 2, 3])],
)
def test_fermionic_contract_matches_oracle(rt, lhs_axes, rhs_axes, out):
    a_o, b_o = _operands(21)
    ref = a_o.contract(b_o, lhs_axes, rhs_axes, out)
    got = _device(rt, a_o).contract(_device(rt, b_o), lhs_axes, rhs_axes, out)
    assert got.space.size == ref.space.size
    _close(got.to_host(), ref.data)


def test_twist_matches_oracle(rt):
    a_o, _ = _operands(4)
    for legs in ([1], [0, 3], [0, 1, 2, 3]):
        np.testing.assert_array_equal(_device(rt, a_o).twist(legs).to_host(), a_o.twist(legs).data)


def test_compose_equals_contract_of_twisted_rhs(rt):
    a_o, b_o = _operands(8)
    a, b = _device(rt, a_o), _device(rt, b_o)
    composed = a.compose(b).to_host()
    twisted = a.contract(b.twist([1]), [2, 3], [0, 1], [0, 1, 2, 3]).to_host()
    np.testing.assert_array_equal(twisted, composed)
    plain = a.contract(b, [2, 3], [0, 1], [0, 1, 2, 3]).to_host()
    assert not np.allclose(plain, composed, rtol=0, atol=1e-12)


def test_transform_chain_on_device_matches_stepwise_oracle(rt):
    """A fused chain (permute, twist, adjoint, repartition) in one device pass."""
    a_o, _ = _operands(31)
    steps = [("permute", [3, 0], [1, 2]), ("twist", [0, 2]), ("adjoint",), ("repartition", 1)]
    ref = a_o.permute([3, 0], [1, 2]).twist([0, 2]).adjoint().repartition(1)
    got = _device(rt, a_o).transform_chain(steps)
    assert got.space.size == ref.space.size
    _close(got.to_host(), ref.data)
