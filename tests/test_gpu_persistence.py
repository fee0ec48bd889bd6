"""Device snapshots: a resident tensor survives to_bytes -> from_bytes bit for bit.

One device-to-host copy encodes, one host-to-device copy restores; a lazy
adjoint snapshot is restored with the device adjoint transform and matches
the oracle's adjoint of the stored body.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

I3 = Rule([FZ2, U1, SU2])
V = Leg.new(I3, [((0, 0, 0), 12), ((1, 1, 1), 9), ((1, -1, 1), 7), ((0, 2, 0), 5), ((0, 0, 2), 4)])
P = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])


@pytest.fixture(scope="module")
def rt():
    import tenet_b200.typed as tb

    return tb.Runtime(0)


def _dev(rt, t_o):
    import tenet_b200.typed as tb

    rule = product_rule(t_o.rule)
    return tb.TensorMap.from_host(rt, [product_leg(rule, l) for l in t_o.space.codomain],
                                  [product_leg(rule, l) for l in t_o.space.domain], t_o.data)


def test_device_snapshot_round_trip_is_bit_exact(rt):
    from tenet_b200 import persistence

    sp = OHom(I3, [V, P], [P, V.dual()])
    t_o = OT(sp, normal_fill(11, sp.size))
    t = _dev(rt, t_o)
    b1 = persistence.tensor_to_bytes(t)
    back = persistence.tensor_from_bytes(rt, b1)
    assert back.space.same_as(t.space)
    assert back.to_host().view(np.uint64).tolist() == t.to_host().view(np.uint64).tolist()
    assert persistence.tensor_to_bytes(back) == b1


def test_lazy_adjoint_snapshot_restores_the_adjoint(rt):
    from tenet_b200 import persistence

    sp = OHom(I3, [V, P], [V])
    t_o = OT(sp, normal_fill(12, sp.size))
    b = persistence.tensor_to_bytes(_dev(rt, t_o))
    h = 20 + int.from_bytes(b[12:20], "little")
    lazy = b[:h] + bytes([persistence.REPR_ADJOINT]) + b[h:]
    got = persistence.tensor_from_bytes(rt, lazy)
    ref = t_o.adjoint()
    assert got.space.size == ref.space.size
    np.testing.assert_array_equal(got.to_host(), ref.data)
