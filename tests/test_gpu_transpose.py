"""Transposing permutes on the device against the oracle.

A single-block group whose source runs along some destination axis other
than axis 0 takes the transposing path of the transform kernel (planes of
axis 0 x that axis staged through shared memory).  Covered here: U(1)
tensors with extents below and above the staging chunks (odd sizes, more
than 64 along the contiguous axis, more rows than one staging pass holds),
several permutes that move axis 0, and alpha / beta through the C ABI
(dst = alpha P(src) + beta dst) -- every result equal to the oracle to
1e-15 relative (the path only scales and moves values).
"""

import ctypes as C

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import U1, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

U1R = Rule([U1])
V = Leg.new(U1R, [((-1,), 5), ((0,), 70), ((1,), 9)])
W = Leg.new(U1R, [((0,), 3), ((1,), 66), ((2,), 40)])


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("p1,p2", [([3, 2], [1, 0]), ([1, 2], [3, 0]), ([2, 0], [1, 3]), ([3], [0, 1, 2]),
                                   ([1, 3, 0], [2])])
def test_transposing_permutes_match_oracle(rt, p1, p2):
    import torch

    from tenet_b200 import _lib, typed

    rule = product_rule(U1R)
    cod, dom = [V, W], [W, V]
    sp = OHom(U1R, cod, dom)
    src = OT(sp, normal_fill(17, sp.size))
    ref = src.permute(p1, p2)
    dev = typed.TensorMap.from_host(rt, [product_leg(rule, l) for l in cod], [product_leg(rule, l) for l in dom],
                                    src.data)
    got = dev.permute(p1, p2)
    assert got.space.block_keys() == [b["key"] for b in ref.space.blocks]
    assert rel(got.to_host(), ref.data) <= 1e-15
    # alpha / beta through the C ABI
    plan = rt.xplan(dev.space, "permute", p1, p2)
    d0 = torch.from_numpy(normal_fill(18, plan.dst.size)).cuda()
    out = d0.clone()
    _lib.call("tnt_transform", rt._h, plan._h, C.c_void_p(out.data_ptr()), C.c_void_p(dev.data.data_ptr()), 2.0, 0.5,
              rt.stream())
    rt.sync()
    want = 2.0 * ref.data + 0.5 * d0.cpu().numpy()
    assert rel(out.cpu().numpy(), want) <= 1e-15
