"""A transform plan imported from exported tables replays on the device bit
for bit like the plan the library compiled (tnt_xplan_from_tables)."""

import ctypes as C

import numpy as np
import pytest

from oracle.fusion import Leg
from oracle.sectors import SU2, Rule
from tests.helpers import product_space

pytestmark = pytest.mark.gpu

SU2R = Rule([SU2])
W = Leg.new(SU2R, [((0,), 24), ((1,), 36), ((2,), 36), ((3,), 24), ((4,), 12)])
P = Leg.new(SU2R, [((1,), 1)])


def test_imported_plan_replays_like_the_native_plan():
    import torch

    from tenet_b200 import Runtime, _lib
    from tenet_b200.typed import TransformPlan

    rt = Runtime(0)
    sp = product_space(SU2R, [W, P], [P, W])
    native = TransformPlan(sp, "permute", [0, 3], [1, 2], (), 0)
    imported = TransformPlan.from_tables(sp.n1 + sp.n2, *native.export(), native.src.size, native.dst.size)
    src = torch.randn(native.src.size, dtype=torch.float64, device="cuda")
    outs = []
    for plan in (native, imported):
        dst = torch.full((native.dst.size,), float("nan"), dtype=torch.float64, device="cuda")
        _lib.call("tnt_transform", rt._h, plan._h, C.c_void_p(dst.data_ptr()), C.c_void_p(src.data_ptr()), 1.0, 0.0,
                  rt.stream())
        outs.append(dst.cpu().numpy())
    assert not np.isnan(outs[1]).any()
    assert outs[0].view(np.uint64).tolist() == outs[1].view(np.uint64).tolist()
