"""CUDA-graph capture of the replay entry points.

After a first (untimed) call has uploaded the plan tables and calibrated the
tile autotuner, tnt_compose (FP64 and split precision) and tnt_transform read
no host memory in stream order, so their launches can be captured once and
replayed; a replay on new operand values must equal a direct call on them.
"""

import ctypes as C

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, Rule
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

SU2R = Rule([SU2])
W = Leg.new(SU2R, [((0,), 24), ((1,), 36), ((2,), 36), ((3,), 24), ((4,), 12)])
P = Leg.new(SU2R, [((1,), 1)])


@pytest.fixture(scope="module")
def setup():
    import torch

    from tenet_b200 import Runtime, typed

    rt = Runtime(0)
    rule = product_rule(SU2R)
    cod, dom = [product_leg(rule, W), product_leg(rule, P)], [product_leg(rule, P), product_leg(rule, W)]
    sp = OHom(SU2R, [W, P], [P, W])
    a = typed.TensorMap.from_host(rt, cod, dom, normal_fill(1, sp.size))
    b = typed.TensorMap.from_host(rt, dom, cod, normal_fill(2, OHom(SU2R, [P, W], [W, P]).size))
    return torch, rt, a, b


def _capture(torch, fn):
    fn()  # first call: plan upload and tuning
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            fn()
    torch.cuda.synchronize()
    return g


@pytest.mark.parametrize("precision,slices", [("fp64", 0), ("bf16x", 6), ("i8x", 6)])
def test_compose_graph_replay_matches_direct(setup, precision, slices):
    from tenet_b200 import _lib

    torch, rt, a, b = setup
    plan = rt.cplan(a.space, b.space)
    out = torch.empty(plan.dst.size, dtype=torch.float64, device="cuda")
    prec = {"fp64": _lib.PREC_FP64, "bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X}[precision]

    def fn(dst=out):
        _lib.call("tnt_compose", rt._h, plan._h, 1, C.c_void_p(dst.data_ptr()), plan.dst.size,
                  C.c_void_p(a.data.data_ptr()), a.space.size, C.c_void_p(b.data.data_ptr()), b.space.size, 1.0, 0.0,
                  prec, slices, C.c_void_p(torch.cuda.current_stream().cuda_stream))

    g = _capture(torch, fn)
    for seed in (7, 8):
        a.data.copy_(torch.as_tensor(normal_fill(seed, a.space.size), device="cuda"))
        g.replay()
        torch.cuda.synchronize()
        ref = torch.empty_like(out)
        fn(ref)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    del g


def test_transform_graph_replay_matches_direct(setup):
    from tenet_b200 import _lib

    torch, rt, a, b = setup
    plan = rt.xplan(a.space, "permute", [0, 3], [2, 1])
    out = torch.empty(plan.dst.size, dtype=torch.float64, device="cuda")

    def fn(dst=out):
        _lib.call("tnt_transform", rt._h, plan._h, C.c_void_p(dst.data_ptr()), C.c_void_p(a.data.data_ptr()), 1.0,
                  0.0, C.c_void_p(torch.cuda.current_stream().cuda_stream))

    g = _capture(torch, fn)
    a.data.copy_(torch.as_tensor(normal_fill(9, a.space.size), device="cuda"))
    g.replay()
    torch.cuda.synchronize()
    ref = torch.empty_like(out)
    fn(ref)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    del g
