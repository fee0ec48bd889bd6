"""Calls on one context from several streams (the header's threading rule).

A context shares its scratch (split-precision slice packs, staging, segment
tables) across streams and orders a call on a new stream after the previous
scratch user's work with an event.  Two split-precision composes issued back
to back on two streams of one context, with no host synchronisation between
them, must each equal the same compose run alone; without the ordering the
second compose's packing would overwrite the first one's packs while the
first one's multiply still reads them.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

I3 = Rule([FZ2, U1, SU2])
V = Leg.new(I3, [((0, 0, 0), 40), ((1, 1, 1), 33), ((0, 2, 0), 27), ((1, -1, 1), 21), ((0, 0, 2), 18)])
P = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])


def _tensor(rt, cod, dom, seed):
    from tenet_b200 import typed

    rule = product_rule(I3)
    sp = OHom(I3, cod, dom)
    return typed.TensorMap.from_host(rt, [product_leg(rule, l) for l in cod], [product_leg(rule, l) for l in dom],
                                     normal_fill(seed, sp.size))


@pytest.mark.parametrize("precision,slices", [("i8x", 5), ("bf16x", 5)])
def test_split_composes_on_two_streams_of_one_context(precision, slices):
    import ctypes as C

    import torch

    from tenet_b200 import Runtime, _lib

    rt = Runtime(0)
    a1, b1 = _tensor(rt, [V, P], [P, V], 1), _tensor(rt, [P, V], [V, P], 2)
    a2, b2 = _tensor(rt, [V, P], [P, V], 3), _tensor(rt, [P, V], [V, P], 4)
    plan = rt.cplan(a1.space, b1.space)
    prec = {"i8x": _lib.PREC_INT8X, "bf16x": _lib.PREC_BF16X}[precision]
    nb = 16  # enough batch entries that the first compose is still running when the second is issued
    ga1, gb1 = a1.data.repeat(nb), b1.data.repeat(nb)
    ga2, gb2 = a2.data.repeat(nb), b2.data.repeat(nb)

    def compose(ga, gb, out, stream):
        _lib.call("tnt_compose", rt._h, plan._h, nb, C.c_void_p(out.data_ptr()), plan.dst.size,
                  C.c_void_p(ga.data_ptr()), a1.space.size, C.c_void_p(gb.data_ptr()), b1.space.size, 1.0, 0.0,
                  prec, slices, C.c_void_p(stream.cuda_stream))

    s0 = torch.cuda.current_stream()
    ref1 = torch.empty(nb * plan.dst.size, dtype=torch.float64, device="cuda")
    ref2 = torch.empty_like(ref1)
    compose(ga1, gb1, ref1, s0)
    compose(ga2, gb2, ref2, s0)
    torch.cuda.synchronize()

    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    for _ in range(3):
        out1, out2 = torch.full_like(ref1, np.nan), torch.full_like(ref2, np.nan)
        torch.cuda.synchronize()
        compose(ga1, gb1, out1, s1)
        compose(ga2, gb2, out2, s2)
        torch.cuda.synchronize()
        assert torch.equal(out1, ref1)
        assert torch.equal(out2, ref2)
    rt.sync()
