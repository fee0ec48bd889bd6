"""Edge cases on the device path: empty results, empty batches, ragged sectors,
rank-0 truncation.  Parity against the oracle where there is a result."""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

U1R = Rule([U1])


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


def dev(rt, orule, ocod, odom, data):
    from tenet_b200 import typed

    rule = product_rule(orule)
    return typed.TensorMap.from_host(rt, [product_leg(rule, l) for l in ocod], [product_leg(rule, l) for l in odom],
                                     data)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_compose_with_no_common_coupled_sector_is_empty(rt):
    V = Leg.new(U1R, [((1,), 2)])
    W = Leg.new(U1R, [((0,), 2), ((2,), 3)])
    X = Leg.new(U1R, [((0,), 1)])
    a_sp, b_sp = OHom(U1R, [V, V], [W]), OHom(U1R, [W], [X, X])
    a = dev(rt, U1R, [V, V], [W], normal_fill(1, a_sp.size))
    b = dev(rt, U1R, [W], [X, X], normal_fill(2, b_sp.size))
    c = a.compose(b)
    assert c.space.size == 0 and c.data.numel() == 0
    rt.sync()


@pytest.mark.parametrize("precision", ["fp64", "bf16x", "i8x"])
def test_empty_batch_is_a_no_op(rt, precision):
    import ctypes as C

    import torch

    from tenet_b200 import _lib

    V = Leg.new(U1R, [((0,), 3), ((1,), 2)])
    sp = OHom(U1R, [V], [V])
    a = dev(rt, U1R, [V], [V], normal_fill(3, sp.size))
    plan = rt.cplan(a.space, a.space)
    out = torch.full((plan.dst.size,), 7.0, dtype=torch.float64, device="cuda")
    prec = {"fp64": _lib.PREC_FP64, "bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X}[precision]
    _lib.call("tnt_compose", rt._h, plan._h, 0, C.c_void_p(out.data_ptr()), plan.dst.size,
              C.c_void_p(a.data.data_ptr()), sp.size, C.c_void_p(a.data.data_ptr()), sp.size, 1.0, 0.0, prec, 6,
              rt.stream())
    rt.sync()
    assert bool((out == 7.0).all())


def test_ragged_sectors_compose_permute_svd(rt):
    """Degeneracies 1 and 257 (one more than four 64-wide tiles) beside ordinary ones."""
    V = Leg.new(U1R, [((-1,), 1), ((0,), 257), ((1,), 1), ((2,), 5)])
    W = Leg.new(U1R, [((0,), 3), ((1,), 4)])
    sp = OHom(U1R, [V, W], [W, V])
    spb = OHom(U1R, [W, V], [V, W])
    a = OT(sp, normal_fill(11, sp.size))
    b = OT(spb, normal_fill(12, spb.size))
    da, db = dev(rt, U1R, [V, W], [W, V], a.data), dev(rt, U1R, [W, V], [V, W], b.data)
    ref = a.compose(b)
    for precision, tol in (("fp64", 1e-12), ("bf16x", 4 * 7 * 2.0 ** -42 + 512 * 2.0 ** -45),
                           ("i8x", 4 * 7 * 2.0 ** -46 + 2.0 ** -50)):
        c = da.compose(db, precision=precision, slices=6)
        assert rel(c.to_host(), ref.data) <= tol, precision
    rt.sync()
    p = da.permute([0, 3], [2, 1])
    assert rel(p.to_host(), a.permute([0, 3], [2, 1]).data) <= 1e-12
    # SVD of blocks of 1 x 1, 257 x 257 (global-memory panel) and 5 x 5
    sq = OHom(U1R, [V], [V])
    m = OT(sq, normal_fill(13, sq.size))
    res = dev(rt, U1R, [V], [V], m.data).svd_compact()
    for (cc, u, s, vh), ent in zip(m.svd_compact(), res.singular_values):
        np.testing.assert_allclose(ent.values, s, rtol=1e-12, atol=1e-12 * s[0])


def test_rank_zero_truncation_discards_everything(rt):
    from tenet_b200 import Truncation

    W = Leg.new(Rule([SU2]), [((0,), 4), ((1,), 6), ((2,), 3)])
    P = Leg.new(Rule([SU2]), [((1,), 1)])
    sp = OHom(Rule([SU2]), [W, P], [P, W])
    src = OT(sp, normal_fill(21, sp.size))
    res = dev(rt, Rule([SU2]), [W, P], [P, W], src.data).svd_trunc(Truncation.rank(0))
    assert all(k == 0 for k in res.kept)
    assert abs(res.error - src.norm()) <= 1e-12 * src.norm()
