"""Transform plans compiled elsewhere (``tnt_xplan_from_tables``), CPU side.

The boundary for a caller that lowers the reference's own
TreeTransformStructure (tenet-operations/src/transform_structure.rs:82-95,
807-811): the tables of a native plan survive export -> import -> export
unchanged, replay identically, and malformed tables (entries or coefficients
out of range, blocks outside the payload, overlapping or missing destination
elements) are rejected before anything runs.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from tests.helpers import product_space, replay_transform

SU2R = Rule([SU2])
I3 = Rule([FZ2, U1, SU2])
V = Leg.new(SU2R, [((0,), 2), ((1,), 2), ((2,), 1)])
V3 = Leg.new(I3, [((0, 0, 0), 2), ((1, 1, 1), 2), ((0, 2, 0), 1)])

CASES = [
    (SU2R, [V, V], [V, V], [1, 0], [3, 2]),
    (SU2R, [V, V], [V, V], [0, 3], [2, 1]),
    (I3, [V3, V3], [V3, V3.dual()], [3, 0], [1, 2]),
]


def _native(rule, cod, dom, p1, p2):
    from tenet_b200.typed import TransformPlan

    sp = product_space(rule, cod, dom)
    return sp, TransformPlan(sp, "permute", p1, p2, (), 0)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_export_import_round_trip(case):
    from tenet_b200.typed import TransformPlan

    rule, cod, dom, p1, p2 = CASES[case]
    sp, plan = _native(rule, cod, dom, p1, p2)
    tables = plan.export()
    imp = TransformPlan.from_tables(sp.n1 + sp.n2, *tables, plan.src.size, plan.dst.size)
    assert imp.ngroups == plan.ngroups and imp.ncoef == plan.ncoef and imp.bytes_moved == plan.bytes_moved
    for a, b in zip(imp.export(), tables):
        np.testing.assert_array_equal(a, b)
    src = np.random.default_rng(1).standard_normal(plan.src.size)
    np.testing.assert_array_equal(replay_transform(imp.export(), src, plan.dst.size),
                                  replay_transform(tables, src, plan.dst.size))


def test_malformed_tables_are_rejected():
    from tenet_b200._lib import TenetError
    from tenet_b200.typed import TransformPlan

    rule, cod, dom, p1, p2 = CASES[0]
    sp, plan = _native(rule, cod, dom, p1, p2)
    g, s, d, c = plan.export()
    n, ns, nd = sp.n1 + sp.n2, plan.src.size, plan.dst.size

    def bad(g=g, s=s, d=d, c=c, ns=ns, nd=nd, rank=n, match=None):
        with pytest.raises(TenetError, match=match):
            TransformPlan.from_tables(rank, g, s, d, c, ns, nd)

    g2 = g.copy()
    g2[0, 5] = len(c)  # coefficients past the end
    bad(g=g2, match="coefficients")
    g2 = g.copy()
    g2[0, 3] = len(s)  # source entries past the end
    bad(g=g2, match="source entries")
    d2 = d.copy()
    d2[0, 0] = nd  # destination block outside the payload
    bad(d=d2, match="outside")
    d2 = d.copy()
    d2[1] = d2[0]  # two blocks on the same destination elements
    bad(d=d2, match="overlap|outside|no group")
    bad(g=g[1:], match="no group")  # a block nothing writes
    g2 = g.copy()
    g2[0, 0] += 1  # element count inconsistent with the extents
    bad(g=g2, match="element count")
    bad(rank=9, match="rank")


def test_imported_plan_has_no_spaces():
    from tenet_b200._lib import TenetError, call
    from tenet_b200.typed import TransformPlan
    import ctypes as C

    rule, cod, dom, p1, p2 = CASES[0]
    sp, plan = _native(rule, cod, dom, p1, p2)
    imp = TransformPlan.from_tables(sp.n1 + sp.n2, *plan.export(), plan.src.size, plan.dst.size)
    assert imp.src is None and imp.dst is None
    with pytest.raises(TenetError, match="no destination space"):
        call("tnt_xplan_dst_space", imp._h, C.byref(C.c_void_p()))
