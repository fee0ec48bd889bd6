"""SU(2) two-site iTEBD update (W spins 0..2, degeneracies [40, 64, 64, 40, 16]) on the device vs the oracle.

Checks the bond matrix after contraction, gate and 6j recoupling (1e-12
relative Frobenius), the per-sector singular values (1e-12 of the largest),
the kept counts of ``Truncation::space(W.truncspace())`` (exact) and the
truncation error (1e-10 relative).
"""

import math

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill

pytestmark = pytest.mark.gpu

W_PAIRS = [((0,), 40), ((1,), 64), ((2,), 64), ((3,), 40), ((4,), 16)]
TAU = 0.05


def oracle_step(seed_a=1, seed_b=2):
    r = Rule([SU2])
    W, P = Leg.new(r, W_PAIRS), Leg.new(r, [((1,), 1)])
    a_sp = OHom(r, [W, P], [W])
    A = OT(a_sp, normal_fill(seed_a, a_sp.size))
    B = OT(a_sp, normal_fill(seed_b, a_sp.size))
    g_sp = OHom(r, [P, P], [P, P])
    G = OT(g_sp)
    for i, (c, rr, cc, off) in enumerate(g_sp.sectors):
        G.data[off] = math.exp(-TAU * (-0.75 if c[0] == 0 else 0.25))
    theta = A.contract(B, [2], [0], [0, 1, 2, 3])
    gated = G.contract(theta, [2, 3], [1, 2], [0, 1, 2, 3])
    th = gated.permute([2, 0], [1, 3])
    prof = {s: d for s, d in W_PAIRS}
    parts, kept, err = th.svd_trunc(("space", prof))
    return A, B, th, parts, kept, err


def test_itebd_bond_update_matches_oracle():
    import tenet_b200 as tb
    from tenet_b200 import itebd

    A_o, B_o, th_o, parts, kept, err = oracle_step()
    rt = tb.Runtime(0)
    rule = tb.SU2FusionRule()
    W = tb.GradedSpace(rule, [(s[0], d) for s, d in W_PAIRS])
    P = tb.GradedSpace(rule, [(1, 1)])
    A = tb.TensorMap.from_host(rt, [W, P], [W], A_o.data)
    B = tb.TensorMap.from_host(rt, [W, P], [W], B_o.data)
    G = itebd.heisenberg_gate(rt, rule, P, TAU)
    th = itebd.bond_theta(A, B, G)
    assert th.space.block_keys() == [b["key"] for b in th_o.space.blocks]
    got = th.to_host()
    assert np.linalg.norm(got - th_o.data) <= 1e-12 * np.linalg.norm(th_o.data)
    res = th.svd_trunc(tb.Truncation.space(W))
    assert res.kept == kept
    smax = max(float(s[0]) for _, _, s, _ in parts if len(s))
    for (c, u, s, vh), ent in zip(parts, res.singular_values):
        np.testing.assert_allclose(ent.values, s, rtol=0, atol=1e-12 * smax)
    assert abs(res.error - err) <= 1e-10 * err
    # the kept bond space is W itself
    assert [k for k in res.kept if k] == [40, 64, 64, 40, 16]
