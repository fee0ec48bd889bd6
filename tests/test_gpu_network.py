"""Contraction networks executed on the device vs the oracle's schedule replay.

One ``tnt_network_execute`` runs the whole schedule: fused operand
transforms, grouped GEMMs, intermediates in a planned workspace.  Parity:
1e-12 relative to the largest entry for FP64; 1e-10 for the BF16-split and
int8-digit composes.  The schedule replays under a CUDA graph.
"""

import math

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.network import execute_schedule
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

SU2R = Rule([SU2])
I3 = Rule([FZ2, U1, SU2])
W = Leg.new(SU2R, [((0,), 40), ((1,), 64), ((2,), 64), ((3,), 40), ((4,), 16)])
P = Leg.new(SU2R, [((1,), 1)])
V3 = Leg.new(I3, [((0, 0, 0), 6), ((1, 1, 1), 8), ((1, -1, 1), 5), ((0, 2, 0), 3), ((0, 0, 2), 4)])
P3 = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])
ITEBD = dict(inputs=[["l", "p1", "m"], ["m", "p2", "r"], ["q1", "q2", "p1", "p2"]],
             output=["l", "q1", "q2", "r"], output_codomain_rank=2)


@pytest.fixture(scope="module")
def rt():
    import tenet_b200.typed as tb

    return tb.Runtime(0)


def _dev(rt, t_o):
    import tenet_b200.typed as tb

    rule = product_rule(t_o.rule)
    return tb.TensorMap.from_host(rt, [product_leg(rule, l) for l in t_o.space.codomain],
                                  [product_leg(rule, l) for l in t_o.space.domain], t_o.data)


def _steps(plan):
    return [(s.lhs_slot, s.rhs_slot, s.result_slot, s.lhs_axes, s.rhs_axes, s.output_axes, s.result_permutation)
            for s in plan.steps]


def _close(got, ref, tol=1e-12):
    np.testing.assert_allclose(got, ref, rtol=0, atol=tol * np.abs(ref).max())


def _itebd(seed_a=1, seed_b=2):
    a_sp = OHom(SU2R, [W, P], [W])
    A, B = OT(a_sp, normal_fill(seed_a, a_sp.size)), OT(a_sp, normal_fill(seed_b, a_sp.size))
    g_sp = OHom(SU2R, [P, P], [P, P])
    G = OT(g_sp)
    for c, r, cc, off in g_sp.sectors:
        G.data[off] = math.exp(-0.05 * (-0.75 if c[0] == 0 else 0.25))
    return A, B, G


def test_itebd_network_matches_oracle(rt):
    from tenet_b200.network import Network

    A, B, G = _itebd()
    ref = G.contract(A.contract(B, [2], [0], [0, 1, 2, 3]), [2, 3], [1, 2], [0, 1, 2, 3]).permute([2, 0], [1, 3])
    ops = [_dev(rt, t) for t in (A, B, G)]
    plan = Network(**ITEBD).plan(ops)
    got = plan.execute(ops)
    assert got.space.size == ref.space.size
    _close(got.to_host(), ref.data)


@pytest.mark.parametrize("precision,slices", [("bf16x", 6), ("i8x", 6)])
def test_itebd_network_split_precision(rt, precision, slices):
    from tenet_b200.network import Network

    A, B, G = _itebd(3, 4)
    ops = [_dev(rt, t) for t in (A, B, G)]
    plan = Network(**ITEBD).plan(ops)
    ref = plan.execute(ops, precision="fp64").to_host()
    got = plan.execute(ops, precision=precision, slices=slices).to_host()
    rt.sync()
    _close(got, ref, 1e-10)


def _fermion_ops(seed):
    rng = np.random.default_rng(seed)
    sp_a = OHom(I3, [V3, P3], [V3])
    sp_g = OHom(I3, [P3, P3], [P3, P3])
    return (OT(sp_a, rng.standard_normal(sp_a.size)), OT(sp_a, rng.standard_normal(sp_a.size)),
            OT(sp_g, rng.standard_normal(sp_g.size)))


@pytest.mark.parametrize("order", [None, ["p1", "m", "p2"]])
def test_fermionic_network_matches_oracle(rt, order):
    from tenet_b200.network import Network

    A, B, G = _fermion_ops(5)
    ops = [_dev(rt, t) for t in (A, B, G)]
    plan = Network(**ITEBD).plan(ops, order=order)
    ref = execute_schedule([A, B, G], [False] * 3, _steps(plan), plan.final_slot, plan.final_permutation)
    _close(plan.execute(ops).to_host(), ref.data)


def test_conjugated_network_matches_oracle(rt):
    from tenet_b200.network import Network

    A, B, G = _fermion_ops(6)
    net = Network([["l", "p", "r"], ["p", "x", "q1", "q2"], ["l", "q1", "s"]], conj=[True, False, False],
                  output=["r", "x", "q2", "s"], output_codomain_rank=2)
    # A^dagger has flat legs (r ; l, p): its domain legs pair with codomain
    # legs of G and B.
    ops_o = [A, G, B]
    ops = [_dev(rt, t) for t in ops_o]
    plan = net.plan(ops)
    ref = execute_schedule(ops_o, [True, False, False], _steps(plan), plan.final_slot, plan.final_permutation)
    _close(plan.execute(ops).to_host(), ref.data)


def test_network_replays_in_a_cuda_graph(rt):
    import torch

    from tenet_b200.network import Network

    A, B, G = _itebd(7, 8)
    ops = [_dev(rt, t) for t in (A, B, G)]
    plan = Network(**ITEBD).plan(ops)
    out = plan.execute(ops)  # first call uploads tables and calibrates
    eager = out.to_host().copy()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        with torch.cuda.graph(graph, stream=stream):
            plan.execute(ops, out=out)
    A2, B2, _ = _itebd(9, 10)
    ops[0].data.copy_(torch.as_tensor(A2.data, device=ops[0].data.device))
    ops[1].data.copy_(torch.as_tensor(B2.data, device=ops[1].data.device))
    graph.replay()
    torch.cuda.synchronize()
    ref = Network(**ITEBD).plan(ops).execute(ops).to_host()
    _close(out.to_host(), ref)
    assert not np.allclose(out.to_host(), eager)


def test_degenerate_networks_match_oracle(rt):
    """Single operand with a final permutation, a conjugated single operand (a
    copy through the adjoint transform), and an outer product."""
    from tenet_b200.network import Network

    A, _, _ = _itebd(13, 14)
    a = _dev(rt, A)
    plan = Network([["a", "b", "c"]], output=["c", "a", "b"], output_codomain_rank=1).plan([a])
    _close(plan.execute([a]).to_host(), A.permute([2], [0, 1]).data)
    plan = Network([["a", "b", "c"]], conj=[True], output=["c", "a", "b"], output_codomain_rank=1).plan([a])
    _close(plan.execute([a]).to_host(), A.adjoint().data)
    ws = Leg.new(SU2R, [((0,), 2), ((1,), 1)])
    small_sp = OHom(SU2R, [ws, P], [ws])
    small = OT(small_sp, normal_fill(15, small_sp.size))
    s = _dev(rt, small)
    plan = Network([["a", "b", "c"], ["d", "e", "f"]], output=list("abcdef"), output_codomain_rank=3).plan([s, s])
    ref = execute_schedule([small, small], [False, False], _steps(plan), plan.final_slot, plan.final_permutation)
    _close(plan.execute([s, s]).to_host(), ref.data)
