"""Contraction networks: label validation, planning and the compiled device
schedule's structure (CPU only; the payload runs in test_gpu_network.py).

The oracle replays schedules with ``TensorMap::contract`` semantics
(tenet-network/src/network.rs:1820-1920).  Checked here: the iTEBD network
equals the hand-written contraction sequence, results do not depend on the
contraction order (SU(2) and fermionic fZ2 x U(1) x SU(2) with conjugated
operands), and the C++ schedule compiler produces the oracle's output space
bit-exactly with every operand transform fused into one pass.
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
from tests.helpers import product_space

SU2R = Rule([SU2])
I3 = Rule([FZ2, U1, SU2])
W = Leg.new(SU2R, [((0,), 4), ((1,), 6), ((2,), 6), ((3,), 4), ((4,), 2)])
P = Leg.new(SU2R, [((1,), 1)])
TAU = 0.05

V3 = Leg.new(I3, [((0, 0, 0), 2), ((1, 1, 1), 3), ((1, -1, 1), 2), ((0, 2, 0), 1)])
P3 = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])


def _steps(plan):
    return [(s.lhs_slot, s.rhs_slot, s.result_slot, s.lhs_axes, s.rhs_axes, s.output_axes, s.result_permutation)
            for s in plan.steps]


def itebd_operands():
    a_sp = OHom(SU2R, [W, P], [W])
    A = OT(a_sp, normal_fill(1, a_sp.size))
    B = OT(a_sp, normal_fill(2, a_sp.size))
    g_sp = OHom(SU2R, [P, P], [P, P])
    G = OT(g_sp)
    for i, (c, r, cc, off) in enumerate(g_sp.sectors):
        G.data[off] = math.exp(-TAU * (-0.75 if c[0] == 0 else 0.25))
    return A, B, G


ITEBD_LABELS = dict(inputs=[["l", "p1", "m"], ["m", "p2", "r"], ["q1", "q2", "p1", "p2"]],
                    output=["l", "q1", "q2", "r"], output_codomain_rank=2)


def test_network_validation():
    from tenet_b200.network import Network

    Network([["a", "b"], ["b", "c"]], output=["a", "c"])
    with pytest.raises(ValueError, match="hyperedge"):
        Network([["a", "b"], ["b", "c"], ["b", "d"]], output=["a", "c", "d"])
    with pytest.raises(ValueError, match="open labels"):
        Network([["a", "b"], ["b", "c"]], output=["a"])
    with pytest.raises(ValueError, match="repeats a label"):
        Network([["a", "a"]], output=[])
    with pytest.raises(ValueError, match="marker lists"):
        Network([["a", "b"], ["b", "c"]], conj=[False], output=["a", "c"])
    with pytest.raises(ValueError, match="exceeds output rank"):
        Network([["a", "b"], ["b", "c"]], output=["a", "c"], output_codomain_rank=3)


@pytest.mark.parametrize("order", [None, ["m", "p1", "p2"], ["p1", "m", "p2"]])
def test_itebd_network_matches_hand_contraction(order):
    from tenet_b200.network import Network

    A, B, G = itebd_operands()
    theta = A.contract(B, [2], [0], [0, 1, 2, 3])
    gated = G.contract(theta, [2, 3], [1, 2], [0, 1, 2, 3])
    ref = gated.permute([2, 0], [1, 3])
    net = Network(**ITEBD_LABELS)
    spaces = [product_space(SU2R, t.space.codomain, t.space.domain) for t in (A, B, G)]
    plan = net.plan(spaces, order=order)
    got = execute_schedule([A, B, G], [False] * 3, _steps(plan), plan.final_slot, plan.final_permutation)
    assert [b["key"] for b in got.space.blocks] == [b["key"] for b in ref.space.blocks]
    np.testing.assert_allclose(got.data, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max())
    # The compiled device schedule: two composes, the output space bit-exact.
    assert plan.n_composes == 2
    assert plan.output_space.block_keys() == [b["key"] for b in ref.space.blocks]
    assert plan.output_space.size == ref.space.size


def _fermion_operands():
    rng = np.random.default_rng(17)
    sp_a = OHom(I3, [V3, P3], [V3])
    sp_g = OHom(I3, [P3, P3], [P3, P3])
    A = OT(sp_a, rng.standard_normal(sp_a.size))
    B = OT(sp_a, rng.standard_normal(sp_a.size))
    G = OT(sp_g, rng.standard_normal(sp_g.size))
    return A, B, G


@pytest.mark.parametrize("order", [["m", "p1", "p2"], ["p1", "m", "p2"], ["p2", "p1", "m"]])
def test_fermionic_network_is_order_independent(order):
    from tenet_b200.network import Network

    A, B, G = _fermion_operands()
    net = Network(**ITEBD_LABELS)
    spaces = [product_space(I3, t.space.codomain, t.space.domain) for t in (A, B, G)]
    base_plan = net.plan(spaces, order=["m", "p1", "p2"])
    base = execute_schedule([A, B, G], [False] * 3, _steps(base_plan), base_plan.final_slot,
                            base_plan.final_permutation)
    plan = net.plan(spaces, order=order)
    got = execute_schedule([A, B, G], [False] * 3, _steps(plan), plan.final_slot, plan.final_permutation)
    np.testing.assert_allclose(got.data, base.data, rtol=0, atol=1e-12 * np.abs(base.data).max())
    assert plan.output_space.block_keys() == [b["key"] for b in base.space.blocks]


def test_conjugated_operand_network():
    """<A|A>-style overlap with a conjugated operand, rank-0 result avoided:
    contract A^dagger with A over the physical and left legs."""
    from tenet_b200.network import Network

    A, _, _ = _fermion_operands()
    net = Network([["l", "p", "r"], ["l", "p", "s"]], conj=[True, False], output=["r", "s"], output_codomain_rank=1)
    spaces = [product_space(I3, A.space.codomain, A.space.domain)] * 2
    plan = net.plan(spaces)
    got = execute_schedule([A, A], [True, False], _steps(plan), plan.final_slot, plan.final_permutation)
    ref = A.adjoint().compose(A)
    assert [b["key"] for b in got.space.blocks] == [b["key"] for b in ref.space.blocks]
    np.testing.assert_allclose(got.data, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max())
    assert plan.output_space.block_keys() == [b["key"] for b in ref.space.blocks]


def test_schedule_fuses_operand_transforms():
    """Three-operand chain: each compose operand gets at most one transform."""
    from tenet_b200.network import Network

    A, B, G = itebd_operands()
    net = Network(**ITEBD_LABELS)
    spaces = [product_space(SU2R, t.space.codomain, t.space.domain) for t in (A, B, G)]
    plan = net.plan(spaces, order=["m", "p1", "p2"])
    assert plan.n_composes == 2
    assert plan.n_transforms <= 2 * plan.n_composes + 1
    assert plan.workspace_elems > 0


def test_schedule_errors():
    from tenet_b200._lib import TenetError
    from tenet_b200.network import PlannedNetwork, Step

    A, B, G = itebd_operands()
    spaces = [product_space(SU2R, t.space.codomain, t.space.domain) for t in (A, B)]
    with pytest.raises(TenetError):
        PlannedNetwork(spaces, [False, False], [Step(0, 0, 2, (2,), (0,), (0, 1, 2, 3))], 2)
    with pytest.raises(TenetError):
        PlannedNetwork(spaces, [False, False], [Step(0, 1, 2, (2,), (0,), (0, 1, 2))], 2)
    with pytest.raises(TenetError):
        PlannedNetwork(spaces, [False, False], [], 0)
    # contracting W against P is a leg mismatch
    with pytest.raises(TenetError):
        PlannedNetwork(spaces, [False, False], [Step(0, 1, 2, (1,), (0,), (0, 1, 2, 3))], 2)


def test_degenerate_networks_compile_to_the_oracle_spaces():
    """A single operand (final permutation only, or a conjugated operand) and
    an outer product (a step with no contracted label) follow the oracle."""
    from tenet_b200.network import Network

    A, _, _ = itebd_operands()
    spA = product_space(SU2R, A.space.codomain, A.space.domain)
    plan = Network([["a", "b", "c"]], output=["c", "a", "b"], output_codomain_rank=1).plan([spA])
    assert plan.steps == [] and plan.n_composes == 0 and plan.n_transforms == 1
    assert plan.output_space.block_keys() == [b["key"] for b in A.permute([2], [0, 1]).space.blocks]
    plan = Network([["a", "b", "c"]], conj=[True], output=["c", "a", "b"], output_codomain_rank=1).plan([spA])
    assert plan.final_permutation is None and plan.n_transforms == 1
    assert plan.output_space.block_keys() == [b["key"] for b in A.adjoint().space.blocks]
    plan = Network([["a", "b", "c"], ["d", "e", "f"]], output=list("abcdef"), output_codomain_rank=3).plan([spA, spA])
    assert len(plan.steps) == 1 and plan.steps[0].lhs_axes == ()
    got = execute_schedule([A, A], [False, False], _steps(plan), plan.final_slot, plan.final_permutation)
    assert plan.output_space.block_keys() == [b["key"] for b in got.space.blocks]


def test_workspace_reuses_dead_intermediates():
    """A four-tensor chain: every intermediate dies at the next step, so the
    planned workspace is smaller than the sum of all intermediates."""
    from tenet_b200.network import Network

    r = SU2R
    v = Leg.new(r, [((0,), 6), ((1,), 8), ((2,), 4)])
    mats = [OT(OHom(r, [v], [v]), normal_fill(40 + i, OHom(r, [v], [v]).size)) for i in range(4)]
    spaces = [product_space(r, m.space.codomain, m.space.domain) for m in mats]
    net = Network([["a", "b"], ["b", "c"], ["c", "d"], ["d", "e"]], output=["a", "e"], output_codomain_rank=1)
    plan = net.plan(spaces, order=["b", "c", "d"])
    assert plan.n_composes == 3
    size = spaces[0].size
    # two intermediates (A.B and (A.B).C) and no operand transforms: at most
    # two live buffers at once, each padded to 32 doubles
    assert plan.workspace_elems <= 2 * ((size + 31) // 32 * 32)
    got = execute_schedule(mats, [False] * 4, _steps(plan), plan.final_slot, plan.final_permutation)
    ref = mats[0].compose(mats[1]).compose(mats[2]).compose(mats[3])
    np.testing.assert_allclose(got.data, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max())
    assert plan.n_transforms == 0


def test_exhaustive_planner_minimises_block_sparse_flops():
    """Every pairwise order is compiled; the kept one has the fewest compose
    flops (then transform bytes), and its result still equals the oracle."""
    from tenet_b200.network import Network, _pair_sequences

    A, B, G = itebd_operands()
    net = Network(**ITEBD_LABELS)
    spaces = [product_space(SU2R, t.space.codomain, t.space.domain) for t in (A, B, G)]
    seqs = list(_pair_sequences({0: ["l", "p1", "m"], 1: ["m", "p2", "r"], 2: ["q1", "q2", "p1", "p2"]}))
    assert len(seqs) == 3  # three pairs to start with, then one
    best = net.plan(spaces, order="exhaustive")
    for order in (None, ["m", "p1", "p2"], ["p1", "m", "p2"], ["p2", "p1", "m"]):
        other = net.plan(spaces, order=order)
        assert (best.flops, best.bytes_moved) <= (other.flops, other.bytes_moved)
    got = execute_schedule([A, B, G], [False] * 3, _steps(best), best.final_slot, best.final_permutation)
    ref = G.contract(A.contract(B, [2], [0], [0, 1, 2, 3]), [2, 3], [1, 2], [0, 1, 2, 3]).permute([2, 0], [1, 3])
    np.testing.assert_allclose(got.data, ref.data, rtol=0, atol=1e-12 * np.abs(ref.data).max())
    with pytest.raises(ValueError):
        net.plan(spaces, order="fastest")
