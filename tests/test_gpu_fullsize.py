"""Full-size checks through size-independent properties.

* hubbard_batch (fZ2 x U(1) x SU(2), 60 W sectors): one full compose against
  the CPU restatement (1e-12), and the grouped FP64 kernel against the
  per-sector cuBLAS route on four tensors at once (1e-13, independent code);
* su2_heff (x: 7.4 M elements, L: 17.9 M): permute round trips and the
  weighted norm under recoupling (SU(2) recoupling is orthogonal), the
  contraction linearity, and <B x, y> = <x, B^dagger y>;
* serving's largest chain (D = 2048, 580 x 580 sectors): the truncated SVD
  of the bond matrix reconstructs it (full rank kept) with orthonormal U.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_hubbard_full_compose_matches_restatement_and_cublas(rt):
    import torch

    import tenet_b200 as tb
    from oracle.fusion import HomSpace as OHom
    from oracle.fusion import Leg
    from oracle.sectors import Rule
    from oracle.tensor import TensorMap as OT
    from tenet_b200 import _lib
    from tenet_b200.workloads import hubbard_batch, splitmix_normal

    cfg = hubbard_batch(0)
    rule = tb.FusionRule(cfg["factors"])
    W, P = tb.GradedSpace(rule, cfg["W"]), tb.GradedSpace(rule, cfg["P"])
    a = tb.TensorMap.from_host(rt, [W, P], [P, W], splitmix_normal(1, rt.space(rule, [W, P], [P, W]).size))
    b = tb.TensorMap.from_host(rt, [P, W], [W, P], splitmix_normal(5001, rt.space(rule, [P, W], [W, P]).size))
    c = a.compose(b)
    r = Rule(cfg["factors"])
    ow, op = Leg.new(r, cfg["W"]), Leg.new(r, cfg["P"])
    ref = OT(OHom(r, [ow, op], [op, ow]), a.to_host()).compose(OT(OHom(r, [op, ow], [ow, op]), b.to_host()))
    assert c.space.block_keys() == [blk["key"] for blk in ref.space.blocks]
    assert rel(c.to_host(), ref.data) <= 1e-12
    # four tensors in one launch vs one cuBLAS DGEMM per coupled sector
    plan = rt.cplan(a.space, b.space)
    nb = 4
    ga = torch.as_tensor(np.concatenate([splitmix_normal(1 + i, a.space.size) for i in range(nb)]), device="cuda")
    gb = torch.as_tensor(np.concatenate([splitmix_normal(5001 + i, b.space.size) for i in range(nb)]), device="cuda")
    outs = []
    for prec in (_lib.PREC_FP64, _lib.PREC_CUBLAS_FP64):
        gc = torch.zeros(nb * plan.dst.size, dtype=torch.float64, device="cuda")
        _lib.call("tnt_compose", rt._h, plan._h, nb, C.c_void_p(gc.data_ptr()), plan.dst.size,
                  C.c_void_p(ga.data_ptr()), a.space.size, C.c_void_p(gb.data_ptr()), b.space.size, 1.0, 0.0, prec,
                  0, rt.stream())
        outs.append(gc.cpu().numpy())
    assert rel(outs[0], outs[1]) <= 1e-13


@pytest.fixture(scope="module")
def heff(rt):
    from tenet_b200 import heff as H
    from tenet_b200 import workloads

    rule, x, L, O, R = H.workload_tensors(rt, workloads.su2_heff(), scale=1)
    return x, L, O, R, H.EffectiveHamiltonian(L, O, R)


def test_heff_permute_round_trip_and_norm(rt, heff):
    x, L, O, R, Hm = heff
    xb = x.permute([0], [1, 2])
    back = xb.permute([0, 1], [2])
    assert back.space.block_keys() == x.space.block_keys()
    assert rel(back.to_host(), x.to_host()) <= 1e-13
    assert abs(xb.norm() - x.norm()) <= 1e-13 * x.norm()
    t1 = L.compose(xb)
    t1p = t1.permute([0, 3], [1, 2])
    assert abs(t1p.norm() - t1.norm()) <= 1e-13 * t1.norm()
    assert rel(t1p.permute([0, 2], [3, 1]).to_host(), t1.to_host()) <= 1e-13


def test_heff_linearity_and_adjoint(rt, heff):
    import tenet_b200 as tb
    from tenet_b200.workloads import splitmix_normal

    torch = tb.typed.torch()
    x, L, O, R, Hm = heff
    y = tb.TensorMap(rt, x.space, torch.as_tensor(splitmix_normal(77, x.space.size), device="cuda"))
    bx, by = Hm.apply_b(x, "fp64", 0), Hm.apply_b(y, "fp64", 0)
    bxy = Hm.apply_b(x.add(y, 2.0, -0.5), "fp64", 0)
    assert rel(bxy.to_host(), 2.0 * bx.to_host() - 0.5 * by.to_host()) <= 1e-12
    bty = Hm.apply_bdag(y, "fp64", 0)

    def wip(a, b):
        s = 0.0
        for lab, r, c, off in a.space.sectors():
            s += a.rule.dim(a.rule.unlabel(lab)) * float(torch.dot(a.data[off:off + r * c], b.data[off:off + r * c]))
        return s

    lhs, rhs = wip(bx, y), wip(x, bty)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_serving_largest_chain_svd_reconstructs(rt):
    import tenet_b200 as tb
    from tenet_b200 import itebd, serving
    from tenet_b200.workloads import splitmix_normal

    rule = tb.SU2FusionRule()
    W = serving.chain_bond_space(rule, 2048)
    P = tb.GradedSpace(rule, [(1, 1)])
    n = rt.space(rule, [W, P], [W]).size
    A = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(3, n))
    B = tb.TensorMap.from_host(rt, [W, P], [W], splitmix_normal(4, n))
    bm = itebd.bond_theta(A, B, itebd.heisenberg_gate(rt, rule, P, 0.05))
    assert max(r for _, r, _, _ in bm.space.sectors()) >= 580
    res = bm.svd_compact()
    U, spectra, Vh = res.factors()
    torch = tb.typed.torch()
    for (lab, m, nn, off), ent in zip(bm.space.sectors(), spectra):
        s = ent.values
        assert np.all(np.diff(s) <= 0)
    ub = {lab: (r, c, off) for lab, r, c, off in U.space.sectors()}
    vb = {lab: (r, c, off) for lab, r, c, off in Vh.space.sectors()}
    for (lab, m, nn, off), ent in zip(bm.space.sectors(), spectra):
        r, k, uo = ub[lab]
        u = U.data[uo:uo + r * k].view(k, r).T
        kr, c, vo = vb[lab]
        vh = Vh.data[vo:vo + kr * c].view(c, kr).T
        a = bm.data[off:off + m * nn].view(nn, m).T
        s = torch.as_tensor(ent.values, device="cuda")
        recon = (u * s) @ vh
        assert float(torch.linalg.norm(recon - a) / torch.linalg.norm(a)) <= 1e-12
        eye = torch.eye(k, dtype=torch.float64, device="cuda")
        assert float(torch.linalg.norm(u.T @ u - eye)) <= 1e-12 * k


@pytest.mark.parametrize("m,n", [(700, 500), (450, 640)], ids=["tall", "wide"])
def test_cluster_svd_matches_lapack(rt, m, n):
    """Sectors with enough column blocks run the blocked Jacobi on a thread-block
    cluster: singular values vs LAPACK within 1e-12 of the largest, factors
    reconstruct the block, U orthonormal."""
    import tenet_b200 as tb
    from tenet_b200.workloads import splitmix_normal

    rule = tb.U1FusionRule()
    X = tb.GradedSpace(rule, [(0, m)])
    Y = tb.GradedSpace(rule, [(0, n)])
    size = rt.space(rule, [X], [Y]).size
    t = tb.TensorMap.from_host(rt, [X], [Y], splitmix_normal(19, size))
    res = t.svd_compact()
    a = t.to_host().reshape(n, m).T
    ref = np.linalg.svd(a, compute_uv=False)
    s = res.singular_values[0].values
    np.testing.assert_allclose(s, ref, rtol=0, atol=1e-12 * ref[0])
    U, _, Vh = res.factors()
    k = min(m, n)
    u = U.to_host().reshape(k, m).T
    vh = Vh.to_host().reshape(n, k).T
    assert rel((u * s) @ vh, a) <= 1e-12
    assert np.linalg.norm(u.T @ u - np.eye(k)) <= 1e-12 * k
