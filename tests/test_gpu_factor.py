"""GPU parity for the batched per-sector QR and eigh kernels vs the oracle.

* QR: Q and R within 1e-12 relative Frobenius error per sector (the
  positive-diagonal gauge makes the factorisation of a full-rank block
  unique), tall and wide sectors, shared-memory and global-memory panels;
* eigh: eigenvalues within 1e-12 relative, eigenvectors within 1e-10
  absolute (non-degenerate random spectra), order and gauge as the
  reference's eigh_full_dyn; eigh_trunc kept counts exact and error within
  1e-10; non-Hermitian input rejected.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

U1R, SU2R = Rule([U1]), Rule([SU2])
X = Leg.new(U1R, [((0,), 20), ((1,), 15)])
Y = Leg.new(U1R, [((0,), 30), ((1,), 60), ((2,), 10)])  # sector 1: 600 x 60 -> global-memory panel
W = Leg.new(SU2R, [((0,), 4), ((1,), 6), ((2,), 6), ((3,), 4), ((4,), 2)])
P = Leg.new(SU2R, [((1,), 1)])
BIG = Leg.new(U1R, [((0,), 150), ((1,), 40)])  # 150 x 150 sector -> global-memory eigh


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


def device_tensor(rt, orule, ocod, odom, data):
    from tenet_b200 import typed

    rule = product_rule(orule)
    return typed.TensorMap.from_host(rt, [product_leg(rule, l) for l in ocod], [product_leg(rule, l) for l in odom],
                                     data)


def sector_blocks(t):
    h = t.to_host()
    return {lab: h[off:off + r * c].reshape(c, r).T for lab, r, c, off in t.space.sectors()}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("cod,dom", [([X, X], [Y]), ([Y], [X, X]), ([W, P], [P, W])], ids=["tall", "wide", "su2"])
def test_qr_matches_oracle(rt, cod, dom):
    rule = cod[0].rule
    sp = OHom(rule, cod, dom)
    src = OT(sp, normal_fill(21, sp.size))
    parts = src.qr_compact()
    Q, R = device_tensor(rt, rule, cod, dom, src.data).qr_compact()
    qb, rb = sector_blocks(Q), sector_blocks(R)
    assert len(qb) == len(parts) == len(rb)
    for key, (c, q, r) in zip(qb, parts):  # both in ascending SectorId order
        assert rel(qb[key], q) <= 1e-12
        assert rel(rb[key], r) <= 1e-12
    # the factors compose back to the input
    back = Q.compose(R)
    assert rel(back.to_host(), src.data) <= 1e-12


def symmetric(orule, legs, seed):
    sp = OHom(orule, legs, legs)
    a = OT(sp, normal_fill(seed, sp.size))
    return OT(sp, a.data + a.adjoint().data)


@pytest.mark.parametrize("orule,legs", [(U1R, [X, X]), (SU2R, [W, P]), (U1R, [BIG])], ids=["u1", "su2", "big"])
def test_eigh_matches_oracle(rt, orule, legs):
    src = symmetric(orule, legs, 31)
    parts = src.eigh_full()
    D, V = device_tensor(rt, orule, legs, legs, src.data).eigh_full()
    vb, db = sector_blocks(V), sector_blocks(D)
    keys = list(vb)
    assert len(keys) == len(parts)
    for key, (c, w, v) in zip(keys, parts):
        np.testing.assert_allclose(np.diag(db[key]), w, rtol=1e-12, atol=1e-12 * np.abs(w).max())
        np.testing.assert_allclose(vb[key], v, atol=1e-10)
    back = V.compose(D).compose(V.adjoint())
    assert rel(back.to_host(), src.data) <= 1e-12


@pytest.mark.parametrize("trunc", [("rank", 20), ("tol", 0.0, 0.3), ("discard", 0.2), ("full",)])
def test_eigh_trunc_matches_oracle(rt, trunc):
    from tenet_b200 import Truncation

    src = symmetric(SU2R, [W, P], 32)
    _, kept, err = src.eigh_trunc(trunc)
    pol = {
        "rank": lambda: Truncation.rank(trunc[1]),
        "tol": lambda: Truncation.tolerance(trunc[1], trunc[2]),
        "discard": lambda: Truncation.discard_weight(trunc[1]),
        "full": Truncation.full,
    }[trunc[0]]()
    res = device_tensor(rt, SU2R, [W, P], [W, P], src.data).eigh_trunc(pol)
    assert res.kept == kept
    assert abs(res.error - err) <= 1e-10 * max(1.0, err)
    D, V = res.factors()
    vb = sector_blocks(V)
    assert [b.shape[1] for b in vb.values()] == [k for k in kept if k > 0]


def test_eigh_rejects_non_hermitian(rt):
    from tenet_b200._lib import TenetError

    sp = OHom(U1R, [X], [X])
    t = device_tensor(rt, U1R, [X], [X], normal_fill(2, sp.size))
    with pytest.raises(TenetError, match="Hermitian"):
        t.eigh_full()


def test_eigh_large_sectors_with_degenerate_spectrum(rt):
    """Sectors beyond the on-chip two-sided Jacobi go through the batched SVD
    of A + ||A||_F I.  A spectrum with repeated eigenvalues and +-lambda pairs
    (so |lambda| is degenerate) is recovered: values within 1e-12 of the
    largest |lambda|, descending |lambda|, V D V^T = A and V orthonormal to
    1e-12."""
    size = OHom(U1R, [BIG], [BIG]).size
    probe = device_tensor(rt, U1R, [BIG], [BIG], np.zeros(size))
    data = np.zeros(probe.space.size)
    rng = np.random.default_rng(5)
    want = {}
    for lab, r, c, off in probe.space.sectors():
        q, _ = np.linalg.qr(rng.standard_normal((r, r)))
        lam = np.concatenate([np.full(r // 3, 2.0), np.full(r // 3, -2.0), rng.standard_normal(r - 2 * (r // 3))])
        a = (q * lam) @ q.T
        a = 0.5 * (a + a.T)
        data[off:off + r * c] = a.T.reshape(-1)  # column-major block
        want[lab] = (a, lam)
    D, V = device_tensor(rt, U1R, [BIG], [BIG], data).eigh_full()
    db, vb = sector_blocks(D), sector_blocks(V)
    for lab, (a, lam) in want.items():
        d, v = np.diag(db[lab]), vb[lab]
        np.testing.assert_allclose(np.sort(d), np.sort(lam), rtol=0, atol=1e-12 * np.abs(lam).max())
        assert np.all(np.diff(np.abs(d)) <= 1e-12)
        assert rel(v @ np.diag(d) @ v.T, a) <= 1e-12
        np.testing.assert_allclose(v.T @ v, np.eye(len(d)), rtol=0, atol=1e-12)


@pytest.mark.parametrize("cod,dom", [([X, X], [Y]), ([Y], [X, X]), ([W, P], [P, W])], ids=["tall", "wide", "su2"])
def test_lq_compact_is_the_adjoint_of_qr(rt, cod, dom):
    """lq_compact (typed.rs:1494) through the adjoint of the device QR: per
    sector L equals R'^T and Q equals Q'^T of the oracle's QR of the adjoint
    (1e-12), L o Q = A, Q Q^T = I, and right_orth / left_orth delegate."""
    rule = cod[0].rule
    sp = OHom(rule, cod, dom)
    src = OT(sp, normal_fill(41, sp.size))
    parts = src.adjoint().qr_compact()
    dev = device_tensor(rt, rule, cod, dom, src.data)
    L, Q = dev.lq_compact()
    lb, qb = sector_blocks(L), sector_blocks(Q)
    assert len(lb) == len(parts) == len(qb)
    for key, (c, q, r) in zip(lb, parts):
        assert rel(lb[key], r.T) <= 1e-12
        assert rel(qb[key], q.T) <= 1e-12
        assert np.allclose(qb[key] @ qb[key].T, np.eye(qb[key].shape[0]), atol=1e-12)
    assert rel(L.compose(Q).to_host(), src.data) <= 1e-12
    L2, Q2 = dev.right_orth()
    assert rel(L2.to_host(), L.to_host()) == 0.0 and rel(Q2.to_host(), Q.to_host()) == 0.0
    Qa, Ra = dev.left_orth()
    Qb, Rb = dev.qr_compact()
    assert rel(Qa.to_host(), Qb.to_host()) == 0.0 and rel(Ra.to_host(), Rb.to_host()) == 0.0
