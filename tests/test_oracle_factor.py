"""Oracle QR / eigh (CPU): reconstruction, gauges, ordering and truncation.

The per-sector factorisations follow qr_compact / eigh_full_dyn /
eigh_trunc_dyn (tenet-matrixalgebra/src/factorize.rs:5158, 3041-3150,
3284-3340); these checks pin the conventions the device kernels are compared
against: Q R = A with R_jj >= 0, V diag(w) V^T = A with w stable-sorted by
descending |w| and each eigenvector's largest-|.| entry positive, and the
truncation of |w| through select_truncation.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace
from oracle.fusion import Leg
from oracle.sectors import SU2, U1, Rule
from oracle.tensor import TensorMap, normal_fill, select_truncation

U1R, SU2R = Rule([U1]), Rule([SU2])
X = Leg.new(U1R, [((0,), 5), ((1,), 4)])
Y = Leg.new(U1R, [((0,), 6), ((1,), 9), ((2,), 3)])
W = Leg.new(SU2R, [((0,), 3), ((1,), 4), ((2,), 3)])
P = Leg.new(SU2R, [((1,), 1)])


def symmetric(rule, legs, seed):
    sp = HomSpace(rule, legs, legs)
    a = TensorMap(sp, normal_fill(seed, sp.size))
    return TensorMap(sp, a.data + a.adjoint().data)


@pytest.mark.parametrize("cod,dom", [([X, X], [Y]), ([Y], [X, X]), ([W, P], [P, W])])
def test_qr_reconstructs_with_positive_diagonal(cod, dom):
    rule = cod[0].rule
    sp = HomSpace(rule, cod, dom)
    t = TensorMap(sp, normal_fill(3, sp.size))
    for i, (c, q, r) in enumerate(t.qr_compact()):
        a = sp.sector_matrix(t.data, i)
        k = min(a.shape)
        assert q.shape == (a.shape[0], k) and r.shape == (k, a.shape[1])
        np.testing.assert_allclose(q @ r, a, atol=1e-12 * np.linalg.norm(a))
        np.testing.assert_allclose(q.T @ q, np.eye(k), atol=1e-12)
        assert np.all(np.diag(r) >= 0)
        assert np.allclose(np.tril(r, -1), 0)


@pytest.mark.parametrize("rule,legs", [(U1R, [X, X]), (SU2R, [W, P])])
def test_eigh_order_gauge_and_reconstruction(rule, legs):
    t = symmetric(rule, legs, 11)
    for i, (c, w, v) in enumerate(t.eigh_full()):
        a = t.space.sector_matrix(t.data, i)
        np.testing.assert_allclose(v @ np.diag(w) @ v.T, a, atol=1e-12 * np.linalg.norm(a))
        assert np.all(np.diff(np.abs(w)) <= 0)
        for j in range(v.shape[1]):
            k = int(np.argmax(np.abs(v[:, j])))
            assert v[k, j] > 0


def test_eigh_tie_order_keeps_ascending_values():
    # |w| ties: -2 and +2 keep LAPACK's ascending order (-2 first).
    sp = HomSpace(U1R, [Leg.new(U1R, [((0,), 3)])], [Leg.new(U1R, [((0,), 3)])])
    t = TensorMap(sp, np.diag([2.0, -2.0, 1.0]).T.ravel())
    (_, w, _), = t.eigh_full()
    assert list(w) == [-2.0, 2.0, 1.0]


def test_eigh_rejects_non_hermitian_and_non_endomorphism():
    sp = HomSpace(U1R, [X], [X])
    with pytest.raises(ValueError, match="Hermitian"):
        TensorMap(sp, normal_fill(1, sp.size)).eigh_full()
    sp2 = HomSpace(U1R, [X, X], [Y])
    with pytest.raises(ValueError, match="endomorphism"):
        TensorMap(sp2, normal_fill(1, sp2.size)).eigh_full()


@pytest.mark.parametrize("trunc", [("rank", 9), ("tol", 0.0, 0.4), ("discard", 0.3), ("full",)])
def test_eigh_trunc_selects_on_magnitudes(trunc):
    t = symmetric(SU2R, [W, P], 12)
    parts = t.eigh_full()
    kept_ref, err_ref = select_truncation([(c, t.rule.dim(c), np.abs(w)) for c, w, _ in parts], trunc)
    out, kept, err = t.eigh_trunc(trunc)
    assert kept == kept_ref and err == err_ref
    for (c, w, v), k in zip(out, kept):
        assert len(w) == k and v.shape[1] == k
