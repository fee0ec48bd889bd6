"""SU(2) effective-Hamiltonian network and device Lanczos.

* the network B x on a reduced configuration (degeneracies / 32) matches the
  oracle's contraction network to 1e-12 relative;
* B^dagger is the adjoint of B under the weighted inner product;
* Lanczos with BF16-split contractions reproduces the FP64 ground energy and
  Ritz vector within the error the slice count allows.
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, Rule
from oracle.tensor import TensorMap as OT

pytestmark = pytest.mark.gpu

SCALE = 32


@pytest.fixture(scope="module")
def setup():
    import tenet_b200 as tb
    from tenet_b200 import heff, workloads

    rt = tb.Runtime(0)
    cfg = workloads.su2_heff()
    rule, x, L, O, R = heff.workload_tensors(rt, cfg, scale=SCALE)
    return rt, cfg, x, L, O, R, heff.EffectiveHamiltonian(L, O, R)


def oracle_b(cfg, x, L, O, R):
    r = Rule([SU2])
    W = Leg.new(r, [(s, max(1, d // SCALE)) for s, d in cfg["W"]])
    M = Leg.new(r, cfg["M"])
    P = Leg.new(r, cfg["P"])
    ox = OT(OHom(r, [W, P], [W]), x.to_host())
    oL = OT(OHom(r, [W, M], [W]), L.to_host())
    oO = OT(OHom(r, [M, P], [P, M]), O.to_host())
    oR = OT(OHom(r, [W, M.dual()], [W]), R.to_host())
    t1 = oL.compose(ox.permute([0], [1, 2]))
    t2 = t1.permute([0, 3], [1, 2]).compose(oO.permute([3, 2], [0, 1]))
    return t2.permute([0, 3], [1, 2]).compose(oR)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_network_matches_oracle(setup):
    rt, cfg, x, L, O, R, H = setup
    ref = oracle_b(cfg, x, L, O, R)
    got = H.apply_b(x, "fp64", 0)
    assert got.space.block_keys() == [b["key"] for b in ref.space.blocks]
    assert rel(got.to_host(), ref.data) <= 1e-12


def test_bdag_is_the_adjoint(setup):
    import tenet_b200 as tb
    from tenet_b200.workloads import splitmix_normal

    rt, cfg, x, L, O, R, H = setup
    y = tb.TensorMap(rt, x.space, tb.typed.torch().as_tensor(splitmix_normal(99, x.space.size), device="cuda"))
    bx = H.apply_b(x, "fp64", 0)
    bty = H.apply_bdag(y, "fp64", 0)

    def wip(a, b):
        s = 0.0
        for lab, r, c, off in a.space.sectors():
            s += a.rule.dim(a.rule.unlabel(lab)) * float(a.data[off:off + r * c].dot(b.data[off:off + r * c]))
        return s

    lhs, rhs = wip(bx, y), wip(x, bty)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_lanczos_split_vs_fp64(setup):
    from tenet_b200 import heff

    rt, cfg, x, L, O, R, H = setup
    e64, v64, a64, b64 = heff.lanczos(H, x, 12, "fp64", 0)
    assert all(b > 0 for b in b64)
    for slices, tol in ((5, 1e-7), (7, 1e-9)):
        e, v, _, _ = heff.lanczos(H, x, 12, "bf16x", slices)
        assert abs(e - e64) <= tol * abs(e64), (slices, e, e64)
        d = v.to_host() - v64.to_host()
        d2 = v.to_host() + v64.to_host()
        err = min(np.linalg.norm(d), np.linalg.norm(d2)) / np.linalg.norm(v64.to_host())
        assert err <= 1e3 * tol, (slices, err)
