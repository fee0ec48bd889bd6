"""The benchmark configurations at full size, held to the path's tolerances.

* hubbard_batch: the whole 64-compose batch of the headline step; every
  split-precision path the benchmark reports as meeting the bar (BF16 slices
  at 5 and 6, 8-bit digits at 5 and 6) is within 1e-10 relative Frobenius
  error of the grouped FP64 result, and the 4-digit path, which the benchmark
  lists but does not claim, is not.
* su2_heff: B x with x of 7.4 M and L, R of 17.9 M elements against the
  oracle's contraction network to 1e-12; then 30 Lanczos iterations of
  H = B^dagger B with the contractions split into BF16 slices k = 3, 5, 7
  (and 8-bit digits at 5) against the FP64 run: ground energy within the
  error the slice count allows (1e-10 from k = 5 on), Ritz vector within a
  looser bound (a Krylov basis amplifies per-product errors).
"""

import ctypes as C

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import SU2, Rule
from oracle.tensor import TensorMap as OT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_hubbard_batch_split_paths_within_1e10(rt):
    import torch

    import tenet_b200 as tb
    from tenet_b200 import _lib
    from tenet_b200.workloads import hubbard_batch, splitmix_normal

    cfg = hubbard_batch(0)
    rule = tb.FusionRule(cfg["factors"])
    W, P = tb.GradedSpace(rule, cfg["W"]), tb.GradedSpace(rule, cfg["P"])
    a_sp, b_sp = rt.space(rule, [W, P], [P, W]), rt.space(rule, [P, W], [W, P])
    plan = rt.cplan(a_sp, b_sp)
    nb = 64
    ga = torch.empty(nb * a_sp.size, dtype=torch.float64, device="cuda")
    gb = torch.empty(nb * b_sp.size, dtype=torch.float64, device="cuda")
    for i in range(nb):  # the benchmark's inputs: seeds 1 + i (A) and 5001 + i (B)
        ga[i * a_sp.size:(i + 1) * a_sp.size] = torch.from_numpy(splitmix_normal(1 + i, a_sp.size))
        gb[i * b_sp.size:(i + 1) * b_sp.size] = torch.from_numpy(splitmix_normal(5001 + i, b_sp.size))

    def compose(prec, slices):
        out = torch.empty(nb * plan.dst.size, dtype=torch.float64, device="cuda")
        _lib.call("tnt_compose", rt._h, plan._h, nb, C.c_void_p(out.data_ptr()), plan.dst.size,
                  C.c_void_p(ga.data_ptr()), a_sp.size, C.c_void_p(gb.data_ptr()), b_sp.size, 1.0, 0.0, prec,
                  slices, rt.stream())
        rt.sync()
        return out

    ref = compose(_lib.PREC_FP64, 0)
    nref = float(torch.linalg.norm(ref))
    errs = {}
    for name, prec, slices in (("bf16x5", _lib.PREC_BF16X, 5), ("bf16x6", _lib.PREC_BF16X, 6),
                               ("i8x5", _lib.PREC_INT8X, 5), ("i8x6", _lib.PREC_INT8X, 6),
                               ("i8x4", _lib.PREC_INT8X, 4)):
        out = compose(prec, slices)
        errs[name] = float(torch.linalg.norm(out - ref)) / nref
        del out
    print("full 64-compose batch, rel. error vs FP64:", {k: f"{v:.2e}" for k, v in errs.items()})
    for name in ("bf16x5", "bf16x6", "i8x5", "i8x6"):
        assert errs[name] <= 1e-10, (name, errs[name])
    assert errs["i8x4"] > 1e-10  # listed, never claimed


@pytest.fixture(scope="module")
def heff(rt):
    from tenet_b200 import heff as H
    from tenet_b200 import workloads

    cfg = workloads.su2_heff()
    rule, x, L, O, R = H.workload_tensors(rt, cfg, scale=1)
    return cfg, x, L, O, R, H.EffectiveHamiltonian(L, O, R)


def test_heff_full_size_b_matches_oracle(heff):
    cfg, x, L, O, R, H = heff
    r = Rule([SU2])
    W, M, P = Leg.new(r, cfg["W"]), Leg.new(r, cfg["M"]), Leg.new(r, cfg["P"])
    ox = OT(OHom(r, [W, P], [W]), x.to_host())
    oL = OT(OHom(r, [W, M], [W]), L.to_host())
    oO = OT(OHom(r, [M, P], [P, M]), O.to_host())
    oR = OT(OHom(r, [W, M.dual()], [W]), R.to_host())
    t1 = oL.compose(ox.permute([0], [1, 2]))
    t2 = t1.permute([0, 3], [1, 2]).compose(oO.permute([3, 2], [0, 1]))
    ref = t2.permute([0, 3], [1, 2]).compose(oR)
    got = H.apply_b(x, "fp64", 0)
    assert got.space.block_keys() == [b["key"] for b in ref.space.blocks]
    assert rel(got.to_host(), ref.data) <= 1e-12


def test_heff_full_size_split_lanczos(heff):
    from tenet_b200 import heff as Hmod

    cfg, x, L, O, R, H = heff
    e64, v64, _, _ = Hmod.lanczos(H, x, 30, "fp64", 0)
    v64h = v64.to_host()
    report = {}
    for precision, k, e_tol, v_tol in (("bf16x", 3, 1e-5, 1e-2), ("bf16x", 5, 1e-10, 1e-6),
                                       ("bf16x", 7, 1e-10, 1e-6), ("i8x", 5, 1e-10, 1e-6)):
        e, v, _, _ = Hmod.lanczos(H, x, 30, precision, k)
        vh = v.to_host()
        e_err = abs(e - e64) / abs(e64)
        v_err = min(np.linalg.norm(vh - v64h), np.linalg.norm(vh + v64h)) / np.linalg.norm(v64h)
        report[f"{precision}{k}"] = (e_err, v_err)
        assert e_err <= e_tol, (precision, k, e_err)
        assert v_err <= v_tol, (precision, k, v_err)
    print("config 4, 30 Lanczos iterations, (energy, vector) rel. error vs FP64:",
          {n: f"{a:.1e}, {b:.1e}" for n, (a, b) in report.items()})
