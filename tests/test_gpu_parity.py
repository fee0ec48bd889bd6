"""GPU parity: device kernels through the C ABI vs the CPU oracle.

Tolerances: payloads within 1e-12 relative Frobenius error for the FP64
paths (the reference's plain-FP64 bar); singular values within 1e-12
relative; block keys and offsets bit-exact (checked on the CPU in
test_host_structure.py and re-checked here on device-built spaces).
"""

import numpy as np
import pytest

from oracle.fusion import HomSpace as OHom
from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from oracle.tensor import TensorMap as OT
from oracle.tensor import normal_fill, select_truncation
from tests.helpers import product_leg, product_rule

pytestmark = pytest.mark.gpu

U1R, SU2R, I3 = Rule([U1]), Rule([SU2]), Rule([FZ2, U1, SU2])
V_U1 = Leg.new(U1R, [((-2,), 4), ((-1,), 8), ((0,), 12), ((1,), 8), ((2,), 4)])
W_SU2 = Leg.new(SU2R, [((0,), 4), ((1,), 6), ((2,), 6), ((3,), 4), ((4,), 2)])
P_SU2 = Leg.new(SU2R, [((1,), 1)])
V_I3 = Leg.new(I3, [((0, 0, 0), 3), ((1, 1, 1), 2), ((0, 2, 0), 2), ((1, -1, 1), 2), ((0, 0, 2), 1)])
P_I3 = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


def device_tensor(rt, orule, ocod, odom, data):
    from tenet_b200 import typed

    rule = product_rule(orule)
    cod = [product_leg(rule, l) for l in ocod]
    dom = [product_leg(rule, l) for l in odom]
    return typed.TensorMap.from_host(rt, cod, dom, data)


CASES = [
    ("u1", U1R, [V_U1, V_U1], [V_U1, V_U1], [0, 3], [2, 1]),
    ("u1_swap", U1R, [V_U1, V_U1], [V_U1, V_U1], [1, 0], [3, 2]),
    ("su2_4", SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2], [0, 3], [2, 1]),
    ("su2_31", SU2R, [W_SU2, P_SU2, P_SU2], [W_SU2], [0, 1], [2, 3]),
    ("su2_31b", SU2R, [W_SU2, P_SU2, P_SU2], [W_SU2], [3, 1], [0, 2]),
    ("i3", I3, [V_I3, P_I3], [P_I3, V_I3], [0, 3], [2, 1]),
]


@pytest.mark.parametrize("name,rule,cod,dom,p1,p2", CASES)
def test_transform_matches_oracle(rt, name, rule, cod, dom, p1, p2):
    sp = OHom(rule, cod, dom)
    src = OT(sp, normal_fill(1, sp.size))
    ref = src.permute(p1, p2)
    t = device_tensor(rt, rule, cod, dom, src.data)
    out = t.permute(p1, p2)
    assert out.space.block_keys() == [b["key"] for b in ref.space.blocks]
    assert rel(out.to_host(), ref.data) <= 1e-12


def test_transform_alpha_beta_accumulate(rt):
    import ctypes as C

    from tenet_b200 import _lib

    sp = OHom(SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2])
    src = OT(sp, normal_fill(3, sp.size))
    ref = src.permute([0, 3], [2, 1])
    t = device_tensor(rt, SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2], src.data)
    plan = rt.xplan(t.space, "permute", [0, 3], [2, 1])
    import torch

    prior = torch.as_tensor(normal_fill(4, plan.dst.size), device="cuda")
    dst = prior.clone()
    _lib.call("tnt_transform", rt._h, plan._h, C.c_void_p(dst.data_ptr()), C.c_void_p(t.data.data_ptr()), 0.5, -2.0,
              rt.stream())
    expect = 0.5 * ref.data - 2.0 * prior.cpu().numpy()
    assert rel(dst.cpu().numpy(), expect) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "cublas"])
@pytest.mark.parametrize("name,rule,cod,dom", [
    ("u1", U1R, [V_U1, V_U1], [V_U1, V_U1]),
    ("su2", SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2]),
    ("i3", I3, [V_I3, P_I3], [P_I3, V_I3]),
])
def test_compose_matches_oracle(rt, precision, name, rule, cod, dom):
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    a = OT(a_sp, normal_fill(1, a_sp.size))
    b = OT(b_sp, normal_fill(2, b_sp.size))
    ref = a.compose(b)
    da = device_tensor(rt, rule, cod, dom, a.data)
    db = device_tensor(rt, rule, dom, cod, b.data)
    out = da.compose(db, precision=precision)
    assert rel(out.to_host(), ref.data) <= 1e-12


def test_compose_batched_and_host_entry_point(rt):
    """nbatch operand triples in one launch, and the host-buffer entry point."""
    import ctypes as C

    import torch

    from tenet_b200 import _lib

    rule, cod, dom = I3, [V_I3, P_I3], [P_I3, V_I3]
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    nb = 5
    A = [OT(a_sp, normal_fill(10 + i, a_sp.size)) for i in range(nb)]
    B = [OT(b_sp, normal_fill(20 + i, b_sp.size)) for i in range(nb)]
    ref = np.concatenate([x.compose(y).data for x, y in zip(A, B)])
    da = device_tensor(rt, rule, cod, dom, A[0].data)
    db = device_tensor(rt, rule, dom, cod, B[0].data)
    plan = rt.cplan(da.space, db.space)
    ga = torch.as_tensor(np.concatenate([x.data for x in A]), device="cuda")
    gb = torch.as_tensor(np.concatenate([x.data for x in B]), device="cuda")
    gc = torch.zeros(nb * plan.dst.size, dtype=torch.float64, device="cuda")
    _lib.call("tnt_compose", rt._h, plan._h, nb, C.c_void_p(gc.data_ptr()), plan.dst.size,
              C.c_void_p(ga.data_ptr()), a_sp.size, C.c_void_p(gb.data_ptr()), b_sp.size, 1.0, 0.0,
              _lib.PREC_FP64, 0, rt.stream())
    assert rel(gc.cpu().numpy(), ref) <= 1e-12
    ha = np.concatenate([x.data for x in A])
    hb = np.concatenate([x.data for x in B])
    hc = np.zeros(nb * plan.dst.size)
    P = lambda x: x.ctypes.data_as(C.c_void_p)
    _lib.call("tnt_compose_host", rt._h, plan._h, nb, P(hc), P(ha), P(hb), _lib.PREC_FP64, 0, rt.stream())
    assert rel(hc, ref) <= 1e-12
    # the host-buffer entry point with split precision (takes the context's
    # scratch while holding its staging buffer)
    hc[:] = 0.0
    _lib.call("tnt_compose_host", rt._h, plan._h, nb, P(hc), P(ha), P(hb), _lib.PREC_BF16X, 6, rt.stream())
    assert rel(hc, ref) <= 4 * 7 * 2.0 ** -42 + 512 * 2.0 ** -45  # the S = 6 split bound
    rt.sync()  # no device-side pipeline timeout was recorded
    # 11 entries: the pipeline's 8 chunks hold one or two entries each
    n11 = 11
    ha11 = np.concatenate([ha] * 3)[: n11 * a_sp.size]
    hb11 = np.concatenate([hb] * 3)[: n11 * b_sp.size]
    hc11 = np.full(n11 * plan.dst.size, np.nan)
    _lib.call("tnt_compose_host", rt._h, plan._h, n11, P(hc11), P(ha11), P(hb11), _lib.PREC_FP64, 0, rt.stream())
    ref11 = np.concatenate([ref] * 3)[: n11 * plan.dst.size]
    assert rel(hc11, ref11) <= 1e-12


def test_svd_matches_oracle_and_gauge(rt):
    rule, cod, dom = SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2]
    sp = OHom(rule, cod, dom)
    src = OT(sp, normal_fill(5, sp.size))
    parts = src.svd_compact()
    t = device_tensor(rt, rule, cod, dom, src.data)
    res = t.svd_compact()
    U, spectra, Vh = res.factors()
    for (c, u, s, vh), ent in zip(parts, spectra):
        np.testing.assert_allclose(ent.values, s, rtol=1e-12, atol=1e-12 * s[0])
    # U and Vh blocks per sector against the oracle (non-degenerate spectra)
    usec = {lab: (r, c, off) for lab, r, c, off in U.space.sectors()}
    vsec = {lab: (r, c, off) for lab, r, c, off in Vh.space.sectors()}
    uh, vhh = U.to_host(), Vh.to_host()
    for c, u, s, vh in parts:
        r, k, off = usec[c]
        np.testing.assert_allclose(uh[off:off + r * k].reshape(k, r).T, u, atol=1e-11)
        kr, n, off = vsec[c]
        np.testing.assert_allclose(vhh[off:off + kr * n].reshape(n, kr).T, vh, atol=1e-11)


@pytest.mark.parametrize("trunc", [("rank", 40), ("rank", 7), ("tol", 0.0, 0.3), ("discard", 0.4), ("full",)])
def test_truncation_matches_oracle(rt, trunc):
    from tenet_b200 import Truncation

    rule, cod, dom = SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2]
    sp = OHom(rule, cod, dom)
    src = OT(sp, normal_fill(6, sp.size))
    _, kept, err = src.svd_trunc(trunc)
    t = device_tensor(rt, rule, cod, dom, src.data)
    pol = {
        "rank": lambda: Truncation.rank(trunc[1]),
        "tol": lambda: Truncation.tolerance(trunc[1], trunc[2]),
        "discard": lambda: Truncation.discard_weight(trunc[1]),
        "full": Truncation.full,
    }[trunc[0]]()
    res = t.svd_trunc(pol)
    assert res.kept == kept
    assert abs(res.error - err) <= 1e-10 * max(1.0, err)


def test_space_truncation(rt):
    from tenet_b200 import Truncation

    rule, cod, dom = SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2]
    sp = OHom(rule, cod, dom)
    src = OT(sp, normal_fill(7, sp.size))
    prof = {(0,): 3, (1,): 2, (2,): 100}
    _, kept, err = src.svd_trunc(("space", prof))
    res = device_tensor(rt, rule, cod, dom, src.data).svd_trunc(Truncation.space(prof))
    assert res.kept == kept
    assert abs(res.error - err) <= 1e-10 * max(1.0, err)


SPLIT_CASES = [
    ("i3", I3, [V_I3, P_I3], [P_I3, V_I3]),
    ("su2", SU2R, [W_SU2, P_SU2], [P_SU2, W_SU2]),
    ("u1", U1R, [V_U1, V_U1], [V_U1, V_U1]),
]


@pytest.mark.parametrize("slices", [3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("name,rule,cod,dom", SPLIT_CASES)
def test_split_precision_compose_error_per_slice_count(rt, slices, name, rule, cod, dom):
    """BF16-split compose: relative Frobenius error vs the FP64 oracle within
    4 (S+1) 2^{-7S} (the dropped-diagonal bound of the slice scheme) plus a
    512 * 2^-45 ~ 1.5e-11 floor (FP32 accumulation of the shared accumulator of
    diagonals >= 3 over one 512-deep K chunk)."""
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    a = OT(a_sp, normal_fill(31, a_sp.size))
    b = OT(b_sp, normal_fill(32, b_sp.size))
    ref = a.compose(b)
    da = device_tensor(rt, rule, cod, dom, a.data)
    db = device_tensor(rt, rule, dom, cod, b.data)
    out = da.compose(db, precision="bf16x", slices=slices)
    err = rel(out.to_host(), ref.data)
    bound = 4 * (slices + 1) * 2.0 ** (-7 * slices) + 512 * 2.0 ** -45
    print(f"split S={slices} {name}: rel err {err:.3e} (bound {bound:.3e})")
    assert err <= bound


def test_split_precision_large_k_chunks(rt):
    """K > 512 exercises the chunked exact accumulation (several TMEM drains)."""
    rule = U1R
    v = Leg.new(rule, [((0,), 700), ((1,), 300)])
    a_sp = OHom(rule, [v], [v])
    a = OT(a_sp, normal_fill(41, a_sp.size))
    b = OT(a_sp, normal_fill(42, a_sp.size))
    ref = a.compose(b)
    da = device_tensor(rt, rule, [v], [v], a.data)
    db = device_tensor(rt, rule, [v], [v], b.data)
    for slices in (6, 7):
        out = da.compose(db, precision="bf16x", slices=slices)
        err = rel(out.to_host(), ref.data)
        assert err <= 4 * (slices + 1) * 2.0 ** (-7 * slices) + 512 * 2.0 ** -45, (slices, err)


def test_split_precision_batched_matches_fp64(rt):
    import ctypes as C

    import torch

    from tenet_b200 import _lib

    rule, cod, dom = I3, [V_I3, P_I3], [P_I3, V_I3]
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    nb = 7
    A = [OT(a_sp, normal_fill(50 + i, a_sp.size)) for i in range(nb)]
    B = [OT(b_sp, normal_fill(70 + i, b_sp.size)) for i in range(nb)]
    ref = np.concatenate([x.compose(y).data for x, y in zip(A, B)])
    da = device_tensor(rt, rule, cod, dom, A[0].data)
    db = device_tensor(rt, rule, dom, cod, B[0].data)
    plan = rt.cplan(da.space, db.space)
    ga = torch.as_tensor(np.concatenate([x.data for x in A]), device="cuda")
    gb = torch.as_tensor(np.concatenate([x.data for x in B]), device="cuda")
    gc = torch.full((nb * plan.dst.size,), 3.0, dtype=torch.float64, device="cuda")
    _lib.call("tnt_compose", rt._h, plan._h, nb, C.c_void_p(gc.data_ptr()), plan.dst.size,
              C.c_void_p(ga.data_ptr()), a_sp.size, C.c_void_p(gb.data_ptr()), b_sp.size, 2.0, -1.0,
              _lib.PREC_BF16X, 6, rt.stream())
    expect = 2.0 * ref - 3.0
    assert rel(gc.cpu().numpy(), expect) <= 1e-11


def i8_bound(slices):
    """Dropped diagonals d >= S and one rounding per operand: 4 (S+1) 2^{2-8S};
    the FP64 recombination adds a few ulps (2^-50)."""
    return 4 * (slices + 1) * 2.0 ** (2 - 8 * slices) + 2.0 ** -50


@pytest.mark.parametrize("slices", [3, 4, 5, 6])
@pytest.mark.parametrize("name,rule,cod,dom", SPLIT_CASES)
def test_int8_digit_compose_error_per_slice_count(rt, slices, name, rule, cod, dom):
    """8-bit-digit compose (kind::i8, exact int32 accumulation per product
    diagonal): relative Frobenius error vs the FP64 oracle within i8_bound."""
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    a = OT(a_sp, normal_fill(31, a_sp.size))
    b = OT(b_sp, normal_fill(32, b_sp.size))
    ref = a.compose(b)
    da = device_tensor(rt, rule, cod, dom, a.data)
    db = device_tensor(rt, rule, dom, cod, b.data)
    out = da.compose(db, precision="i8x", slices=slices)
    rt.sync()
    err = rel(out.to_host(), ref.data)
    print(f"int8 S={slices} {name}: rel err {err:.3e} (bound {i8_bound(slices):.3e})")
    assert err <= i8_bound(slices)


@pytest.mark.parametrize("slices", [1, 2, 5, 6])
@pytest.mark.parametrize("name,rule,cod,dom", SPLIT_CASES)
def test_int8_digit_compose_is_bit_exact_to_the_restated_scheme(rt, slices, name, rule, cod, dom):
    """Every digit, integer sum and FP64 recombination step of the device
    product is restated in numpy (tests.split_restate): the payload must agree
    bit for bit, which pins the packing, the stacked MMAs and the epilogue."""
    from tests.split_restate import replay_compose_i8

    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    a = normal_fill(131, a_sp.size)
    b = normal_fill(132, b_sp.size)
    da = device_tensor(rt, rule, cod, dom, a)
    db = device_tensor(rt, rule, dom, cod, b)
    out = da.compose(db, precision="i8x", slices=slices)
    rt.sync()
    plan = rt.cplan(da.space, db.space)
    expect = replay_compose_i8(plan.export(), a, b, plan.dst.size, slices)
    got = out.to_host()
    assert np.array_equal(got, expect), float(np.abs(got - expect).max())


def test_int8_digits_large_k_and_batched_alpha_beta(rt):
    """K = 1000 in one exact chunk, and nbatch entries with alpha/beta."""
    import ctypes as C

    import torch

    from tenet_b200 import _lib

    rule = U1R
    v = Leg.new(rule, [((0,), 700), ((1,), 300)])
    a_sp = OHom(rule, [v], [v])
    nb = 3
    A = [OT(a_sp, normal_fill(81 + i, a_sp.size)) for i in range(nb)]
    B = [OT(a_sp, normal_fill(91 + i, a_sp.size)) for i in range(nb)]
    ref = np.concatenate([x.compose(y).data for x, y in zip(A, B)])
    da = device_tensor(rt, rule, [v], [v], A[0].data)
    plan = rt.cplan(da.space, da.space)
    ga = torch.as_tensor(np.concatenate([x.data for x in A]), device="cuda")
    gb = torch.as_tensor(np.concatenate([x.data for x in B]), device="cuda")
    gc = torch.full((nb * plan.dst.size,), 3.0, dtype=torch.float64, device="cuda")
    _lib.call("tnt_compose", rt._h, plan._h, nb, C.c_void_p(gc.data_ptr()), plan.dst.size,
              C.c_void_p(ga.data_ptr()), a_sp.size, C.c_void_p(gb.data_ptr()), a_sp.size, 2.0, -1.0,
              _lib.PREC_INT8X, 6, rt.stream())
    rt.sync()
    assert rel(gc.cpu().numpy(), 2.0 * ref - 3.0) <= i8_bound(6)


def test_int8_digits_k_beyond_one_exact_chunk(rt):
    """K = 16400 > 16384: two int32 accumulation chunks recombined in FP64,
    bit-exact to the restatement and within the bound of the FP64 product.
    The dropped-diagonal error grows with the square of sigma / rms of the
    rows and columns: over 16400 normal entries the row maximum is about 4.3
    rms, so the power-of-two scale is 8 rms (at most 4 rms for the short rows
    i8_bound is calibrated on), hence the factor 4."""
    from tests.split_restate import replay_compose_i8

    rule = U1R
    w = Leg.new(rule, [((0,), 5), ((1,), 3)])
    v = Leg.new(rule, [((0,), 16400), ((1,), 40)])
    a_sp, b_sp = OHom(rule, [w], [v]), OHom(rule, [v], [w])
    a = OT(a_sp, normal_fill(141, a_sp.size))
    b = OT(b_sp, normal_fill(142, b_sp.size))
    da = device_tensor(rt, rule, [w], [v], a.data)
    db = device_tensor(rt, rule, [v], [w], b.data)
    out = da.compose(db, precision="i8x", slices=5)
    rt.sync()
    got = out.to_host()
    assert rel(got, a.compose(b).data) <= 4 * i8_bound(5)
    plan = rt.cplan(da.space, db.space)
    assert np.array_equal(got, replay_compose_i8(plan.export(), a.data, b.data, plan.dst.size, 5))


def test_int8_digits_refuse_more_than_six(rt):
    from tenet_b200 import _lib

    rule, cod, dom = I3, [V_I3, P_I3], [P_I3, V_I3]
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    da = device_tensor(rt, rule, cod, dom, normal_fill(1, a_sp.size))
    db = device_tensor(rt, rule, dom, cod, normal_fill(2, b_sp.size))
    with pytest.raises(_lib.TenetError):
        da.compose(db, precision="i8x", slices=7)


@pytest.mark.parametrize("precision,slices", [("bf16x", 5), ("i8x", 6)])
def test_compose_with_caller_scratch_matches(rt, precision, slices):
    """tnt_compose_ws (slice packs in a caller buffer of tnt_cplan_scratch_bytes) equals tnt_compose."""
    import ctypes as C

    import torch

    from tenet_b200 import _lib

    rule, cod, dom = I3, [V_I3, P_I3], [P_I3, V_I3]
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    da = device_tensor(rt, rule, cod, dom, normal_fill(61, a_sp.size))
    db = device_tensor(rt, rule, dom, cod, normal_fill(62, b_sp.size))
    plan = rt.cplan(da.space, db.space)
    prec = {"bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X}[precision]
    nb = C.c_size_t()
    _lib.call("tnt_cplan_scratch_bytes", plan._h, 1, prec, slices, C.byref(nb))
    assert nb.value > 0
    scratch = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    ref = da.compose(db, precision=precision, slices=slices)
    out = torch.zeros(plan.dst.size, dtype=torch.float64, device="cuda")
    _lib.call("tnt_compose_ws", rt._h, plan._h, 1, C.c_void_p(out.data_ptr()), plan.dst.size,
              C.c_void_p(da.data.data_ptr()), a_sp.size, C.c_void_p(db.data.data_ptr()), b_sp.size, 1.0, 0.0, prec,
              slices, C.c_void_p(scratch.data_ptr()), nb.value, rt.stream())
    rt.sync()
    assert torch.equal(out, ref.data)
    # a buffer below the stated size is refused
    with pytest.raises(_lib.TenetError):
        _lib.call("tnt_compose_ws", rt._h, plan._h, 1, C.c_void_p(out.data_ptr()), plan.dst.size,
                  C.c_void_p(da.data.data_ptr()), a_sp.size, C.c_void_p(db.data.data_ptr()), b_sp.size, 1.0, 0.0,
                  prec, slices, C.c_void_p(scratch.data_ptr()), 1024, rt.stream())


@pytest.mark.parametrize("side", ["lhs", "rhs", "both"])
def test_packed_operand_compose_is_bit_identical(rt, side):
    """An operand packed once (tnt_split_pack_operand) gives the same bits as
    packing it inside every compose, on either side and on both, twice in a
    row (the packed buffer is only read)."""
    rule, cod, dom = I3, [V_I3, P_I3], [P_I3, V_I3]
    a_sp, b_sp = OHom(rule, cod, dom), OHom(rule, dom, cod)
    da = device_tensor(rt, rule, cod, dom, normal_fill(151, a_sp.size))
    db = device_tensor(rt, rule, dom, cod, normal_fill(152, b_sp.size))
    for slices in (5, 6):
        ref = da.compose(db, precision="i8x", slices=slices)
        pa = da.pack_split(db.space, 0, slices) if side in ("lhs", "both") else da
        pb = db.pack_split(da.space, 1, slices) if side in ("rhs", "both") else db
        for _ in range(2):
            out = type(da).compose_packed(pa, pb, slices)
            rt.sync()
            assert np.array_equal(out.to_host(), ref.to_host())
