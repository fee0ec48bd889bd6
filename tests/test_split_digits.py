"""The digit schemes of the split-precision packing, restated on the CPU.

``csrc/gemm_split.cu`` cuts each scaled value x' in (-1, 1) into S digits of
one rounded integer.

* BF16 slices: X = rint(x' 2^{7S}), balanced base-128 digits,
  Y = X + 64 (1 + 128 + ... + 128^{S-1}), d_0 = floor(Y / 128^{S-1}) - 64,
  d_s = (floor(Y / 128^{S-1-s}) mod 128) - 64.
* int8 digits: X = rint(x' 2^{8S-2}), balanced base-256 digits,
  d_0 in [-64, 64] and d_s in [-128, 127], read off the bit pattern of
  x' 2^{8S-2} + 1.5 2^52 + C (``tests.split_restate``).

Checked here with exact integer arithmetic: the digits reproduce X, stay in
their int8 / BF16-exact ranges, and the represented value is within half a
unit of the last digit of x'.
"""

import numpy as np
import pytest


def digits(xp, S, shift):
    X = np.rint(np.ldexp(xp, shift)).astype(np.int64)
    C = 0
    for _ in range(S):
        C = C * 128 + 64
    Y = X + C
    out = []
    for s in range(S):
        sh = 7 * (S - 1 - s)
        u = Y >> sh  # arithmetic shift: floor division
        out.append((u if s == 0 else (u & 127)) - 64)
    return X, out


@pytest.mark.parametrize("S", [1, 2, 3, 5, 6, 8])
def test_bf16_balanced_digits_reproduce_the_rounded_integer(S):
    rng = np.random.default_rng(S)
    xp = np.concatenate([rng.uniform(-1, 1, 20000), [0.0, -0.0, 1 - 2.0 ** -53, -(1 - 2.0 ** -53), 0.5, -0.5]])
    shift = 7 * S
    X, d = digits(xp, S, shift)
    acc = np.zeros_like(X)
    for s in range(S):
        acc = acc * 128 + d[s]
    assert np.array_equal(acc, X)
    assert d[0].min() >= -128 and d[0].max() <= 128
    for s in range(1, S):
        assert d[s].min() >= -64 and d[s].max() <= 63
    # one rounding: within half a unit of the last digit
    err = np.abs(np.ldexp(X.astype(np.float64), -shift) - xp)
    assert err.max() <= 2.0 ** -(shift + 1)


def _edge_values(rng):
    edge = [0.0, -0.0, 1 - 2.0 ** -53, -(1 - 2.0 ** -53), 0.5, -0.5, 2.0 ** -60, -(2.0 ** -60), 0.25 - 2.0 ** -40]
    return np.concatenate([rng.uniform(-1, 1, 20000), rng.uniform(-1e-3, 1e-3, 2000), edge])


@pytest.mark.parametrize("S", [1, 2, 3, 4, 5, 6])
def test_int8_digits_reproduce_the_rounded_integer(S):
    from tests.split_restate import digits8

    xp = _edge_values(np.random.default_rng(100 + S))
    X, d = digits8(xp, S)
    acc = np.zeros_like(X)
    for s in range(S):
        acc = acc * 256 + d[s]
    assert np.array_equal(acc, X)
    assert d[0].min() >= -64 and d[0].max() <= 64
    for s in range(1, S):
        assert d[s].min() >= -128 and d[s].max() <= 127
    err = np.abs(np.ldexp(X.astype(np.float64), -(8 * S - 2)) - xp)
    assert err.max() <= 2.0 ** -(8 * S - 1)


@pytest.mark.parametrize("S", [1, 2, 3, 4, 5, 6])
def test_int8_digits_from_the_bit_pattern_match(S):
    """The device reads the digits off the bytes of one FMA result; the same
    bytes give the same digits as the integer cut, edge values included."""
    from tests.split_restate import digits8, digits8_from_bits

    xp = _edge_values(np.random.default_rng(200 + S))
    _, d = digits8(xp, S)
    e = digits8_from_bits(xp, S)
    for s in range(S):
        assert np.array_equal(d[s], e[s]), s


def test_bf16_slices_are_exact():
    """q * 2^{-7s} with |q| <= 128 has at most 8 significant bits: exact in BF16."""
    for q in range(-128, 129):
        for s in range(8):
            v = np.float32(q) * np.float32(2.0 ** (-7 * s))
            bits = np.array([v], dtype=np.float32).view(np.uint32)[0]
            assert bits & 0xFFFF == 0  # the low 16 bits a BF16 drops are zero


def _split_product(a, b, S):
    """The int8-digit product of the device kernel (tests.split_restate)."""
    from tests.split_restate import split_product_i8

    return split_product_i8(a, b, S)


@pytest.mark.parametrize("S", [3, 4, 5, 6])
def test_split_product_meets_the_documented_error_bound(S):
    """Relative Frobenius error below 4 (S + 1) 2^{2-8S} (dropped diagonals
    d >= S and one rounding per operand); 8.7e-11 at S = 5."""
    rng = np.random.default_rng(7 + S)
    a, b = rng.standard_normal((24, 40)), rng.standard_normal((40, 16))
    ref = a @ b
    got = _split_product(a, b, S)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= 4 * (S + 1) * 2.0 ** (2 - 8 * S)


def test_split_product_scales_rows_and_columns_independently():
    """Rows of very different magnitude (and zero rows) keep their own relative accuracy."""
    rng = np.random.default_rng(3)
    a = rng.standard_normal((6, 30)) * np.array([1e-200, 1.0, 1e150, 0.0, 3.0, 1e-5])[:, None]
    b = rng.standard_normal((30, 5))
    ref = a @ b
    got = _split_product(a, b, 5)
    for r in range(6):
        den = max(np.linalg.norm(ref[r]), 1e-300)
        assert np.linalg.norm(got[r] - ref[r]) <= 4 * 6 * 2.0 ** -38 * max(den, np.linalg.norm(a[r]) * np.linalg.norm(b))


def test_split_product_long_k_is_chunked_exactly():
    """K beyond one 16384-deep chunk: the chunks are recombined in FP64."""
    rng = np.random.default_rng(11)
    a, b = rng.standard_normal((3, 16400)), rng.standard_normal((16400, 2))
    got = _split_product(a, b, 5)
    ref = a @ b
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 4 * 6 * 2.0 ** -38


def test_restated_compose_over_a_plan_meets_the_bound():
    """The restated int8-digit compose over a real plan's job table (the
    device's bit-exact reference in the GPU tests) is within the bound of the
    oracle's FP64 compose for every digit count."""
    from oracle.fusion import HomSpace as OHom
    from oracle.fusion import Leg
    from oracle.sectors import FZ2, SU2, U1, Rule
    from oracle.tensor import TensorMap as OT
    from oracle.tensor import normal_fill
    from tenet_b200.typed import ComposePlan
    from tests.helpers import product_space
    from tests.split_restate import replay_compose_i8

    I3 = Rule([FZ2, U1, SU2])
    V = Leg.new(I3, [((0, 0, 0), 3), ((1, 1, 1), 2), ((0, 2, 0), 2), ((1, -1, 1), 2), ((0, 0, 2), 1)])
    P = Leg.new(I3, [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)])
    a_sp, b_sp = OHom(I3, [V, P], [P, V]), OHom(I3, [P, V], [V, P])
    a, b = OT(a_sp, normal_fill(131, a_sp.size)), OT(b_sp, normal_fill(132, b_sp.size))
    ref = a.compose(b).data
    plan = ComposePlan(product_space(I3, [V, P], [P, V]), product_space(I3, [P, V], [V, P]))
    for S in range(1, 7):
        got = replay_compose_i8(plan.export(), a.data, b.data, plan.dst.size, S)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 4 * (S + 1) * 2.0 ** (2 - 8 * S), S
