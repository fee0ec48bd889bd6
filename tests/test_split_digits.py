"""The digit scheme of the split-precision packing, restated on the CPU.

``csrc/gemm_split.cu`` cuts each scaled value x' in (-1, 1) into S balanced
base-128 digits of one rounded integer: X = rint(x' 2^{6 + 7(S-1)}) for int8
digits (X = rint(x' 2^{7S}) for BF16 slices), Y = X + 64 (1 + 128 + ... +
128^{S-1}), d_0 = floor(Y / 128^{S-1}) - 64, d_s = (floor(Y / 128^{S-1-s})
mod 128) - 64.  Checked here with exact integer arithmetic: the digits
reproduce X, stay in their int8 / BF16-exact ranges, and the represented
value is within half a unit of the last digit of x'.
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
@pytest.mark.parametrize("kind", ["int8", "bf16"])
def test_balanced_digits_reproduce_the_rounded_integer(S, kind):
    rng = np.random.default_rng(S)
    xp = np.concatenate([rng.uniform(-1, 1, 20000), [0.0, -0.0, 1 - 2.0 ** -53, -(1 - 2.0 ** -53), 0.5, -0.5]])
    shift = 6 + 7 * (S - 1) if kind == "int8" else 7 * S
    X, d = digits(xp, S, shift)
    acc = np.zeros_like(X)
    for s in range(S):
        acc = acc * 128 + d[s]
    assert np.array_equal(acc, X)
    lo0 = -64 if kind == "int8" else -128
    hi0 = 64 if kind == "int8" else 128
    assert d[0].min() >= lo0 and d[0].max() <= hi0
    for s in range(1, S):
        assert d[s].min() >= -64 and d[s].max() <= 63
    # one rounding: within half a unit of the last digit
    err = np.abs(np.ldexp(X.astype(np.float64), -shift) - xp)
    assert err.max() <= 2.0 ** -(shift + 1)


def test_bf16_slices_are_exact():
    """q * 2^{-7s} with |q| <= 128 has at most 8 significant bits: exact in BF16."""
    for q in range(-128, 129):
        for s in range(8):
            v = np.float32(q) * np.float32(2.0 ** (-7 * s))
            bits = np.array([v], dtype=np.float32).view(np.uint32)[0]
            assert bits & 0xFFFF == 0  # the low 16 bits a BF16 drops are zero


def _split_product(a, b, S):
    """The int8-digit product of the device kernel, restated exactly: rows of
    A and columns of B scaled by powers of two below 1, cut into S digits,
    digit products summed per diagonal d = s + t < S in exact integers, the
    diagonals weighted by 2^{-7d}, times 2^{-12} sigma tau."""
    shift = 6 + 7 * (S - 1)

    def scale(m, axis):
        amax = np.abs(m).max(axis=axis, keepdims=True)
        e = np.where(amax > 0, np.frexp(np.where(amax > 0, amax, 1.0))[1], 0)
        return np.ldexp(1.0, e)

    sa, sb = scale(a, 1), scale(b, 0)
    _, da = digits(a / sa, S, shift)
    _, db = digits(b / sb, S, shift)
    acc = np.zeros((a.shape[0], b.shape[1]))
    for dg in range(S):
        diag = sum((da[s].astype(object) @ db[dg - s].astype(object)) for s in range(dg + 1))
        acc += np.ldexp(np.asarray(diag, dtype=np.float64), -7 * dg)
    return acc * 2.0 ** -12 * sa * sb


@pytest.mark.parametrize("S", [3, 5, 6])
def test_split_product_meets_the_documented_error_bound(S):
    """Relative Frobenius error below about (S + 1) 2^{-7S} (dropped diagonals d >= S)."""
    rng = np.random.default_rng(7 + S)
    a, b = rng.standard_normal((24, 40)), rng.standard_normal((40, 16))
    ref = a @ b
    got = _split_product(a, b, S)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= 4 * (S + 1) * 2.0 ** (-7 * S)
