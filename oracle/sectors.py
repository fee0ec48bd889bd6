"""Sector labels, SectorId codecs and multiplicity-free symbols (oracle).

Test infrastructure only; see ``oracle/__init__.py``.

A rule is an ordered list of factors (``U1``, ``SU2``, ``FZ2``, ``Z2``).  A
sector label is a tuple with one integer per factor: the U(1) charge, the
doubled SU(2) spin ``2j``, or the Z2 / fermion parity.  Products of several
factors follow ``tenet-sectors/src/product_rule.rs``: fusion channels are the
Cartesian product of the factor channels with the *first* factor varying
fastest (``product_rule.rs:287-302``), and every symbol is the product of the
factor symbols (``product_rule.rs:420-470``).
"""

from __future__ import annotations

from fractions import Fraction
from functools import lru_cache
from itertools import product as _cartesian
from math import factorial, isqrt

U1, SU2, FZ2, Z2 = "U1", "SU2", "FZ2", "Z2"

# Packed codec widths per factor (tenet-sectors/src/algebra.rs:1500-1560).
_PACKED_BITS = {FZ2: 1, Z2: 1, U1: 32, SU2: 8}


def u1_zigzag(charge: int) -> int:
    """``u1_charge_to_zigzag_u32`` (tenet-sectors/src/abelian.rs:570-572)."""
    return ((charge << 1) ^ (charge >> 31)) & 0xFFFFFFFF


def u1_unzigzag(code: int) -> int:
    """``u1_charge_from_zigzag_u32`` (tenet-sectors/src/abelian.rs:574-576)."""
    return (code >> 1) ^ -(code & 1)


def cantor_pair(left: int, right: int) -> int:
    """``TensorKitProductCodec::try_encode`` (tenet-sectors/src/algebra.rs:1436-1447)."""
    s = left + right
    return s * (s + 1) // 2 + left


class Rule:
    """A (possibly product) multiplicity-free fusion rule.

    ``codec`` is ``"packed"`` (``PackedProductCodec``, algebra.rs:1581-1620,
    the layout the built-in product spaces use) or ``"cantor"`` (the
    left-nested ``TensorKitProductCodec``, algebra.rs:1432-1479).
    """

    def __init__(self, factors, codec="packed"):
        self.factors = tuple(factors)
        self.codec = codec
        self.fermionic = FZ2 in self.factors
        self.unique = SU2 not in self.factors

    def __repr__(self):
        return f"Rule({'x'.join(self.factors)}, {self.codec})"

    def __eq__(self, other):
        return isinstance(other, Rule) and self.factors == other.factors and self.codec == other.codec

    def __hash__(self):
        return hash((self.factors, self.codec))

    # -- codec ---------------------------------------------------------
    def leaf_id(self, kind, value):
        if kind == U1:
            return u1_zigzag(value)
        return value  # SU2: 2j (su2.rs:41-43); Z2/fZ2: parity

    def sector_id(self, label) -> int:
        ids = [self.leaf_id(k, v) for k, v in zip(self.factors, label)]
        if len(ids) == 1:
            return ids[0]
        if self.codec == "packed":
            out, shift = 0, 0
            for k, i in zip(self.factors, ids):
                out |= i << shift
                shift += _PACKED_BITS[k]
            return out
        out = ids[0]
        for i in ids[1:]:
            out = cantor_pair(out, i)
        return out

    def sort_key(self, label):
        return self.sector_id(label)

    # -- fusion --------------------------------------------------------
    def vacuum(self):
        return tuple(0 for _ in self.factors)

    def dual(self, a):
        return tuple(-v if k == U1 else v for k, v in zip(self.factors, a))

    @staticmethod
    def _factor_channels(kind, a, b):
        if kind == U1:
            return [a + b]
        if kind == SU2:
            return list(range(abs(a - b), a + b + 1, 2))
        return [a ^ b]

    def fusion_channels(self, a, b):
        per = [self._factor_channels(k, x, y) for k, x, y in zip(self.factors, a, b)]
        # first factor fastest: iterate the last factor outermost.
        out = []
        for combo in _cartesian(*reversed(per)):
            out.append(tuple(reversed(combo)))
        return out

    def nsymbol(self, a, b, c) -> int:
        for k, x, y, z in zip(self.factors, a, b, c):
            if z not in self._factor_channels(k, x, y):
                return 0
        return 1

    # -- symbols ---------------------------------------------------------
    def dim(self, a) -> float:
        d = 1
        for k, v in zip(self.factors, a):
            if k == SU2:
                d *= v + 1
        return float(d)

    def twist(self, a) -> float:
        t = 1.0
        for k, v in zip(self.factors, a):
            if k == FZ2 and v == 1:
                t = -t
        return t

    def fs(self, a) -> float:
        """Frobenius-Schur phase: (-1)^(2j) for SU(2) (su2.rs:366-369), 1 otherwise."""
        t = 1.0
        for k, v in zip(self.factors, a):
            if k == SU2 and v % 2 == 1:
                t = -t
        return t

    def R(self, a, b, c) -> float:
        """R symbol, product over factors (abelian.rs:477-484, su2.rs:333-358)."""
        r = 1.0
        for k, x, y, z in zip(self.factors, a, b, c):
            if k == FZ2:
                if x == 1 and y == 1:
                    r = -r
            elif k == SU2:
                if z not in self._factor_channels(SU2, x, y):
                    return 0.0
                if ((x + y - z) // 2) % 2 == 1:
                    r = -r
        return r

    def F(self, a, b, c, d, e, f) -> float:
        """F(a,b,c; d; e, f) with e in a(x)b and f in b(x)c (algebra.rs:570-578).

        Abelian factors contribute 1 (abelian.rs:334-345, 465-475); SU(2)
        contributes the Racah coefficient in the Condon-Shortley gauge
        (su2.rs:300-318 -> racah::su2_f_symbol).
        """
        v = 1.0
        for i, k in enumerate(self.factors):
            if k == SU2:
                v *= su2_f(a[i], b[i], c[i], d[i], e[i], f[i])
                if v == 0.0:
                    return 0.0
        return v

    def A(self, a, b, c) -> float:
        """A symbol default (tenet-sectors/src/algebra.rs:603-613)."""
        factor = (self.dim(a) * self.dim(b)) ** 0.5 / self.dim(c) ** 0.5
        return factor * self.fs(a) * self.F(self.dual(a), a, b, b, self.vacuum(), c)

    def B(self, a, b, c) -> float:
        """B symbol default (tenet-sectors/src/algebra.rs:615-623)."""
        return (
            self.dim(a) ** 0.5
            * self.dim(b) ** 0.5
            / self.dim(c) ** 0.5
            * self.F(a, b, self.dual(b), a, c, self.vacuum())
        )


class TableRule(Rule):
    """A rule given by provider tables (labels 0 .. n-1, 0 the vacuum), the
    restatement of the table-provider branch of the device rule: the
    reference's checked Generic providers (tenet-sectors/src/algebra.rs:
    743-910) restricted to multiplicity-free, real, symmetric data.  Labels
    are 1-tuples ``(i,)``; SectorId = i; channels ascend by label.  The A and
    B symbols keep the defaults of ``Rule`` (algebra.rs:603-623)."""

    def __init__(self, dual, nsym, dims, fs, rsym, fsym):
        self.factors = ("TABLE",)
        self.codec = "packed"
        self.fermionic = False
        self.unique = False
        self._dual = [int(x) for x in dual]
        self._N = nsym
        self._dims = [float(x) for x in dims]
        self._fs = [float(x) for x in fs]
        self._R = rsym
        self._F = fsym
        self.n = len(self._dims)

    def __repr__(self):
        return f"TableRule(n={self.n})"

    def __eq__(self, other):
        return isinstance(other, TableRule) and self is other

    def __hash__(self):
        return id(self)

    def sector_id(self, label) -> int:
        return int(label[0])

    def vacuum(self):
        return (0,)

    def dual(self, a):
        return (self._dual[a[0]],)

    def fusion_channels(self, a, b):
        return [(c,) for c in range(self.n) if self._N[a[0], b[0], c]]

    def nsymbol(self, a, b, c) -> int:
        return int(self._N[a[0], b[0], c[0]])

    def dim(self, a) -> float:
        return self._dims[a[0]]

    def twist(self, a) -> float:
        return 1.0

    def fs(self, a) -> float:
        return self._fs[a[0]]

    def R(self, a, b, c) -> float:
        return float(self._R[a[0], b[0], c[0]]) if self._N[a[0], b[0], c[0]] else 0.0

    def F(self, a, b, c, d, e, f) -> float:
        return float(self._F[a[0], b[0], c[0], d[0], e[0], f[0]])


def product(*factors, codec="packed") -> Rule:
    return Rule(factors, codec)


# ---------------------------------------------------------------------------
# SU(2) recoupling in exact rational arithmetic
# ---------------------------------------------------------------------------


def _triad(a, b, c):
    return (a + b - c) >= 0 and (a - b + c) >= 0 and (-a + b + c) >= 0 and (a + b + c) % 2 == 0


def _delta2(a, b, c) -> Fraction:
    """Squared triangle coefficient, arguments are doubled spins."""
    return Fraction(
        factorial((a + b - c) // 2) * factorial((a - b + c) // 2) * factorial((-a + b + c) // 2),
        factorial((a + b + c) // 2 + 1),
    )


def _sqrt_fraction(x: Fraction) -> float:
    """Correctly rounded sqrt of a non-negative rational (128 guard bits)."""
    if x == 0:
        return 0.0
    k = 160
    r = isqrt((x.numerator << (2 * k)) // x.denominator)
    return float(Fraction(r, 1 << k))


@lru_cache(maxsize=None)
def su2_6j_exact(j1, j2, j3, j4, j5, j6):
    """Wigner 6j {j1 j2 j3; j4 j5 j6} (doubled spins) as (sign, square) rationals.

    Racah's single-sum formula.  Returns ``(s, q)`` with the 6j value equal
    to ``s * sqrt(q)`` (``s`` rational, ``q`` non-negative rational).
    """
    if not (_triad(j1, j2, j3) and _triad(j1, j5, j6) and _triad(j4, j2, j6) and _triad(j4, j5, j3)):
        return Fraction(0), Fraction(0)
    q = _delta2(j1, j2, j3) * _delta2(j1, j5, j6) * _delta2(j4, j2, j6) * _delta2(j4, j5, j3)
    a1 = (j1 + j2 + j3) // 2
    a2 = (j1 + j5 + j6) // 2
    a3 = (j4 + j2 + j6) // 2
    a4 = (j4 + j5 + j3) // 2
    b1 = (j1 + j2 + j4 + j5) // 2
    b2 = (j2 + j3 + j5 + j6) // 2
    b3 = (j3 + j1 + j6 + j4) // 2
    s = Fraction(0)
    for z in range(max(a1, a2, a3, a4), min(b1, b2, b3) + 1):
        term = Fraction(
            factorial(z + 1),
            factorial(z - a1)
            * factorial(z - a2)
            * factorial(z - a3)
            * factorial(z - a4)
            * factorial(b1 - z)
            * factorial(b2 - z)
            * factorial(b3 - z),
        )
        s += -term if z % 2 else term
    return s, q


@lru_cache(maxsize=None)
def su2_f(a, b, c, d, e, f) -> float:
    """SU(2) F-symbol F(a,b,c; d; e, f), doubled spins.

    F = sqrt((2e+1)(2f+1)) (-1)^(a+b+c+d) {a b e; c d f}: the gauge whose
    values TensorKit tabulates (benchmarks/tensorkit_semantic_oracle.out,
    section 1, ``F SU2`` rows) and whose frozen values su2.rs:377-430 pins.
    """
    if not (_triad(a, b, e) and _triad(e, c, d) and _triad(b, c, f) and _triad(a, f, d)):
        return 0.0
    s, q = su2_6j_exact(a, b, e, c, d, f)
    if s == 0:
        return 0.0
    sq = s * s * q * (e + 1) * (f + 1)
    sign = -1 if s < 0 else 1
    if ((a + b + c + d) // 2) % 2 == 1:
        sign = -sign
    return sign * _sqrt_fraction(sq)
