"""v1 typed snapshots (CPU): framing, canonical bytes, round trips, rejections.

Mirrors the reference's own serialization tests
(tenet/tests/typed_serialization.rs:382-410, 670-712, 963-1117): the header
ends at 20 + key length, the leg and block-count offsets follow the wire
layout, a round trip reproduces spaces, payload bits and bytes, and malformed
framing, unsupported versions, limits, missing or mismatched providers,
missing and duplicate blocks are rejected with the matching error kind.
"""

import struct

import numpy as np
import pytest

from oracle.fusion import Leg
from oracle.sectors import FZ2, SU2, U1, Rule
from tests.helpers import product_space


def _u64(b, off):
    return struct.unpack_from("<Q", b, off)[0]


def _header_end(b):
    return 20 + _u64(b, 12)


@pytest.fixture(scope="module")
def p():
    from tenet_b200 import persistence

    return persistence


def _su2_leg(dual):
    from tenet_b200 import typed

    leg = typed.GradedSpace(typed.SU2FusionRule(), [(0, 1), (1, 2)])
    return leg.dual() if dual else leg


SPACES = {
    "su2": (Rule([SU2]), [Leg.new(Rule([SU2]), [((0,), 2), ((1,), 3), ((2,), 1)])] * 2,
            [Leg.new(Rule([SU2]), [((0,), 2), ((1,), 3), ((2,), 1)]).dual()] * 2),
    "u1_dual": (Rule([U1]), [Leg.new(Rule([U1]), [((-1,), 2), ((0,), 3), ((1,), 2)]),
                             Leg.new(Rule([U1]), [((-1,), 1), ((1,), 2)]).dual()],
                [Leg.new(Rule([U1]), [((-1,), 2), ((0,), 3), ((1,), 2)])]),
    "fz2_u1_su2": (Rule([FZ2, U1, SU2]),
                   [Leg.new(Rule([FZ2, U1, SU2]), [((0, 0, 0), 2), ((1, 1, 1), 2), ((0, 2, 0), 1)]),
                    Leg.new(Rule([FZ2, U1, SU2]), [((0, 0, 0), 1), ((1, 1, 1), 1)])],
                   [Leg.new(Rule([FZ2, U1, SU2]), [((1, 1, 1), 1), ((0, 0, 0), 1)]),
                    Leg.new(Rule([FZ2, U1, SU2]), [((0, 0, 0), 2), ((1, 1, 1), 2), ((0, 2, 0), 1)]).dual()]),
}


def test_space_round_trip_keeps_duality_and_deterministic_bytes(p):
    for dual in (False, True):
        leg = _su2_leg(dual)
        b = p.space_to_bytes(leg)
        assert b[:8] == b"TENETTS\x00" and struct.unpack_from("<H", b, 8)[0] == 1
        assert b[10] == 1 and b[11] == 0 and b[20:_header_end(b)] == b"su2"
        back = p.space_from_bytes(b)
        assert back == leg and back.is_dual == dual
        assert p.space_to_bytes(back) == b


def test_u1_space_round_trip_does_not_dualize_twice(p):
    from tenet_b200 import typed

    leg = typed.GradedSpace(typed.U1FusionRule(), [(-1, 2), (2, 1)]).dual()
    back = p.space_from_bytes(p.space_to_bytes(leg))
    assert back == leg and back.sectors() == leg.sectors()


@pytest.mark.parametrize("name", sorted(SPACES))
def test_dense_round_trip_exact_bits_and_bytes(p, name):
    rule, cod, dom = SPACES[name]
    sp = product_space(rule, cod, dom)
    rng = np.random.default_rng(3)
    payload = rng.standard_normal(sp.size)
    payload[0] = -0.0
    b = p.payload_to_bytes(sp, payload)
    sp2, back, adjoint = p.payload_from_bytes(b)
    assert not adjoint and sp2.same_as(sp)
    assert back.view(np.uint64).tolist() == payload.view(np.uint64).tolist()
    assert p.payload_to_bytes(sp2, back) == b
    # The leg-degeneracy offsets of the wire layout point at the degeneracies.
    pos = _header_end(b) + 1
    rank = _u64(b, pos) + _u64(b, pos + 8)
    pos += 16
    legs = list(sp.codomain) + list(sp.domain)
    assert rank == len(legs)
    for leg in legs:
        pos += 1
        n = _u64(b, pos)
        pos += 8
        degs = []
        for _ in range(n):
            pos += 8 + _u64(b, pos)
            degs.append(_u64(b, pos))
            pos += 8
        assert sorted(degs) == sorted(leg.degeneracies())


def test_blocks_are_sorted_by_key_bytes_and_values_first_axis_fastest(p):
    rule, cod, dom = SPACES["u1_dual"]
    sp = product_space(rule, cod, dom)
    payload = np.arange(sp.size, dtype=np.float64)
    b = p.payload_to_bytes(sp, payload)
    pos = _header_end(b) + 1 + 16
    for _ in range(sp.n1 + sp.n2):
        pos += 1
        n = _u64(b, pos)
        pos += 8
        for _ in range(n):
            pos += 8 + _u64(b, pos) + 8
    nblocks = _u64(b, pos)
    pos += 8
    assert nblocks == sp.nblocks
    keys = []
    for _ in range(nblocks):
        klen = _u64(b, pos)
        keys.append(b[pos + 8:pos + 8 + klen])
        pos += 8 + klen
        r = _u64(b, pos)
        shape = [_u64(b, pos + 8 + 8 * i) for i in range(r)]
        pos += 8 + 8 * r
        cnt = _u64(b, pos)
        vals = np.frombuffer(b[pos + 8:pos + 8 + 8 * cnt], dtype="<f8")
        pos += 8 + 8 * cnt
        assert cnt == int(np.prod(shape))
        # first axis fastest: consecutive values along axis 0 differ by its stride
        blk = [x for x in sp.blocks() if tuple(x[1]) == tuple(shape) and x[0] == int(vals[0])]
        assert blk and (shape[0] < 2 or vals[1] - vals[0] == blk[0][2][0])
    assert keys == sorted(keys)
    assert pos == len(b)


def test_malformed_space_framing_limits_and_providers(p):
    leg = _su2_leg(True)
    b = p.space_to_bytes(leg)
    for off, val in [(0, ord("X")), (10, 2), (11, 1)]:
        m = bytearray(b)
        m[off] = val
        with pytest.raises(p.DecodeError) as e:
            p.space_from_bytes(bytes(m))
        assert e.value.kind == "invalid_format"
    m = bytearray(b)
    m[8:10] = struct.pack("<H", 2)
    with pytest.raises(p.DecodeError) as e:
        p.space_from_bytes(bytes(m))
    assert e.value.kind == "unsupported_version"
    m = bytearray(b)
    m[_header_end(b)] = 2
    with pytest.raises(p.DecodeError, match="duality"):
        p.space_from_bytes(bytes(m))
    for bad in (b[:-1], b + b"\x00"):
        with pytest.raises(p.DecodeError) as e:
            p.space_from_bytes(bad)
        assert e.value.kind == "invalid_format"

    class Counting(p.LabelCodec):
        calls = 0

        def resolve_provider(self, key):
            Counting.calls += 1
            return super().resolve_provider(key)

    c = Counting()
    with pytest.raises(p.DecodeError) as e:
        p.space_from_bytes(b, c, p.DecodeLimits(max_bytes=len(b) - 1))
    assert e.value.kind == "limit_exceeded" and Counting.calls == 0
    m = bytearray(b)
    m[0] = 0
    with pytest.raises(p.DecodeError) as e:
        p.space_from_bytes(bytes(m), c)
    assert e.value.kind == "invalid_format" and Counting.calls == 0

    class Missing(p.LabelCodec):
        def resolve_provider(self, key):
            raise p.DecodeError("codec", "missing provider")

    with pytest.raises(p.DecodeError) as e:
        p.space_from_bytes(b, Missing())
    assert e.value.kind == "codec"

    class Foreign(p.LabelCodec):
        def resolve_provider(self, key):
            from tenet_b200 import typed

            return typed.SU2FusionRule()

    m = bytearray(b)
    m[20:23] = b"bad"
    with pytest.raises(p.DecodeError) as e:
        p.space_from_bytes(bytes(m), Foreign())
    assert e.value.kind == "provider_mismatch"


def test_malformed_tensor_tags_missing_duplicate_blocks_and_limits(p):
    from tenet_b200 import typed

    rule = typed.SU2FusionRule()
    leg = typed.GradedSpace(rule, [(0, 1)])
    sp = typed.HomSpace(rule, [leg], [])
    assert sp.size == 1
    b = p.payload_to_bytes(sp, np.array([3.0]))
    for off, val in [(10, 1), (11, 2), (_header_end(b), 99)]:
        m = bytearray(b)
        m[off] = val
        with pytest.raises(p.DecodeError) as e:
            p.payload_from_bytes(bytes(m))
        assert e.value.kind == "invalid_format"
    count_at = _header_end(b) + 1 + 16 + 1 + 8 + 8 + 1 + 8
    assert _u64(b, count_at) == 1
    first = count_at + 8
    missing = bytearray(b[:first])
    missing[count_at:first] = struct.pack("<Q", 0)
    with pytest.raises(p.DecodeError, match="missing an admitted block"):
        p.payload_from_bytes(bytes(missing))
    dup = bytearray(b)
    dup[count_at:first] = struct.pack("<Q", 2)
    dup += b[first:]
    with pytest.raises(p.DecodeError, match="duplicate"):
        p.payload_from_bytes(bytes(dup))
    for lim in (dict(max_rank=0), dict(max_sectors_per_leg=0), dict(max_blocks=0), dict(max_elements=0),
                dict(max_blob_bytes=0)):
        with pytest.raises(p.DecodeError) as e:
            p.payload_from_bytes(b, limits=p.DecodeLimits(**lim))
        assert e.value.kind == "limit_exceeded"
    _, back, _ = p.payload_from_bytes(b)
    assert back.tolist() == [3.0]


def test_product_provider_keys_round_trip(p):
    codec = p.LabelCodec()
    for factors, cdc in ((["FZ2", "U1", "SU2"], "packed"), (["U1", "SU2"], "cantor"), (["Z2"], "packed")):
        from tenet_b200 import typed

        rule = typed.FusionRule(factors, cdc)
        assert codec.resolve_provider(codec.provider_key(rule)) == rule


def test_compact_spectrum_and_lazy_adjoint_snapshots_decode_dense(p):
    """Representation 2 (a compact spectrum on a rank-(1,1) bond space,
    serialization.rs:872-910) decodes into dense diagonal blocks; representation
    3 wraps a parent body and marks the result as its adjoint."""
    from tenet_b200 import typed

    rule = typed.SU2FusionRule()
    leg = typed.GradedSpace(rule, [(0, 2), (1, 3)])
    codec = p.LabelCodec()
    body = p._encode_space(codec, rule, typed.HomSpace(rule, [leg], [leg]))
    spectra = {(0,): [2.0, 1.0], (1,): [5.0, 4.0, 3.0]}
    entries = sorted((codec.encode_sector(rule, k), v) for k, v in spectra.items())
    enc = p._u64(len(entries)) + b"".join(p._blob(k) + p._u64(len(v)) + np.asarray(v, "<f8").tobytes()
                                          for k, v in entries)
    head = p._header(p.KIND_TENSOR, p.SCALAR_F64, codec.provider_key(rule))
    sp, payload, adjoint = p.payload_from_bytes(head + bytes([p.REPR_DIAGONAL]) + body + enc)
    assert not adjoint
    for lab, r, c, off in sp.sectors():
        np.testing.assert_array_equal(payload[off:off + r * c].reshape(c, r), np.diag(spectra[tuple(lab)]))
    dense = p.payload_to_bytes(sp, payload)
    lazy = dense[:_header_end(dense)] + bytes([p.REPR_ADJOINT]) + dense[_header_end(dense):]
    sp2, payload2, adjoint2 = p.payload_from_bytes(lazy)
    assert adjoint2 and sp2.same_as(sp) and payload2.tolist() == payload.tolist()
    bad = head + bytes([p.REPR_DIAGONAL]) + body + enc[:-8] + np.asarray([1.0], "<f8").tobytes()[:0]
    with pytest.raises(p.DecodeError):
        p.payload_from_bytes(bad)
