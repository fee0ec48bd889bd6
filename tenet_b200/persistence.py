"""Snapshots of device tensors in TeNeT's v1 typed persistence format.

Restates the wire format of ``TypedPersistenceCodec`` snapshots
(tenet/src/typed/serialization.rs:17-26, 301-360, 657-960, 980-1456) so a
serving loop can checkpoint resident tensors and restore them on a device:

* header: ``b"TENETTS\\0"``, version u16 (1), kind u8 (1 space, 2 tensor),
  scalar u8 (0 none, 1 f64), provider-key blob;
* a blob is a u64 length and its bytes; every integer is little-endian u64
  unless stated;
* a leg: dual flag u8, sector count, then per sector (sorted by label bytes)
  the label blob and the degeneracy;
* a dense tensor: representation u8 (1 dense, 3 adjoint + inner
  representation), codomain and domain ranks, the legs, the block count, then
  per block (sorted by key bytes) the key blob -- codomain tree then domain
  tree, each coupled label blob, uncoupled labels, inner lines, vertex labels
  (all one for multiplicity-free rules) -- its shape and its values in
  first-axis-fastest order as f64 bits.

Decoding applies ``DecodeLimits`` before any allocation, checks the provider
key, requires every admitted block exactly once with its admitted shape, and
rejects trailing bytes.  Compact diagonal payloads (representation 2) decode
into dense diagonal blocks.  The payload crosses the PCIe link once per
snapshot (one device-to-host copy to encode, one host-to-device copy to
restore); the byte work is host work, as in the reference.
"""

from __future__ import annotations

import struct
from dataclasses import dataclass
import numpy as np

from .typed import FusionRule, GradedSpace, HomSpace

MAGIC = b"TENETTS\x00"
VERSION = 1
KIND_SPACE, KIND_TENSOR = 1, 2
SCALAR_NONE, SCALAR_F64, SCALAR_C64 = 0, 1, 2
REPR_DENSE, REPR_DIAGONAL, REPR_ADJOINT = 1, 2, 3


@dataclass(frozen=True)
class DecodeLimits:
    """Resource ceilings checked before lengths drive allocation (serialization.rs:72-100)."""

    max_bytes: int = 1 << 30
    max_rank: int = 64
    max_sectors_per_leg: int = 1 << 20
    max_blocks: int = 1 << 20
    max_elements: int = 1 << 32
    max_blob_bytes: int = 1 << 20


class DecodeError(ValueError):
    """A snapshot that cannot be decoded; ``kind`` is one of ``invalid_format``,
    ``unsupported_version``, ``limit_exceeded``, ``codec``, ``provider_mismatch``."""

    def __init__(self, kind: str, message: str):
        super().__init__(message)
        self.kind = kind


class LabelCodec:
    """Canonical sector-label bytes for the rules of this package.

    Per factor: U(1) charge as i32, SU(2) twice the spin as u8, fermion
    parity and Z2 parity as u8, concatenated in factor order.  The provider
    key names the factors (``b"u1"``, ``b"su2"``, ``b"fz2"``, ``b"z2"`` for a
    single factor -- the keys and label bytes of the reference's own
    serialization tests -- and ``b"fz2*u1*su2;packed"`` style keys for
    products, which include the product codec).
    """

    _NAMES = {"U1": b"u1", "SU2": b"su2", "FZ2": b"fz2", "Z2": b"z2"}

    def provider_key(self, rule: FusionRule) -> bytes:
        names = [self._NAMES[f] for f in rule.factors]
        if len(names) == 1:
            return names[0]
        return b"*".join(names) + b";" + rule.codec.encode()

    def resolve_provider(self, key: bytes) -> FusionRule:
        inv = {v: k for k, v in self._NAMES.items()}
        if key in inv:
            return FusionRule([inv[key]])
        head, sep, codec = key.partition(b";")
        parts = head.split(b"*")
        if not sep or len(parts) < 2 or any(p not in inv for p in parts) or codec not in (b"packed", b"cantor"):
            raise DecodeError("codec", f"unknown provider key {key!r}")
        return FusionRule([inv[p] for p in parts], codec.decode())

    def encode_sector(self, rule: FusionRule, label) -> bytes:
        out = b""
        for f, v in zip(rule.factors, label):
            out += struct.pack("<i", v) if f == "U1" else struct.pack("<B", v)
        return out

    def decode_sector(self, rule: FusionRule, data: bytes):
        vals, pos = [], 0
        for f in rule.factors:
            width = 4 if f == "U1" else 1
            if pos + width > len(data):
                raise DecodeError("codec", "sector label is too short")
            vals.append(struct.unpack_from("<i" if f == "U1" else "<B", data, pos)[0])
            pos += width
        if pos != len(data):
            raise DecodeError("codec", "sector label has trailing bytes")
        for f, v in zip(rule.factors, vals):
            if f in ("FZ2", "Z2") and v > 1:
                raise DecodeError("codec", "parity label is not 0 or 1")
        return tuple(vals)


# ---------------------------------------------------------------------------
# encoding
# ---------------------------------------------------------------------------


def _u64(n: int) -> bytes:
    return struct.pack("<Q", n)


def _blob(b: bytes) -> bytes:
    return _u64(len(b)) + b


def _header(kind: int, scalar: int, key: bytes) -> bytes:
    return MAGIC + struct.pack("<HBB", VERSION, kind, scalar) + _blob(key)


def _encode_leg(codec, rule, leg: GradedSpace) -> bytes:
    entries = sorted((codec.encode_sector(rule, s), d) for s, d in zip(leg._sectors, leg._degs))
    out = bytes([1 if leg.is_dual else 0]) + _u64(len(entries))
    for lab, d in entries:
        out += _blob(lab) + _u64(d)
    return out


def _encode_tree(codec, rule, tree) -> bytes:
    uncoupled, _duals, coupled, inner = tree
    out = _blob(codec.encode_sector(rule, coupled))
    for labels in (uncoupled, inner):
        out += _u64(len(labels)) + b"".join(_blob(codec.encode_sector(rule, s)) for s in labels)
    nv = max(0, len(uncoupled) - 1)
    return out + _u64(nv) + _u64(1) * nv


def _encode_space(codec, rule, space: HomSpace) -> bytes:
    out = _u64(space.n1) + _u64(space.n2)
    for leg in tuple(space.codomain) + tuple(space.domain):
        out += _encode_leg(codec, rule, leg)
    return out


def _block_view(payload: np.ndarray, offset: int, shape, strides) -> np.ndarray:
    return np.lib.stride_tricks.as_strided(payload[offset:], shape=tuple(shape),
                                           strides=tuple(8 * s for s in strides), writeable=True)


def space_to_bytes(leg: GradedSpace, codec=None) -> bytes:
    """``GradedSpace::to_bytes_with`` (serialization.rs:1701-1712)."""
    codec = codec or LabelCodec()
    return _header(KIND_SPACE, SCALAR_NONE, codec.provider_key(leg.rule)) + _encode_leg(codec, leg.rule, leg)


def payload_to_bytes(space: HomSpace, payload: np.ndarray, codec=None) -> bytes:
    """A dense f64 tensor snapshot of ``payload`` laid out in ``space``
    (``TensorMap::to_bytes_with``, encode_tensor / encode_dense_body)."""
    codec = codec or LabelCodec()
    rule = space.rule
    payload = np.ascontiguousarray(payload, dtype=np.float64)
    if payload.shape != (space.size,):
        raise ValueError("dense storage length does not match the layout")
    out = bytearray(_header(KIND_TENSOR, SCALAR_F64, codec.provider_key(rule)))
    out.append(REPR_DENSE)
    out += _encode_space(codec, rule, space)
    blocks = []
    for (off, shape, strides, _), (ct, dt) in zip(space.blocks(), space.block_keys()):
        key = _encode_tree(codec, rule, ct) + _encode_tree(codec, rule, dt)
        blocks.append((key, off, shape, strides))
    blocks.sort(key=lambda b: b[0])
    out += _u64(len(blocks))
    for key, off, shape, strides in blocks:
        out += _blob(key) + _u64(len(shape)) + b"".join(_u64(d) for d in shape)
        vals = _block_view(payload, off, shape, strides).ravel(order="F")
        out += _u64(vals.size) + vals.astype("<f8").tobytes()
    return bytes(out)


# ---------------------------------------------------------------------------
# decoding
# ---------------------------------------------------------------------------


class _Reader:
    def __init__(self, data: bytes, limits: DecodeLimits):
        self.b, self.pos, self.limits = data, 0, limits

    def take(self, n: int) -> bytes:
        if n < 0 or self.pos + n > len(self.b):
            raise DecodeError("invalid_format", "truncated input")
        out = self.b[self.pos:self.pos + n]
        self.pos += n
        return out

    def u8(self) -> int:
        return self.take(1)[0]

    def u64(self) -> int:
        return struct.unpack("<Q", self.take(8))[0]

    def blob(self, what: str) -> bytes:
        n = self.u64()
        _limit(what, n, self.limits.max_blob_bytes)
        return self.take(n)

    def finish(self):
        if self.pos != len(self.b):
            raise DecodeError("invalid_format", "trailing bytes")


def _limit(what: str, actual: int, limit: int):
    if actual > limit:
        raise DecodeError("limit_exceeded", f"typed snapshot {what} {actual} exceeds decode limit {limit}")


def _read_header(data: bytes, limits: DecodeLimits, kind: int, codec):
    _limit("bytes", len(data), limits.max_bytes)
    r = _Reader(data, limits)
    if r.take(8) != MAGIC:
        raise DecodeError("invalid_format", "not a typed snapshot")
    version = struct.unpack("<H", r.take(2))[0]
    if version != VERSION:
        raise DecodeError("unsupported_version",
                          f"unsupported typed snapshot version {version}; this decoder supports {VERSION}")
    k, scalar = r.u8(), r.u8()
    if k != kind:
        raise DecodeError("invalid_format", f"snapshot kind {k} where {kind} was expected")
    key = r.blob("provider key bytes")
    rule = codec.resolve_provider(key)
    if codec.provider_key(rule) != key:
        raise DecodeError("provider_mismatch", "resolved provider key does not match")
    return r, rule, scalar


def _read_leg(r: _Reader, codec, rule) -> GradedSpace:
    dual = r.u8()
    if dual not in (0, 1):
        raise DecodeError("invalid_format", "duality flag is not 0 or 1")
    n = r.u64()
    _limit("sectors per leg", n, r.limits.max_sectors_per_leg)
    pairs = []
    for _ in range(n):
        lab = codec.decode_sector(rule, r.blob("sector label bytes"))
        d = r.u64()
        if d == 0:
            raise DecodeError("invalid_format", "zero-degeneracy sector is not canonical")
        pairs.append((lab, d))
    if len({p[0] for p in pairs}) != len(pairs):
        raise DecodeError("invalid_format", "duplicate sector label on one leg")
    return GradedSpace(rule, pairs, bool(dual))


def _read_labels(r: _Reader, codec, rule, what: str):
    n = r.u64()
    _limit(what, n, r.limits.max_rank)
    return tuple(codec.decode_sector(rule, r.blob("sector label bytes")) for _ in range(n))


def _read_tree(r: _Reader, codec, rule):
    coupled = codec.decode_sector(rule, r.blob("sector label bytes"))
    uncoupled = _read_labels(r, codec, rule, "fusion-tree labels")
    inner = _read_labels(r, codec, rule, "fusion-tree labels")
    nv = r.u64()
    _limit("fusion vertices", nv, r.limits.max_rank)
    for _ in range(nv):
        if r.u64() != 1:
            raise DecodeError("invalid_format", "a multiplicity-free vertex label is not one")
    if nv != max(0, len(uncoupled) - 1):
        raise DecodeError("invalid_format", "vertex count does not match the tree")
    return (uncoupled, coupled, inner)


def _read_legs(r: _Reader, codec, rule):
    n1, n2 = r.u64(), r.u64()
    _limit("rank", n1 + n2, r.limits.max_rank)
    legs = [_read_leg(r, codec, rule) for _ in range(n1 + n2)]
    return legs[:n1], legs[n1:]


def space_from_bytes(data: bytes, codec=None, limits: DecodeLimits = DecodeLimits()) -> GradedSpace:
    """``GradedSpace::from_bytes_with`` (serialization.rs:1726-1740)."""
    codec = codec or LabelCodec()
    r, rule, scalar = _read_header(data, limits, KIND_SPACE, codec)
    if scalar != SCALAR_NONE:
        raise DecodeError("invalid_format", "a space snapshot carries no scalar type")
    leg = _read_leg(r, codec, rule)
    r.finish()
    return leg


def _read_dense_records(r: _Reader, codec, rule, rank: int):
    n = r.u64()
    _limit("dense blocks", n, r.limits.max_blocks)
    total, records = 0, {}
    for _ in range(n):
        kr = _Reader(r.blob("block key bytes"), r.limits)
        ct, dt = _read_tree(kr, codec, rule), _read_tree(kr, codec, rule)
        kr.finish()
        if ct[1] != dt[1]:
            raise DecodeError("invalid_format", "fusion-tree pair has unequal coupled sectors")
        if r.u64() != rank:
            raise DecodeError("invalid_format", "block shape rank does not match tensor rank")
        shape = tuple(r.u64() for _ in range(rank))
        count = r.u64()
        total += count
        _limit("payload elements", total, r.limits.max_elements)
        vals = np.frombuffer(r.take(8 * count), dtype="<f8")
        if count != int(np.prod(shape, dtype=np.int64)):
            raise DecodeError("invalid_format", "block value count does not match shape")
        if (ct, dt) in records:
            raise DecodeError("invalid_format", "duplicate semantic block key")
        records[(ct, dt)] = (shape, vals)
    return records


def _read_diagonal_records(r: _Reader, codec, rule):
    n = r.u64()
    _limit("sectors per leg", n, r.limits.max_sectors_per_leg)
    total, records = 0, {}
    for _ in range(n):
        lab = codec.decode_sector(rule, r.blob("sector label bytes"))
        count = r.u64()
        total += count
        _limit("payload elements", total, r.limits.max_elements)
        if lab in records:
            raise DecodeError("invalid_format", "duplicate spectrum sector")
        records[lab] = np.frombuffer(r.take(8 * count), dtype="<f8")
    return records


def payload_from_bytes(data: bytes, codec=None, limits: DecodeLimits = DecodeLimits()):
    """Decode a tensor snapshot into ``(space, payload, adjoint)``: the
    admitted HomSpace, the FP64 payload in its coupled-sector layout, and
    whether the snapshot is a lazy adjoint of that tensor (``TensorMap::
    from_bytes_with``, decode_tensor / build_dense / build_diagonal)."""
    codec = codec or LabelCodec()
    r, rule, scalar = _read_header(data, limits, KIND_TENSOR, codec)
    if scalar == SCALAR_C64:
        raise DecodeError("invalid_format", "complex payloads are not supported by this backend")
    if scalar != SCALAR_F64:
        raise DecodeError("invalid_format", f"unknown scalar tag {scalar}")
    rep = r.u8()
    adjoint = rep == REPR_ADJOINT
    if adjoint:
        rep = r.u8()
    if rep not in (REPR_DENSE, REPR_DIAGONAL):
        raise DecodeError("invalid_format", f"unknown representation {rep}")
    cod, dom = _read_legs(r, codec, rule)
    rank = len(cod) + len(dom)
    if rep == REPR_DENSE:
        records = _read_dense_records(r, codec, rule, rank)
    else:
        if len(cod) != 1 or len(dom) != 1:
            raise DecodeError("invalid_format", "a compact spectrum needs a rank-(1,1) space")
        records = _read_diagonal_records(r, codec, rule)
    r.finish()
    space = HomSpace(rule, cod, dom)
    _limit("admitted dense blocks", space.nblocks, limits.max_blocks)
    _limit("admitted dense elements", space.size, limits.max_elements)
    payload = np.zeros(space.size)
    if rep == REPR_DENSE:
        for (off, shape, strides, _), (ct, dt) in zip(space.blocks(), space.block_keys()):
            key = ((ct[0], ct[2], ct[3]), (dt[0], dt[2], dt[3]))
            rec = records.pop(key, None)
            if rec is None:
                raise DecodeError("invalid_format", "dense payload is missing an admitted block")
            if tuple(rec[0]) != tuple(shape):
                raise DecodeError("invalid_format", "serialized block shape differs from admitted shape")
            _block_view(payload, off, shape, strides)[...] = rec[1].reshape(shape, order="F")
        if records:
            raise DecodeError("invalid_format", "dense payload contains an unadmitted block")
    else:
        for lab, rows, cols, off in space.sectors():
            vals = records.pop(tuple(lab), None)
            if vals is None or rows != cols or vals.size != rows:
                raise DecodeError("invalid_format", "spectrum does not match its bond space")
            payload[off:off + rows * cols].reshape(cols, rows)[np.arange(rows), np.arange(rows)] = vals
        if records:
            raise DecodeError("invalid_format", "spectrum contains an unadmitted sector")
    return space, payload, adjoint


def tensor_to_bytes(tensor, codec=None) -> bytes:
    """Snapshot of a device-resident TensorMap: one device-to-host copy of the payload."""
    return payload_to_bytes(tensor.space, tensor.to_host(), codec)


def tensor_from_bytes(runtime, data: bytes, codec=None, limits: DecodeLimits = DecodeLimits()):
    """Restore a snapshot onto ``runtime``'s device: one host-to-device copy;
    a lazy-adjoint snapshot is materialised with the device adjoint transform."""
    from .typed import TensorMap

    space, payload, adjoint = payload_from_bytes(data, codec, limits)
    t = TensorMap.from_host(runtime, list(space.codomain), list(space.domain), payload)
    return t.adjoint() if adjoint else t
