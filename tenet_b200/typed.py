"""Typed facade mirroring TeNeT's ``tenet::typed`` layer over the C ABI.

Names, argument meaning and error behaviour follow the reference facade
(tenet/src/typed.rs): ``GradedSpace::try_new`` (typed.rs:7777),
``TensorMap::{zeros, from_block_fn}`` (typed.rs:12230, 12262), ``permute`` /
``braid`` / ``repartition`` (typed.rs:13163-13250), ``contract``
(typed.rs:13653), ``compose`` (typed.rs:13842) and ``svd_trunc``
(typed.rs:1806), with ``Truncation`` from
tenet-matrixalgebra/src/truncation.rs:69-93.  Storage is always device
resident (the reference's ``CudaStorage`` placement); every hot operation runs
through ``libtenet_b200.so`` kernels.  Device memory and streams are torch
tensors and torch streams (plumbing only).
"""

from __future__ import annotations

import ctypes as C
import itertools
from dataclasses import dataclass
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import arr, call, i32, i64, u64, f64

_torch = None


def _release(fn, handle):
    """Destroy a C handle; a no-op once the interpreter is tearing modules down."""
    if not handle:
        return
    try:
        getattr(_lib.lib(), fn)(handle)
    except Exception:
        pass


def torch():
    global _torch
    if _torch is None:
        import torch as t

        _torch = t
    return _torch


# ---------------------------------------------------------------------------
# fusion rules
# ---------------------------------------------------------------------------


class FusionRule:
    """A product of U(1) / SU(2) / fermion-parity / Z2 factors.

    ``codec`` selects the SectorId packing: ``"packed"`` (PackedProductCodec,
    tenet-sectors/src/algebra.rs:1581-1620) or ``"cantor"``
    (TensorKitProductCodec, algebra.rs:1432-1479).
    """

    _KIND = {"U1": _lib.U1, "SU2": _lib.SU2, "FZ2": _lib.FZ2, "Z2": _lib.Z2}

    def __init__(self, factors: Sequence[str], codec: str = "packed"):
        self.factors = tuple(factors)
        self.codec = codec
        kinds = [self._KIND[f] for f in self.factors]
        h = C.c_void_p()
        call("tnt_rule_create", len(kinds), arr(i32, kinds), 0 if codec == "packed" else 1, C.byref(h))
        self._h = h

    def __del__(self):
        _release("tnt_rule_destroy", getattr(self, "_h", None))

    def __eq__(self, other):
        return isinstance(other, FusionRule) and self.factors == other.factors and self.codec == other.codec

    def __hash__(self):
        return hash((self.factors, self.codec))

    def __repr__(self):
        return "FusionRule(" + " x ".join(self.factors) + ")"

    @property
    def nfactors(self):
        return len(self.factors)

    def label(self, sector) -> Tuple[int, ...]:
        if isinstance(sector, (int, np.integer)):
            return (int(sector),)
        return tuple(int(x) for x in sector)

    def unlabel(self, label):
        return label[0] if self.nfactors == 1 else tuple(label)

    def sector_id(self, sector) -> int:
        out = u64()
        call("tnt_rule_sector_id", self._h, arr(i32, self.label(sector)), C.byref(out))
        return out.value

    def dual(self, sector):
        lab = self.label(sector)
        return self.unlabel(tuple(-v if f == "U1" else v for f, v in zip(self.factors, lab)))

    def dim(self, sector) -> float:
        out = f64()
        call("tnt_rule_dim", self._h, arr(i32, self.label(sector)), C.byref(out))
        return out.value

    def fsymbol(self, a, b, c, d, e, f) -> float:
        out = f64()
        lab = [x for s in (a, b, c, d, e, f) for x in self.label(s)]
        call("tnt_rule_fsymbol", self._h, arr(i32, lab), C.byref(out))
        return out.value

    def rsymbol(self, a, b, c) -> float:
        out = f64()
        lab = [x for s in (a, b, c) for x in self.label(s)]
        call("tnt_rule_rsymbol", self._h, arr(i32, lab), C.byref(out))
        return out.value


def U1FusionRule():
    return FusionRule(["U1"])


def SU2FusionRule():
    return FusionRule(["SU2"])


def FermionParityFusionRule():
    return FusionRule(["FZ2"])


def Z2FusionRule():
    return FusionRule(["Z2"])


class TableFusionRule(FusionRule):
    """A fusion rule given by a checked table provider (``providers.TableProvider``).

    The library checks the tables when the rule is created (vacuum and dual
    laws, no outer multiplicity, dimensions, orthogonal F moves, pentagon,
    symmetric R and hexagon; ``tnt_rule_create_table``) and then runs every
    recoupling and contraction on them like on a built-in rule.  Sectors are
    the labels 0 .. n-1."""

    def __init__(self, provider, tol: float = 1e-10):
        p = provider
        self.provider = p
        self.factors = ("TABLE",)
        self.codec = "packed"
        n = p.n
        h = C.c_void_p()
        as_c = lambda a, ct: np.ascontiguousarray(a, dtype=ct)
        self._tables = (as_c(p.dual, np.int32), as_c(p.nsym, np.uint8), as_c(p.dims, np.float64),
                        as_c(p.fs, np.float64), as_c(p.rsym, np.float64), as_c(p.fsym, np.float64))
        dual, nsym, dims, fs, rs, fsym = self._tables
        call("tnt_rule_create_table", n, dual.ctypes.data_as(C.POINTER(i32)), nsym.ctypes.data_as(C.POINTER(C.c_uint8)),
             dims.ctypes.data_as(C.POINTER(f64)), fs.ctypes.data_as(C.POINTER(f64)), rs.ctypes.data_as(C.POINTER(f64)),
             fsym.ctypes.data_as(C.POINTER(f64)), tol, C.byref(h))
        self._h = h
        self._key = hash((dual.tobytes(), nsym.tobytes(), dims.tobytes(), fs.tobytes(), rs.tobytes(), fsym.tobytes()))

    def __eq__(self, other):
        return isinstance(other, TableFusionRule) and self._key == other._key

    def __hash__(self):
        return self._key

    def __repr__(self):
        return f"TableFusionRule(n={self.provider.n})"

    def dual(self, sector):
        return int(self.provider.dual[int(sector)])


def product(*factors: str, codec: str = "packed") -> FusionRule:
    """``ProductFusionRuleExt::product`` (tenet-sectors/src/product_rule.rs:185-215)."""
    return FusionRule(list(factors), codec)


# ---------------------------------------------------------------------------
# graded spaces
# ---------------------------------------------------------------------------


class GradedSpace:
    """One tensor leg: ``GradedSpace`` / ``SectorLeg`` (tenet-core/src/sector.rs:147-237).

    Sectors are stored sorted by SectorId with zero degeneracies dropped; a
    dual space stores the dualized sectors and a dual flag.
    """

    def __init__(self, rule: FusionRule, pairs, is_dual: bool = False):
        pairs = [(rule.label(s), int(d)) for s, d in (pairs.items() if isinstance(pairs, dict) else pairs)]
        ids = [rule.sector_id(s) for s, _ in pairs]
        if len(set(ids)) != len(ids):
            raise ValueError("sector appears multiple times on one leg")
        if any(d < 0 for _, d in pairs):
            raise ValueError("negative degeneracy")
        order = sorted(range(len(pairs)), key=lambda i: ids[i])
        self.rule = rule
        self._sectors = tuple(pairs[i][0] for i in order if pairs[i][1] != 0)
        self._degs = tuple(pairs[i][1] for i in order if pairs[i][1] != 0)
        self.is_dual = bool(is_dual)

    @staticmethod
    def try_new(rule, pairs):
        return GradedSpace(rule, pairs)

    def sectors(self):
        return [self.rule.unlabel(s) for s in self._sectors]

    def degeneracies(self):
        return list(self._degs)

    def degeneracy(self, sector):
        lab = self.rule.label(sector)
        for s, d in zip(self._sectors, self._degs):
            if s == lab:
                return d
        return 0

    def dual(self) -> "GradedSpace":
        return GradedSpace(
            self.rule, [(self.rule.label(self.rule.dual(self.rule.unlabel(s))), d) for s, d in zip(self._sectors, self._degs)],
            not self.is_dual,
        )

    def dim(self) -> int:
        return int(sum(self.rule.dim(self.rule.unlabel(s)) * d for s, d in zip(self._sectors, self._degs)))

    def reduced_dim(self) -> int:
        return int(sum(self._degs))

    def _key(self):
        return (self.rule, self._sectors, self._degs, self.is_dual)

    def __eq__(self, other):
        return isinstance(other, GradedSpace) and self._key() == other._key()

    def __hash__(self):
        return hash(self._key())

    def __repr__(self):
        inner = ", ".join(f"{self.rule.unlabel(s)}=>{d}" for s, d in zip(self._sectors, self._degs))
        return f"GradedSpace({inner}){'*' if self.is_dual else ''}"


# ---------------------------------------------------------------------------
# hom spaces (block structures)
# ---------------------------------------------------------------------------


class HomSpace:
    """``codomain <- domain`` compiled by the C++ structure compiler."""

    def __init__(self, rule: FusionRule, codomain, domain, handle=None):
        self.rule = rule
        self.codomain = tuple(codomain)
        self.domain = tuple(domain)
        if handle is None:
            legs = list(self.codomain) + list(self.domain)
            for l in legs:
                if l.rule != rule:
                    raise ValueError("legs use different fusion rules")
            nsec = [len(l._sectors) for l in legs]
            labels = [x for l in legs for s in l._sectors for x in s]
            degs = [d for l in legs for d in l._degs]
            dual = [1 if l.is_dual else 0 for l in legs]
            h = C.c_void_p()
            call(
                "tnt_space_create", rule._h, len(self.codomain), len(self.domain), arr(i32, nsec), arr(i32, labels),
                arr(i64, degs), arr(C.c_uint8, dual), C.byref(h),
            )
            handle = h
        self._h = handle
        size, ns, nb, n1, n2 = i64(), i32(), i32(), i32(), i32()
        call("tnt_space_info", self._h, C.byref(size), C.byref(ns), C.byref(nb), C.byref(n1), C.byref(n2))
        self.size, self.nsectors, self.nblocks = size.value, ns.value, nb.value
        self.n1, self.n2 = n1.value, n2.value

    @staticmethod
    def from_handle(rule, handle):
        n1, n2 = i32(), i32()
        call("tnt_space_info", handle, None, None, None, C.byref(n1), C.byref(n2))
        legs = []
        for axis in range(n1.value + n2.value):
            ns = i32()
            call("tnt_space_leg", handle, axis, C.byref(ns), None, None, None)
            labels = (i32 * max(1, ns.value * rule.nfactors))()
            degs = (i64 * max(1, ns.value))()
            dual = C.c_uint8()
            call("tnt_space_leg", handle, axis, C.byref(ns), labels, degs, C.byref(dual))
            nf = rule.nfactors
            pairs = [(tuple(labels[i * nf:(i + 1) * nf]), degs[i]) for i in range(ns.value)]
            legs.append(GradedSpace(rule, pairs, bool(dual.value)))
        return HomSpace(rule, legs[: n1.value], legs[n1.value:], handle=handle)

    def __del__(self):
        _release("tnt_space_destroy", getattr(self, "_h", None))

    def key(self):
        return (self.rule, self.codomain, self.domain)

    def same_as(self, other):
        return self.key() == other.key()

    def sectors(self):
        """``[(coupled label, rows, cols, offset)]`` in storage order."""
        nf = self.rule.nfactors
        labels = (i32 * max(1, self.nsectors * nf))()
        rows, cols, offs = (i64 * max(1, self.nsectors))(), (i64 * max(1, self.nsectors))(), (i64 * max(1, self.nsectors))()
        call("tnt_space_sectors", self._h, labels, rows, cols, offs)
        return [
            (tuple(labels[i * nf:(i + 1) * nf]), rows[i], cols[i], offs[i]) for i in range(self.nsectors)
        ]

    def blocks(self):
        """``[(offset, shape, strides, sector_index)]`` in storage order."""
        r = self.n1 + self.n2
        n = max(1, self.nblocks)
        offs, shapes, strides, sidx = (i64 * n)(), (i64 * (n * max(1, r)))(), (i64 * (n * max(1, r)))(), (i32 * n)()
        call("tnt_space_blocks", self._h, offs, shapes, strides, sidx)
        return [
            (offs[b], tuple(shapes[b * r:(b + 1) * r]), tuple(strides[b * r:(b + 1) * r]), sidx[b])
            for b in range(self.nblocks)
        ]

    def block_keys(self):
        """Block keys: ``((cod uncoupled, cod duals, coupled, cod inner), (dom ...))`` per block."""
        length = i64()
        call("tnt_space_block_keys", self._h, None, 0, C.byref(length))
        buf = (i32 * max(1, length.value))()
        call("tnt_space_block_keys", self._h, buf, length.value, C.byref(length))
        nf = self.rule.nfactors
        out, pos = [], 0

        def tree():
            nonlocal pos
            n = buf[pos]
            pos += 1
            u = tuple(tuple(buf[pos + i * nf: pos + (i + 1) * nf]) for i in range(n))
            pos += n * nf
            d = tuple(bool(buf[pos + i]) for i in range(n))
            pos += n
            c = tuple(buf[pos:pos + nf])
            pos += nf
            ni = max(0, n - 2)
            inner = tuple(tuple(buf[pos + i * nf: pos + (i + 1) * nf]) for i in range(ni))
            pos += ni * nf
            return (u, d, c, inner)

        for _ in range(self.nblocks):
            a = tree()
            b = tree()
            out.append((a, b))
        return out


# ---------------------------------------------------------------------------
# runtime (device context + plan caches)
# ---------------------------------------------------------------------------


class Runtime:
    """Device execution context: ``Runtime::builder().cuda(device)`` (tenet/src/runtime.rs:1031-1275).

    Owns a ``tnt_ctx`` and the compiled-plan caches (the reference's Runtime
    LRU of completed tree-transform structures, tenet-tensors/src/tree_transform/cache.rs:98-123).
    ``precision`` selects the compose arithmetic: ``"fp64"``, ``"bf16x"``
    (split precision with ``slices`` BF16 slices) or ``"cublas"``.
    """

    def __init__(self, device: int = 0, precision: str = "fp64", slices: int = 6, cache_entries: int = 256):
        self.device = device
        self.precision = precision
        self.slices = slices
        self.cache_entries = cache_entries
        h = C.c_void_p()
        call("tnt_ctx_create", device, C.byref(h))
        self._h = h
        self._xplans: Dict = {}
        self._cplans: Dict = {}
        self._fplans: Dict = {}
        self._spaces: Dict = {}

    @staticmethod
    def builder():
        return _RuntimeBuilder()

    def __del__(self):
        for d in (getattr(self, "_xplans", {}), getattr(self, "_cplans", {}), getattr(self, "_fplans", {})):
            d.clear()
        _release("tnt_ctx_destroy", getattr(self, "_h", None))

    def stream(self):
        return C.c_void_p(torch().cuda.current_stream(self.device).cuda_stream)

    def sync(self):
        """Synchronise the current stream; raises if a device-side pipeline wait gave up since the last sync."""
        call("tnt_ctx_sync", self._h, self.stream())

    def space(self, rule, codomain, domain) -> HomSpace:
        key = (rule, tuple(codomain), tuple(domain))
        sp = self._spaces.get(key)
        if sp is None:
            sp = HomSpace(rule, codomain, domain)
            self._spaces[key] = sp
        return sp

    def _evict(self, d):
        while len(d) > self.cache_entries:
            d.pop(next(iter(d)))

    def xplan(self, space: HomSpace, kind: str, p1=(), p2=(), levels=(), nrep=0) -> "TransformPlan":
        key = (space.key(), kind, tuple(p1), tuple(p2), tuple(levels), nrep)
        plan = self._xplans.get(key)
        if plan is None:
            plan = TransformPlan(space, kind, p1, p2, levels, nrep)
            self._xplans[key] = plan
            self._evict(self._xplans)
        return plan

    def cplan(self, lhs: HomSpace, rhs: HomSpace) -> "ComposePlan":
        key = (lhs.key(), rhs.key())
        plan = self._cplans.get(key)
        if plan is None:
            plan = ComposePlan(lhs, rhs)
            self._cplans[key] = plan
            self._evict(self._cplans)
        return plan

    def fplan(self, space: HomSpace) -> "FactorPlan":
        key = space.key()
        plan = self._fplans.get(key)
        if plan is None:
            plan = FactorPlan(space)
            self._fplans[key] = plan
            self._evict(self._fplans)
        return plan


class _RuntimeBuilder:
    def __init__(self):
        self._device = 0
        self._precision = "fp64"
        self._slices = 6

    def cuda(self, device: int):
        self._device = device
        return self

    def gemm_backend(self, precision: str, slices: int = 6):
        self._precision = precision
        self._slices = slices
        return self

    def build(self):
        return Runtime(self._device, self._precision, self._slices)


class TransformPlan:
    def __init__(self, space: HomSpace, kind, p1, p2, levels, nrep):
        h = C.c_void_p()
        if kind == "permute":
            call("tnt_permute_plan", space._h, len(p1), arr(i32, p1), len(p2), arr(i32, p2), C.byref(h))
        elif kind == "braid":
            call("tnt_braid_plan", space._h, len(p1), arr(i32, p1), len(p2), arr(i32, p2), arr(i32, levels), C.byref(h))
        elif kind == "repartition":
            call("tnt_repartition_plan", space._h, nrep, C.byref(h))
        elif kind == "adjoint":
            call("tnt_adjoint_plan", space._h, C.byref(h))
        elif kind == "twist":
            call("tnt_twist_plan", space._h, len(p1), arr(i32, p1), 0, C.byref(h))
        elif kind == "contract_rhs":
            call("tnt_contract_rhs_plan", space._h, len(p1), arr(i32, p1), len(p2), arr(i32, p2), C.byref(h))
        elif kind == "chain":  # p1: the step program, nrep: the step count
            call("tnt_transform_chain_plan", space._h, nrep, arr(i32, p1), len(p1), C.byref(h))
        else:
            raise ValueError(kind)
        self._h = h
        self.src = space
        dh = C.c_void_p()
        call("tnt_xplan_dst_space", h, C.byref(dh))
        self.dst = HomSpace.from_handle(space.rule, dh)
        ng, nc, nb = i64(), i64(), i64()
        call("tnt_xplan_info", h, C.byref(ng), C.byref(nc), C.byref(nb))
        self.ngroups, self.ncoef, self.bytes_moved = ng.value, nc.value, nb.value

    def __del__(self):
        _release("tnt_xplan_destroy", getattr(self, "_h", None))

    @staticmethod
    def from_tables(rank, groups, src_entries, dst_entries, coef, src_size, dst_size) -> "TransformPlan":
        """A plan from tables compiled elsewhere, in the ``export`` layout
        (``tnt_xplan_from_tables``); it has no spaces (``src`` / ``dst`` are None)."""
        g = np.ascontiguousarray(groups, dtype=np.int64).reshape(-1, 14)
        se = np.ascontiguousarray(src_entries, dtype=np.int64).reshape(-1, 9)
        de = np.ascontiguousarray(dst_entries, dtype=np.int64).reshape(-1, 9)
        cf = np.ascontiguousarray(coef, dtype=np.float64).reshape(-1)
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
        h = C.c_void_p()
        call("tnt_xplan_from_tables", int(rank), len(g), P(g, i64), len(se), P(se, i64), len(de), P(de, i64), len(cf),
             P(cf, f64), int(src_size), int(dst_size), C.byref(h))
        plan = TransformPlan.__new__(TransformPlan)
        plan._h = h
        plan.src = plan.dst = None
        ng, nc, nb = i64(), i64(), i64()
        call("tnt_xplan_info", h, C.byref(ng), C.byref(nc), C.byref(nb))
        plan.ngroups, plan.ncoef, plan.bytes_moved = ng.value, nc.value, nb.value
        return plan

    def export(self):
        """Compiled tables as numpy arrays (groups, src entries, dst entries, coefficients)."""
        ns, nd = i64(), i64()
        call("tnt_xplan_entries", self._h, C.byref(ns), C.byref(nd))
        g = np.zeros((self.ngroups, 14), dtype=np.int64)
        s = np.zeros((max(1, ns.value), 9), dtype=np.int64)
        d = np.zeros((max(1, nd.value), 9), dtype=np.int64)
        c = np.zeros(max(1, self.ncoef), dtype=np.float64)
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
        call("tnt_xplan_export", self._h, P(g, i64), P(s, i64), P(d, i64), P(c, f64))
        return g, s[: ns.value], d[: nd.value], c[: self.ncoef]


class ComposePlan:
    def __init__(self, lhs: HomSpace, rhs: HomSpace):
        h = C.c_void_p()
        call("tnt_compose_plan", lhs._h, rhs._h, C.byref(h))
        self._h = h
        dh = C.c_void_p()
        call("tnt_cplan_dst_space", h, C.byref(dh))
        self.dst = HomSpace.from_handle(lhs.rule, dh)
        nj, fl = i64(), f64()
        call("tnt_cplan_info", h, C.byref(nj), C.byref(fl))
        self.njobs, self.flops = nj.value, fl.value

    def __del__(self):
        _release("tnt_cplan_destroy", getattr(self, "_h", None))

    def export(self):
        j = np.zeros((max(1, self.njobs), 9), dtype=np.int64)
        call("tnt_cplan_export", self._h, j.ctypes.data_as(C.POINTER(i64)))
        return j[: self.njobs]

    @property
    def suits_split(self) -> bool:
        """True when most of the plan's flops sit in products with K >= 32.

        Split precision pads K to 64-deep digit blocks, so a thinner product
        (an MPO or gate contraction over a physical leg, K of 1 to 4) would
        move many times its operand bytes in digit packs for no tensor-core
        gain; callers run such plans in FP64."""
        if not hasattr(self, "_suits_split"):
            j = self.export().astype(np.float64)
            fl = 2.0 * j[:, 0] * j[:, 1] * j[:, 2]
            self._suits_split = bool(fl.sum() > 0 and fl[j[:, 2] >= 32].sum() >= 0.5 * fl.sum())
        return self._suits_split


class FactorPlan:
    def __init__(self, space: HomSpace):
        h = C.c_void_p()
        call("tnt_factor_plan", space._h, C.byref(h))
        self._h = h
        self.space = space
        ns, us, ss, vs = i32(), i64(), i64(), i64()
        call("tnt_fplan_info", h, C.byref(ns), C.byref(us), C.byref(ss), C.byref(vs))
        self.nsectors, self.u_size, self.s_size, self.v_size = ns.value, us.value, ss.value, vs.value
        rec = np.zeros((max(1, self.nsectors), 8), dtype=np.int64)
        w = np.zeros(max(1, self.nsectors), dtype=np.float64)
        call("tnt_fplan_export", h, rec.ctypes.data_as(C.POINTER(i64)), w.ctypes.data_as(C.POINTER(f64)))
        self.records = rec[: self.nsectors]
        self.weights = w[: self.nsectors]
        we = i64()
        call("tnt_fplan_work", h, C.byref(we))
        self.work_elems = we.value

    def __del__(self):
        _release("tnt_fplan_destroy", getattr(self, "_h", None))


# ---------------------------------------------------------------------------
# truncation policies
# ---------------------------------------------------------------------------


@dataclass
class Truncation:
    """``Truncation`` (tenet-matrixalgebra/src/truncation.rs:69-93)."""

    policy: int
    p0: float = 0.0
    p1: float = 0.0
    ranks: Optional[Dict] = None

    @staticmethod
    def full():
        return Truncation(_lib.TRUNC_FULL)

    @staticmethod
    def rank(n: int):
        return Truncation(_lib.TRUNC_RANK, float(n))

    @staticmethod
    def tolerance(atol: float = 0.0, rtol: float = 0.0):
        return Truncation(_lib.TRUNC_TOL, float(atol), float(rtol))

    @staticmethod
    def discard_weight(rtol: float):
        return Truncation(_lib.TRUNC_DISCARD, float(rtol))

    @staticmethod
    def space(profile):
        """``Truncation::space`` over a GradedSpace (``truncspace``) or a {sector: rank} map."""
        if isinstance(profile, GradedSpace):
            ranks = {s: d for s, d in zip(profile._sectors, profile._degs)}
        else:
            ranks = {tuple(k) if not isinstance(k, int) else (k,): int(v) for k, v in profile.items()}
        return Truncation(_lib.TRUNC_SPACE, ranks=ranks)


# ---------------------------------------------------------------------------
# tensor maps
# ---------------------------------------------------------------------------


class TensorMap:
    """Device-resident block-sparse ``TensorMap`` (tenet/src/typed.rs:9044-9047, CUDA placement)."""

    def __init__(self, runtime: Runtime, space: HomSpace, data=None):
        t = torch()
        self.runtime = runtime
        self.space = space
        if data is None:
            data = t.zeros(space.size, dtype=t.float64, device=f"cuda:{runtime.device}")
        if data.dtype != t.float64 or data.numel() != space.size or not data.is_cuda:
            raise ValueError("payload must be a CUDA float64 tensor of the space size")
        self.data = data.contiguous()

    # -- construction ---------------------------------------------------------
    @staticmethod
    def zeros(runtime, codomain, domain):
        rule = (list(codomain) + list(domain))[0].rule
        return TensorMap(runtime, runtime.space(rule, codomain, domain))

    @staticmethod
    def from_host(runtime, codomain, domain, values):
        rule = (list(codomain) + list(domain))[0].rule
        sp = runtime.space(rule, codomain, domain)
        t = torch()
        data = t.as_tensor(np.ascontiguousarray(values, dtype=np.float64)).to(f"cuda:{runtime.device}")
        return TensorMap(runtime, sp, data)

    @staticmethod
    def from_block_fn(runtime, codomain, domain, fn):
        """``TensorMap::from_block_fn`` (typed.rs:12262): ``fn(block_key, idx)`` per element."""
        rule = (list(codomain) + list(domain))[0].rule
        sp = runtime.space(rule, codomain, domain)
        host = np.zeros(sp.size)
        for (off, shape, strides, _), key in zip(sp.blocks(), sp.block_keys()):
            for idx in itertools.product(*[range(s) for s in shape]):
                host[off + sum(i * s for i, s in zip(idx, strides))] = fn(key, idx)
        return TensorMap.from_host(runtime, codomain, domain, host)

    def to_host(self) -> np.ndarray:
        return self.data.detach().cpu().numpy()

    @property
    def rule(self):
        return self.space.rule

    def codomain(self):
        return list(self.space.codomain)

    def domain(self):
        return list(self.space.domain)

    # -- recoupling ---------------------------------------------------------------
    def _apply(self, plan: TransformPlan):
        out = TensorMap(self.runtime, plan.dst)
        call(
            "tnt_transform", self.runtime._h, plan._h, C.c_void_p(out.data.data_ptr()),
            C.c_void_p(self.data.data_ptr()), 1.0, 0.0, self.runtime.stream(),
        )
        return out

    def permute(self, codomain_axes, domain_axes):
        """``TensorMap::permute`` (typed.rs:13163): identity returns a copy."""
        n1, n2 = self.space.n1, self.space.n2
        if list(codomain_axes) == list(range(n1)) and list(domain_axes) == list(range(n1, n1 + n2)):
            return TensorMap(self.runtime, self.space, self.data.clone())
        return self._apply(self.runtime.xplan(self.space, "permute", codomain_axes, domain_axes))

    def braid(self, codomain_axes, domain_axes, levels):
        if len(levels) != self.space.n1 + self.space.n2:
            raise ValueError("braid levels must list one level per source axis")
        return self._apply(self.runtime.xplan(self.space, "braid", codomain_axes, domain_axes, levels))

    def repartition(self, num_codomain):
        if num_codomain == self.space.n1:
            return TensorMap(self.runtime, self.space, self.data.clone())
        return self._apply(self.runtime.xplan(self.space, "repartition", nrep=num_codomain))

    def adjoint(self):
        """Materialised adjoint: block(t', c) = block(t, c)^T (real payloads)."""
        return self._apply(self.runtime.xplan(self.space, "adjoint"))

    def twist(self, legs):
        """``TensorMap::twist`` (typed.rs:4599): each block times the product of
        the ribbon twists of its uncoupled sectors on ``legs`` (flat axes,
        codomain first).  A rule without a fermion-parity factor returns a copy."""
        n = self.space.n1 + self.space.n2
        for a in legs:
            if not 0 <= a < n:
                raise ValueError(f"twist leg {a} out of range for rank {n}")
        if not legs or "FZ2" not in self.rule.factors:
            return TensorMap(self.runtime, self.space, self.data.clone())
        return self._apply(self.runtime.xplan(self.space, "twist", list(legs)))

    def transform_chain(self, steps):
        """Several recoupling steps in one device pass (``tnt_transform_chain_plan``).

        ``steps``: ``("permute", codomain, domain)``, ``("braid", codomain,
        domain, levels)``, ``("repartition", n)``, ``("adjoint",)`` or
        ``("twist", legs)``, each applied to the previous step's result; the
        result equals applying them one by one, with one read and one write of
        the payload instead of one per step.
        """
        prog = []
        for st in steps:
            kind = st[0]
            if kind in ("permute", "braid"):
                prog += [0 if kind == "permute" else 1, len(st[1]), *st[1], len(st[2]), *st[2]]
                if kind == "braid":
                    prog += list(st[3])
            elif kind == "repartition":
                prog += [2, int(st[1])]
            elif kind == "adjoint":
                prog += [3]
            elif kind == "twist":
                prog += [4, len(st[1]), *st[1]]
            else:
                raise ValueError(f"unknown step {kind!r}")
        if not steps:
            return TensorMap(self.runtime, self.space, self.data.clone())
        return self._apply(self.runtime.xplan(self.space, "chain", tuple(prog), (), (), len(steps)))

    def twist_inverse(self, legs):
        """``TensorMap::twist_inverse`` (typed.rs:4604); the twists in scope are +-1."""
        return self.twist(legs)

    # -- contraction --------------------------------------------------------------
    def compose(self, other: "TensorMap", precision: Optional[str] = None, slices: Optional[int] = None):
        """``TensorMap::compose`` (typed.rs:13842): one GEMM per coupled sector."""
        plan = self.runtime.cplan(self.space, other.space)
        out = TensorMap(self.runtime, plan.dst)
        prec = {"fp64": _lib.PREC_FP64, "bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X,
                "cublas": _lib.PREC_CUBLAS_FP64}[
            precision or self.runtime.precision
        ]
        call(
            "tnt_compose", self.runtime._h, plan._h, 1, C.c_void_p(out.data.data_ptr()), plan.dst.size,
            C.c_void_p(self.data.data_ptr()), self.space.size, C.c_void_p(other.data.data_ptr()), other.space.size,
            1.0, 0.0, prec, slices or self.runtime.slices, self.runtime.stream(),
        )
        return out

    def pack_split(self, partner_space: "HomSpace", side: int, slices: int) -> "PackedOperand":
        """This tensor's 8-bit digit packs for composes with tensors of
        ``partner_space``: as the left operand (side 0) or the right one
        (side 1).  A constant operand of many composes (an environment across
        Lanczos iterations) is then sliced once."""
        lhs, rhs = (self.space, partner_space) if side == 0 else (partner_space, self.space)
        plan = self.runtime.cplan(lhs, rhs)
        nb = C.c_size_t()
        call("tnt_split_operand_bytes", plan._h, side, _lib.PREC_INT8X, slices, C.byref(nb))
        buf = torch().empty(max(1, nb.value), dtype=torch().uint8, device=self.data.device)
        call("tnt_split_pack_operand", self.runtime._h, plan._h, side, C.c_void_p(self.data.data_ptr()),
             _lib.PREC_INT8X, slices, C.c_void_p(buf.data_ptr()), nb.value, self.runtime.stream())
        return PackedOperand(self, plan, side, slices, buf)

    def compose_packed(self, other, slices: int):
        """``compose`` with 8-bit digits where ``self`` or ``other`` is a
        PackedOperand of this plan (bit-identical to ``compose(..., "i8x")``)."""
        lhs = self.tensor if isinstance(self, PackedOperand) else self
        rhs = other.tensor if isinstance(other, PackedOperand) else other
        plan = lhs.runtime.cplan(lhs.space, rhs.space)
        for p_ in (self, other):
            if isinstance(p_, PackedOperand) and (p_.plan is not plan or p_.slices != slices):
                raise ValueError("packed operand made for another plan or digit count")
        out = TensorMap(lhs.runtime, plan.dst)
        ptr = lambda t: C.c_void_p(t.data_ptr())
        lp = ptr(self.buf) if isinstance(self, PackedOperand) else None
        rp = ptr(other.buf) if isinstance(other, PackedOperand) else None
        call("tnt_compose_packed", lhs.runtime._h, plan._h, ptr(out.data), None if lp else ptr(lhs.data), lp,
             None if rp else ptr(rhs.data), rp, 1.0, 0.0, _lib.PREC_INT8X, slices, lhs.runtime.stream())
        return out

    def contract(self, other: "TensorMap", lhs_axes, rhs_axes, output_axes):
        """``TensorMap::contract`` (typed.rs:13653).

        Lowered as the reference's DynamicTree resolution
        (tenet-tensors/src/contract/dynamic.rs:330-390): permute ``self`` to
        (open ; contracted), ``other`` to (contracted ; open) with the fermionic
        supertrace twist on its dual contracted legs folded into the same
        transform, compose, and permute the result by ``output_axes``; the
        result's codomain is every open axis of ``self`` and its domain every
        open axis of ``other``.
        """
        ra, rb = self.space.n1 + self.space.n2, other.space.n1 + other.space.n2
        open_a = [i for i in range(ra) if i not in lhs_axes]
        open_b = [i for i in range(rb) if i not in rhs_axes]
        a = self.permute(open_a, list(lhs_axes))
        b = other._apply(self.runtime.xplan(other.space, "contract_rhs", list(rhs_axes), open_b))
        c = a.compose(b)
        na = len(open_a)
        out_axes = list(output_axes)
        if out_axes == list(range(na + len(open_b))):
            return c
        return c.permute(out_axes[:na], out_axes[na:])

    # -- reductions (TensorKit semantics) ------------------------------------
    def _sector_weights(self):
        t = torch()
        w = np.zeros(self.space.size)
        for lab, r, c, off in self.space.sectors():
            w[off:off + r * c] = self.rule.dim(self.rule.unlabel(lab))
        return t.as_tensor(w, device=self.data.device)

    def norm(self) -> float:
        return float(torch().sqrt(torch().sum(self._sector_weights() * self.data * self.data)))

    def tr(self) -> float:
        s = 0.0
        for lab, r, c, off in self.space.sectors():
            blk = self.data[off:off + r * c].view(c, r)
            s += self.rule.dim(self.rule.unlabel(lab)) * float(torch().trace(blk))
        return s

    def add(self, other, alpha=1.0, beta=1.0):
        if not self.space.same_as(other.space):
            raise ValueError("add: spaces differ")
        return TensorMap(self.runtime, self.space, alpha * self.data + beta * other.data)

    # -- factorisation ------------------------------------------------------------
    def svd_compact(self):
        return self.svd_trunc(Truncation.full())

    def svd_trunc(self, truncation: Truncation):
        """``TensorMap::svd_trunc`` (typed.rs:1806): device SVD + device truncation."""
        t = torch()
        rt = self.runtime
        plan = rt.fplan(self.space)
        dev = self.data.device
        u = t.empty(max(1, plan.u_size), dtype=t.float64, device=dev)
        s = t.empty(max(1, plan.s_size), dtype=t.float64, device=dev)
        vh = t.empty(max(1, plan.v_size), dtype=t.float64, device=dev)
        call("tnt_svd", rt._h, plan._h, C.c_void_p(self.data.data_ptr()), C.c_void_p(u.data_ptr()),
             C.c_void_p(s.data_ptr()), C.c_void_p(vh.data_ptr()), rt.stream())
        kept_d = t.empty(max(1, plan.nsectors), dtype=t.int64, device=dev)
        err_d = t.empty(1, dtype=t.float64, device=dev)
        ranks = None
        sectors = self.space.sectors()
        if truncation.policy == _lib.TRUNC_SPACE:
            ranks = arr(i64, [truncation.ranks.get(lab, 0) for lab, _, _, _ in sectors])
        call("tnt_truncate", rt._h, plan._h, C.c_void_p(s.data_ptr()), truncation.policy, truncation.p0,
             truncation.p1, ranks, C.c_void_p(kept_d.data_ptr()), C.c_void_p(err_d.data_ptr()), rt.stream())
        return SvdResult(self, plan, u, s, vh, kept_d, err_d)


    def qr_compact(self):
        """``TensorMap::qr_compact`` (typed.rs:1393): ``self = Q o R`` per coupled sector on the device.

        Q : codomain <- W is an isometry, R : W <- domain is upper trapezoidal
        with a non-negative diagonal; W carries min(rows, cols) per sector.
        """
        t = torch()
        rt = self.runtime
        plan = rt.fplan(self.space)
        dev = self.data.device
        q = t.empty(max(1, plan.u_size), dtype=t.float64, device=dev)
        r = t.empty(max(1, plan.v_size), dtype=t.float64, device=dev)
        call("tnt_qr", rt._h, plan._h, C.c_void_p(self.data.data_ptr()), C.c_void_p(q.data_ptr()),
             C.c_void_p(r.data_ptr()), rt.stream())
        ranks = [int(rec[2]) for rec in plan.records]
        return _bond_factors(self, plan, ranks, q, r)

    def lq_compact(self):
        """``TensorMap::lq_compact`` (typed.rs:1494): ``self = L o Q`` per coupled sector on the device.

        L : codomain <- W is lower trapezoidal with a non-negative diagonal, Q :
        W <- domain has orthonormal rows; W carries min(rows, cols) per sector.
        Computed as the adjoint of the QR of the adjoint (two fused transform
        passes around one batched QR): self^T = Q' R' gives L = R'^T, Q = Q'^T.
        """
        q, r = self.adjoint().qr_compact()
        return r.adjoint(), q.adjoint()

    def left_orth(self):
        """``TensorMap::left_orth`` (TensorKit's default ``:qr``): ``qr_compact``."""
        return self.qr_compact()

    def right_orth(self):
        """``TensorMap::right_orth`` (typed.rs:1507, TensorKit's default ``:lq``): ``lq_compact``."""
        return self.lq_compact()

    def eigh_full(self):
        """``TensorMap::eigh_full`` (typed.rs:1884): ``(d, v)`` with ``self = v d v^dagger``."""
        res = self.eigh_trunc(Truncation.full())
        return res.factors()

    def eigh_trunc(self, truncation: Truncation):
        """``TensorMap::eigh_trunc`` (typed.rs:1907): device eigh + truncation on |lambda| on the device."""
        t = torch()
        rt = self.runtime
        if list(self.space.codomain) != list(self.space.domain):
            raise ValueError("eigh requires an endomorphism (codomain == domain)")
        plan = rt.fplan(self.space)
        dev = self.data.device
        vecs = t.empty(max(1, plan.u_size), dtype=t.float64, device=dev)
        vals = t.empty(max(1, plan.s_size), dtype=t.float64, device=dev)
        mags = t.empty(max(1, plan.s_size), dtype=t.float64, device=dev)
        call("tnt_eigh", rt._h, plan._h, C.c_void_p(self.data.data_ptr()), C.c_void_p(vecs.data_ptr()),
             C.c_void_p(vals.data_ptr()), C.c_void_p(mags.data_ptr()), rt.stream())
        kept_d = t.empty(max(1, plan.nsectors), dtype=t.int64, device=dev)
        err_d = t.empty(1, dtype=t.float64, device=dev)
        ranks = None
        if truncation.policy == _lib.TRUNC_SPACE:
            ranks = arr(i64, [truncation.ranks.get(lab, 0) for lab, _, _, _ in self.space.sectors()])
        call("tnt_truncate", rt._h, plan._h, C.c_void_p(mags.data_ptr()), truncation.policy, truncation.p0,
             truncation.p1, ranks, C.c_void_p(kept_d.data_ptr()), C.c_void_p(err_d.data_ptr()), rt.stream())
        return EighResult(self, plan, vecs, vals, kept_d, err_d)


def _bond_factors(src: "TensorMap", plan: "FactorPlan", ranks, left, right):
    """Left factor (codomain <- W) and right factor (W <- domain) over the bond W
    with ``ranks[i]`` states in coupled sector i, cut from the plan's U / Vh
    layouts (column-major m x k and k x n per sector, leading columns / rows kept)."""
    rt = src.runtime
    rule = src.rule
    sectors = src.space.sectors()
    bond = GradedSpace(rule, [(lab, k) for (lab, _, _, _), k in zip(sectors, ranks) if k > 0])
    L = TensorMap.zeros(rt, src.space.codomain, [bond])
    R = TensorMap.zeros(rt, [bond], src.space.domain)
    lsec = {lab: off for lab, _, _, off in L.space.sectors()}
    rsec = {lab: off for lab, _, _, off in R.space.sectors()}
    for (lab, m, n, _), rec, k in zip(sectors, plan.records, ranks):
        if k == 0:
            continue
        kk = int(rec[2])
        L.data[lsec[lab]: lsec[lab] + m * k] = left[rec[4]: rec[4] + m * k]
        full = right[rec[6]: rec[6] + kk * n].view(n, kk)  # column-major kk x n
        R.data[rsec[lab]: rsec[lab] + k * n] = full[:, :k].contiguous().view(-1)
    return L, R


@dataclass
class SpectrumEntry:
    sector: object
    values: np.ndarray


class SvdResult:
    """Truncated SVD factors: ``u`` (codomain <- bond), ``s`` per sector, ``vh`` (bond <- domain)."""

    def __init__(self, src: TensorMap, plan: FactorPlan, u, s, vh, kept_d, err_d):
        self._src, self._plan = src, plan
        self._u, self._s, self._vh = u, s, vh
        self.kept = [int(x) for x in kept_d.cpu().numpy()[: plan.nsectors]]
        self.error = float(err_d.cpu().numpy()[0])
        s_host = s.cpu().numpy()
        self.singular_values = []
        rule = src.rule
        for (lab, r, c, off), rec, k in zip(src.space.sectors(), plan.records, self.kept):
            self.singular_values.append(SpectrumEntry(rule.unlabel(lab), s_host[rec[5]: rec[5] + k].copy()))

    def bond_space(self) -> GradedSpace:
        rule = self._src.rule
        return GradedSpace(rule, [(lab, k) for (lab, _, _, _), k in zip(self._src.space.sectors(), self.kept)])

    def factors(self):
        """Materialise ``(U, S-values, Vh)`` as TensorMaps over the kept bond space."""
        U, Vh = _bond_factors(self._src, self._plan, self.kept, self._u, self._vh)
        return U, self.singular_values, Vh


class EighResult:
    """Truncated eigendecomposition: kept eigenvalues per sector (signed, descending |lambda|),
    the eigenvector isometry ``v`` (codomain <- W) and the diagonal ``d`` (W <- W)."""

    def __init__(self, src: TensorMap, plan: FactorPlan, vecs, vals, kept_d, err_d):
        self._src, self._plan = src, plan
        self._vecs, self._vals = vecs, vals
        self.kept = [int(x) for x in kept_d.cpu().numpy()[: plan.nsectors]]
        self.error = float(err_d.cpu().numpy()[0])
        v_host = vals.cpu().numpy()
        rule = src.rule
        self.eigenvalues = []
        for (lab, _, _, _), rec, k in zip(src.space.sectors(), plan.records, self.kept):
            if k > 0:
                self.eigenvalues.append(SpectrumEntry(rule.unlabel(lab), v_host[rec[5]: rec[5] + k].copy()))

    def factors(self):
        """``(d, v)``: the diagonal of kept eigenvalues and the kept eigenvectors."""
        t = torch()
        src, plan = self._src, self._plan
        V, _ = _bond_factors(src, plan, self.kept, self._vecs, t.zeros(max(1, plan.v_size), dtype=t.float64,
                                                                         device=self._vecs.device))
        bond = V.space.domain
        D = TensorMap.zeros(src.runtime, bond, bond)
        dsec = {lab: (r, off) for lab, r, _, off in D.space.sectors()}
        for (lab, _, _, _), rec, k in zip(src.space.sectors(), plan.records, self.kept):
            if k == 0:
                continue
            r, off = dsec[lab]
            D.data[off: off + r * r].view(r, r).diagonal().copy_(self._vals[rec[5]: rec[5] + k])
        return D, V


class PackedOperand:
    """A tensor's 8-bit digit packs for one compose plan and side (``TensorMap.pack_split``)."""

    def __init__(self, tensor, plan, side, slices, buf):
        self.tensor, self.plan, self.side, self.slices, self.buf = tensor, plan, side, slices, buf

    def compose_packed(self, other, slices):
        return TensorMap.compose_packed(self, other, slices)
