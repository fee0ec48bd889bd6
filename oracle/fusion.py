"""Graded legs, fusion-tree enumeration and coupled-sector block layout (oracle).

Test infrastructure only; see ``oracle/__init__.py``.

A fusion tree is a tuple ``(uncoupled, is_dual, coupled, inner)`` where
``inner`` lists the inner lines innermost-first, exactly the field layout of
``FusionTreeKey`` (tenet-core/src/fusion_tree.rs:1225).  For uncoupled
``(u0, ..., u_{n-1})`` the tree fuses ``u0 x u1 -> inner[0]``,
``inner[0] x u2 -> inner[1]`` ... ``inner[n-3] x u_{n-1} -> coupled``.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import reduce

import numpy as np


@dataclass(frozen=True)
class Leg:
    """One tensor axis: ``SectorLeg`` (tenet-core/src/sector.rs:80-197).

    ``sectors`` holds the labels *as stored* (already dualized for a dual
    leg), sorted by SectorId with zero degeneracies dropped.
    """

    rule: object
    sectors: tuple
    degeneracies: tuple
    is_dual: bool = False

    @staticmethod
    def new(rule, pairs, is_dual=False):
        """``SectorLeg::try_new`` (sector.rs:147-197): sort by id, drop zeros."""
        pairs = sorted(((tuple(s), int(d)) for s, d in pairs), key=lambda p: rule.sector_id(p[0]))
        ids = [rule.sector_id(s) for s, _ in pairs]
        if len(set(ids)) != len(ids):
            raise ValueError("duplicate sector")
        kept = [(s, d) for s, d in pairs if d != 0]
        return Leg(rule, tuple(s for s, _ in kept), tuple(d for _, d in kept), is_dual)

    def dual(self):
        """``SectorLeg::dual`` (sector.rs:226-237)."""
        r = self.rule
        return Leg.new(r, [(r.dual(s), d) for s, d in zip(self.sectors, self.degeneracies)], not self.is_dual)

    def degeneracy(self, sector):
        for s, d in zip(self.sectors, self.degeneracies):
            if s == sector:
                return d
        return 0

    def dim(self):
        return int(sum(self.rule.dim(s) * d for s, d in zip(self.sectors, self.degeneracies)))

    def reduced_dim(self):
        return int(sum(self.degeneracies))


def _leg_tuples(legs):
    """``try_visit_selected_leg_tuples`` (fusion_tree.rs:491-510): first leg fastest."""
    n = len(legs)
    if n == 0:
        yield ()
        return
    # recursion peels the last leg in the outermost loop
    def rec(remaining, current):
        if remaining == 0:
            yield tuple(current)
            return
        idx = remaining - 1
        for s in legs[idx].sectors:
            current[idx] = s
            yield from rec(remaining - 1, current)

    yield from rec(n, [None] * n)


def _reachable_coupled(rule, effective):
    """``reachable_coupled_sectors`` (fusion_tree.rs:970-990)."""
    if not effective:
        return [rule.vacuum()]
    acc = {effective[0]}
    for last in effective[1:]:
        nxt = set()
        for front in acc:
            nxt.update(rule.fusion_channels(front, last))
        acc = nxt
    return sorted(acc, key=rule.sector_id)


def _visit_trees(rule, effective, coupled, inner_rev, out):
    """``visit_fusion_trees_where`` / ``try_visit_fusion_trees_checked`` (fusion_tree.rs:699-750, 1076-1130)."""
    n = len(effective)
    if n == 0:
        if coupled == rule.vacuum():
            out.append(tuple(reversed(inner_rev)))
        return
    if n == 1:
        if effective[0] == coupled:
            out.append(tuple(reversed(inner_rev)))
        return
    if n == 2:
        if rule.nsymbol(effective[0], effective[1], coupled):
            out.append(tuple(reversed(inner_rev)))
        return
    last = effective[-1]
    for front in rule.fusion_channels(coupled, rule.dual(last)):
        if not rule.nsymbol(front, last, coupled):
            continue
        inner_rev.append(front)
        _visit_trees(rule, effective[:-1], front, inner_rev, out)
        inner_rev.pop()


def trees_by_coupled(rule, legs):
    """``fusion_trees_by_coupled_for_space`` (fusion_tree.rs:512-560).

    Returns ``[(coupled, [tree, ...]), ...]`` sorted by coupled SectorId;
    within a group trees follow leg-tuple order, then inner-line order.
    """
    groups = {}
    order = []
    is_dual = tuple(l.is_dual for l in legs)
    for tup in _leg_tuples(legs):
        for coupled in _reachable_coupled(rule, list(tup)):
            inners = []
            _visit_trees(rule, list(tup), coupled, [], inners)
            trees = [(tup, is_dual, coupled, inner) for inner in inners]
            if coupled not in groups:
                groups[coupled] = []
                order.append(coupled)
            groups[coupled].extend(trees)
    return sorted(((c, groups[c]) for c in order), key=lambda g: rule.sector_id(g[0]))


class HomSpace:
    """``codomain <- domain`` with its coupled-sector column-major layout.

    Layout follows ``fusion_tree_layout_data_from_groups``
    (tenet-core/src/fusion_space.rs:2211-2262: keys domain-major inside a
    sector) and ``coupled_sector_matrix_block_specs_after_dimension_validation``
    (fusion_space.rs:3953-4104: one r_C x r_D column-major matrix per coupled
    sector, sectors in ascending SectorId order; block strides
    ``1, d0, d0 d1 ...`` over codomain axes and ``r_C, r_C d_n1 ...`` over
    domain axes; offset = sector_off + row_start + r_C * col_start).
    """

    def __init__(self, rule, codomain, domain):
        self.rule = rule
        self.codomain = tuple(codomain)
        self.domain = tuple(domain)
        self.n1 = len(self.codomain)
        self.n2 = len(self.domain)
        cod_groups = dict(trees_by_coupled(rule, self.codomain))
        dom_groups = dict(trees_by_coupled(rule, self.domain))
        coupled = sorted(set(cod_groups) & set(dom_groups), key=rule.sector_id)
        self.sectors = []  # (coupled, rows, cols, offset)
        self.blocks = []  # dicts: key, shape, strides, offset, sector index
        self.block_index = {}
        self.row_trees = {}
        self.col_trees = {}
        offset = 0
        for c in coupled:
            rtrees = cod_groups[c]
            ctrees = dom_groups[c]
            if not rtrees or not ctrees:
                continue
            rstarts, r = [], 0
            for t in rtrees:
                rstarts.append(r)
                r += self._tree_dim(self.codomain, t)
            cstarts, cc = [], 0
            for t in ctrees:
                cstarts.append(cc)
                cc += self._tree_dim(self.domain, t)
            sidx = len(self.sectors)
            self.sectors.append((c, r, cc, offset))
            self.row_trees[c] = list(zip(rtrees, rstarts))
            self.col_trees[c] = list(zip(ctrees, cstarts))
            for dt, cs in zip(ctrees, cstarts):
                for ct, rs in zip(rtrees, rstarts):
                    shape = tuple(self._shape(self.codomain, ct) + self._shape(self.domain, dt))
                    strides = []
                    s = 1
                    for d in shape[: self.n1]:
                        strides.append(s)
                        s *= d
                    s = r
                    for d in shape[self.n1 :]:
                        strides.append(s)
                        s *= d
                    key = (ct, dt)
                    self.block_index[key] = len(self.blocks)
                    self.blocks.append(
                        dict(key=key, shape=shape, strides=tuple(strides), offset=offset + rs + r * cs, sector=sidx)
                    )
            offset += r * cc
        self.size = offset

    @staticmethod
    def _shape(legs, tree):
        return [leg.degeneracy(s) for leg, s in zip(legs, tree[0])]

    @classmethod
    def _tree_dim(cls, legs, tree):
        return int(reduce(lambda x, y: x * y, cls._shape(legs, tree), 1))

    def sector_of(self, c):
        for i, s in enumerate(self.sectors):
            if s[0] == c:
                return i
        return None

    def block_view(self, data, b):
        """Strided view of block ``b`` inside flat ``data``."""
        blk = self.blocks[b]
        item = data.itemsize
        return np.lib.stride_tricks.as_strided(
            data[blk["offset"] :],
            shape=blk["shape"],
            strides=tuple(s * item for s in blk["strides"]),
            writeable=True,
        )

    def sector_matrix(self, data, i):
        c, r, cc, off = self.sectors[i]
        return data[off : off + r * cc].reshape((cc, r)).T

    def same_as(self, other):
        return (
            self.rule == other.rule
            and self.codomain == other.codomain
            and self.domain == other.domain
        )
