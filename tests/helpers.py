"""Shared test helpers: oracle <-> product conversions and a numpy replay of plan tables."""

from __future__ import annotations

import numpy as np

from oracle.fusion import Leg as OLeg
from oracle.sectors import Rule as ORule

FACTOR_NAMES = {"U1": "U1", "SU2": "SU2", "FZ2": "FZ2", "Z2": "Z2"}


_TABLE_RULES = {}


def product_rule(orule: ORule):
    """The device rule of an oracle rule (a table rule maps to the
    TableFusionRule of the same provider tables, made once)."""
    from tenet_b200 import typed

    if orule.factors == ("TABLE",):
        if id(orule) not in _TABLE_RULES:
            _TABLE_RULES[id(orule)] = (orule, typed.TableFusionRule(orule.provider))
        return _TABLE_RULES[id(orule)][1]
    return typed.FusionRule([FACTOR_NAMES[f] for f in orule.factors], orule.codec)


def table_rules(provider):
    """(oracle rule, device rule) over one provider's tables."""
    from oracle.sectors import TableRule

    p = provider
    orule = TableRule(p.dual, p.nsym, p.dims, p.fs, p.rsym, p.fsym)
    orule.provider = p
    return orule, product_rule(orule)


def product_leg(rule, oleg: OLeg):
    from tenet_b200 import typed

    return typed.GradedSpace(rule, list(zip(oleg.sectors, oleg.degeneracies)), oleg.is_dual)


def product_space(orule, ocod, odom):
    from tenet_b200 import typed

    rule = product_rule(orule)
    return typed.HomSpace(rule, [product_leg(rule, l) for l in ocod], [product_leg(rule, l) for l in odom])


def replay_transform(tables, src: np.ndarray, dst_size: int) -> np.ndarray:
    """Apply exported transform tables on the CPU (reference semantics of the kernel)."""
    groups, s_e, d_e, coef = tables
    dst = np.zeros(dst_size)
    for g in groups:
        nelem, nsrc, ndst, sf, df, co = (int(x) for x in g[:6])
        dims = [int(x) for x in g[6:14]]
        multi = np.unravel_index(np.arange(nelem), dims, order="F")

        def pos(entry):
            p = np.full(nelem, entry[0], dtype=np.int64)
            for k in range(8):
                p += multi[k].astype(np.int64) * entry[1 + k]
            return p

        if nsrc == 0:
            for d in range(ndst):
                dst[pos(d_e[df + d])] = 0.0
            continue
        U = coef[co: co + ndst * nsrc].reshape(ndst, nsrc)
        S = np.stack([src[pos(s_e[sf + s])] for s in range(nsrc)])
        D = U @ S
        for d in range(ndst):
            dst[pos(d_e[df + d])] = D[d]
    return dst


def replay_compose(jobs, a, b, c_size):
    c = np.zeros(c_size)
    for m, n, k, ao, bo, co, lda, ldb, ldc in jobs:
        if m == 0 or n == 0:
            continue
        if k == 0:
            continue
        A = a[ao: ao + lda * k].reshape(k, lda).T[:m]
        B = b[bo: bo + ldb * n].reshape(n, ldb).T[:k]
        c[co: co + ldc * n].reshape(n, ldc).T[:m][:] = A @ B
    return c
