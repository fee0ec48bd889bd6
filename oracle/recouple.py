"""Fusion-tree-pair recoupling: Artin braids, bends, repartition, permute (oracle).

Test infrastructure only; see ``oracle/__init__.py``.

Trees are ``(uncoupled, is_dual, coupled, inner)`` tuples (see
``oracle/fusion.py``); a tree pair is ``(codomain_tree, domain_tree)``.  Each
operation returns a list of ``(tree_pair, coefficient)`` terms.
"""

from __future__ import annotations


class _Acc:
    """``FusionTermAccumulator`` (fusion_tree.rs:3888-3980): merge equal keys, keep first-seen order."""

    def __init__(self):
        self.order = []
        self.coef = {}

    def push(self, key, c):
        if key in self.coef:
            self.coef[key] += c
        else:
            self.order.append(key)
            self.coef[key] = c

    def items(self):
        return [(k, self.coef[k]) for k in self.order]


def _ext(tree, index, first):
    """``PreparedMultiplicityFreeArtin::inner_extended`` (fusion_tree.rs:8255-8275)."""
    rank = len(tree[0])
    if index == 0:
        return first
    if index + 1 == rank:
        return tree[2]
    return tree[3][index - 1]


def artin(rule, tree, index, inverse):
    """Elementary braid of legs ``index``/``index+1``.

    ``PreparedMultiplicityFreeArtin::apply`` (fusion_tree.rs:8154-8253).
    """
    u, dual, coupled, inner = tree
    rank = len(u)
    left, right = u[index], u[index + 1]
    nu = list(u)
    nu[index], nu[index + 1] = nu[index + 1], nu[index]
    nd = list(dual)
    nd[index], nd[index + 1] = nd[index + 1], nd[index]
    nu, nd = tuple(nu), tuple(nd)
    first = nu[0]
    vac = rule.vacuum()
    if left == vac or right == vac:
        ninner = list(inner)
        if index > 0:
            src = _ext(tree, index + 1, first) if left == vac else _ext(tree, index - 1, first)
            ninner[index - 1] = src
        return [((nu, nd, coupled, tuple(ninner)), 1.0)]
    if index == 0:
        c = inner[0] if rank > 2 else coupled
        coef = rule.R(right, left, c) if inverse else rule.R(left, right, c)
        return [((nu, nd, coupled, inner), coef)]
    a = _ext(tree, index - 1, first)
    b = left
    c = _ext(tree, index, first)
    d = right
    e = _ext(tree, index + 1, first)
    out = []
    for cp in rule.fusion_channels(a, d):
        if not rule.nsymbol(cp, b, e):
            continue
        ninner = list(inner)
        ninner[index - 1] = cp
        f = rule.F(d, a, b, e, cp, c)
        if inverse:
            coef = (rule.R(d, c, e) * f) * rule.R(d, a, cp)
        else:
            coef = rule.R(c, d, e) * (f * rule.R(a, d, cp))
        out.append(((nu, nd, coupled, tuple(ninner)), coef))
    return out


def bendright(rule, pair):
    """Move the last codomain leg to the end of the domain.

    ``PreparedMultiplicityFreeBendRight`` (fusion_tree.rs:8744-8921):
    coefficient sqrt(d_c)/sqrt(d_a) B(a, b, c), times the conjugated
    Frobenius-Schur phase of dual(b) when the bent leg is dual.
    """
    (u, ud, c, ui), (v, vd, c2, vi) = pair
    n1, n2 = len(u), len(v)
    if n1 == 0:
        raise ValueError("bendright requires a codomain leg")
    b, bdual = u[-1], ud[-1]
    if n1 == 1:
        a = rule.vacuum()
    elif n1 == 2:
        a = u[0]
    else:
        a = ui[-1]
    new_cod = (u[:-1], ud[:-1], a, ui[:-1] if n1 > 2 else ())
    new_dom = (v + (rule.dual(b),), vd + (not bdual,), a, vi + ((c,) if n2 > 1 else ()))
    coef = rule.dim(c) ** 0.5 / rule.dim(a) ** 0.5 * rule.B(a, b, c)
    if bdual:
        coef *= rule.fs(rule.dual(b))
    return [((new_cod, new_dom), coef)]


def bendleft(rule, pair):
    """Move the last domain leg to the end of the codomain (fusion_tree.rs:8923-8998, 9024-9040)."""
    cod, dom = pair
    ((ncod, ndom), coef), = bendright(rule, (dom, cod))
    return [((ndom, ncod), coef)]


def _compose(rule, terms, op):
    acc = _Acc()
    for key, c in terms:
        for k2, c2 in op(rule, key):
            acc.push(k2, c * c2)
    return acc.items()


def repartition(rule, pair, target):
    """``multiplicity_free_repartition_tree_pair_validated`` (fusion_tree.rs:3785-3812)."""
    terms = [(pair, 1.0)]
    n1 = len(pair[0][0])
    while n1 < target:
        terms = _compose(rule, terms, bendleft)
        n1 += 1
    while n1 > target:
        terms = _compose(rule, terms, bendright)
        n1 -= 1
    return terms


def linearize(p1, p2, n1, n2):
    """``linearize_tree_pair_permutation`` (fusion_tree.rs:6936-6963, 12537-12543)."""
    def lin(a):
        return a if a < n1 else n2 + 2 * n1 - 1 - a

    return [lin(a) for a in p1] + [lin(a) for a in reversed(p2)]


def artin_steps(perm, levels):
    """``PreparedTreeBraid::new`` (fusion_tree.rs:2477-2507)."""
    rank = len(perm)
    work = list(perm)
    lv = list(levels)
    steps = []
    for target in range(rank - 1):
        source = work[target]
        for index in range(source - 1, target - 1, -1):
            steps.append((index, lv[index] > lv[index + 1]))
            lv[index], lv[index + 1] = lv[index + 1], lv[index]
        for k in range(target + 1, rank):
            if work[k] < source:
                work[k] += 1
        work[target] = target
    return steps


def braid_tree(rule, tree, steps):
    """``execute_multiplicity_free_tree_braid_steps`` (fusion_tree.rs:3691-3726)."""
    current = [(tree, 1.0)]
    for index, inverse in steps:
        acc = _Acc()
        for t, c in current:
            for t2, c2 in artin(rule, t, index, inverse):
                acc.push(t2, c * c2)
        current = acc.items()
    return current


def braid_pair(rule, pair, p1, p2, levels1, levels2):
    """Tree-pair braid (``prepare_braid_lowered`` fusion_tree.rs:2763-2870 and
    ``execute_multiplicity_free_validated`` fusion_tree.rs:3319-3355)."""
    n1, n2 = len(pair[0][0]), len(pair[1][0])
    n = n1 + n2
    if list(p1) == list(range(n1)) and list(p2) == list(range(n1, n)):
        return [(pair, 1.0)]
    lin = linearize(p1, p2, n1, n2)
    if lin == list(range(n)):
        return repartition(rule, pair, len(p1))
    levels = list(levels1) + list(reversed(list(levels2)))
    steps = artin_steps(lin, levels)
    acc = _Acc()
    for key, c in repartition(rule, pair, n):
        for t2, c2 in braid_tree(rule, key[0], steps):
            acc.push((t2, key[1]), c * c2)
    out = _Acc()
    for key, c in acc.items():
        for k2, c2 in repartition(rule, key, len(p1)):
            out.push(k2, c * c2)
    return out.items()


def permute_pair(rule, pair, p1, p2):
    """Tree-pair permute: a braid with levels ``0..rank`` (``prepare_permute``, fusion_tree.rs:2929-3060)."""
    n1, n2 = len(pair[0][0]), len(pair[1][0])
    return braid_pair(rule, pair, p1, p2, list(range(n1)), list(range(n1, n1 + n2)))
