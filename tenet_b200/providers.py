"""Table-backed fusion providers: a rule given as tables instead of built-in factors.

The reference admits fusion categories beyond U(1), SU(2) and the parities
through a checked provider: the rule's fusion multiplicities, duals, quantum
dimensions, Frobenius-Schur phases and F / R symbols come from the provider
and are validated before any plan is compiled
(``CheckedGenericFusion`` / ``CheckedGenericRigidSymbols``,
tenet-sectors/src/algebra.rs:743-910; the transform path
tenet-tensors/src/tree_context.rs:38-110 and tree_transform/plan.rs:250-330).

This backend takes the multiplicity-free, real, symmetric (bosonic) case of
that idea: ``TableProvider`` holds the tables, ``tnt_rule_create_table``
checks them (vacuum and duality laws, N in {0, 1}, dimension consistency,
orthogonal F moves, the pentagon, symmetric R with the hexagon) and the
whole recoupling machinery -- tree enumeration, Artin moves, bends, the
device transform tables -- runs on them unchanged.  Sectors are labelled
0 .. n-1 with 0 the vacuum; the SectorId of label i is i.

``finite_group_provider`` derives the tables of Rep(G) for a finite group G
from real orthogonal irreducible representations given on generators (the
Clebsch-Gordan isometries are the one-dimensional intertwiner spaces, so the
rule must be multiplicity free); ``rep_s3`` is Rep(S3) (irreps: trivial,
sign, the two-dimensional standard representation), the smallest
non-abelian example, whose 2 x 2 -> 1 + sign + 2 fusion has three channels.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np


@dataclass
class TableProvider:
    """Tables of a multiplicity-free fusion rule with real symmetric braiding.

    * ``dual[a]``; ``nsym[a, b, c]`` in {0, 1};
    * ``dims[a]`` (quantum dimensions), ``fs[a]`` (Frobenius-Schur phases);
    * ``rsym[a, b, c]`` (R symbols, +-1 on admissible triples);
    * ``fsym[a, b, c, d, e, f]`` = F(a, b, c; d; e, f): the coefficient of the
      tree a (x) (b (x) c -> f) -> d in the tree (a (x) b -> e) (x) c -> d.
    """

    dual: np.ndarray
    nsym: np.ndarray
    dims: np.ndarray
    fs: np.ndarray
    rsym: np.ndarray
    fsym: np.ndarray

    @property
    def n(self) -> int:
        return len(self.dims)


def _intertwiner(rho_c: Sequence[np.ndarray], rho_ab: Sequence[np.ndarray]) -> np.ndarray:
    """The isometry C : V_c -> V_a (x) V_b with rho_ab(g) C = C rho_c(g) on the
    generators, or None when the intertwiner space is zero.  Raises if it has
    more than one dimension (an outer multiplicity)."""
    dc, dab = rho_c[0].shape[0], rho_ab[0].shape[0]
    rows = []
    for gc, gab in zip(rho_c, rho_ab):
        # vec(rho_ab C - C rho_c) = (I (x) rho_ab - rho_c^T (x) I) vec(C), column-major vec
        rows.append(np.kron(np.eye(dc), gab) - np.kron(gc.T, np.eye(dab)))
    M = np.vstack(rows)
    _, s, vt = np.linalg.svd(M)
    null = vt[np.sum(s > 1e-9 * max(1.0, s.max())):]
    if len(null) == 0:
        return None
    if len(null) > 1:
        raise ValueError("fusion with outer multiplicity: the table provider is multiplicity free")
    C = null[0].reshape(dc, dab).T  # column-major un-vec: dab x dc
    CtC = C.T @ C
    C = C / np.sqrt(CtC[0, 0])
    # the sign of each isometry is a gauge choice: first non-negligible entry positive
    flat = C.ravel()
    if flat[np.argmax(np.abs(flat) > 1e-12)] < 0:
        C = -C
    return C


def finite_group_provider(irreps: Sequence[Sequence[np.ndarray]]) -> TableProvider:
    """Tables of Rep(G) from real orthogonal irreps given on the same list of
    generators; irreps[0] must be the trivial representation."""
    n = len(irreps)
    irreps = [[np.asarray(g, dtype=np.float64) for g in rep] for rep in irreps]
    dims = np.array([rep[0].shape[0] for rep in irreps], dtype=np.float64)
    ngen = len(irreps[0])
    C = {}
    nsym = np.zeros((n, n, n), dtype=np.uint8)
    for a, b, c in itertools.product(range(n), repeat=3):
        rho_ab = [np.kron(irreps[a][g], irreps[b][g]) for g in range(ngen)]
        iso = _intertwiner(irreps[c], rho_ab)
        if iso is not None:
            C[a, b, c] = iso
            nsym[a, b, c] = 1
    # real irreps are self-dual
    dual = np.arange(n, dtype=np.int32)
    # R(a, b, c): swap . C^{ab}_c = R C^{ba}_c
    rsym = np.zeros((n, n, n))
    for (a, b, c), iso in C.items():
        da, db = int(dims[a]), int(dims[b])
        swap = np.zeros((da * db, da * db))
        for i in range(da):
            for j in range(db):
                swap[j * da + i, i * db + j] = 1.0
        rsym[a, b, c] = np.trace(C[b, a, c].T @ swap @ iso) / dims[c]
    fsym = np.zeros((n,) * 6)
    for a, b, c, d in itertools.product(range(n), repeat=4):
        da, db, dcc = (int(dims[x]) for x in (a, b, c))
        for e in range(n):
            if not (nsym[a, b, e] and nsym[e, c, d]):
                continue
            left = np.kron(C[a, b, e], np.eye(dcc)) @ C[e, c, d]
            for f in range(n):
                if not (nsym[b, c, f] and nsym[a, f, d]):
                    continue
                right = np.kron(np.eye(da), C[b, c, f]) @ C[a, f, d]
                fsym[a, b, c, d, e, f] = np.trace(right.T @ left) / dims[d]
    fs = np.array([dims[a] * fsym[a, a, a, a, 0, 0] for a in range(n)])
    return TableProvider(dual, nsym, dims, np.round(fs), rsym, fsym)


def rep_s3() -> TableProvider:
    """Rep(S3): 0 trivial, 1 sign, 2 standard (two-dimensional), from the
    generators r (rotation by 2 pi / 3) and s (a reflection)."""
    c, s_ = np.cos(2 * np.pi / 3), np.sin(2 * np.pi / 3)
    r2 = np.array([[c, -s_], [s_, c]])
    s2 = np.array([[1.0, 0.0], [0.0, -1.0]])
    one = np.array([[1.0]])
    return finite_group_provider([[one, one], [one, -one], [r2, s2]])


def check_tables(p: TableProvider, tol: float = 1e-10) -> List[str]:
    """Host restatement of the provider checks ``tnt_rule_create_table`` runs;
    returns the failed laws (empty when the tables are admissible)."""
    n, N, F, R, d = p.n, p.nsym, p.fsym, p.rsym, p.dims
    bad = []
    for a in range(n):
        if not (N[0, a, a] and N[a, 0, a] and N[a, p.dual[a], 0]) or p.dual[p.dual[a]] != a:
            bad.append(f"vacuum or dual law at {a}")
    if np.any(N > 1):
        bad.append("outer multiplicity")
    for a, b in itertools.product(range(n), repeat=2):
        if abs(d[a] * d[b] - sum(N[a, b, c] * d[c] for c in range(n))) > tol * d[a] * d[b]:
            bad.append(f"dimensions at {a},{b}")
    for a, b, c, x in itertools.product(range(n), repeat=4):
        es = [e for e in range(n) if N[a, b, e] and N[e, c, x]]
        fs_ = [f for f in range(n) if N[b, c, f] and N[a, f, x]]
        if len(es) != len(fs_):
            bad.append(f"F block shape at {a},{b},{c},{x}")
            continue
        if es:
            M = F[a, b, c, x][np.ix_(es, fs_)]
            if np.abs(M @ M.T - np.eye(len(es))).max() > tol:
                bad.append(f"F orthogonality at {a},{b},{c},{x}")
    # pentagon: F(f,c,d;e;g,l) F(a,b,l;e;f,k) = sum_h F(a,b,c;g;f,h) F(a,h,d;e;g,k) F(b,c,d;k;h,l)
    for a, b, c, dd, e in itertools.product(range(n), repeat=5):
        for f, g, k, l in itertools.product(range(n), repeat=4):
            lhs = F[f, c, dd, e, g, l] * F[a, b, l, e, f, k]
            rhs = sum(F[a, b, c, g, f, h] * F[a, h, dd, e, g, k] * F[b, c, dd, k, h, l] for h in range(n))
            if abs(lhs - rhs) > tol:
                bad.append(f"pentagon at {(a, b, c, dd, e, f, g, k, l)}")
                return bad
    for a, b, c in itertools.product(range(n), repeat=3):
        if N[a, b, c] and abs(R[a, b, c] * R[b, a, c] - 1.0) > tol:
            bad.append(f"symmetric braiding at {a},{b},{c}")
    # hexagon: R(c,a,e) F(a,c,b;d;e,g) R(c,b,g) = sum_f F(c,a,b;d;e,f) R(c,f,d) F(a,b,c;d;f,g)
    for a, b, c, dd, e, g in itertools.product(range(n), repeat=6):
        lhs = R[c, a, e] * F[a, c, b, dd, e, g] * R[c, b, g]
        rhs = sum(F[c, a, b, dd, e, f] * R[c, f, dd] * F[a, b, c, dd, f, g] for f in range(n))
        if abs(lhs - rhs) > tol:
            bad.append(f"hexagon at {(a, b, c, dd, e, g)}")
            return bad
    return bad
