"""Block-sparse symmetric tensor maps on the CPU (oracle).

Test infrastructure only; see ``oracle/__init__.py``.

``TensorMap`` holds a ``HomSpace`` and one flat float64 payload in the
coupled-sector layout.  Operations restate TeNeT's Host path:

* ``compose``: one GEMM per coupled sector (tenet-operations/src/fusion_replay.rs:457-556);
* ``permute`` / ``braid`` / ``repartition``: per source tree-pair block,
  ``dst += coef * transpose(src, p1 + p2)`` over the recoupling terms
  (tenet-operations/src/transform_replay.rs:4428-4517 for single blocks,
  4519-4800 for multi-tree groups; both compute the same sum);
* ``norm`` / ``tr``: quantum-dimension-weighted sector sums (TensorKit
  semantics asserted by tenet/tests/semantic_suite.rs:835-905);
* ``svd_compact`` / ``svd_trunc``: per-sector SVD with the largest-|U| gauge
  (tenet-matrixalgebra/src/factorize.rs:3836-3852, 3945-3962) and
  ``select_truncation`` (tenet-matrixalgebra/src/truncation.rs:257-560);
* ``qr_compact``: per-sector thin QR with the positive-diagonal gauge
  (factorize.rs:5158, 3789-3830);
* ``eigh_full`` / ``eigh_trunc``: per-sector symmetric eigendecomposition,
  eigenvalues stable-sorted by descending magnitude, largest-entry-positive
  eigenvectors (factorize.rs:3041-3150, 3902-3913), truncation on the
  magnitudes (factorize.rs:3284-3340, 2332-2377).
"""

from __future__ import annotations

import heapq
import math

import numpy as np

from . import recouple
from .fusion import HomSpace
from .sectors import FZ2


# ---------------------------------------------------------------------------
# seeded fills
# ---------------------------------------------------------------------------

_M64 = 0xFFFFFFFFFFFFFFFF


def splitmix_uniform(state: int):
    """``random_unit`` (tenet/src/typed.rs:2086-2093): returns (new_state, U[-1,1))."""
    state = (state + 0x9E3779B97F4A7C15) & _M64
    v = state
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & _M64
    v ^= v >> 31
    return state, float(v >> 11) / float(1 << 52) - 1.0


def splitmix_uniform_array(seed: int, n: int) -> np.ndarray:
    """Vectorised ``random_unit`` stream of length ``n`` (identical values)."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    return (v >> np.uint64(11)).astype(np.float64) / float(1 << 52) - 1.0


def normal_fill(seed: int, n: int) -> np.ndarray:
    """N(0,1) entries in flat storage order from the splitmix64 stream.

    The reference has no normal sampler; this is the project-defined
    Box-Muller map over consecutive ``random_unit`` pairs ``(x1, x2)``:
    ``u1 = (1 - x1) / 2`` in (0, 1], ``u2 = (x2 + 1) / 2`` in [0, 1),
    value ``sqrt(-2 ln u1) cos(2 pi u2)``.  The product computes the same map.
    """
    u = splitmix_uniform_array(seed, 2 * n)
    u1 = (1.0 - u[0::2]) * 0.5
    u2 = (u[1::2] + 1.0) * 0.5
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


class TensorMap:
    def __init__(self, space: HomSpace, data=None):
        self.space = space
        self.data = np.zeros(space.size) if data is None else np.ascontiguousarray(data, dtype=np.float64)
        assert self.data.shape == (space.size,)

    # -- construction ----------------------------------------------------
    @staticmethod
    def zeros(rule, codomain, domain):
        return TensorMap(HomSpace(rule, codomain, domain))

    @staticmethod
    def randn(rule, codomain, domain, seed):
        sp = HomSpace(rule, codomain, domain)
        return TensorMap(sp, normal_fill(seed, sp.size))

    @staticmethod
    def from_block_fn(rule, codomain, domain, fn):
        """``TensorMap::from_block_fn`` (tenet/src/typed.rs:12262): ``fn(key, idx)`` per element."""
        t = TensorMap.zeros(rule, codomain, domain)
        for b, blk in enumerate(t.space.blocks):
            view = t.space.block_view(t.data, b)
            for idx in np.ndindex(*blk["shape"]):
                view[idx] = fn(blk["key"], idx)
        return t

    @property
    def rule(self):
        return self.space.rule

    def copy(self):
        return TensorMap(self.space, self.data.copy())

    # -- linear algebra --------------------------------------------------
    def compose(self, other: "TensorMap") -> "TensorMap":
        """C = self o other: per coupled sector C_c = A_c B_c.

        ``FusionBlockContractPlan::try_from_canonical_coupled_regions_impl``
        (fusion_replay.rs:457-530) zips the two sorted sector lists; sectors
        present in only one operand contribute a zero block.
        """
        a, b = self.space, other.space
        if a.domain != b.codomain:
            raise ValueError("compose: domain/codomain mismatch")
        out = TensorMap.zeros(a.rule, a.codomain, b.domain)
        for i, (c, r, cc, off) in enumerate(out.space.sectors):
            ia, ib = a.sector_of(c), b.sector_of(c)
            if ia is None or ib is None:
                continue
            out.space.sector_matrix(out.data, i)[:] = a.sector_matrix(self.data, ia) @ b.sector_matrix(other.data, ib)
        return out

    def norm(self) -> float:
        s = 0.0
        for i, (c, r, cc, off) in enumerate(self.space.sectors):
            m = self.space.sector_matrix(self.data, i)
            s += self.rule.dim(c) * float(np.sum(m * m))
        return math.sqrt(s)

    def tr(self) -> float:
        s = 0.0
        for i, (c, r, cc, off) in enumerate(self.space.sectors):
            m = self.space.sector_matrix(self.data, i)
            s += self.rule.dim(c) * float(np.trace(m))
        return s

    def add(self, other, alpha=1.0, beta=1.0):
        assert self.space.same_as(other.space)
        return TensorMap(self.space, alpha * self.data + beta * other.data)

    def adjoint(self) -> "TensorMap":
        """Materialised adjoint: block(t', c) = block(t, c)^T for real data."""
        sp = self.space
        out = TensorMap.zeros(sp.rule, sp.domain, sp.codomain)
        for i, (c, r, cc, off) in enumerate(out.space.sectors):
            j = sp.sector_of(c)
            out.space.sector_matrix(out.data, i)[:] = sp.sector_matrix(self.data, j).T
        return out

    # -- recoupling -------------------------------------------------------
    def _transformed(self, p1, p2, pair_terms):
        sp = self.space
        legs = list(sp.codomain) + [l.dual() for l in sp.domain]
        cod = [legs[p] for p in p1]
        dom = [legs[p].dual() for p in p2]
        out = TensorMap.zeros(sp.rule, cod, dom)
        axes = tuple(p1) + tuple(p2)
        for b, blk in enumerate(sp.blocks):
            src = sp.block_view(self.data, b)
            perm = np.transpose(src, axes)
            for key, coef in pair_terms(blk["key"]):
                if coef == 0.0:
                    continue
                d = out.space.block_index[key]
                view = out.space.block_view(out.data, d)
                view += coef * perm
        return out

    def permute(self, p1, p2):
        """``TensorMap::permute`` (tenet/src/typed.rs:13163-13180)."""
        if list(p1) == list(range(self.space.n1)) and list(p2) == list(
            range(self.space.n1, self.space.n1 + self.space.n2)
        ):
            return self.copy()
        rule = self.rule
        return self._transformed(p1, p2, lambda key: recouple.permute_pair(rule, key, p1, p2))

    def braid(self, p1, p2, levels):
        n1 = self.space.n1
        rule = self.rule
        return self._transformed(
            p1, p2, lambda key: recouple.braid_pair(rule, key, p1, p2, levels[:n1], levels[n1:])
        )

    def repartition(self, n):
        """``TensorMap::repartition`` (tenet/src/typed.rs:13250): planar order kept."""
        n1, n2 = self.space.n1, self.space.n2
        rank = n1 + n2
        planar = list(range(n1)) + list(reversed(range(n1, rank)))
        p1 = planar[:n]
        p2 = list(reversed(planar[n:]))
        rule = self.rule
        return self._transformed(p1, p2, lambda key: recouple.repartition(rule, key, n))

    def twist(self, legs):
        """``TensorMap::twist`` (tenet/src/typed.rs:4599-4601): every block times
        the product over ``legs`` (flat axes, codomain first) of the ribbon
        twist of that leg's uncoupled sector in the block's tree pair."""
        sp = self.space
        out = self.copy()
        for b, blk in enumerate(sp.blocks):
            cod, dom = blk["key"]
            f = 1.0
            for a in legs:
                f *= self.rule.twist(cod[0][a] if a < sp.n1 else dom[0][a - sp.n1])
            if f != 1.0:
                sp.block_view(out.data, b)[...] *= f
        return out

    def contract(self, other, lhs_axes, rhs_axes, output_axes):
        """``TensorMap::contract`` (tenet/src/typed.rs:13653).

        The reference's DynamicTree resolution (tenet-tensors/src/contract/
        resolution.rs:28-40, dynamic.rs:330-390): permute ``self`` to
        (open ; contracted), ``other`` to (contracted ; open), twist the
        permuted ``other`` on each contracted codomain leg that is dual when
        the rule is fermionic (the supertrace twist, contract/fusion/
        block_specs.rs:683-716), compose, then permute the result by
        ``output_axes``; the result's codomain holds every open axis of
        ``self`` and its domain every open axis of ``other``.
        """
        ra = self.space.n1 + self.space.n2
        rb = other.space.n1 + other.space.n2
        open_a = [i for i in range(ra) if i not in lhs_axes]
        open_b = [i for i in range(rb) if i not in rhs_axes]
        a = self.permute(open_a, list(lhs_axes))
        b = other.permute(list(rhs_axes), open_b)
        if FZ2 in self.rule.factors:
            dual = [p for p in range(len(rhs_axes)) if b.space.codomain[p].is_dual]
            if dual:
                b = b.twist(dual)
        c = a.compose(b)
        na = len(open_a)
        out = list(output_axes)
        if out == list(range(na + len(open_b))):
            return c
        return c.permute(out[:na], out[na:])

    # -- factorisation ---------------------------------------------------
    def svd_compact(self):
        """Per-sector thin SVD with the largest-|U| column gauge.

        Returns ``[(coupled, U, S, Vh), ...]`` in sector order.
        """
        out = []
        for i, (c, r, cc, off) in enumerate(self.space.sectors):
            m = self.space.sector_matrix(self.data, i)
            u, s, vh = np.linalg.svd(m, full_matrices=False)
            for j in range(len(s)):
                col = u[:, j]
                k = int(np.argmax(np.abs(col)))  # first maximum (factorize.rs:3953-3959)
                if col[k] < 0:
                    u[:, j] *= -1
                    vh[j, :] *= -1
            out.append((c, u, s, vh))
        return out

    def svd_trunc(self, truncation):
        parts = self.svd_compact()
        spectra = [(c, self.rule.dim(c), s) for c, _, s, _ in parts]
        kept, err = select_truncation(spectra, truncation)
        return [(c, u[:, :k], s[:k], vh[:k, :]) for (c, u, s, vh), k in zip(parts, kept)], kept, err

    def qr_compact(self):
        """Per-sector thin QR, ``R_jj >= 0`` (positive_diagonal_gauge, factorize.rs:3808-3830:
        a zero diagonal entry keeps phase 1).  Returns ``[(coupled, Q, R), ...]``."""
        out = []
        for i, (c, r, cc, off) in enumerate(self.space.sectors):
            m = self.space.sector_matrix(self.data, i)
            q, rr = np.linalg.qr(m, mode="reduced")
            for j in range(min(q.shape[1], rr.shape[0])):
                if rr[j, j] < 0:
                    q[:, j] *= -1
                    rr[j, :] *= -1
            out.append((c, q, rr))
        return out

    def eigh_full(self):
        """Per-sector symmetric eigendecomposition (eigh_full_dyn, factorize.rs:3041-3150).

        LAPACK's ascending eigenvalues are stable-sorted by descending absolute
        value (ties keep the ascending order), then every eigenvector's first
        largest-|.| entry is made positive (eigenvector_gauge, :3902-3913).
        Returns ``[(coupled, values, vectors), ...]``.
        """
        if list(self.space.codomain) != list(self.space.domain):
            raise ValueError("eigh requires an endomorphism (codomain == domain)")
        out = []
        for i, (c, r, cc, off) in enumerate(self.space.sectors):
            m = self.space.sector_matrix(self.data, i)
            if np.linalg.norm(m - m.T) > 128 * np.finfo(float).eps * np.linalg.norm(m):
                raise ValueError("eigh requires Hermitian coupled-sector blocks")
            w, v = np.linalg.eigh(m)
            order = sorted(range(len(w)), key=lambda j: -abs(w[j]))  # stable: ties keep ascending order
            w = w[order]
            v = v[:, order]
            for j in range(v.shape[1]):
                k = int(np.argmax(np.abs(v[:, j])))
                if v[k, j] < 0:
                    v[:, j] *= -1
            out.append((c, w, v))
        return out

    def eigh_trunc(self, truncation):
        """``eigh_trunc_dyn`` (factorize.rs:3284-3340): select_truncation on |lambda|."""
        parts = self.eigh_full()
        spectra = [(c, self.rule.dim(c), np.abs(w)) for c, w, _ in parts]
        kept, err = select_truncation(spectra, truncation)
        return [(c, w[:k], v[:, :k]) for (c, w, v), k in zip(parts, kept)], kept, err


# ---------------------------------------------------------------------------
# truncation selection
# ---------------------------------------------------------------------------


def select_truncation(spectra, truncation):
    """``select_truncation`` (tenet-matrixalgebra/src/truncation.rs:257-271).

    ``spectra``: list of ``(sector, weight, descending values)``.
    ``truncation``: ``("full",)``, ``("rank", n)``, ``("tol", atol, rtol)``,
    ``("discard", rtol)`` or ``("space", {sector: rank})``.
    Returns ``(kept_counts, error)`` with error = sqrt(sum_c w_c sum_disc s^2)
    (truncation.rs:558-570).
    """
    kind = truncation[0]
    n = [len(s) for _, _, s in spectra]
    if kind == "full":
        kept = list(n)
    elif kind == "rank":
        budget = float(truncation[1])
        # descending_candidates (truncation.rs:477-520): value desc, then sector asc, index asc
        heap = [(-s[0], k, 0) for k, (_, _, s) in enumerate(spectra) if len(s)]
        heapq.heapify(heap)
        kept = [0] * len(spectra)
        used = 0.0
        while heap:
            v, k, i = heapq.heappop(heap)
            w = spectra[k][1]
            if used + w > budget + 1e-12:
                break
            used += w
            kept[k] += 1
            if i + 1 < n[k]:
                heapq.heappush(heap, (-spectra[k][2][i + 1], k, i + 1))
    elif kind == "tol":
        atol, rtol = truncation[1], truncation[2]
        full = math.sqrt(sum(w * float(np.sum(np.asarray(s) ** 2)) for _, w, s in spectra))
        thr = max(atol, rtol * full)
        kept = [int(np.sum(np.asarray(s) >= thr)) for _, _, s in spectra]
    elif kind == "discard":
        rtol = truncation[1]
        full = math.sqrt(sum(w * float(np.sum(np.asarray(s) ** 2)) for _, w, s in spectra))
        budget = (rtol * full) ** 2
        kept = list(n)
        disc = 0.0
        while True:
            best = None
            for k, (_, w, s) in enumerate(spectra):
                if kept[k] == 0:
                    continue
                v = s[kept[k] - 1]
                if best is None or v < best[1]:
                    best = (k, v)
            if best is None:
                break
            k, v = best
            nxt = disc + spectra[k][1] * v * v
            if nxt > budget + 1e-15:
                break
            disc = nxt
            kept[k] -= 1
    elif kind == "space":
        prof = truncation[1]
        kept = [min(prof.get(c, 0), len(s)) for c, _, s in spectra]
    else:
        raise ValueError(kind)
    err = 0.0
    for (c, w, s), k in zip(spectra, kept):
        tail = np.asarray(s[k:], dtype=np.float64)
        err += w * float(np.sum(tail * tail))
    return kept, math.sqrt(err)
