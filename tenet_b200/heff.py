"""SU(2) effective-Hamiltonian matvec and a device-resident FP64 Lanczos.

Workload: MPS tensor x : (W x P) <- W, environments L : (W x M) <- W and
R : (W x M*) <- W, MPO tensor O : (M x P) <- (P x M).  The single-site network

    B x = R-contract( O-contract( L-contract(x) ) )

is three pairwise contractions lowered like the reference's ``contract``
(tenet/src/typed.rs:13653; permute the open legs out, compose, permute):

    xb  = x.permute([0], [1, 2])          W <- (P* x W)
    t1  = L o xb                          (W x M) <- (P* x W)
    t1p = t1.permute([0, 3], [1, 2])      (W x W*) <- (M* x P*)
    t2  = t1p o Op,  Op = O.permute([3, 2], [0, 1])
    t2p = t2.permute([0, 3], [1, 2])      (W x P) <- (W x M*)
    B x = t2p o R                         (W x P) <- W

R carries the MPO bond as M* so the network closes on x's space.  With random
environments B is not self-adjoint, so the Lanczos operator is the symmetric
positive semi-definite H = B^dagger B; B^dagger runs the same chain backwards
with the adjoint operands and the inverse permutes (SU(2) recoupling is
orthogonal, so a permute's inverse is its adjoint).  Every compose runs the
selected arithmetic (plain FP64, BF16 slices or 8-bit digits, ``slices`` per
operand; with digits the constant operands are packed once); the
recoupling transforms, the Lanczos orthogonalisation (weighted inner products
and axpys) and the tridiagonal eigenproblem stay in FP64 on the GPU.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, typed
from ._lib import call


class EffectiveHamiltonian:
    """B and B^dagger of the single-site network.  With 8-bit digits
    (``precision="i8x"``) the six constant operands (L, O, R and their
    adjoints) are packed once per digit count and reused by every matvec;
    only the Krylov vector's side is packed per compose."""

    def __init__(self, L, O, R):
        self.L = L
        self.R = R
        self.Op = O.permute([3, 2], [0, 1])
        self.Ld = L.adjoint()
        self.Rd = R.adjoint()
        self.Opd = self.Op.adjoint()
        self._packed = {}

    def _mul(self, lhs, rhs, const, precision, slices):
        """lhs o rhs, where ``const`` ("lhs" or "rhs") is the constant operand.

        The MPO step (O contracted over M x P, K <= 3: 0.2 of the 166 GFLOP
        of a matvec) stays in FP64 at every precision: slicing a product
        that thin pads K to the 64-deep digit block, so its packs would move
        twenty times the operand's bytes for no tensor-core gain."""
        if precision != "fp64" and not lhs.runtime.cplan(lhs.space, rhs.space).suits_split:
            return lhs.compose(rhs, "fp64", 0)
        if precision != "i8x":
            return lhs.compose(rhs, precision, slices)
        c, other, side = (lhs, rhs, 0) if const == "lhs" else (rhs, lhs, 1)
        key = (id(c), side, slices)
        pk = self._packed.get(key)
        if pk is None:
            pk = c.pack_split(other.space, side, slices)
            self._packed[key] = pk
        return pk.compose_packed(rhs, slices) if side == 0 else lhs.compose_packed(pk, slices)

    def apply_b(self, x, precision, slices):
        xb = x.permute([0], [1, 2])
        t1 = self._mul(self.L, xb, "lhs", precision, slices)
        t2 = self._mul(t1.permute([0, 3], [1, 2]), self.Op, "rhs", precision, slices)
        return self._mul(t2.permute([0, 3], [1, 2]), self.R, "rhs", precision, slices)

    def apply_bdag(self, y, precision, slices):
        t2p = self._mul(y, self.Rd, "rhs", precision, slices)
        t2 = t2p.permute([0, 2], [3, 1])
        t1p = self._mul(t2, self.Opd, "rhs", precision, slices)
        t1 = t1p.permute([0, 2], [3, 1])
        xb = self._mul(self.Ld, t1, "lhs", precision, slices)
        return xb.permute([0, 1], [2])

    def apply(self, x, precision="fp64", slices=6):
        return self.apply_bdag(self.apply_b(x, precision, slices), precision, slices)


def lanczos(H: EffectiveHamiltonian, x0: "typed.TensorMap", iterations: int = 30, precision="fp64", slices=6):
    """``iterations`` Lanczos steps with full (twice-iterated) reorthogonalisation.

    Returns (lowest Ritz value, Ritz vector as a TensorMap, tridiagonal alphas, betas).
    """
    torch = typed.torch()
    rt = x0.runtime
    space = x0.space
    n = space.size
    m = iterations
    if m > 48:
        raise ValueError("at most 48 Lanczos steps (device eigensolver limit)")
    fplan = rt.fplan(space)
    dev = x0.data.device
    V = torch.empty((m, n), dtype=torch.float64, device=dev)
    h = torch.empty(m, dtype=torch.float64, device=dev)
    h2 = torch.empty(m, dtype=torch.float64, device=dev)
    nrm = torch.empty(1, dtype=torch.float64, device=dev)
    st = rt.stream()
    P = lambda t: C.c_void_p(t.data_ptr())

    def wdot(k, vecs, y, out):
        call("tnt_wdot", rt._h, fplan._h, k, P(vecs), n, P(y), P(out), st)

    v = x0.data.clone()
    wdot(1, v, v, nrm)
    v /= torch.sqrt(nrm[0])
    alphas, betas = [], []
    for j in range(m):
        V[j].copy_(v)
        w = H.apply(typed.TensorMap(rt, space, V[j].clone()), precision, slices).data
        for hv in (h, h2):  # classical Gram-Schmidt, twice
            wdot(j + 1, V, w, hv)
            neg = -hv[: j + 1]
            call("tnt_axpy_many", rt._h, n, j + 1, P(V), n, P(neg), 1.0, None, P(w), st)
        alpha = float(h[j] + h2[j])
        wdot(1, w, w, nrm)
        beta = float(torch.sqrt(nrm[0]))
        alphas.append(alpha)
        betas.append(beta)
        if j + 1 < m:
            v = w / beta
    T = np.diag(alphas) + np.diag(betas[:-1], 1) + np.diag(betas[:-1], -1)
    Td = torch.as_tensor(np.asfortranarray(T).ravel(order="F"), device=dev)
    evals = torch.empty(m, dtype=torch.float64, device=dev)
    evecs = torch.empty(m * m, dtype=torch.float64, device=dev)
    call("tnt_symeig", rt._h, m, P(Td), P(evals), P(evecs), st)
    c0 = evecs[:m].contiguous()
    ritz = torch.zeros(n, dtype=torch.float64, device=dev)
    call("tnt_axpy_many", rt._h, n, m, P(V), n, P(c0), 0.0, None, P(ritz), st)
    return float(evals[0]), typed.TensorMap(rt, space, ritz), alphas, betas


def workload_tensors(rt, cfg, scale=1, seed0=1):
    """x, L, O, R of the effective-Hamiltonian configuration, degeneracies divided by ``scale``."""
    from .workloads import splitmix_normal

    rule = typed.FusionRule(cfg["factors"])
    W = typed.GradedSpace(rule, [(s[0], max(1, d // scale)) for s, d in cfg["W"]])
    M = typed.GradedSpace(rule, [(s[0], d) for s, d in cfg["M"]])
    P = typed.GradedSpace(rule, [(s[0], d) for s, d in cfg["P"]])
    Md = M.dual()
    mk = lambda cod, dom, seed: typed.TensorMap.from_host(
        rt, cod, dom, splitmix_normal(seed, rt.space(rule, cod, dom).size)
    )
    x = mk([W, P], [W], seed0)
    L = mk([W, M], [W], seed0 + 1)
    O = mk([M, P], [P, M], seed0 + 2)
    R = mk([W, Md], [W], seed0 + 3)
    return rule, x, L, O, R
