"""Two-site iTEBD bond update on the device path.

The update of the reference's ``bond_update``
(tenet-network/examples/itebd_heisenberg.rs:63-82), written as the pairwise
contractions its ``tensor!`` network lowers to
(tenet-network/src/network.rs:1609-1925):

1. theta = A . B over the shared virtual leg:
   ``contract(A, B, [2], [0])`` -> (W x P) <- (P* x W);
2. the two-site gate G = exp(-tau S.S) on both physical legs:
   ``contract(G, theta, [2, 3], [1, 2])`` -> (P x P) <- (W* x W);
3. recoupling into the bond matrix form (W x P) <- (P* x W) by one permute
   (F/R/B symbols of SU(2), 6j recoupling);
4. truncated SVD over all coupled sectors with the truncation chosen on the
   device.

A and B are (W x P) <- W MPS tensors; every hot operation is a
``libtenet_b200.so`` kernel (transform, grouped GEMM, batched SVD,
truncation).
"""

from __future__ import annotations

import math

import numpy as np

from . import network, typed


def heisenberg_gate(rt, rule, P, tau):
    """exp(-tau S.S) on two spin-1/2 legs as a (P x P) <- (P x P) map.

    S.S is -3/4 on the singlet (coupled 2j = 0) and +1/4 on the triplet
    (coupled 2j = 2), so the gate is diagonal over the coupled sectors.
    """
    sp = rt.space(rule, [P, P], [P, P])
    vals = []
    for lab, r, c, off in sp.sectors():
        e = -0.75 if lab[0] == 0 else 0.25
        vals.append(np.full(r * c, 0.0))
        vals[-1][:: r + 1] = math.exp(-tau * e)
    return typed.TensorMap(rt, sp, typed.torch().as_tensor(np.concatenate(vals), device=f"cuda:{rt.device}"))


# Steps 1-3 as one network: labels of A, B, G and of theta.
BOND_NETWORK = dict(inputs=[["l", "p1", "m"], ["m", "p2", "r"], ["q1", "q2", "p1", "p2"]],
                    output=["l", "q1", "q2", "r"], output_codomain_rank=2)
_plans = {}


def bond_plan(A, B, G):
    """The compiled schedule of steps 1-3 for these spaces (cached)."""
    key = (A.runtime.device, A.space.key(), B.space.key(), G.space.key())
    plan = _plans.get(key)
    if plan is None:
        plan = network.Network(**BOND_NETWORK).plan([A, B, G], order=["m", "p1", "p2"])
        _plans[key] = plan
    return plan


def bond_theta(A, B, G):
    """theta in the bond-matrix form (W x P) <- (P* x W) (steps 1-3), one
    device schedule: the operand transforms of both contractions and the final
    recoupling are fused into three recoupling passes around two grouped GEMMs."""
    return bond_plan(A, B, G).execute([A, B, G])


def bond_update(A, B, G, truncation):
    """One two-site update: returns the truncated SVD result of theta."""
    return bond_theta(A, B, G).svd_trunc(truncation)
