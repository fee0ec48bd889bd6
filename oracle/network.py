"""Host replay of a compiled contraction schedule (test infrastructure only).

Restates ``PlannedNetwork::execute`` (tenet-network/src/network.rs:1820-1920):
slots 0..n-1 hold the inputs (their adjoint where ``conj[i]``), each step
contracts two slots with ``TensorMap::contract`` semantics (supertrace twist
included) and applies its optional result permutation, and the final slot is
permuted by the optional final permutation.  Steps are tuples
``(lhs_slot, rhs_slot, result_slot, lhs_axes, rhs_axes, output_axes,
result_permutation_or_None)``.
"""

from __future__ import annotations


def execute_schedule(tensors, conj, steps, final_slot, final_permutation=None):
    slots = {i: (t.adjoint() if c else t) for i, (t, c) in enumerate(zip(tensors, conj))}
    for ls, rs, res, la, ra, out, perm in steps:
        lhs, rhs = slots.pop(ls), slots.pop(rs)
        r = lhs.contract(rhs, list(la), list(ra), list(out))
        if perm is not None:
            r = r.permute(list(perm[0]), list(perm[1]))
        slots[res] = r
    result = slots.pop(final_slot)
    if slots:
        raise ValueError("a tensor is left uncontracted outside the final slot")
    if final_permutation is not None:
        result = result.permute(list(final_permutation[0]), list(final_permutation[1]))
    return result
