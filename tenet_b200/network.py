"""Contraction networks on the device: ``tenet-network``'s ``Network`` /
``PlannedNetwork`` (tenet-network/src/network.rs:87-110, 235-340, 909-941)
lowered to one ``tnt_network_execute`` call.

``Network`` validates written label lists (each label open once or contracted
exactly twice, output labels the open ones); ``Network.plan`` picks a pairwise
order (greedy on reduced sizes, or contraction in a given label order as in
``LabelOrderDenseOptimizer``) and compiles it with ``tnt_network_plan``, whose
schedule steps mirror the reference's ``CompiledStep``.  ``PlannedNetwork``
can also be built from an explicit schedule, which is the boundary a caller
holding the reference planner's ``CompiledSchedule`` uses.  Execution fuses
every operand transform into one recoupling pass and keeps intermediates in a
planned workspace; it makes no device allocation after the first call and is
capturable in a CUDA graph.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

from . import _lib
from ._lib import arr, call, i32, i64
from .typed import HomSpace, TensorMap, _release, torch

_PREC = {"fp64": _lib.PREC_FP64, "bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X, "cublas": _lib.PREC_CUBLAS_FP64}


@dataclass
class Step:
    """One pairwise contraction (``CompiledStep``, network.rs:931-941)."""

    lhs_slot: int
    rhs_slot: int
    result_slot: int
    lhs_axes: Tuple[int, ...]
    rhs_axes: Tuple[int, ...]
    output_axes: Tuple[int, ...]
    result_permutation: Optional[Tuple[Tuple[int, ...], Tuple[int, ...]]] = None


def _program(steps: Sequence[Step]) -> List[int]:
    prog: List[int] = []
    for s in steps:
        prog += [s.lhs_slot, s.rhs_slot, s.result_slot, len(s.lhs_axes), *s.lhs_axes, *s.rhs_axes]
        prog += [len(s.output_axes), *s.output_axes]
        if s.result_permutation is None:
            prog.append(-1)
        else:
            cod, dom = s.result_permutation
            prog += [len(cod), *cod, len(dom), *dom]
    return prog


class PlannedNetwork:
    """A compiled schedule over fixed input spaces (``PlannedNetwork``, network.rs:909)."""

    def __init__(self, spaces: Sequence[HomSpace], conj: Sequence[bool], steps: Sequence[Step], final_slot: int,
                 final_permutation=None):
        self.spaces = list(spaces)
        self.conj = [bool(c) for c in conj]
        self.steps = list(steps)
        self.final_slot = final_slot
        self.final_permutation = final_permutation
        prog = _program(self.steps)
        fin = [] if final_permutation is None else [len(final_permutation[0]), *final_permutation[0],
                                                     len(final_permutation[1]), *final_permutation[1]]
        handles = (C.c_void_p * len(self.spaces))(*[C.cast(s._h, C.c_void_p).value for s in self.spaces])
        h = C.c_void_p()
        call("tnt_network_plan", len(self.spaces), handles, arr(C.c_uint8, [1 if c else 0 for c in self.conj]),
             len(self.steps), arr(i32, prog), len(prog), final_slot, arr(i32, fin), len(fin), C.byref(h))
        self._h = h
        oh = C.c_void_p()
        call("tnt_nplan_output_space", h, C.byref(oh))
        self.output_space = HomSpace.from_handle(self.spaces[0].rule, oh)
        nx, nc, nb, nw = i64(), i64(), i64(), i64()
        fl = C.c_double()
        call("tnt_nplan_info", h, C.byref(nx), C.byref(nc), C.byref(fl), C.byref(nb), C.byref(nw))
        self.n_transforms, self.n_composes, self.flops = nx.value, nc.value, fl.value
        self.bytes_moved, self.workspace_elems = nb.value, nw.value
        self._ws = {}

    def __del__(self):
        _release("tnt_nplan_destroy", getattr(self, "_h", None))

    def workspace_bytes(self, precision: str = "fp64", slices: int = 6) -> int:
        b = C.c_size_t()
        call("tnt_nplan_workspace_bytes", self._h, _PREC[precision], slices, C.byref(b))
        return b.value

    def _workspace(self, runtime, precision, slices):
        key = (runtime.device, precision, slices)
        ws = self._ws.get(key)
        if ws is None:
            t = torch()
            n = max(1, self.workspace_bytes(precision, slices))
            ws = t.empty(n, dtype=t.uint8, device=f"cuda:{runtime.device}")
            self._ws[key] = ws
        return ws

    def execute(self, tensors: Sequence[TensorMap], precision: Optional[str] = None, slices: Optional[int] = None,
                out: Optional[TensorMap] = None) -> TensorMap:
        """``PlannedNetwork::execute`` (network.rs:1609): device-resident, no fallback."""
        if len(tensors) != len(self.spaces):
            raise ValueError(f"plan has {len(self.spaces)} operands but {len(tensors)} tensors were given")
        rt = tensors[0].runtime
        for i, (t, sp) in enumerate(zip(tensors, self.spaces)):
            if t.runtime is not rt:
                raise ValueError(f"operand {i} uses a different Runtime")
            if not t.space.same_as(sp):
                raise ValueError(f"operand {i} does not match the planned space")
        prec = precision or rt.precision
        sl = slices or rt.slices
        if out is None:
            out = TensorMap(rt, self.output_space)
        elif not out.space.same_as(self.output_space):
            raise ValueError("out does not have the network's output space")
        ws = self._workspace(rt, prec, sl)
        ptrs = (C.c_void_p * len(tensors))(*[t.data.data_ptr() for t in tensors])
        call("tnt_network_execute", rt._h, self._h, len(tensors), ptrs, C.c_void_p(out.data.data_ptr()),
             C.c_void_p(ws.data_ptr()), ws.numel(), _PREC[prec], sl, rt.stream())
        return out


class Network:
    """Written label lists (``Network::new``, network.rs:235-266).

    ``inputs[i]`` are operand i's labels in flat leg order (codomain then
    domain of the tensor as passed), ``conj[i]`` marks adjoint operands,
    ``codomain_splits[i]`` is the written ``;`` position (checked against the
    tensor at planning), ``output`` the result's labels and
    ``output_codomain_rank`` how many of them form its codomain (None: all).
    """

    def __init__(self, inputs, conj=None, codomain_splits=None, output=(), output_codomain_rank=None):
        self.inputs = [list(l) for l in inputs]
        n = len(self.inputs)
        self.conj = [False] * n if conj is None else [bool(c) for c in conj]
        self.codomain_splits = [None] * n if codomain_splits is None else list(codomain_splits)
        if len(self.conj) != n or len(self.codomain_splits) != n:
            raise ValueError("operand marker lists must match operand count")
        self.output = list(output)
        if output_codomain_rank is not None and output_codomain_rank > len(self.output):
            raise ValueError(f"output codomain rank {output_codomain_rank} exceeds output rank {len(self.output)}")
        self.output_codomain_rank = output_codomain_rank
        count = {}
        for i, labels in enumerate(self.inputs):
            if len(set(labels)) != len(labels):
                raise ValueError(f"operand {i} repeats a label (traces are not contractions)")
            for l in labels:
                count[l] = count.get(l, 0) + 1
        bad = [l for l, c in count.items() if c > 2]
        if bad:
            raise ValueError(f"label {bad[0]!r} appears more than twice (hyperedge)")
        open_labels = [l for l, c in count.items() if c == 1]
        if len(set(self.output)) != len(self.output):
            raise ValueError("output labels repeat")
        if sorted(map(repr, open_labels)) != sorted(map(repr, self.output)):
            raise ValueError("output labels must be exactly the open labels")

    def _lowered_labels(self, spaces):
        labels = []
        for i, (sp, written) in enumerate(zip(spaces, self.inputs)):
            n1, n = sp.n1, sp.n1 + sp.n2
            if len(written) != n:
                raise ValueError(f"operand {i} has rank {n} but {len(written)} labels")
            split = self.codomain_splits[i]
            if split is not None and split != n1:
                raise ValueError(f"operand {i}: written split {split} differs from the tensor's codomain rank {n1}")
            labels.append(written[n1:] + written[:n1] if self.conj[i] else list(written))
        return labels

    def plan(self, tensors, order=None) -> PlannedNetwork:
        """Pick a pairwise order and compile it (``Network::plan`` / ``plan_with``).

        ``tensors`` are TensorMaps or their HomSpaces (planning reads only the
        structure, as the reference's planner reads only metadata).

        ``order=None`` contracts greedily: at each stage the pair sharing a
        label whose result has the fewest reduced entries (ties: lowest slot
        indices).  ``order`` as a label list contracts, for each label not yet
        contracted, the two operands holding it (all their shared labels at
        once), as ``LabelOrderDenseOptimizer`` does.  ``order="exhaustive"``
        compiles every pairwise order of up to six operands and keeps the one
        with the fewest block-sparse compose flops, then the fewest transform
        bytes (the reference's block-sparse cost, tenet-network/src/cost.rs).
        """
        if len(tensors) != len(self.inputs):
            raise ValueError(f"network has {len(self.inputs)} operands but {len(tensors)} tensors were given")
        spaces = [t.space if isinstance(t, TensorMap) else t for t in tensors]
        labels = self._lowered_labels(spaces)
        dims, cod_rank0 = {}, {}
        for i, sp in enumerate(spaces):
            legs = list(sp.codomain) + list(sp.domain)
            n1 = sp.n1
            if self.conj[i]:
                legs, n1 = legs[n1:] + legs[:n1], sp.n2
            cod_rank0[i] = n1
            for lab, leg in zip(labels[i], legs):
                dims[lab] = leg.reduced_dim()
        if isinstance(order, str):
            if order != "exhaustive":
                raise ValueError(f"unknown order {order!r}")
            if len(spaces) > 6:
                raise ValueError("exhaustive planning is limited to six operands")
            best = None
            for seq in _pair_sequences({i: list(l) for i, l in enumerate(labels)}):
                plan = self._build(spaces, labels, cod_rank0, dims, None, seq)
                key = (plan.flops, plan.bytes_moved)
                if best is None or key < best[0]:
                    best = (key, plan)
            return best[1]
        return self._build(spaces, labels, cod_rank0, dims, order, None)

    def _build(self, spaces, labels, cod_rank0, dims, order, seq) -> PlannedNetwork:
        """Compile one pairwise order: label order ``order``, pair-choice
        sequence ``seq`` (indices into each stage's candidate pairs), or greedy."""
        cod_rank = dict(cod_rank0)
        slots = {i: list(labels[i]) for i in range(len(spaces))}
        steps: List[Step] = []

        def transforms(x, y):
            """Operand permutes a contraction x . y needs (0, 1 or 2)."""
            a, b = slots[x], slots[y]
            shared = [lab for lab in a if lab in b]
            k = len(shared)
            la = [a.index(lab) for lab in shared]
            ra = [b.index(lab) for lab in shared]
            lhs_ok = la == list(range(len(a) - k, len(a))) and cod_rank[x] == len(a) - k
            rhs_ok = ra == list(range(k)) and cod_rank[y] == k
            return (not lhs_ok) + (not rhs_ok)

        def contract(i, j):
            # the orientation needing fewer operand permutes, lower slot first on ties
            if transforms(j, i) < transforms(i, j):
                i, j = j, i
            a, b = slots.pop(i), slots.pop(j)
            shared = [lab for lab in a if lab in b]
            res = [lab for lab in a if lab not in shared] + [lab for lab in b if lab not in shared]
            r = len(spaces) + len(steps)
            steps.append(Step(i, j, r, tuple(a.index(x) for x in shared), tuple(b.index(x) for x in shared),
                              tuple(range(len(res)))))
            slots[r] = res
            cod_rank[r] = len(a) - len(shared)

        for lab in order or ():
            holders = sorted(s for s, ls in slots.items() if lab in ls)
            if len(holders) == 2:
                contract(*holders)
        stage = 0
        while len(slots) > 1:
            pairs = _candidate_pairs(slots)
            if seq is not None:
                contract(*pairs[seq[stage]])
                stage += 1
                continue

            def cost(pair):
                a, b = slots[pair[0]], slots[pair[1]]
                size = 1
                for lab in a + b:
                    if not (lab in a and lab in b):
                        size *= dims[lab]
                return (size, pair)

            contract(*min(pairs, key=cost))
        final_slot = next(iter(slots))
        final = slots[final_slot]
        k = len(self.output) if self.output_codomain_rank is None else self.output_codomain_rank
        cod = tuple(final.index(lab) for lab in self.output[:k])
        dom = tuple(final.index(lab) for lab in self.output[k:])
        perm = None if (cod_rank[final_slot] == k and cod + dom == tuple(range(len(final)))) else (cod, dom)
        return PlannedNetwork(spaces, self.conj, steps, final_slot, perm)


def _candidate_pairs(slots):
    """Pairs of live slots that share a label (all pairs when none do), in slot order."""
    keys = sorted(slots)
    pairs = [(x, y) for x in keys for y in keys if x < y and any(lab in slots[y] for lab in slots[x])]
    return pairs or [(x, y) for x in keys for y in keys if x < y]


def _pair_sequences(slots, nxt=None):
    """Every sequence of candidate-pair choices that contracts ``slots`` to one."""
    if len(slots) <= 1:
        yield []
        return
    nxt = max(slots) + 1 if nxt is None else nxt
    for idx, (x, y) in enumerate(_candidate_pairs(slots)):
        a, b = slots[x], slots[y]
        rest = {k: v for k, v in slots.items() if k not in (x, y)}
        rest[nxt] = [lab for lab in a if lab not in b] + [lab for lab in b if lab not in a]
        for tail in _pair_sequences(rest, nxt + 1):
            yield [idx] + tail
