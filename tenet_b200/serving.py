"""Continuous-batching service of iTEBD bond updates for many independent chains.

Each chain is an SU(2) Heisenberg iTEBD simulation with its own bond space W
(spins 0..3, a total reduced bond dimension D split evenly over the seven
spins) and its own Trotter step tau; its MPS tensors A, B : (W x P) <- W stay
resident on the device.  A request is one two-site update of a chain, the
iTEBD bond update of ``itebd.bond_update``: theta = A . B, the gate
exp(-tau S.S), 6j recoupling into the
bond matrix, truncated SVD back to W (``Truncation::space(W)``), and the
publish step A <- U, B <- (S Vh) recoupled to (W x P) <- W.

All tensors of all chains and every in-flight request's intermediates live in
one device arena (``Arena``) of the configured byte budget; a request is
admitted when its chain is idle and its intermediates fit (admission by
memory budget).  Two schedulers:

* ``serve`` (continuous batching, the default): requests are admitted the
  moment a lane and memory free up and run on one of several lanes (a CUDA
  stream with its own context), each request as its own short launch
  sequence over the chain's cached plans with every host table and result
  moved asynchronously, so nothing on the host waits for the GPU.  Requests
  that arrive while others are on the GPU start at once and run beside them:
  a small chain's update finishes while a large chain's SVD is still running.
  Completion is observed by polling each request's event.
* ``serve_ticks``: ticks; each tick runs the admitted batch as ONE grouped
  launch per stage (plans concatenated over arena offsets,
  ``tnt_*plan_concat``), and requests that arrive during a tick wait for the
  next one.

Results do not depend on the scheduler or on which other requests run
beside a request: every kernel computes each request's blocks independently.
Products whose K is too thin for split precision (the gate contraction over
the physical legs, K = 1) run in FP64 at every precision.
"""

from __future__ import annotations

import bisect
import ctypes as C
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _lib, typed
from ._lib import call, i32, i64

PREC = {"fp64": _lib.PREC_FP64, "bf16x": _lib.PREC_BF16X, "i8x": _lib.PREC_INT8X}


class Arena:
    """First-fit allocator of float64 elements over one device buffer."""

    def __init__(self, device: int, capacity_elems: int):
        t = typed.torch()
        self.capacity = int(capacity_elems)
        self.buf = t.empty(self.capacity, dtype=t.float64, device=f"cuda:{device}")
        self.free = [(0, self.capacity)]  # sorted (offset, length)
        self.used = 0

    @staticmethod
    def _round(n):
        return (int(n) + 31) // 32 * 32  # 256-byte granules

    def alloc(self, n: int) -> Optional[int]:
        n = self._round(max(n, 1))
        for i, (off, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (off + n, ln - n)
                self.used += n
                return off
        return None

    def release(self, off: int, n: int):
        n = self._round(max(n, 1))
        self.used -= n
        i = bisect.bisect_left(self.free, (off, 0))
        self.free.insert(i, (off, n))
        # coalesce neighbours
        if i + 1 < len(self.free) and self.free[i][0] + self.free[i][1] == self.free[i + 1][0]:
            self.free[i] = (self.free[i][0], self.free[i][1] + self.free[i + 1][1])
            self.free.pop(i + 1)
        if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == self.free[i][0]:
            self.free[i - 1] = (self.free[i - 1][0], self.free[i - 1][1] + self.free[i][1])
            self.free.pop(i)

    def ptr(self, off=0):
        return C.c_void_p(self.buf.data_ptr() + 8 * off)

    def view(self, off, n):
        return self.buf[off: off + n]


@dataclass
class ChainPlans:
    """Compiled plans of one chain's update (cached per chain, reused by every request)."""

    W: "typed.GradedSpace"
    a_space: "typed.HomSpace"
    g_off: int  # gate tensor in the arena
    x_b: "typed.TransformPlan"     # B -> W <- (P* x W)
    c_theta: "typed.ComposePlan"   # A o xb
    x_t: "typed.TransformPlan"     # theta -> (P* x W) <- ... for the gate
    c_gate: "typed.ComposePlan"    # G o theta'
    x_bond: "typed.TransformPlan"  # gated -> (W x P) <- (P* x W)
    f_bond: "typed.FactorPlan"
    x_back: "typed.TransformPlan"  # S Vh : W <- (P* x W)  ->  (W x P) <- W
    svh_space: "typed.HomSpace"
    ranks: List[int]
    sizes: Dict[str, int] = field(default_factory=dict)
    split_doubles: int = 0  # slice-pack scratch of this chain's composes (split precisions), in doubles
    publish: List[Tuple] = field(default_factory=list)  # (rec, m, n, k, A sector offset, S Vh sector offset)
    ranks_dev: object = None  # the per-sector ranks on the device (continuous scheduler)


@dataclass
class Chain:
    cid: int
    D: int
    tau: float
    plans: ChainPlans
    a_off: int
    b_off: int
    busy: bool = False


@dataclass
class Request:
    rid: int
    cid: int
    arrival: float
    start: float = 0.0
    done: float = 0.0
    err: float = 0.0
    offs: Dict[str, int] = field(default_factory=dict)
    lane: int = -1
    pending: Dict = field(default_factory=dict)  # device / pinned buffers alive until completion


@dataclass
class Lane:
    """A CUDA stream with its own context (so lanes share no scratch)."""

    ctx: object
    stream: object
    inflight: List[Request] = field(default_factory=list)
    work: float = 0.0


def chain_bond_space(rule, D):
    """Split D evenly over the seven spins 0..3 (D rounded to a multiple of 7)."""
    d = max(1, int(round(D / 7.0)))
    return typed.GradedSpace(rule, [(tj, d) for tj in range(7)])


class ServingLoop:
    def __init__(self, rt: "typed.Runtime", budget_bytes: int, precision="fp64", slices=6, lanes: int = 4):
        self.rt = rt
        self.rule = typed.SU2FusionRule()
        self.P = typed.GradedSpace(self.rule, [(1, 1)])
        self.arena = Arena(rt.device, budget_bytes // 8)
        self.precision = precision
        self.slices = slices
        self.chains: List[Chain] = []
        self._plan_cache: Dict = {}
        self.stream = rt.stream()
        self.nlanes = lanes
        self.lanes: List[Lane] = []

    def __del__(self):
        for ln in getattr(self, "lanes", []):
            try:
                ln.stream.synchronize()
                _lib.lib().tnt_ctx_destroy(ln.ctx)
            except Exception:
                pass

    def _prec(self, plan):
        """The chain precision for plans that suit it, FP64 for thin-K ones."""
        return PREC[self.precision] if self.precision == "fp64" or plan.suits_split else PREC["fp64"]

    # -- chain setup -------------------------------------------------------
    def _plans(self, D, tau):
        key = (chain_bond_space(self.rule, D)._degs, tau)
        if key in self._plan_cache:
            return self._plan_cache[key]
        rt, rule, P = self.rt, self.rule, self.P
        W = chain_bond_space(rule, D)
        a_sp = rt.space(rule, [W, P], [W])
        x_b = rt.xplan(a_sp, "permute", [0], [1, 2])
        c_theta = rt.cplan(a_sp, x_b.dst)
        x_t = rt.xplan(c_theta.dst, "permute", [1, 2], [0, 3])
        g_sp = rt.space(rule, [P, P], [P, P])
        c_gate = rt.cplan(g_sp, x_t.dst)
        x_bond = rt.xplan(c_gate.dst, "permute", [2, 0], [1, 3])
        f_bond = rt.fplan(x_bond.dst)
        bond_secs = x_bond.dst.sectors()
        ranks = [W.degeneracy(rule.unlabel(lab)) for lab, _, _, _ in bond_secs]
        svh_sp = rt.space(rule, [W], list(x_bond.dst.domain))
        x_back = rt.xplan(svh_sp, "permute", [0, 1], [2])
        g_off = self.arena.alloc(g_sp.size)
        gate = np.zeros(g_sp.size)
        for lab, r, c, off in g_sp.sectors():
            gate[off] = math.exp(-tau * (-0.75 if lab[0] == 0 else 0.25))
        self.arena.view(g_off, g_sp.size).copy_(typed.torch().as_tensor(gate))
        plans = ChainPlans(W, a_sp, g_off, x_b, c_theta, x_t, c_gate, x_bond, f_bond, x_back, svh_sp, ranks)
        a_secs = {lab: off for lab, _, _, off in a_sp.sectors()}
        svh_secs = {lab: off for lab, _, _, off in svh_sp.sectors()}
        for (lab, m, nn, _), rec, k in zip(bond_secs, f_bond.records, ranks):
            if k == 0:
                continue
            if lab not in a_secs or k > int(rec[2]):
                raise RuntimeError("truncated bond differs from the chain's bond space")
            plans.publish.append((rec, m, nn, k, a_secs[lab], svh_secs[lab]))
        plans.sizes = dict(
            xb=x_b.dst.size, theta=c_theta.dst.size, thp=x_t.dst.size, gated=c_gate.dst.size,
            bond=x_bond.dst.size, u=f_bond.u_size, s=f_bond.s_size, v=f_bond.v_size, svh=svh_sp.size,
            svdw=f_bond.work_elems,
        )
        if self.precision != "fp64":
            need = 0
            for cp in (c_theta, c_gate):
                nb = C.c_size_t()
                call("tnt_cplan_scratch_bytes", cp._h, 1, PREC[self.precision], self.slices, C.byref(nb))
                need = max(need, nb.value)
            plans.split_doubles = (need + 7) // 8
        self._plan_cache[key] = plans
        return plans

    def add_chain(self, D: int, tau: float, seed: int) -> Chain:
        from .workloads import splitmix_normal

        plans = self._plans(D, tau)
        n = plans.a_space.size
        a_off, b_off = self.arena.alloc(n), self.arena.alloc(n)
        if a_off is None or b_off is None:
            raise MemoryError("arena too small for the chain states")
        t = typed.torch()
        for off, sd in ((a_off, 2 * seed + 1), (b_off, 2 * seed + 2)):
            v = splitmix_normal(sd, n)
            self.arena.view(off, n).copy_(t.as_tensor(v / np.linalg.norm(v)))
        ch = Chain(len(self.chains), D, tau, plans, a_off, b_off)
        self.chains.append(ch)
        return ch

    # -- checkpoints ---------------------------------------------------------
    def checkpoint_chain(self, cid: int, codec=None) -> Tuple[bytes, bytes]:
        """v1 typed snapshots of a chain's resident MPS tensors A and B (one
        device-to-host copy each), for checkpointing a live service."""
        from . import persistence

        ch = self.chains[cid]
        n = ch.plans.a_space.size
        return tuple(persistence.payload_to_bytes(ch.plans.a_space, self.arena.view(off, n).cpu().numpy(), codec)
                     for off in (ch.a_off, ch.b_off))

    def restore_chain(self, cid: int, snapshots: Tuple[bytes, bytes], codec=None):
        """Write snapshots back into a chain's arena slots.  Each must decode to
        exactly the chain's MPS space (a dense, non-adjoint body)."""
        from . import persistence

        ch = self.chains[cid]
        if ch.busy:
            raise RuntimeError("chain has an update in flight")
        payloads = []
        for data in snapshots:
            sp, payload, adjoint = persistence.payload_from_bytes(data, codec)
            if adjoint or not sp.same_as(ch.plans.a_space):
                raise persistence.DecodeError("invalid_format", "snapshot does not hold this chain's MPS space")
            payloads.append(payload)
        t = typed.torch()
        n = ch.plans.a_space.size
        for off, payload in zip((ch.a_off, ch.b_off), payloads):
            self.arena.view(off, n).copy_(t.as_tensor(payload))

    def request_bytes(self, ch: Chain) -> int:
        return 8 * sum(Arena._round(v) for v in ch.plans.sizes.values())

    # -- one tick ------------------------------------------------------------
    def _alloc_request(self, req: Request) -> bool:
        ch = self.chains[req.cid]
        got = {}
        for name, n in ch.plans.sizes.items():
            off = self.arena.alloc(n)
            if off is None:
                for k, o in got.items():
                    self.arena.release(o, ch.plans.sizes[k])
                return False
            got[name] = off
        req.offs = got
        return True

    def _release_request(self, req: Request):
        ch = self.chains[req.cid]
        for k, o in req.offs.items():
            self.arena.release(o, ch.plans.sizes[k])
        req.offs = {}

    def _tick_scratch(self, batch: List[Request]):
        """Arena block for the slice packs of one tick's grouped composes.

        The packs of a concatenated plan are the per-chain packs side by side,
        so the sum of the chains' needs (plus alignment slack) bounds them.
        Returns (offset, doubles), (None, 0) for FP64, or None if it does not fit.
        """
        if self.precision == "fp64":
            return (None, 0)
        n = sum(self.chains[r.cid].plans.split_doubles for r in batch) + 8192
        off = self.arena.alloc(n)
        return None if off is None else (off, n)

    def run_tick(self, batch: List[Request], scratch=(None, 0)):
        """Execute one grouped update of every request in ``batch``."""
        if not batch:
            return
        rt, ar, st = self.rt, self.arena, self.stream
        base = ar.ptr(0)
        chs = [self.chains[r.cid] for r in batch]
        n = len(batch)
        H = lambda objs: (C.c_void_p * n)(*[o._h for o in objs])
        I64 = lambda vals: (i64 * n)(*vals)

        def xform(plans, srcs, dsts):
            h = C.c_void_p()
            call("tnt_xplan_concat", n, H(plans), I64(srcs), I64(dsts), C.byref(h))
            try:
                call("tnt_transform", rt._h, h, base, base, 1.0, 0.0, st)
            finally:
                _lib.lib().tnt_xplan_destroy(h)

        def compose(plans, a, b, c):
            # one grouped launch per arithmetic: chains whose plan suits the
            # split precision, and (FP64) those whose products are too thin
            groups: Dict[int, List[int]] = {}
            for i, pl in enumerate(plans):
                groups.setdefault(self._prec(pl), []).append(i)
            for prec, idx in groups.items():
                m = len(idx)
                h = C.c_void_p()
                call("tnt_cplan_concat", m, (C.c_void_p * m)(*[plans[i]._h for i in idx]),
                     (i64 * m)(*[a[i] for i in idx]), (i64 * m)(*[b[i] for i in idx]),
                     (i64 * m)(*[c[i] for i in idx]), C.byref(h))
                try:
                    if scratch[0] is None or prec == PREC["fp64"]:
                        call("tnt_compose", rt._h, h, 1, base, 0, base, 0, base, 0, 1.0, 0.0, prec, self.slices, st)
                    else:
                        call("tnt_compose_ws", rt._h, h, 1, base, 0, base, 0, base, 0, 1.0, 0.0, prec,
                             self.slices, ar.ptr(scratch[0]), 8 * scratch[1], st)
                finally:
                    _lib.lib().tnt_cplan_destroy(h)

        xform([c.plans.x_b for c in chs], [c.b_off for c in chs], [r.offs["xb"] for r in batch])
        compose([c.plans.c_theta for c in chs], [c.a_off for c in chs], [r.offs["xb"] for r in batch],
                [r.offs["theta"] for r in batch])
        xform([c.plans.x_t for c in chs], [r.offs["theta"] for r in batch], [r.offs["thp"] for r in batch])
        compose([c.plans.c_gate for c in chs], [c.plans.g_off for c in chs], [r.offs["thp"] for r in batch],
                [r.offs["gated"] for r in batch])
        xform([c.plans.x_bond for c in chs], [r.offs["gated"] for r in batch], [r.offs["bond"] for r in batch])

        # batched SVD of every request's bond matrix, truncation per request
        fh = C.c_void_p()
        call("tnt_fplan_concat", n, H([c.plans.f_bond for c in chs]), I64([r.offs["bond"] for r in batch]),
             I64([r.offs["u"] for r in batch]), I64([r.offs["s"] for r in batch]), I64([r.offs["v"] for r in batch]),
             I64([r.offs["svdw"] for r in batch]), C.byref(fh))
        try:
            call("tnt_svd_ws", rt._h, fh, base, base, base, base, base, st)
            seg = [0]
            ranks = []
            for c in chs:
                seg.append(seg[-1] + c.plans.f_bond.nsectors)
                ranks.extend(c.plans.ranks)
            t = typed.torch()
            kept = t.empty(seg[-1], dtype=t.int64, device=ar.buf.device)
            err = t.empty(n, dtype=t.float64, device=ar.buf.device)
            call("tnt_truncate_segments", rt._h, fh, n, (i32 * (n + 1))(*seg), base, _lib.TRUNC_SPACE, 0.0, 0.0,
                 (i64 * len(ranks))(*ranks), C.c_void_p(kept.data_ptr()), C.c_void_p(err.data_ptr()), st)
        finally:
            _lib.lib().tnt_fplan_destroy(fh)
        kept_h = kept.cpu().numpy()
        err_h = err.cpu().numpy()

        # publish: A <- U[:, :kept] per sector; SVh <- S Vh[:kept, :]; B <- permute(SVh)
        table = []
        pos = 0
        for r, c in zip(batch, chs):
            a_secs = {lab: off for lab, _, _, off in c.plans.a_space.sectors()}
            svh_secs = {lab: off for lab, _, _, off in c.plans.svh_space.sectors()}
            for (lab, m, nn, _), rec in zip(c.plans.x_bond.dst.sectors(), c.plans.f_bond.records):
                k = int(kept_h[pos])
                pos += 1
                if k == 0:
                    continue
                kk = int(rec[2])
                if lab not in a_secs or k != c.plans.W.degeneracy(c.plans.W.rule.unlabel(lab)):
                    raise RuntimeError("truncated bond differs from the chain's bond space")
                table.append([r.offs["u"] + int(rec[4]), c.a_off + a_secs[lab], m, k, m, m, -1])
                table.append([r.offs["v"] + int(rec[6]), r.offs["svh"] + svh_secs[lab], k, nn, kk, k,
                              r.offs["s"] + int(rec[5])])
        arr = np.asarray(table, dtype=np.int64).ravel()
        call("tnt_copy_segments", rt._h, len(table), arr.ctypes.data_as(C.POINTER(i64)), base, base, base, st)
        xform([c.plans.x_back for c in chs], [r.offs["svh"] for r in batch], [c.b_off for c in chs])
        typed.torch().cuda.synchronize(self.rt.device)
        for i, r in enumerate(batch):
            r.err = float(err_h[i])

    # -- continuous scheduler: lanes -----------------------------------------------
    def _ensure_lanes(self):
        t = typed.torch()
        while len(self.lanes) < self.nlanes:
            h = C.c_void_p()
            call("tnt_ctx_create", self.rt.device, C.byref(h))
            self.lanes.append(Lane(h, t.cuda.Stream(self.rt.device)))

    def _launch(self, req: Request, lane: Lane):
        """Enqueue one request's whole update on a lane; no host synchronisation."""
        t = typed.torch()
        ch = self.chains[req.cid]
        p, o, ar = ch.plans, req.offs, self.arena
        ctx, st = lane.ctx, C.c_void_p(lane.stream.cuda_stream)
        ptr = ar.ptr
        dev = ar.buf.device
        with t.cuda.stream(lane.stream):
            if p.ranks_dev is None:
                p.ranks_dev = t.tensor(p.ranks, dtype=t.int64).to(dev)
            status = t.empty(2, dtype=t.int32, device=dev)
            kept = t.empty(p.f_bond.nsectors, dtype=t.int64, device=dev)
            err = t.empty(1, dtype=t.float64, device=dev)
            rows = []
            for rec, m, nn, k, a_sec, svh_sec in p.publish:
                kk = int(rec[2])
                rows.append([o["u"] + int(rec[4]), ch.a_off + a_sec, m, k, m, m, -1])
                rows.append([o["v"] + int(rec[6]), o["svh"] + svh_sec, k, nn, kk, k, o["s"] + int(rec[5])])
            table = t.tensor(np.asarray(rows, dtype=np.int64).ravel()).pin_memory().to(dev, non_blocking=True)
        call("tnt_transform", ctx, p.x_b._h, ptr(o["xb"]), ptr(ch.b_off), 1.0, 0.0, st)
        call("tnt_compose", ctx, p.c_theta._h, 1, ptr(o["theta"]), 0, ptr(ch.a_off), 0, ptr(o["xb"]), 0, 1.0, 0.0,
             self._prec(p.c_theta), self.slices, st)
        call("tnt_transform", ctx, p.x_t._h, ptr(o["thp"]), ptr(o["theta"]), 1.0, 0.0, st)
        call("tnt_compose", ctx, p.c_gate._h, 1, ptr(o["gated"]), 0, ptr(p.g_off), 0, ptr(o["thp"]), 0, 1.0, 0.0,
             self._prec(p.c_gate), self.slices, st)
        call("tnt_transform", ctx, p.x_bond._h, ptr(o["bond"]), ptr(o["gated"]), 1.0, 0.0, st)
        P = lambda x: C.c_void_p(x.data_ptr())
        call("tnt_svd_ws_async", ctx, p.f_bond._h, ptr(o["bond"]), ptr(o["u"]), ptr(o["s"]), ptr(o["v"]),
             ptr(o["svdw"]), P(status), st)
        call("tnt_truncate_async", ctx, p.f_bond._h, ptr(o["s"]), _lib.TRUNC_SPACE, 0.0, 0.0, P(p.ranks_dev),
             P(kept), P(err), st)
        call("tnt_copy_segments_async", ctx, len(rows), P(table), ptr(0), ptr(0), ptr(0), st)
        call("tnt_transform", ctx, p.x_back._h, ptr(ch.b_off), ptr(o["svh"]), 1.0, 0.0, st)
        with t.cuda.stream(lane.stream):
            host = {k_: t.empty(v.shape, dtype=v.dtype, pin_memory=True) for k_, v in
                    (("status", status), ("kept", kept), ("err", err))}
            for k_, v in (("status", status), ("kept", kept), ("err", err)):
                host[k_].copy_(v, non_blocking=True)
            ev = t.cuda.Event()
            ev.record(lane.stream)
        req.pending = {"event": ev, "host": host, "dev": (status, kept, err, table)}

    def _finish(self, req: Request):
        """Read a completed request's status and truncation (already on the host)."""
        h = req.pending["host"]
        p = self.chains[req.cid].plans
        if int(h["status"][0]) != 0:
            raise RuntimeError("Jacobi SVD did not converge within the sweep limit")
        if [int(k) for k in h["kept"].tolist()] != list(p.ranks):
            raise RuntimeError("truncated bond differs from the chain's bond space")
        req.err = float(h["err"][0])
        req.pending = {}

    def serve(self, requests: List[Request], max_inflight_per_lane: int = 2):
        """Serve ``requests`` (sorted by arrival, seconds from now) with the
        continuous scheduler; returns them with timings.

        Every loop iteration retires the requests whose events completed,
        then admits arrived requests in arrival order while their chain is
        idle, a lane has fewer than ``max_inflight_per_lane`` requests in
        flight and the arena has room; an admitted request goes to the lane
        with the least estimated outstanding work (D^3)."""
        self._ensure_lanes()
        t0 = time.perf_counter()
        pending: List[Request] = []
        queue = list(requests)
        qi = 0
        done = []
        while qi < len(queue) or pending or any(ln.inflight for ln in self.lanes):
            now = time.perf_counter() - t0
            while qi < len(queue) and queue[qi].arrival <= now:
                pending.append(queue[qi])
                qi += 1
            progressed = False
            for ln in self.lanes:
                still = []
                for r in ln.inflight:
                    if r.pending["event"].query():
                        self._finish(r)
                        r.done = time.perf_counter() - t0
                        ln.work -= self.chains[r.cid].D ** 3
                        self._release_request(r)
                        self.chains[r.cid].busy = False
                        done.append(r)
                        progressed = True
                    else:
                        still.append(r)
                ln.inflight = still
            rest = []
            for r in pending:
                ch = self.chains[r.cid]
                free = [ln for ln in self.lanes if len(ln.inflight) < max_inflight_per_lane]
                if free and not ch.busy and self._alloc_request(r):
                    ln = min(free, key=lambda l_: l_.work)
                    ch.busy = True
                    r.lane = self.lanes.index(ln)
                    r.start = time.perf_counter() - t0
                    self._launch(r, ln)
                    ln.inflight.append(r)
                    ln.work += ch.D ** 3
                    progressed = True
                else:
                    rest.append(r)
            pending = rest
            if not progressed:
                time.sleep(5e-5)
        return done, time.perf_counter() - t0

    # -- the tick scheduler ---------------------------------------------------------
    def serve_ticks(self, requests: List[Request], max_batch: int = 1 << 30):
        """Serve ``requests`` (sorted by arrival, seconds from now) in ticks; returns them with timings."""
        t0 = time.perf_counter()
        pending: List[Request] = []
        queue = list(requests)
        qi = 0
        done = []
        while qi < len(queue) or pending:
            now = time.perf_counter() - t0
            while qi < len(queue) and queue[qi].arrival <= now:
                pending.append(queue[qi])
                qi += 1
            batch = []
            rest = []
            for r in pending:
                ch = self.chains[r.cid]
                if len(batch) < max_batch and not ch.busy and self._alloc_request(r):
                    ch.busy = True
                    batch.append(r)
                else:
                    rest.append(r)
            # the tick's slice-pack scratch also comes out of the budget:
            # shrink the tick until it fits
            scratch = None
            while batch:
                scratch = self._tick_scratch(batch)
                if scratch is not None:
                    break
                r = batch.pop()
                self._release_request(r)
                self.chains[r.cid].busy = False
                rest.insert(0, r)
            pending = rest
            if not batch:
                if qi < len(queue):
                    wait = queue[qi].arrival - (time.perf_counter() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.002))
                continue
            start = time.perf_counter() - t0
            self.run_tick(batch, scratch)
            if scratch[0] is not None:
                self.arena.release(scratch[0], scratch[1])
            end = time.perf_counter() - t0
            for r in batch:
                r.start, r.done = start, end
                self._release_request(r)
                self.chains[r.cid].busy = False
                done.append(r)
        return done, time.perf_counter() - t0


def poisson_requests(nchains, nreq, rate, seed=0):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
    cids = rng.integers(0, nchains, size=nreq)
    return [Request(i, int(c), float(a)) for i, (c, a) in enumerate(zip(cids, t))]


def chain_mix(nchains, seed=0):
    """Per-chain D log-uniform in [32, 2048] and tau from {0.01, 0.05, 0.1}."""
    rng = np.random.default_rng(seed)
    D = np.exp(rng.uniform(math.log(32), math.log(2048), size=nchains))
    tau = rng.choice([0.01, 0.05, 0.1], size=nchains)
    return [(int(round(d)), float(t)) for d, t in zip(D, tau)]
