"""Multi-GPU replicas host logic on CPU: two gloo ranks.

The path shards by independent tensors with no data-path collective; the
ranks meet only in the timing barrier and in the maximum of their device
times.  Run as two processes over gloo on 127.0.0.1.
"""

import os

import numpy as np
import pytest


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tenet_b200 import replicas

        replicas.barrier()
        t = replicas.max_over_ranks(10.0 + rank, device="cpu")
        seeds = replicas.replica_seeds(rank, 64)
        # each replica composes its own tensors with the CPU restatement
        from oracle.fusion import HomSpace, Leg
        from oracle.sectors import U1, Rule
        from oracle.tensor import TensorMap, normal_fill

        r = Rule([U1])
        v = Leg.new(r, [((-1,), 2), ((0,), 3), ((1,), 2)])
        sp = HomSpace(r, [v, v], [v, v])
        sa, sb = seeds[0]
        c = TensorMap(sp, normal_fill(sa, sp.size)).compose(TensorMap(sp, normal_fill(sb, sp.size)))
        out.put((rank, t, seeds, float(c.norm())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_max_and_disjoint_replicas():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, s0, n0), (r1, t1, s1, n1) = res
    assert t0 == t1 == 11.0  # every rank sees the slowest replica's time
    assert not set(x for pair in s0 for x in pair) & set(x for pair in s1 for x in pair)
    assert n0 != n1 and np.isfinite(n0) and np.isfinite(n1)


def test_single_process_is_its_own_maximum():
    from tenet_b200 import replicas

    assert replicas.max_over_ranks(3.5) == 3.5
    with pytest.raises(ValueError):
        replicas.replica_seeds(0, 1001)
