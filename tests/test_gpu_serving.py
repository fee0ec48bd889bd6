"""Continuous-batching iTEBD service: batching and lanes do not change
results, a request that arrives during a large update runs beside it, and the
published state equals the single-request device update."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_loop(chains, budget=2 << 30, precision="fp64"):
    import tenet_b200 as tb
    from tenet_b200 import serving

    rt = tb.Runtime(0)
    loop = serving.ServingLoop(rt, budget, precision)
    for i, (D, tau) in enumerate(chains):
        loop.add_chain(D, tau, seed=100 + i)
    return loop


def snapshot(loop):
    return [(loop.arena.view(c.a_off, c.plans.a_space.size).clone(),
             loop.arena.view(c.b_off, c.plans.a_space.size).clone()) for c in loop.chains]


def restore(loop, snap):
    for c, (a, b) in zip(loop.chains, snap):
        loop.arena.view(c.a_off, a.numel()).copy_(a)
        loop.arena.view(c.b_off, b.numel()).copy_(b)


@pytest.mark.parametrize("precision", ["fp64", "bf16x", "i8x"])
def test_result_is_the_same_alone_and_in_the_mix(precision):
    """Bit-identical: every sector's arithmetic is independent of the tick it runs in."""
    from tenet_b200 import serving

    loop = make_loop([(40, 0.05), (90, 0.1), (140, 0.01), (64, 0.05), (210, 0.1)], precision=precision)
    snap = snapshot(loop)
    target = 2
    alone_req = serving.Request(0, target, 0.0)
    assert loop._alloc_request(alone_req)
    scratch = loop._tick_scratch([alone_req])
    loop.run_tick([alone_req], scratch)
    if scratch[0] is not None:
        loop.arena.release(*scratch)
    loop._release_request(alone_req)
    alone = snapshot(loop)[target]
    restore(loop, snap)
    mix = [serving.Request(i, cid, 0.0) for i, cid in enumerate([0, 1, 2, 3, 4])]
    for r in mix:
        assert loop._alloc_request(r)
    loop.run_tick(mix, loop._tick_scratch(mix))
    mixed = snapshot(loop)[target]
    assert np.array_equal(alone[0].cpu().numpy(), mixed[0].cpu().numpy())
    assert np.array_equal(alone[1].cpu().numpy(), mixed[1].cpu().numpy())
    assert alone_req.err == mix[target].err


def test_published_state_matches_device_update():
    import tenet_b200 as tb
    from tenet_b200 import itebd, serving

    loop = make_loop([(70, 0.05)])
    ch = loop.chains[0]
    rt = loop.rt
    n = ch.plans.a_space.size
    A = tb.TensorMap(rt, ch.plans.a_space, loop.arena.view(ch.a_off, n).clone())
    B = tb.TensorMap(rt, ch.plans.a_space, loop.arena.view(ch.b_off, n).clone())
    G = itebd.heisenberg_gate(rt, loop.rule, loop.P, ch.tau)
    res = itebd.bond_update(A, B, G, tb.Truncation.space(ch.plans.W))
    U, spectra, Vh = res.factors()
    r = serving.Request(0, 0, 0.0)
    assert loop._alloc_request(r)
    loop.run_tick([r])
    A_new = loop.arena.view(ch.a_off, n).cpu().numpy()
    np.testing.assert_allclose(A_new, U.to_host(), rtol=0, atol=1e-13)
    assert abs(r.err - res.error) <= 1e-12 * max(1.0, res.error)


def test_poisson_serving_completes_every_request():
    from tenet_b200 import serving

    chains = serving.chain_mix(12, seed=1)
    chains = [(min(D, 256), tau) for D, tau in chains]
    loop = make_loop(chains)
    reqs = serving.poisson_requests(len(chains), 60, rate=400.0, seed=2)
    done, wall = loop.serve(reqs)
    assert len(done) == 60
    lat = np.array([r.done - r.arrival for r in done])
    assert (lat > 0).all()
    assert all(np.isfinite(r.err) for r in done)


def test_chain_checkpoint_restores_and_replays_bit_for_bit():
    """A checkpoint taken from the live arena (v1 typed snapshots) restores the
    chain exactly: the update after a restore equals the update after the
    checkpoint, and the snapshot of the restored state equals the original."""
    from tenet_b200 import persistence, serving

    loop = make_loop([(90, 0.05), (140, 0.1)])

    def update(cid):
        req = serving.Request(0, cid, 0.0)
        assert loop._alloc_request(req)
        scratch = loop._tick_scratch([req])
        loop.run_tick([req], scratch)
        if scratch[0] is not None:
            loop.arena.release(*scratch)
        loop._release_request(req)
        return snapshot(loop)[cid]

    ckpt = loop.checkpoint_chain(1)
    first = update(1)
    loop.restore_chain(1, ckpt)
    assert loop.checkpoint_chain(1) == ckpt
    second = update(1)
    for x, y in zip(first, second):
        assert np.array_equal(x.cpu().numpy(), y.cpu().numpy())
    with pytest.raises(persistence.DecodeError):
        loop.restore_chain(0, ckpt)  # chain 0 has another bond space


def test_poisson_serving_in_ticks_completes_every_request():
    from tenet_b200 import serving

    chains = serving.chain_mix(12, seed=1)
    chains = [(min(D, 256), tau) for D, tau in chains]
    loop = make_loop(chains)
    reqs = serving.poisson_requests(len(chains), 60, rate=400.0, seed=2)
    done, wall = loop.serve_ticks(reqs)
    assert len(done) == 60
    assert all(np.isfinite(r.err) for r in done)


@pytest.mark.parametrize("precision", ["fp64", "i8x"])
def test_continuous_lanes_overlap_and_match_ticks(precision):
    """Continuous batching: a small chain's request that arrives while a large
    chain's update (a D = 2048 SVD of ~0.2 s) is on the GPU is admitted at
    once on another lane and finishes before the large one; and every chain
    state the continuous scheduler publishes is bit-identical to the tick
    scheduler's (and so to the request run alone)."""
    from tenet_b200 import serving

    chains = [(2048, 0.05), (64, 0.1), (96, 0.01)]
    loop = make_loop(chains, budget=8 << 30, precision=precision)
    snap = snapshot(loop)
    # warm up: plans, tile calibration and lane scratch, outside the measured run
    loop.serve([serving.Request(i, cid, 0.0) for i, cid in enumerate([0, 1, 2])])
    restore(loop, snap)
    reqs = [serving.Request(0, 0, 0.0), serving.Request(1, 1, 0.02), serving.Request(2, 2, 0.03)]
    done, _ = loop.serve(reqs)
    by = {r.rid: r for r in done}
    big, small = by[0], by[1]
    assert small.start < big.done  # admitted while the large update was in flight
    assert small.done < big.done, (small.done, big.done)  # and finished first
    assert by[1].lane != by[0].lane
    cont = snapshot(loop)
    errs = {r.cid: r.err for r in done}
    restore(loop, snap)
    tdone, _ = loop.serve_ticks([serving.Request(i, cid, 0.0) for i, cid in enumerate([0, 1, 2])])
    ticks = snapshot(loop)
    for (a1, b1), (a2, b2) in zip(cont, ticks):
        assert np.array_equal(a1.cpu().numpy(), a2.cpu().numpy())
        assert np.array_equal(b1.cpu().numpy(), b2.cpu().numpy())
    for r in tdone:
        assert r.err == errs[r.cid]
