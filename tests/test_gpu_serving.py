"""Continuous-batching iTEBD service: batching does not change results, and the
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
