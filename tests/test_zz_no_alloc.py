"""The allocation-free SVD entry point agrees with the allocating one.

``tnt_svd_static`` exists for callers that cannot allocate device memory
where they factorise: a serving loop holding a fixed device-memory budget, or
a foreign host whose own allocator owns every device byte.  It keeps its
scratch in a library-owned static device array instead.  This file is
collected last on purpose, so a run that stops at the first failure has
already run every other test; it also passes when run alone in a fresh
process.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _space_and_inputs(rt, seed):
    from oracle.tensor import normal_fill
    from tenet_b200 import typed

    rule = typed.SU2FusionRule()
    w = typed.GradedSpace(rule, [(0, 6), (1, 8), (2, 8), (3, 5), (4, 3)])
    p = typed.GradedSpace(rule, [(1, 1)])
    sp = rt.space(rule, [w, p], [p, w])
    return sp, normal_fill(seed, sp.size)


def _svd(rt, plan, data, static):
    import torch

    from tenet_b200 import _lib

    a = torch.as_tensor(data, device="cuda")
    u = torch.full((plan.u_size,), np.nan, dtype=torch.float64, device="cuda")
    s = torch.full((plan.s_size,), np.nan, dtype=torch.float64, device="cuda")
    vh = torch.full((plan.v_size,), np.nan, dtype=torch.float64, device="cuda")
    ptr = lambda x: C.c_void_p(x.data_ptr())
    if static:
        _lib.call("tnt_svd_static", plan._h, ptr(a), ptr(u), ptr(s), ptr(vh), rt.stream())
    else:
        _lib.call("tnt_svd", rt._h, plan._h, ptr(a), ptr(u), ptr(s), ptr(vh), rt.stream())
    torch.cuda.synchronize()
    return u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy()


def test_static_scratch_svd_matches_allocating_svd_twice():
    from tenet_b200 import Runtime

    rt = Runtime(0)
    for seed in (11, 12):  # two calls in a row: the second must not see the first's leftovers
        sp, data = _space_and_inputs(rt, seed)
        plan = rt.fplan(sp)
        u0, s0, v0 = _svd(rt, plan, data, static=False)
        u1, s1, v1 = _svd(rt, plan, data, static=True)
        assert np.isfinite(u1).all() and np.isfinite(s1).all() and np.isfinite(v1).all()
        np.testing.assert_allclose(s1, s0, rtol=1e-12, atol=1e-12 * np.abs(s0).max())
        np.testing.assert_allclose(u1, u0, atol=1e-11)
        np.testing.assert_allclose(v1, v0, atol=1e-11)


def test_static_scratch_svd_with_sectors_beyond_shared_memory_twice():
    """Sectors of 300 and 250 rows do not fit the 200 KB on-chip panel, so the
    static path runs the blocked kernel on work panels inside the static
    array (at non-zero offsets); about 0.31 Mi of its 1 Mi doubles.  The
    allocating path may run the same sectors on thread-block clusters, so the
    two agree to rounding: singular values to 1e-12 relative, singular vectors
    (same largest-entry gauge) to 1e-9, reconstructions to 1e-12."""
    from oracle.tensor import normal_fill
    from tenet_b200 import Runtime, typed

    rt = Runtime(0)
    rule = typed.U1FusionRule()
    v = typed.GradedSpace(rule, [(0, 300), (1, 250), (2, 7)])
    sp = rt.space(rule, [v], [v])
    plan = rt.fplan(sp)
    for seed in (21, 22):
        data = normal_fill(seed, sp.size)
        u0, s0, v0 = _svd(rt, plan, data, static=False)
        u1, s1, v1 = _svd(rt, plan, data, static=True)
        assert np.isfinite(u1).all() and np.isfinite(s1).all() and np.isfinite(v1).all()
        np.testing.assert_allclose(s1, s0, rtol=1e-12, atol=1e-12 * np.abs(s0).max())
        np.testing.assert_allclose(u1, u0, atol=1e-9)
        np.testing.assert_allclose(v1, v0, atol=1e-9)
        off_u = off_s = off_v = off_a = 0
        for d in (300, 250, 7):
            a = data[off_a: off_a + d * d].reshape(d, d).T
            uu = u1[off_u: off_u + d * d].reshape(d, d).T
            vv = v1[off_v: off_v + d * d].reshape(d, d).T
            ss = s1[off_s: off_s + d]
            rec = (uu * ss) @ vv
            assert np.linalg.norm(rec - a) <= 1e-12 * np.linalg.norm(a) * d ** 0.5
            off_u, off_v, off_a, off_s = off_u + d * d, off_v + d * d, off_a + d * d, off_s + d


def test_static_scratch_svd_rejects_plans_beyond_its_limit():
    from tenet_b200 import Runtime, _lib, typed

    rt = Runtime(0)
    rule = typed.U1FusionRule()
    big = typed.GradedSpace(rule, [(0, 1100)])
    plan = rt.fplan(rt.space(rule, [big], [big]))
    import torch

    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = _lib.lib().tnt_svd_static(plan._h, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                   C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), rt.stream())
    assert st == 1  # TNT_INVALID_ARGUMENT
    assert "static array" in _lib.last_error()
