"""The TensorKit invariant stream run entirely through the device path.

Same op sequence and tolerances as tenet/tests/semantic_suite.rs:835-905
(norm / tr to 1e-9, singular values to 1e-8) and the weighted-rank truncation
fixture (semantic_suite.rs:762-830); expected values from
tests/golden/tensorkit_semantic.json.
"""

import numpy as np
import pytest

from tests.test_oracle_golden import STREAMS, oracle_fill

pytestmark = pytest.mark.gpu


def build(rt, name):
    from tenet_b200 import typed

    orule, pairs, label = STREAMS[name]
    rule = typed.FusionRule(list(orule.factors), orule.codec)
    v = typed.GradedSpace(rule, pairs)

    def tensor(c0):
        def fn(key, idx):
            (cu, _, cc, _), (du, _, _, _) = key
            return oracle_fill(c0, [label(cu[0]), label(cu[1]), label(du[0]), label(du[1]), label(cc)], idx)

        return typed.TensorMap.from_block_fn(rt, [v, v], [v, v], fn)

    return rule, label, tensor(3), tensor(5)


@pytest.fixture(scope="module")
def rt():
    from tenet_b200 import Runtime

    return Runtime(0)


@pytest.mark.parametrize("name", sorted(STREAMS))
def test_invariant_stream_on_device(rt, golden, name):
    rule, label, a, b = build(rt, name)
    c = a.compose(b)
    d = a.permute([1, 0], [3, 2])
    e = d.compose(c)
    g = a.adjoint().compose(a)
    h = e.add(a, 1.0, 0.5)
    hh = h.compose(h).tr()
    got = dict(
        s1a=(a.norm(), a.tr()), s1b=(b.norm(), b.tr()), s2=(c.norm(), c.tr()), s3=(d.norm(), d.tr()),
        s4=(e.norm(), e.tr()), s5=(g.norm(), g.tr()), s7=(h.norm(), h.tr()), s8=(hh, hh),
    )
    exp = golden["streams"][name]
    for step, (n, t) in got.items():
        en, et = exp["steps"][step]
        assert abs(n - en) <= 1e-9 * max(1.0, abs(en)), (step, n, en)
        assert abs(t - et) <= 1e-9 * max(1.0, abs(et)), (step, t, et)
    res = e.svd_compact()
    values = sorted(np.concatenate([s.values for s in res.singular_values]), reverse=True)
    assert len(values) == exp["svdcount"]
    sv = np.array(exp["svd"])
    sig = sv[sv > 1e-6 * sv[0]]
    np.testing.assert_allclose(values[: len(sig)], sig, rtol=1e-8)


@pytest.mark.parametrize("name", ["U1", "SU2"])
def test_weighted_rank_truncation_on_device(rt, golden, name):
    from tenet_b200 import Truncation

    rule, label, a, b = build(rt, name)
    e = a.permute([1, 0], [3, 2]).compose(a.compose(b))
    res = e.svd_trunc(Truncation.rank(5))
    got = sorted((label(rule.label(ent.sector)), len(ent.values)) for ent in res.singular_values if len(ent.values))
    exp = golden["truncation"][name]
    assert got == sorted(tuple(x) for x in exp["kept"])
    assert abs(res.error - exp["error"]) <= 1e-10 * exp["error"]


def test_qspace_spin_half_operator_on_device(rt):
    """The QSpace spin-half known answers (benchmarks/qspace_su2_oracle.out)
    through the device compose, adjoint and weighted norm."""
    from tenet_b200 import typed

    rule = typed.SU2FusionRule()
    p, a = typed.GradedSpace(rule, [(1, 1)]), typed.GradedSpace(rule, [(2, 1)])
    s = typed.TensorMap.from_host(rt, [p], [p, a], np.array([-8.660254037844387e-01]))
    assert abs(s.norm() ** 2 - 1.5) <= 1e-14
    cas = s.compose(s.adjoint())
    assert abs(cas.to_host()[0] - 0.75) <= 1e-14
