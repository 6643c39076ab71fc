"""Serving request streams (host only): sessions of cohesive load steps."""
import numpy as np


def test_session_stream_orders_steps():
    """With session_steps > 1 every cohesive request opens a session: its steps 0..n-1 share one
    problem description (Ortiz-Pandolfi interfaces), arrive in step order and keep their session's
    seed; request ids stay unique and follow arrival order."""
    from pigfem_b200 import capi, serving
    reqs = serving.poisson_stream(12, rate=4.0, seed=7, scale=0.2, session_steps=4)
    assert [q.rid for q in reqs] == list(range(len(reqs)))
    assert all(a.arrival <= b.arrival for a, b in zip(reqs, reqs[1:]))
    sess = {}
    for q in reqs:
        if q.session >= 0:
            sess.setdefault(q.session, []).append(q)
    assert sess
    n_first = sum(1 for q in reqs if q.session < 0) + len(sess)
    assert n_first == 12
    for v in sess.values():
        assert [q.step for q in v] == [0, 1, 2, 3]
        assert all(q.steps == 4 and q.kind == "cohesive_step" for q in v)
        assert all(q.desc is v[0].desc for q in v)
        assert v[0].desc.coh_law == capi.COH_OP
    plain = serving.poisson_stream(12, rate=4.0, seed=7, scale=0.2)
    assert all(q.session < 0 for q in plain) and len(plain) == 12
